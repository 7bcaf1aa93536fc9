"""Nonlinear conjugate gradient with the vectors on the device.

PyFWI's ``FWI.cg`` (src/PyFWI/fwi.py:162-195) hands its misfit to SciPy's
``fmin_cg(fun, m, jac, gtol=1e-8, maxiter=ITER)`` (SciPy 1.7.3 in the
reference's requirements.txt:4).  This module restates that method:

* Polak-Ribiere+ directions, p_{k+1} = -g_{k+1} + max(0, y'g_{k+1} / g'g) p_k
  (Gilbert & Nocedal, SIAM J. Optim. 2 (1992)), starting from p_0 = -g_0;
* each step from a line search for the strong Wolfe conditions with
  c1 = 1e-4, c2 = 0.4, accepted only if the new direction is a sufficient
  descent direction, p'g <= -0.01 g'g, or the gradient already meets gtol;
* the line search is first the Moré-Thuente search (MINPACK-2 dcsrch, as in
  ``lbfgs.LineSearch``; xtol = 1e-14, steps in [1e-100, 1e100], at most 100
  rounds, a warning counts as failure), its first trial
  min(1, 2.02 (f_k - f_{k-1}) / g'p) (f_{-1} = f_0 + ||g_0|| / 2); if it
  fails or its step is not a descent step, the bracketing and zoom search of
  Nocedal & Wright, Numerical Optimization, algorithms 3.5 and 3.6 (trial
  steps doubled up to 10 times, then at most 11 cubic / quadratic /
  bisection zoom trials with the safeguards 0.2 and 0.1 of the interval);
  if that fails too the run stops;
* the run stops when max|g| <= gtol or after maxiter iterations.

x, g and p stay where x0 is (the GPU in FWI), in float64; the function and
the directional derivatives reach the host for the line-search decisions.
Each distinct point is evaluated once (function and gradient together)."""
import math

import torch

from .lbfgs import LineSearch

SIGMA3 = 0.01  # sufficient-descent constant of the Polak-Ribiere+ test


class _Evaluations:
    """(f, g) of the last point asked for; a point equal to it bit for bit
    is not evaluated again."""

    def __init__(self, fun):
        self.fun = fun
        self.x = None
        self.nfev = 0

    def __call__(self, x):
        if self.x is None or not torch.equal(x, self.x):
            f, g = self.fun(x)
            self.x, self.f, self.g = x.clone(), float(f), g.to(torch.float64)
            self.nfev += 1
        return self.f, self.g


def _cubic_min(a, fa, fpa, b, fb, c, fc):
    """Minimiser of the cubic through (a, fa) with slope fpa at a, (b, fb)
    and (c, fc); None when it does not exist."""
    try:
        db, dc = b - a, c - a
        denom = (db * dc) ** 2 * (db - dc)
        rb, rc = fb - fa - fpa * db, fc - fa - fpa * dc
        A = (dc ** 2 * rb - db ** 2 * rc) / denom
        B = (-dc ** 3 * rb + db ** 3 * rc) / denom
        radical = B * B - 3 * A * fpa
        x = a + (-B + math.sqrt(radical)) / (3 * A)
    except (ArithmeticError, ValueError):
        return None
    return x if math.isfinite(x) else None


def _quad_min(a, fa, fpa, b, fb):
    """Minimiser of the parabola through (a, fa) with slope fpa and (b, fb)."""
    try:
        db = b - a
        B = (fb - fa - fpa * db) / (db * db)
        x = a - fpa / (2.0 * B)
    except ArithmeticError:
        return None
    return x if math.isfinite(x) else None


def _zoom(a_lo, a_hi, phi_lo, phi_hi, dphi_lo, phi, dphi, phi0, dphi0, c1, c2, accept):
    """Nocedal & Wright algorithm 3.6 (the interpolation and the stopping
    rule of SciPy's line_search_wolfe2): (step, phi, dphi) or (None, ...)."""
    a_rec, phi_rec = 0.0, phi0
    for i in range(11):
        dalpha = a_hi - a_lo
        lo, hi = (a_hi, a_lo) if dalpha < 0 else (a_lo, a_hi)
        a_j = None
        if i > 0:
            a_j = _cubic_min(a_lo, phi_lo, dphi_lo, a_hi, phi_hi, a_rec, phi_rec)
            cchk = 0.2 * dalpha
        if i == 0 or a_j is None or a_j > hi - cchk or a_j < lo + cchk:
            qchk = 0.1 * dalpha
            a_j = _quad_min(a_lo, phi_lo, dphi_lo, a_hi, phi_hi)
            if a_j is None or a_j > hi - qchk or a_j < lo + qchk:
                a_j = a_lo + 0.5 * dalpha
        phi_j = phi(a_j)
        if phi_j > phi0 + c1 * a_j * dphi0 or phi_j >= phi_lo:
            a_rec, phi_rec = a_hi, phi_hi
            a_hi, phi_hi = a_j, phi_j
        else:
            dphi_j = dphi(a_j)
            if abs(dphi_j) <= -c2 * dphi0 and accept(a_j, phi_j):
                return a_j, phi_j, dphi_j
            if dphi_j * (a_hi - a_lo) >= 0:
                a_rec, phi_rec = a_hi, phi_hi
                a_hi, phi_hi = a_lo, phi_lo
            else:
                a_rec, phi_rec = a_lo, phi_lo
            a_lo, phi_lo, dphi_lo = a_j, phi_j, dphi_j
    return None, None, None


def _bracket_zoom(phi, dphi, phi0, old_phi0, dphi0, c1, c2, amax, accept):
    """Nocedal & Wright algorithm 3.5 with SciPy's line_search_wolfe2
    choices: (step, phi) or (None, None)."""
    a0 = 0.0
    a1 = min(1.0, 1.01 * 2 * (phi0 - old_phi0) / dphi0) if old_phi0 is not None and dphi0 != 0 else 1.0
    if a1 < 0:
        a1 = 1.0
    a1 = min(a1, amax)
    phi_a1, phi_a0, dphi_a0 = phi(a1), phi0, dphi0
    for i in range(10):
        if a1 == 0 or a0 > amax:
            return None, None
        if phi_a1 > phi0 + c1 * a1 * dphi0 or (phi_a1 >= phi_a0 and i > 0):
            a, p, _ = _zoom(a0, a1, phi_a0, phi_a1, dphi_a0, phi, dphi, phi0, dphi0, c1, c2, accept)
            return a, p
        dphi_a1 = dphi(a1)
        if abs(dphi_a1) <= -c2 * dphi0 and accept(a1, phi_a1):
            return a1, phi_a1
        if dphi_a1 >= 0:
            a, p, _ = _zoom(a1, a0, phi_a1, phi_a0, dphi_a1, phi, dphi, phi0, dphi0, c1, c2, accept)
            return a, p
        a0, a1 = a1, min(2 * a1, amax)
        phi_a0, dphi_a0 = phi_a1, dphi_a1
        phi_a1 = phi(a1)
    # no conforming step after the doublings: SciPy reports a warning and
    # returns the last trial, whose gradient it has not checked
    return a1, phi_a1


class Result:
    """Outcome of ``minimize``: x, f, iterations, evaluations, status (0
    converged, 1 maxiter, 2 line search failed), and how many iterations
    needed the bracketing search."""

    def __init__(self, x, f, nit, nfev, status, fallbacks):
        self.x, self.f, self.nit, self.nfev, self.status = x, f, nit, nfev, status
        self.fallbacks = fallbacks


def minimize(fun, x0, gtol=1e-5, maxiter=None, c1=1e-4, c2=0.4, callback=None):
    """Minimise ``fun`` (x -> (f, g)) from ``x0`` (float64 tensor, any
    device) as described in the module docstring; returns a ``Result``."""
    ev = _Evaluations(fun)
    xk = x0.detach().clone().to(torch.float64)
    if maxiter is None:
        maxiter = xk.numel() * 200
    old_fval, gfk = ev(xk)
    old_old_fval = old_fval + float(torch.linalg.vector_norm(gfk)) / 2
    pk = -gfk
    gnorm = float(gfk.abs().max())
    k, status, fallbacks = 0, 0, 0
    while gnorm > gtol and k < maxiter:
        deltak = float(torch.dot(gfk, gfk))

        def pr_step(alpha, gfkp1):
            xkp1 = xk + alpha * pk
            beta = max(0.0, float(torch.dot(gfkp1 - gfk, gfkp1)) / deltak)
            pkp1 = -gfkp1 + beta * pk
            return alpha, xkp1, pkp1, gfkp1, float(gfkp1.abs().max())

        cached = [None]

        def descent(alpha, gfkp1):
            cached[0] = pr_step(alpha, gfkp1)
            _, _, p1, g1, gn = cached[0]
            return gn <= gtol or float(torch.dot(p1, g1)) <= -SIGMA3 * float(torch.dot(g1, g1))

        last_g = [None]

        def phi(s):
            return ev(xk + s * pk)[0]

        def dphi(s):
            last_g[0] = (s, ev(xk + s * pk)[1])
            return float(torch.dot(last_g[0][1], pk))

        dphi0 = float(torch.dot(gfk, pk))
        # Moré-Thuente first
        alpha1 = 1.0
        if dphi0 != 0:
            alpha1 = min(1.0, 1.01 * 2 * (old_fval - old_old_fval) / dphi0)
            if alpha1 < 0:
                alpha1 = 1.0
        search = LineSearch(ftol=c1, gtol=c2, xtol=1e-14, stpmin=1e-100, stpmax=1e100)
        phi1, d1, stp = old_fval, dphi0, alpha1
        for i in range(100):
            task, stp = search.start(phi1, d1, stp) if i == 0 else search.step(stp, phi1, d1)
            if not math.isfinite(stp):
                task = "WARN"
                break
            if task != "FG":
                break
            phi1, d1 = phi(stp), dphi(stp)
        else:
            task = "WARN"  # no conforming step within 100 rounds
        alpha_k = stp if task == "CONV" else None
        new_f, gfkp1 = phi1, (last_g[0][1] if last_g[0] is not None else None)
        if alpha_k is not None and not descent(alpha_k, gfkp1):
            alpha_k = None
        if alpha_k is None:
            fallbacks += 1
            # bracketing and zoom, as SciPy's fallback
            def accept(alpha, phi_a):
                if last_g[0] is None or last_g[0][0] != alpha:
                    dphi(alpha)
                return descent(alpha, last_g[0][1])
            alpha_k, new_f = _bracket_zoom(phi, dphi, old_fval, old_old_fval, dphi0, c1, c2, 1e100, accept)
            if alpha_k is None:
                status = 2
                break
            gfkp1 = last_g[0][1] if last_g[0] is not None and last_g[0][0] == alpha_k else None
        old_old_fval, old_fval = old_fval, new_f
        if cached[0] is not None and alpha_k == cached[0][0]:
            _, xk, pk, gfk, gnorm = cached[0]
        else:
            if gfkp1 is None:
                gfkp1 = ev(xk + alpha_k * pk)[1]
            _, xk, pk, gfk, gnorm = pr_step(alpha_k, gfkp1)
        k += 1
        if callback is not None:
            callback(xk)
    if status == 0 and k >= maxiter:
        status = 1
    return Result(xk, old_fval, k, ev.nfev, status, fallbacks)
