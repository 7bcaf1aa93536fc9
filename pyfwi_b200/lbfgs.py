"""L-BFGS with the model, gradient and history vectors on the device.

PyFWI's ``FWI.lbfgs`` (src/PyFWI/fwi.py:197-226) hands its misfit to SciPy's
``fmin_l_bfgs_b`` with ``m=10, factr=1e7, pgtol=1e-8, bounds=None,
maxfun=15000, maxiter=ITER, maxls=10`` (SciPy 1.7.3 in the reference's
requirements.txt:4: L-BFGS-B 3.0, Zhu, Byrd, Lu & Nocedal, ACM TOMS 23
(1997), with the Morales & Nocedal (2011) update).  This module restates
that method for the case the reference uses, no bounds, where it reduces to:

* after a start or a reset of the memory, the generalised Cauchy point
  x - g / theta with theta = 1, so d = (x - g) - x; the first trial step of
  the first iteration is 1 / ||d||, every other trial starts at 1;
* with stored pairs, d = (x - H g) - x, H the limited-memory BFGS inverse
  of the last m accepted pairs (s, y) with H0 = I / theta, theta = y'y / s'y
  of the newest pair.  L-BFGS-B forms the compact representation of
  B = H^-1 and solves with it; here H is applied by the two-loop recursion
  (Nocedal, Math. Comp. 35 (1980)): the same matrix in exact arithmetic;
* a direction with g'd >= 0 resets the memory (or ends the run when the
  memory is empty);
* the Moré-Thuente line search (MINPACK-2 dcsrch / dcstep, Moré & Thuente,
  ACM TOMS 20 (1994)) with ftol = 1e-3, gtol = 0.9, xtol = 0.1,
  stpmin = 0, stpmax = 1e10; when it has not converged after ``maxls``
  evaluations the previous iterate is restored and the memory reset;
* the pair (s, y) = (stp d, g_new - g_old) is stored only when
  s'y > eps * stp * (-g'd);
* the run ends when max|g| <= pgtol, when (f_old - f) <= factr * eps *
  max(|f_old|, |f|, 1), after ``maxiter`` iterations, or when the number of
  evaluations exceeds ``maxfun``.

x, g, d and the 2m history vectors stay where x0 is (the GPU in FWI), in
float64 as in SciPy.  Per evaluation two scalars, f and g'd, reach the host,
where the line search chooses the next trial step."""
import math

import torch

EPS = 2.220446049250313e-16  # float64 machine epsilon (L-BFGS-B's epsmch)
STPMAX = 1e10
FTOL, GTOL, XTOL = 1e-3, 0.9, 0.1


def _cstep(stx, fx, dx, sty, fy, dy, stp, fp, dp, brackt, stpmin, stpmax):
    """One safeguarded step of the Moré-Thuente search (MINPACK-2 dcstep):
    the new trial step from the best point (stx), the other end of the
    interval (sty) and the current trial (stp), each with its function value
    and derivative.  Returns the updated (stx, fx, dx, sty, fy, dy, stp,
    brackt)."""
    sgnd = dp * (dx / abs(dx))
    if fp > fx:
        # higher value: the minimum is bracketed; cubic or cubic/quadratic mean
        theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp
        s = max(abs(theta), abs(dx), abs(dp))
        gamma = s * math.sqrt((theta / s) ** 2 - (dx / s) * (dp / s))
        if stp < stx:
            gamma = -gamma
        p = (gamma - dx) + theta
        q = ((gamma - dx) + gamma) + dp
        stpc = stx + (p / q) * (stp - stx)
        stpq = stx + ((dx / ((fx - fp) / (stp - stx) + dx)) / 2.0) * (stp - stx)
        stpf = stpc if abs(stpc - stx) < abs(stpq - stx) else stpc + (stpq - stpc) / 2.0
        brackt = True
    elif sgnd < 0.0:
        # lower value, derivatives of opposite sign: bracketed; cubic or secant
        theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp
        s = max(abs(theta), abs(dx), abs(dp))
        gamma = s * math.sqrt((theta / s) ** 2 - (dx / s) * (dp / s))
        if stp > stx:
            gamma = -gamma
        p = (gamma - dp) + theta
        q = ((gamma - dp) + gamma) + dx
        stpc = stp + (p / q) * (stx - stp)
        stpq = stp + (dp / (dp - dx)) * (stx - stp)
        stpf = stpc if abs(stpc - stp) > abs(stpq - stp) else stpq
        brackt = True
    elif abs(dp) < abs(dx):
        # lower value, same sign, the derivative shrinks
        theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp
        s = max(abs(theta), abs(dx), abs(dp))
        gamma = s * math.sqrt(max(0.0, (theta / s) ** 2 - (dx / s) * (dp / s)))
        if stp > stx:
            gamma = -gamma
        p = (gamma - dp) + theta
        q = (gamma + (dx - dp)) + gamma
        r = p / q
        if r < 0.0 and gamma != 0.0:
            stpc = stp + r * (stx - stp)
        elif stp > stx:
            stpc = stpmax
        else:
            stpc = stpmin
        stpq = stp + (dp / (dp - dx)) * (stx - stp)
        if brackt:
            stpf = stpc if abs(stpc - stp) < abs(stpq - stp) else stpq
            if stp > stx:
                stpf = min(stp + 0.66 * (sty - stp), stpf)
            else:
                stpf = max(stp + 0.66 * (sty - stp), stpf)
        else:
            stpf = stpc if abs(stpc - stp) > abs(stpq - stp) else stpq
            stpf = max(stpmin, min(stpmax, stpf))
    else:
        # lower value, same sign, the derivative does not shrink
        if brackt:
            theta = 3.0 * (fp - fy) / (sty - stp) + dy + dp
            s = max(abs(theta), abs(dy), abs(dp))
            gamma = s * math.sqrt((theta / s) ** 2 - (dy / s) * (dp / s))
            if stp > sty:
                gamma = -gamma
            p = (gamma - dp) + theta
            q = ((gamma - dp) + gamma) + dy
            stpf = stp + (p / q) * (sty - stp)
        elif stp > stx:
            stpf = stpmax
        else:
            stpf = stpmin
    if fp > fx:
        sty, fy, dy = stp, fp, dp
    else:
        if sgnd < 0.0:
            sty, fy, dy = stx, fx, dx
        stx, fx, dx = stp, fp, dp
    return stx, fx, dx, sty, fy, dy, stpf, brackt


class LineSearch:
    """Moré-Thuente search for a step satisfying f(stp) <= f(0) + ftol stp
    g(0) and |g(stp)| <= gtol |g(0)| (MINPACK-2 dcsrch).  ``start`` takes
    f(0), g(0) and the first trial; each ``step`` takes f and the
    directional derivative at the last trial and returns ('FG', next trial),
    ('CONV', stp) or ('WARN', stp)."""

    def __init__(self, ftol=FTOL, gtol=GTOL, xtol=XTOL, stpmin=0.0, stpmax=STPMAX):
        self.ftol, self.gtol, self.xtol = ftol, gtol, xtol
        self.stpmin, self.stpmax = stpmin, stpmax

    def start(self, f, g, stp):
        if stp < self.stpmin or stp > self.stpmax or g >= 0.0:
            raise ValueError("line search started with an invalid step or an ascent direction")
        self.brackt, self.stage = False, 1
        self.finit, self.ginit = f, g
        self.gtest = self.ftol * g
        self.width = self.stpmax - self.stpmin
        self.width1 = self.width / 0.5
        self.stx, self.fx, self.gx = 0.0, f, g
        self.sty, self.fy, self.gy = 0.0, f, g
        self.stmin, self.stmax = 0.0, stp + 4.0 * stp
        return "FG", stp

    def step(self, stp, f, g):
        ftest = self.finit + stp * self.gtest
        if self.stage == 1 and f <= ftest and g >= 0.0:
            self.stage = 2
        task = None
        if self.brackt and (stp <= self.stmin or stp >= self.stmax):
            task = "WARN"  # rounding errors prevent progress
        if self.brackt and self.stmax - self.stmin <= self.xtol * self.stmax:
            task = "WARN"  # xtol test satisfied
        if stp == self.stpmax and f <= ftest and g <= self.gtest:
            task = "WARN"  # stp = stpmax
        if stp == self.stpmin and (f > ftest or g >= self.gtest):
            task = "WARN"  # stp = stpmin
        if f <= ftest and abs(g) <= self.gtol * (-self.ginit):
            task = "CONV"
        if task is not None:
            return task, stp
        if self.stage == 1 and f <= self.fx and f > ftest:
            # modified function psi(stp) = f - f(0) - ftol stp g(0) until stage 2
            gt = self.gtest
            stx, fxm, gxm, sty, fym, gym, stp, self.brackt = _cstep(
                self.stx, self.fx - self.stx * gt, self.gx - gt, self.sty, self.fy - self.sty * gt, self.gy - gt,
                stp, f - stp * gt, g - gt, self.brackt, self.stmin, self.stmax)
            self.stx, self.sty = stx, sty
            self.fx, self.fy = fxm + stx * gt, fym + sty * gt
            self.gx, self.gy = gxm + gt, gym + gt
        else:
            (self.stx, self.fx, self.gx, self.sty, self.fy, self.gy, stp,
             self.brackt) = _cstep(self.stx, self.fx, self.gx, self.sty, self.fy, self.gy, stp, f, g,
                                   self.brackt, self.stmin, self.stmax)
        if self.brackt:
            if abs(self.sty - self.stx) >= 0.66 * self.width1:
                stp = self.stx + 0.5 * (self.sty - self.stx)
            self.width1 = self.width
            self.width = abs(self.sty - self.stx)
            self.stmin, self.stmax = min(self.stx, self.sty), max(self.stx, self.sty)
        else:
            self.stmin = stp + 1.1 * (stp - self.stx)
            self.stmax = stp + 4.0 * (stp - self.stx)
        stp = min(max(stp, self.stpmin), self.stpmax)
        if (self.brackt and (stp <= self.stmin or stp >= self.stmax)) or \
                (self.brackt and self.stmax - self.stmin <= self.xtol * self.stmax):
            stp = self.stx
        return "FG", stp


class Memory:
    """The last m accepted pairs (s, y) and 1/(y's), newest last."""

    def __init__(self, m):
        self.m = m
        self.reset()

    def reset(self):
        self.s, self.y, self.rho = [], [], []
        self.theta = 1.0

    def __len__(self):
        return len(self.s)

    def push(self, s, y, sy, yy):
        if len(self.s) == self.m:
            self.s.pop(0), self.y.pop(0), self.rho.pop(0)
        self.s.append(s)
        self.y.append(y)
        self.rho.append(1.0 / sy)
        self.theta = yy / sy

    def apply_inverse(self, g):
        """H g by the two-loop recursion with H0 = I / theta.  Every scalar
        stays a device tensor, so the loop queues without host round trips."""
        q = g.clone()
        alpha = []
        for s, y, rho in zip(reversed(self.s), reversed(self.y), reversed(self.rho)):
            a = rho * torch.dot(s, q)
            q.sub_(a * y)
            alpha.append(a)
        q.div_(self.theta)
        for s, y, rho, a in zip(self.s, self.y, self.rho, reversed(alpha)):
            b = rho * torch.dot(y, q)
            q.add_((a - b) * s)
        return q


class Result:
    """Outcome of ``minimize``: final x and f, iterations, evaluations, why
    it stopped, f after each iteration, and how often a failed line search
    reset the memory."""

    def __init__(self, x, f, nit, nfev, task, history, resets=0):
        self.x, self.f, self.nit, self.nfev, self.task, self.history = x, f, nit, nfev, task, history
        self.resets = resets


def minimize(fun, x0, m=10, factr=1e7, pgtol=1e-8, maxfun=15000, maxiter=15000, maxls=10, callback=None):
    """Minimise ``fun`` from ``x0`` (a float64 tensor on any device) with the
    unbounded L-BFGS-B iteration described in the module docstring.

    ``fun(x) -> (f, g)``: the float misfit and its gradient, a tensor shaped
    like x.  ``callback(x)`` runs after every iteration.  Returns a
    ``Result``."""
    x = x0.detach().clone().to(torch.float64)
    f, g = fun(x)
    g = g.to(torch.float64)
    nfev = 1
    tol = factr * EPS
    mem = Memory(m)
    nit = resets = 0
    history = []
    if float(g.abs().max()) <= pgtol:
        return Result(x, f, 0, nfev, "CONVERGENCE: NORM_OF_PROJECTED_GRADIENT_<=_PGTOL", history, resets)
    search = LineSearch()
    while True:
        # search direction, written as (x + step) - x as L-BFGS-B forms it
        z = x - g if len(mem) == 0 else x - mem.apply_inverse(g)
        d = z - x
        dnorm = math.sqrt(float(torch.dot(d, d)))
        stp = min(1.0 / dnorm, STPMAX) if nit == 0 else 1.0
        x_old, g_old, f_old = x, g, f
        gd0 = float(torch.dot(g, d))
        failed = gd0 >= 0.0
        if not failed:
            task, stp = search.start(f, gd0, stp)
            evals = 0
            while True:
                if evals >= maxls:
                    failed = True
                    break
                x = z if stp == 1.0 else torch.add(x_old, d, alpha=stp)
                f, g = fun(x)
                g = g.to(torch.float64)
                nfev += 1
                evals += 1
                gd = float(torch.dot(g, d))
                task, stp = search.step(stp, f, gd)
                if task != "FG":
                    break
        if failed:
            x, g, f = x_old, g_old, f_old
            if len(mem) == 0:
                return Result(x, f, nit, nfev, "ABNORMAL_TERMINATION_IN_LNSRCH", history, resets)
            mem.reset()
            resets += 1
            continue
        nit += 1
        history.append(f)
        if callback is not None:
            callback(x)
        if nit >= maxiter:
            return Result(x, f, nit, nfev, "STOP: TOTAL NO. of ITERATIONS REACHED LIMIT", history, resets)
        if nfev > maxfun:
            return Result(x, f, nit, nfev, "STOP: TOTAL NO. of F,G EVALUATIONS EXCEEDS LIMIT", history, resets)
        if float(g.abs().max()) <= pgtol:
            return Result(x, f, nit, nfev, "CONVERGENCE: NORM_OF_PROJECTED_GRADIENT_<=_PGTOL", history, resets)
        if f_old - f <= tol * max(abs(f_old), abs(f), 1.0):
            return Result(x, f, nit, nfev, "CONVERGENCE: REL_REDUCTION_OF_F_<=_FACTR*EPSMCH", history, resets)
        y = g - g_old
        if stp == 1.0:
            dr, ddum, s = gd - gd0, -gd0, d
        else:
            dr, ddum, s = (gd - gd0) * stp, -gd0 * stp, d * stp
        if dr <= EPS * ddum:
            continue  # curvature too small: keep the memory as it is
        mem.push(s, y, dr, float(torch.dot(y, y)))
