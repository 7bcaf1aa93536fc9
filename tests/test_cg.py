"""The device conjugate gradient (pyfwi_b200.cg) against SciPy's fmin_cg, the
optimiser PyFWI's FWI.cg calls (src/PyFWI/fwi.py:180-182: gtol=1e-8,
maxiter=ITER), with the reference's evaluation pattern (MemoizeJac: one
evaluation of misfit and gradient per point).

Run on CPU float64 tensors: the same evaluations in the same order and the
same iterates to rounding, including an iteration that needs the
bracketing-and-zoom search and a run the line search ends; on Rosenbrock's
valley and ill-conditioned quadratics rounding differences grow with the
iterations, so those are compared over their first iterations."""
import numpy as np
import pytest
import torch
from scipy.optimize import fmin_cg
from scipy.optimize._optimize import MemoizeJac

from pyfwi_b200 import cg


def rosenbrock(x):
    r = x[1:] - x[:-1] ** 2
    f = np.sum(100.0 * r ** 2 + (1 - x[:-1]) ** 2)
    g = np.zeros_like(x)
    g[1:] += 200 * r
    g[:-1] += -400 * x[:-1] * r - 2 * (1 - x[:-1])
    return f, g


def quadratic(seed=0, n=60):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n))
    a = a @ a.T + np.diag(np.logspace(0, 4, n))
    b = rng.standard_normal(n)
    return lambda x: (0.5 * x @ a @ x - b @ x, a @ x - b)


def wavy(x):
    return np.sum(x ** 2) + 10 * np.sum(np.sin(3 * x)), 2 * x + 30 * np.cos(3 * x)


def softplus_like(x):
    return np.sum(np.log(np.cosh(3 * x))) + 0.01 * np.sum(x ** 4), 3 * np.tanh(3 * x) + 0.04 * x ** 3


def _both(fun, x0, maxiter):
    ev_s, xs_s = [], []

    def f_and_g(x):
        ev_s.append(np.copy(x))
        return fun(x)
    m = MemoizeJac(f_and_g)
    out = fmin_cg(m, x0, m.derivative, gtol=1e-8, maxiter=maxiter, full_output=True, disp=False,
                  callback=lambda xk: xs_s.append(np.copy(xk)))
    ev_t, xs_t = [], []

    def ft(t):
        ev_t.append(t.numpy().copy())
        f, g = fun(t.numpy())
        return float(f), torch.from_numpy(np.asarray(g, np.float64))
    res = cg.minimize(ft, torch.from_numpy(x0), gtol=1e-8, maxiter=maxiter,
                      callback=lambda t: xs_t.append(t.numpy().copy()))
    return (out, ev_s, xs_s), (res, ev_t, xs_t)


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("fun,x0,maxiter", [(softplus_like, np.linspace(-3, 4, 30), 100),
                                            (rosenbrock, np.array([-1.2, 1.0]), 200)])
def test_converging_runs_match_scipy(fun, x0, maxiter):
    (out, ev_s, xs_s), (res, ev_t, xs_t) = _both(fun, x0, maxiter)
    assert res.status == out[4] == 0
    assert len(ev_t) == len(ev_s) and res.nit == len(xs_s)
    # on the start's scale (iterates shrink towards the minimum); trial points
    # of a line search in Rosenbrock's valley magnify rounding differences
    scale = np.abs(x0).max()
    for a, b in zip(ev_t, ev_s):
        assert np.abs(a - b).max() <= 1e-6 * scale
    assert np.abs(res.x.numpy() - out[0]).max() <= 1e-9 * scale


def test_bracketing_search_is_used_and_matches():
    """On the 2-D Rosenbrock function one iteration needs the fallback
    search (the Moré-Thuente step fails the descent test)."""
    (out, ev_s, xs_s), (res, ev_t, xs_t) = _both(rosenbrock, np.array([-1.2, 1.0]), 200)
    assert res.fallbacks >= 1
    assert len(ev_t) == len(ev_s)
    assert _rel(res.x.numpy(), out[0]) < 1e-9


def test_failed_line_search_ends_the_run():
    (out, ev_s, xs_s), (res, ev_t, xs_t) = _both(wavy, np.linspace(-4, 4, 12), 200)
    assert res.status == out[4] == 2 and res.fallbacks >= 1
    for a, b in zip(xs_t, xs_s):
        assert _rel(a, b) < 1e-9
    assert _rel(res.x.numpy(), out[0]) < 1e-9


@pytest.mark.parametrize("fun,x0,iters", [(quadratic(), np.zeros(60), 60),
                                          (rosenbrock, np.array([-1.2, 1.0] * 10), 30)])
def test_first_iterations_match_scipy(fun, x0, iters):
    (out, ev_s, xs_s), (res, ev_t, xs_t) = _both(fun, x0, iters)
    assert res.nit == len(xs_s) == iters and len(ev_t) == len(ev_s)
    for a, b in zip(xs_t, xs_s):
        assert _rel(a, b) < 1e-8
