"""The device L-BFGS (pyfwi_b200.lbfgs) against SciPy's L-BFGS-B, the
optimiser PyFWI's FWI.lbfgs calls (src/PyFWI/fwi.py:214-218, same settings:
m=10, factr=1e7, pgtol=1e-8, bounds=None, maxls=10).

Run on CPU float64 tensors: the same evaluations in the same order, the
same iteration and evaluation counts and stopping reason, iterates equal to
rounding (on Rosenbrock's valley rounding differences grow with the
iterations, so its iterates are compared over the first 30)."""
import numpy as np
import pytest
import torch
from scipy.optimize import fmin_l_bfgs_b

from pyfwi_b200 import lbfgs

SETTINGS = dict(m=10, factr=1e7, pgtol=1e-8, maxfun=15000, maxls=10)


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


def _both(fun, x0, maxiter, fresh=None):
    """(scipy: iterates, evaluations, info), (ours: iterates, evaluations,
    result); ``fresh()`` makes a new objective for each run when it keeps
    state."""
    xs_s, ev_s = [], []

    def fs(x):
        ev_s.append(np.copy(x))
        return fun(x)

    _, _, info = fmin_l_bfgs_b(fs, x0, None, maxiter=maxiter, callback=lambda xk: xs_s.append(np.copy(xk)),
                               **SETTINGS)
    xs_t, ev_t = [], []
    fun = fresh() if fresh is not None else fun

    def ft(t):
        ev_t.append(t.numpy().copy())
        f, g = fun(t.numpy())
        return float(f), torch.from_numpy(np.asarray(g, np.float64))

    res = lbfgs.minimize(ft, torch.from_numpy(x0), maxiter=maxiter, callback=lambda t: xs_t.append(t.numpy().copy()),
                         **SETTINGS)
    return (xs_s, ev_s, info), (xs_t, ev_t, res)


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _same_reason(info, res):
    words = {"CONVERGENCE: REL_REDUCTION_OF_F": "RELATIVE REDUCTION", "NORM_OF_PROJECTED": "PROJECTED",
             "ITERATIONS REACHED LIMIT": "ITERATIONS", "ABNORMAL": "ABNORMAL"}
    msg = str(info.get("task", info.get("message", ""))).upper()
    for ours, theirs in words.items():
        if ours in res.task:
            return theirs.replace("_", " ") in msg.replace("_", " ")
    return False


def test_quadratic_matches_scipy():
    (xs_s, ev_s, info), (xs_t, ev_t, res) = _both(quadratic(), np.zeros(60), 500)
    assert res.nit == info["nit"] and res.nfev == info["funcalls"] == len(ev_s) == len(ev_t)
    assert _same_reason(info, res), (info, res.task)
    for a, b in zip(xs_t, xs_s):
        assert _rel(a, b) < 1e-9
    for a, b in zip(ev_t, ev_s):
        assert _rel(a, b) < 1e-9


def test_rosenbrock_matches_scipy_over_30_iterations():
    x0 = np.array([-1.2, 1.0] * 10)
    (xs_s, ev_s, _), (xs_t, ev_t, _) = _both(rosenbrock, x0, 30)
    assert len(xs_s) == len(xs_t) == 30 and len(ev_s) == len(ev_t)
    for a, b in zip(xs_t, xs_s):
        assert _rel(a, b) < 1e-9


def test_maxiter_and_first_step():
    """The first trial is x0 - g / ||g||; maxiter stops after that many
    accepted iterations."""
    fun = quadratic(1, 20)
    x0 = np.ones(20)
    (xs_s, ev_s, info), (xs_t, ev_t, res) = _both(fun, x0, 3)
    g0 = fun(x0)[1]
    assert _rel(ev_t[1], x0 - g0 / np.linalg.norm(g0)) < 1e-14
    assert res.nit == 3 == info["nit"] and res.nfev == len(ev_s)
    assert res.task.startswith("STOP: TOTAL NO. of ITERATIONS")


def test_zero_gradient_stops_at_once():
    res = lbfgs.minimize(lambda x: (float(x @ x), 2 * x), torch.zeros(5, dtype=torch.float64))
    assert res.nit == 0 and res.nfev == 1 and "PGTOL" in res.task


def _liar(after):
    """f = |x|^2 whose gradient turns to the wrong sign after `after`
    evaluations: the line search cannot meet its conditions, so the memory
    is reset and the run then ends abnormally."""
    count = [0]

    def fun(x):
        count[0] += 1
        sign = 1.0 if count[0] <= after else -1.0
        return float(x @ x + 0.1 * np.sum(x ** 4)), sign * (2 * x + 0.4 * x ** 3)
    return fun


@pytest.mark.parametrize("after", [1, 6])
def test_failed_line_search_resets_then_stops(after):
    x0 = np.linspace(-2, 3, 12)
    (xs_s, ev_s, info), (xs_t, ev_t, res) = _both(_liar(after), x0, 50, fresh=lambda: _liar(after))
    assert len(ev_t) == len(ev_s) and res.nit == info["nit"]
    assert res.task.startswith("ABNORMAL") and _same_reason(info, res), (info, res.task)
    assert res.resets == 1  # once with pairs stored, then the empty memory ends the run
    for a, b in zip(ev_t, ev_s):
        assert _rel(a, b) < 1e-9
    assert _rel(res.x.numpy(), xs_s[-1] if xs_s else x0) < 1e-9


def test_line_search_matches_minpack_dcsrch():
    """The Moré-Thuente search step by step against SciPy's restatement of
    MINPACK-2 dcsrch on 1-D functions of different shapes."""
    dcsrch = pytest.importorskip("scipy.optimize._dcsrch")
    funcs = [(lambda a: (a - 3.0) ** 2 - 9.0, lambda a: 2 * (a - 3.0), 1.0),
             (lambda a: -np.sin(a) + 0.05 * a * a, lambda a: -np.cos(a) + 0.1 * a, 0.01),
             (lambda a: np.exp(-a) + a ** 4 / 100, lambda a: -np.exp(-a) + a ** 3 / 25, 40.0),
             (lambda a: (1 - a) ** 3 + a, lambda a: -3 * (1 - a) ** 2 + 1, 0.1)]
    for phi, dphi, a0 in funcs:
        calls_s = []
        ref = dcsrch.DCSRCH(lambda a: calls_s.append(a) or phi(a), dphi, lbfgs.FTOL, lbfgs.GTOL, lbfgs.XTOL, 0.0,
                            lbfgs.STPMAX)
        stp_s = ref(a0, phi0=phi(0.0), derphi0=dphi(0.0), maxiter=30)[0]
        ls = lbfgs.LineSearch()
        task, stp = ls.start(phi(0.0), dphi(0.0), a0)
        calls_t = []
        while task == "FG" and len(calls_t) < 30:
            calls_t.append(stp)
            task, stp = ls.step(stp, phi(stp), dphi(stp))
        assert np.allclose(calls_t, calls_s, rtol=1e-13, atol=0), (calls_t, calls_s)
        assert stp == pytest.approx(stp_s, rel=1e-13)
