"""The oracle's exact discrete adjoint against central finite differences of
the misfit, in double precision.

J(m) = 1/2 sum over every raw trace of (trace(m) - observed)^2.  For a
direction d, (J(m + e d) - J(m - e d)) / 2 must equal <dJ/dm, e d> up to the
O(e^2) truncation of the central difference.  The absorbing profiles scale
with max(vp) (a kink, not a derivative), so the directions leave every cell
that the perturbation could lift to the maximum unchanged."""
import numpy as np
import pytest
from scipy.ndimage import gaussian_filter

import cases
from helpers import fp64_propagator

FIELDS = ["vx", "vz", "taux", "tauz", "tauxz"]
EPS = 1e-6
TOL = 1e-6


def _misfit(W, m, obs):
    tr = W.raw_traces(m)
    return 0.5 * sum(np.sum((tr[f] - obs[f]) ** 2) for f in FIELDS), tr


@pytest.mark.parametrize("name", [f.__name__ for f in cases.TINY])
def test_exact_gradient_matches_central_differences(name):
    case = cases.by_name(name)
    W = fp64_propagator(case)
    obs = W.raw_traces({k: v.astype(np.float64) for k, v in case["model_obs"].items()})
    m0 = {k: v.astype(np.float64) for k, v in case["model_est"].items()}
    _, tr = _misfit(W, m0, obs)
    g = W.model_gradient(m0, *W.exact_gradient(m0, {f: tr[f] - obs[f] for f in FIELDS}))
    keep = m0["vp"] * (1 + 3 * EPS) < m0["vp"].max()
    rng = np.random.default_rng(11)
    for p in ("vp", "vs", "rho"):
        d = gaussian_filter(rng.standard_normal(m0[p].shape), 2.0)
        d *= keep / np.abs(d).max()
        dm = EPS * m0[p] * d
        fd = (_misfit(W, dict(m0, **{p: m0[p] + dm}), obs)[0] - _misfit(W, dict(m0, **{p: m0[p] - dm}), obs)[0]) / 2
        pred = float(np.sum(g[p] * dm))
        assert abs(pred - fd) <= TOL * abs(fd), (p, pred, fd)
