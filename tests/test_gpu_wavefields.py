"""WavePropagator.W on the GPU: the wavefields the reference keeps at its
checkpoint steps (src/PyFWI/wave_propagation.py:150-156, filled at
:710-727), against the reference's own W (tests/golden/wavefields.npz, which
the oracle reproduces bit for bit, tests/test_wavefields.py).  Read from the
plan's checkpoint store in reverse mode (chpr < 100) and from a reverse-mode
re-run in exact mode (chpr = 100); within the seismogram bar (1e-5 relative
L2) of the reference."""
import numpy as np
import pytest
import torch

import cases
from conftest import load_golden, rel_l2
from helpers import product

pytestmark = pytest.mark.gpu
FIELDS = ("vx", "vz", "taux", "tauz", "tauxz")
TOL = 1e-5


def _check(W, g, name):
    ks = g[name + "_ks"]
    assert np.array_equal(np.asarray(W.chp), g[name + "_chp"])
    Wf = W.W
    for f in FIELDS:
        ref = g[name + "_" + f]
        assert Wf[f].dtype == np.float32 and Wf[f].shape == (int(W.tnz), int(W.tnx), int(W.ns), int(W.nchp))
        got = Wf[f][:, :, :, ks]
        assert rel_l2(got, ref) <= TOL, (f, rel_l2(got, ref))
    return Wf


@pytest.mark.parametrize("name", ["tiny_chpr", "tiny_dxr", "tiny_dtscale", "tiny_water"])
def test_W_matches_the_reference(name):
    g = load_golden("wavefields")
    case = cases.by_name(name)
    W = product(case)
    W.forward_modeling({k: v.copy() for k, v in case["model_est"].items()})
    assert W.checkpoint == ("reverse" if case["chpr"] < 100 else "exact")
    _check(W, g, name)


def test_W_is_zero_before_a_forward_run():
    W = product(cases.tiny_chpr())
    Wf = W.W
    assert set(Wf) == set(FIELDS)
    assert all(v.shape == (int(W.tnz), int(W.tnx), int(W.ns), int(W.nchp)) and not v.any() for v in Wf.values())


def test_W_follows_the_last_model_run():
    """W is rebuilt after each forward run (forward_modeling or the fused
    misfit_gradient), from the model of that run, even if the caller edits its
    tensors afterwards; both ways of building it give the same bits."""
    case = cases.tiny_chpr()
    g = load_golden("wavefields")
    W = product(case)
    est = {k: torch.from_numpy(v.copy()).cuda() for k, v in case["model_est"].items()}
    obs = W.forward_modeling({k: v.copy() for k, v in case["model_obs"].items()})
    W_obs = {k: v.copy() for k, v in W.W.items()}
    d_est = W.forward_modeling(est)
    W_plan = {k: v.copy() for k, v in W.W.items()}  # from the plan's store
    assert any(not np.array_equal(W_obs[k], W_plan[k]) for k in FIELDS)
    W.misfit_gradient(est, obs)
    est["vp"].mul_(1.1)  # edits after the run do not reach W
    W_rerun = W.W  # from a reverse-mode re-run of the same model
    for k in FIELDS:
        assert np.array_equal(W_rerun[k], W_plan[k]), k
    for f in FIELDS:
        assert rel_l2(W_plan[f][:, :, :, g["tiny_chpr_ks"]], g["tiny_chpr_" + f]) <= TOL
    assert d_est is not None
