"""The multiscale low-pass on the device (pyfwi_lowpass: FFT convolution of
every trace with the filter's response, one kernel) against the reference's
outputs, and the
band-limited FWI misfit and gradient (FWI.fprime with a frequency) against
the oracle's restatement of the reference pipeline: forward modelling,
lowpass of both data, L2 residual, adj_lowpass, gradient."""
import os

import numpy as np
import pytest

import cases
from conftest import GOLDEN, load_golden, rel_l2

pytestmark = pytest.mark.gpu

FN = 1.0 / 2.0 / 0.0006
FIELDS = ["vx", "vz", "taux", "tauz", "tauxz"]


def test_device_lowpass_matches_reference():
    import torch
    from pyfwi_b200 import fwi_tools
    with np.load(os.path.join(GOLDEN, "lowpass.npz")) as d:
        f = {k: d[k] for k in d.files}
    for q in range(2):
        hc = float(f["hc%d" % q])
        y = fwi_tools.lowpass(f["x%d" % q], hc, FN, order=3, axis=1)
        assert isinstance(y, np.ndarray) and rel_l2(y, f["low%d" % q]) < 1e-5
        a = fwi_tools.adj_lowpass(torch.from_numpy(f["r%d" % q]).cuda(), hc, FN, 3, axis=1)
        assert a.is_cuda and rel_l2(a.cpu().numpy(), f["adj%d" % q]) < 1e-5


def _oracle_fprime(case, d_obs, freq):
    import oracle as O
    inpa = case["inpa"]
    src = O.Ricker(case["src_loc"], inpa["dh"], inpa["dt"], case["src_type"])
    src.Ricker(case["fdom"])
    W = O.OracleWavePropagator(inpa, src, case["rec_loc"], case["model_est"]["vp"].shape,
                               components=case["components"], n_well_rec=case["n_well_rec"], chpr=case["chpr"])
    d_est = W.forward_modeling({k: v.copy() for k, v in case["model_est"].items()})
    pe, po = O.prepare_residual(d_est, 1), O.prepare_residual(d_obs, 1)
    lp = lambda d: O.lowpass(np.stack([d[k] for k in FIELDS]), freq, W.fn, 3)
    res = np.float32(lp(pe) - lp(po))
    rms = sum(0.5 * float(r.reshape(-1) @ r.reshape(-1)) for r in res)
    adj = O.lowpass(res, freq, W.fn, 3).astype(np.float32)
    grad = W.gradient({k: adj[q] for q, k in enumerate(FIELDS)}, parameterization="dv")
    return rms, np.concatenate([grad[k].reshape(-1) for k in ("vp", "vs", "rho")])


@pytest.mark.parametrize("name,freq", [("tiny_dtscale", 30.0), ("c1", 80.0)])
def test_band_limited_fprime_matches_oracle(name, freq):
    from pyfwi_b200 import acquisition as acq
    from pyfwi_b200 import fwi_tools
    from pyfwi_b200.fwi import FWI
    case = cases.by_name(name)
    g = load_golden(name)
    d_obs = {k[6:]: v for k, v in g.items() if k.startswith("d_obs_")}
    inpa = case["inpa"]
    src = acq.Source(case["src_loc"], inpa["dh"], inpa["dt"], case["src_type"])
    src.Ricker(case["fdom"])
    F = FWI(d_obs, inpa, src, case["rec_loc"], case["model_est"]["vp"].shape, components=case["components"],
            chpr=case["chpr"], n_well_rec=case["n_well_rec"])
    rms, grad = F.fprime(fwi_tools.vel_dict2vec(case["model_est"]), freq)
    rms_o, grad_o = _oracle_fprime(case, d_obs, freq)
    assert abs(rms - rms_o) <= 1e-4 * abs(rms_o), (rms, rms_o)
    assert rel_l2(grad, grad_o) <= 1e-4, rel_l2(grad, grad_o)


@pytest.mark.parametrize("planes,nt,ncols,hc", [(2, 6000, 7, 6.0), (3, 1537, 33, 25.0), (1, 150, 64, 60.0),
                                                (2, 1, 5, 60.0), (1, 4000, 2001, 8.0)])
def test_device_lowpass_shapes_match_oracle(planes, nt, ncols, hc):
    """The FFT kernel on record lengths from 1 to 6000 samples (FFTs of 2 to
    16384 points, 1 to 4 trace pairs per CTA), odd trace counts (a CTA with
    an unpaired trace) and several planes, against the oracle's
    restatement of the reference's filter."""
    import torch
    import oracle as O
    from pyfwi_b200 import fwi_tools
    rng = np.random.default_rng(nt + ncols)
    x = rng.standard_normal((planes, nt, ncols)).astype(np.float32)
    y = fwi_tools.lowpass(torch.from_numpy(x).cuda(), hc, FN, order=3, axis=1)
    ref = O.lowpass(x, hc, FN, 3)
    assert rel_l2(y.cpu().numpy(), ref) < 1e-5, rel_l2(y.cpu().numpy(), ref)
    for p in range(planes):  # each plane on its own too
        assert rel_l2(y[p].cpu().numpy(), ref[p]) < 1e-5
