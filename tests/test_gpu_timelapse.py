"""The time-lapse drivers (pyfwi_b200.tl_fwi.TimeLapse) against the
reference's own (tests/golden/tl_<method>.npz, made by
tests/golden/make_fwi.py: PyFWI.tl_fwi.TimeLapse with SciPy's L-BFGS-B on
PyFWI's kernels), for all eight methods on cases.timelapse: the same number
of misfit evaluations; misfits within 5e-4 relative (the bound of
tests/test_gpu_lbfgs.py, for the same reason: gradient-level differences
compound through the L-BFGS memory); every returned model's update from the
start within 1e-4 relative L2 per inversion stage that made it (a model
inverted from, or on data modelled from, an earlier inversion's result
carries that stage's error too); every time-lapse difference ('dm...')
within 1e-4 per stage of the updates' size."""
import numpy as np
import pytest

import cases
from conftest import GOLDEN, load_golden, rel_l2

pytestmark = pytest.mark.gpu

KEYS = ("vp", "vs", "rho")
# inversion stages behind each returned model (tl_fwi.py): 'pa' inverts both
# vintages from the start; 'cc' / 'dd' the monitor from / with data of the
# baseline result; 'sim' runs its joint inversion from an FWI result; 'wa',
# 'cd', 'cu' chain further cascades; 'cj' repeats the joint inversion from
# the first one's average
STAGES = {"pa": {"b1": 1, "m1": 1}, "cc": {"b1": 1, "m1": 2}, "dd": {"b1": 1, "m1": 2}, "sim": {"b1": 2, "m1": 2},
          "wa": {"b1": 1, "m1": 2, "b2": 3}, "cj": {"b1": 1, "m1": 1, "b2": 2, "m2": 2},
          "cd": {"b1": 1, "m2": 2, "m1": 1, "b2": 2}, "cu": {"b1": 1, "m1": 2, "b2": 3, "m2": 4}}


def _timelapse(case):
    from pyfwi_b200 import acquisition as acq
    from pyfwi_b200.processing import prepare_residual
    from pyfwi_b200.tl_fwi import TimeLapse
    from pyfwi_b200.wave_propagation import WavePropagator
    g = load_golden("tiny_dxr")
    b_obs = {k[6:]: v for k, v in g.items() if k.startswith("d_obs_")}
    inpa = case["inpa"]
    src = acq.Source(case["src_loc"], inpa["dh"], inpa["dt"], case["src_type"])
    src.Ricker(case["fdom"])
    shape = case["model_est"]["vp"].shape
    kw = dict(components=case["components"], n_well_rec=case["n_well_rec"])
    m_obs = WavePropagator(inpa, src, case["rec_loc"], shape, chpr=0, **kw).forward_modeling(case["model_mon"])
    return TimeLapse(prepare_residual(b_obs), prepare_residual(m_obs), inpa, src, case["rec_loc"], shape,
                     chpr=case["chpr"], **kw)


@pytest.mark.parametrize("method", cases.TL_METHODS)
def test_timelapse_matches_reference(method):
    case = cases.timelapse(method)
    with np.load("%s/tl_%s.npz" % (GOLDEN, method)) as f:
        ref = {k: f[k] for k in f.files}
    T = _timelapse(case)
    evals = []
    for obj, name in ((T, "tl_fprime"), (T.inv_obj, "fprime")):
        inner = getattr(obj, name)

        def recorded(*a, _inner=inner):
            rms, grad = _inner(*a)
            evals.append(rms)
            return rms, grad
        setattr(obj, name, recorded)
    s = case["tl"]
    out, _ = T({k: v.copy() for k, v in case["model_est"].items()}, iter=s["iter"], freqs=s["freqs"],
               tl_method=method, n_params=s["n_params"], k_0=s["k_0"], k_end=s["k_end"])
    assert len(evals) == len(ref["evals_rms"]), (len(evals), len(ref["evals_rms"]))
    for q, (a, b) in enumerate(zip(evals, ref["evals_rms"])):
        assert abs(a - b) <= 5e-4 * abs(b), (q, a, b)
    m0 = case["model_est"]
    stages = STAGES[method]
    models = {n for n in stages}
    diffs = sorted({k.rsplit("_", 1)[0] for k in ref if k.startswith("dm")})
    assert set(out) >= models | set(diffs)
    size = 0.0
    for name in sorted(models):
        for k in KEYS:
            upd, upd_ref = out[name][k] - m0[k], ref["%s_%s" % (name, k)] - m0[k]
            size = max(size, float(np.linalg.norm(upd_ref)))
            if np.any(upd_ref):
                err = rel_l2(upd, upd_ref)
                print("%s %s %s update vs reference: rel-L2 %.2e" % (method, name, k, err))
                assert err <= 1e-4 * stages[name], (name, k, err)
            else:
                assert not np.any(upd), (name, k)
    worst = max(stages.values())
    for name in diffs:
        for k in KEYS:
            err = float(np.linalg.norm(out[name][k] - ref["%s_%s" % (name, k)]))
            assert err <= 1e-4 * worst * size, (name, k, err, size)
