"""The time-lapse drivers (pyfwi_b200.tl_fwi.TimeLapse) against the
reference's own (tests/golden/tl_<method>.npz, made by
tests/golden/make_fwi.py: PyFWI.tl_fwi.TimeLapse with SciPy's L-BFGS-B on
PyFWI's kernels), for the cascaded ('cc'), double-difference ('dd') and
simultaneous ('sim') methods on cases.timelapse: the same number of misfit
evaluations, misfits within 5e-4 relative (the bound of
tests/test_gpu_lbfgs.py, for the same reason: gradient-level differences
compound through the L-BFGS memory), every returned model's update from the
start within 1e-4 relative L2 for a model one inversion makes and 2e-4 for
a model whose inversion starts from, or inverts data modelled from, an
earlier inversion's result (each stage adds its own gradient-level error),
and the time-lapse difference dm within 2e-4 of the updates' size."""
import numpy as np
import pytest

import cases
from conftest import GOLDEN, load_golden, rel_l2

pytestmark = pytest.mark.gpu

KEYS = ("vp", "vs", "rho")
# models made by a second inversion stage: 'cc' and 'dd' invert the monitor
# from / with data of the baseline result; 'sim' starts its joint inversion
# from an FWI result
SECOND_STAGE = {"cc": ("m1",), "dd": ("m1",), "sim": ("b1", "m1")}


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
    size = 0.0
    for name in ("b1", "m1"):
        for k in KEYS:
            upd, upd_ref = out[name][k] - m0[k], ref["%s_%s" % (name, k)] - m0[k]
            size = max(size, float(np.linalg.norm(upd_ref)))
            if np.any(upd_ref):
                tol = 2e-4 if name in SECOND_STAGE[method] else 1e-4
                print("%s %s %s update vs reference: rel-L2 %.2e" % (method, name, k, rel_l2(upd, upd_ref)))
                assert rel_l2(upd, upd_ref) <= tol, (name, k, rel_l2(upd, upd_ref))
            else:
                assert not np.any(upd), (name, k)
    for k in KEYS:
        err = float(np.linalg.norm(out["dm"][k] - ref["dm_" + k]))
        assert err <= 2e-4 * size, ("dm", k, err, size)
