"""Shared helpers for the tests: build inputs of a case the way a PyFWI user
would, and run the oracle on them."""
import numpy as np

import cases


def oracle_run(case, precision="fp32", d_obs=None, gradient=True):
    """Run the CPU oracle on a case: (d_obs, d_est, grad, propagator)."""
    import oracle as O
    inpa = case["inpa"]
    src = O.Ricker(case["src_loc"], inpa["dh"], inpa["dt"], case["src_type"])
    src.Ricker(case["fdom"])
    kw = dict(components=case["components"], n_well_rec=case["n_well_rec"], precision=precision)
    shape = case["model_est"]["vp"].shape
    if d_obs is None:
        Wo = O.OracleWavePropagator(inpa, src, case["rec_loc"], shape, chpr=0, **kw)
        d_obs = Wo.forward_modeling({k: v.copy() for k, v in case["model_obs"].items()})
    W = O.OracleWavePropagator(inpa, src, case["rec_loc"], shape, chpr=case["chpr"], **kw)
    d_est = W.forward_modeling({k: v.copy() for k, v in case["model_est"].items()})
    grad = None
    if gradient:
        pe, po = O.prepare_residual(d_est, 1), O.prepare_residual(d_obs, 1)
        res = {k: (pe[k] - po[k]).astype(W.real) for k in O.FIELDS}
        grad = W.gradient(res, parameterization=case["param"])
    return d_obs, d_est, grad, W


def product(case, **extra):
    """The product's WavePropagator for a case (extra inpa keys allowed)."""
    from pyfwi_b200 import acquisition as acq
    from pyfwi_b200.wave_propagation import WavePropagator
    inpa = dict(case["inpa"])
    inpa.update(extra)
    src = acq.Source(case["src_loc"], inpa["dh"], inpa["dt"], case["src_type"])
    src.Ricker(case["fdom"])
    return WavePropagator(inpa, src, case["rec_loc"], case["model_est"]["vp"].shape, components=case["components"],
                          n_well_rec=case["n_well_rec"], chpr=case["chpr"])


def l2_residual_np(d_est, d_obs):
    """CostFunction('l2') of the reference on prepared dicts: float32(est - obs)."""
    import oracle as O
    pe, po = O.prepare_residual(d_est, 1), O.prepare_residual(d_obs, 1)
    return {k: np.float32(pe[k] - po[k]) for k in O.FIELDS}


def fp64_propagator(case, precision="fp64"):
    """The oracle propagator of a case (FP64 unless asked), storing every
    step (chpr 100)."""
    import oracle as O
    inpa = case["inpa"]
    src = O.Ricker(case["src_loc"], inpa["dh"], inpa["dt"], case["src_type"])
    src.Ricker(case["fdom"])
    return O.OracleWavePropagator(inpa, src, case["rec_loc"], case["model_est"]["vp"].shape,
                                  components=case["components"], n_well_rec=case["n_well_rec"], chpr=100,
                                  precision=precision)


def input_digest(case):
    """sha256 over the models, geometry and wavelet parameters of a case: a
    fixture stores it so a test can tell that tests/cases.py still builds
    the survey the fixture was made from."""
    import hashlib
    h = hashlib.sha256()
    for key in ("model_obs", "model_est"):
        for k in ("vp", "vs", "rho"):
            h.update(np.ascontiguousarray(case[key][k], np.float32).tobytes())
    h.update(np.ascontiguousarray(case["src_loc"], np.float32).tobytes())
    h.update(np.ascontiguousarray(case["rec_loc"], np.float32).tobytes())
    h.update(repr(sorted(case["inpa"].items())).encode())
    h.update(repr((case["fdom"], case["src_type"], case["components"], case["chpr"])).encode())
    return h.hexdigest()


def section_error(ours, ref, f64=None, tol=1e-5):
    """(passes, description) for a section against the reference's float32
    one: within `tol` relative L2; or, where the reference's own float32
    rounding puts it further than tol / 2 from the FP64 oracle's section
    (traces next to a source over long records), no further from the FP64
    answer than the reference is, and within twice the reference's own error
    of it."""
    from conftest import rel_l2
    e_ref = rel_l2(ours, ref)
    if e_ref < tol:
        return True, "%.2e from the reference" % e_ref
    if f64 is None:
        return False, "%.2e from the reference" % e_ref
    noise, e_64 = rel_l2(ref, f64), rel_l2(ours, f64)
    ok = noise > tol / 2 and e_64 <= noise and e_ref <= 2 * noise
    return ok, "%.2e from the reference, whose own float32 error is %.2e; ours %.2e from FP64" % (e_ref, noise, e_64)
