"""TEST INFRASTRUCTURE ONLY -- runs the unmodified PyFWI propagator on the CPU.

    python oracle/run_reference.py CASE.pkl OUT.npz [REFERENCE_SRC]

Imports PyFWI from the reference tree (default /root/reference/src) with the
stand-in modules of ``oracle/standin`` first on ``sys.path``, so that
``WavePropagator`` runs its own host loops and its own OpenCL C kernels
(compiled for the CPU by ``oracle/ref_build.py``).  It models the observed
data on ``model_obs`` and the estimate on ``model_est``, forms the L2
residual with ``CostFunction('l2')``, and takes ``WavePropagator.gradient``.
The set-up values it reads back (time-step split, checkpoint list, index
constants, damping arrays, wavelet) pin the product's host logic.

Used by tests/golden/make_golden.py; it needs the reference tree, so it runs
only on a machine that has it.
"""
import os
import pickle
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    case_path, out_path = sys.argv[1], sys.argv[2]
    ref_src = sys.argv[3] if len(sys.argv) > 3 else "/root/reference/src"
    sys.path[:0] = [os.path.join(HERE, "standin"), ref_src]
    import numpy as np
    import PyFWI.acquisition as acq
    import PyFWI.fwi_tools as tools
    import PyFWI.wave_propagation as wave
    from PyFWI.processing import prepare_residual

    with open(case_path, "rb") as f:
        case = pickle.load(f)
    inpa = dict(case["inpa"])
    src = acq.Source(case["src_loc"], inpa["dh"], inpa["dt"], src_type=case.get("src_type", 0))
    src.Ricker(case["fdom"])
    shape = case["model_est"]["vp"].shape
    kw = dict(components=case["components"], n_well_rec=case.get("n_well_rec", 0))
    out = {}
    W_obs = wave.WavePropagator(inpa, src, case["rec_loc"], shape, chpr=0, **kw)
    d_obs = W_obs.forward_modeling({k: v.copy() for k, v in case["model_obs"].items()}, show=False)
    W = wave.WavePropagator(inpa, src, case["rec_loc"], shape, chpr=case["chpr"], **kw)
    d_est = W.forward_modeling({k: v.copy() for k, v in case["model_est"].items()}, show=False)
    for k, v in d_obs.items():
        out["d_obs_" + k] = np.asarray(v)
    for k, v in d_est.items():
        out["d_est_" + k] = np.asarray(v)
    for k, v in W.seismogram.items():
        out["seis_" + k] = np.asarray(v)
    if case.get("gradient", True):
        CF = tools.CostFunction("l2")
        rms, res = CF(prepare_residual(d_est, 1), prepare_residual(d_obs, 1))
        out["rms"] = np.asarray(rms)
        grad = W.gradient(res, show=False, parameterization=case.get("param", "dv"))
        for k, v in grad.items():
            out["grad_" + k] = np.asarray(v)
    # set-up values, for the host-logic checks
    out["setup_dt_scale"] = np.asarray(W.dt_scale)
    out["setup_nt"] = np.asarray(W.nt)
    out["setup_nt_ext"] = np.asarray(W.nt_ext)
    out["setup_dt"] = np.asarray(W.dt)
    out["setup_chp"] = np.asarray(W.chp)
    out["setup_srcx"] = np.asarray(W.srcx)
    out["setup_srcz"] = np.asarray(W.srcz)
    out["setup_dxr"] = np.asarray(W.dxr)
    out["setup_sdo"] = np.asarray(W.sdo)
    for k in ("rec_top_left_const", "rec_top_left_var", "rec_top_right_const", "rec_top_right_var",
              "rec_surface_const", "rec_surface_var", "src_cts"):
        out["setup_" + k] = np.asarray(getattr(W, k))
    out["setup_dx_pml"] = W.dx_pml
    out["setup_dz_pml"] = W.dz_pml
    out["setup_wavelet"] = np.asarray(src.w)
    np.savez_compressed(out_path, **out)


if __name__ == "__main__":
    main()
