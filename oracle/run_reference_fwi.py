"""TEST INFRASTRUCTURE ONLY -- runs the unmodified PyFWI inversion driver on
the CPU.

    python oracle/run_reference_fwi.py CASE.pkl OUT.npz [REFERENCE_SRC]

Like oracle/run_reference.py (same stand-in modules, the reference's own
OpenCL C kernels compiled for the CPU), but drives ``PyFWI.fwi.FWI``: the
observed data come from ``model_obs`` through ``WavePropagator``, then
``FWI(...)(model_est, method, iter, freqs, n_params, k_0, k_end)`` runs with
the case's ``fwi`` settings.  Stores the final model (``m_vp``, ``m_vs``,
``m_rho``), the misfit of every evaluation in order (``evals_rms``) and
the model vector of every evaluation (``evals_m``).

SciPy here is newer than the reference's pin (1.7.3), so two of the
reference's imports are pointed at their current places before PyFWI.fwi is
imported: ``MemoizeJac`` (moved from scipy.optimize.optimize to
scipy.optimize._optimize) and ``fmin_l_bfgs_b`` (which no longer takes the
printing-only ``iprint`` / ``disp`` arguments the reference passes).  The
optimiser itself is SciPy's L-BFGS-B either way.
"""
import os
import pickle
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _scipy_compat():
    import scipy.optimize as so
    import scipy.optimize._optimize as new_optimize
    import scipy.optimize.lbfgsb as lbfgsb_module
    import scipy.optimize.optimize as old_optimize
    old_optimize.MemoizeJac = new_optimize.MemoizeJac
    fmin = so.fmin_l_bfgs_b

    def fmin_l_bfgs_b(*args, iprint=None, disp=None, **kwargs):
        return fmin(*args, **kwargs)
    lbfgsb_module.fmin_l_bfgs_b = fmin_l_bfgs_b


def main():
    case_path, out_path = sys.argv[1], sys.argv[2]
    ref_src = sys.argv[3] if len(sys.argv) > 3 else "/root/reference/src"
    sys.path[:0] = [os.path.join(HERE, "standin"), ref_src]
    import warnings
    warnings.simplefilter("ignore", DeprecationWarning)
    _scipy_compat()
    import numpy as np
    import PyFWI.acquisition as acq
    import PyFWI.fwi as fwi
    import PyFWI.wave_propagation as wave

    with open(case_path, "rb") as f:
        case = pickle.load(f)
    inpa = dict(case["inpa"])
    src = acq.Source(case["src_loc"], inpa["dh"], inpa["dt"], src_type=case.get("src_type", 0))
    src.Ricker(case["fdom"])
    shape = case["model_est"]["vp"].shape
    kw = dict(components=case["components"], n_well_rec=case.get("n_well_rec", 0))
    W_obs = wave.WavePropagator(inpa, src, case["rec_loc"], shape, chpr=0, **kw)
    d_obs = W_obs.forward_modeling({k: v.copy() for k, v in case["model_obs"].items()}, show=False)

    if "tl" in case:
        return _timelapse(case, inpa, src, shape, kw, d_obs, out_path)
    s = case["fwi"]
    m0 = {k: v.copy() for k, v in case["model_est"].items()}
    param_functions = None
    if "param_scale" in s:
        # the model in units of `scale`: PyFWI's param_functions hooks
        import PyFWI.fwi_tools as tools
        scale = s["param_scale"]
        param_functions = {"dict2vec": tools.vel_dict2vec, "vec2dict": tools.vec2vel_dict,
                           "model_to_dv": lambda m, args: {k: v * args[0] for k, v in m.items()},
                           "grad_from_dv": lambda g, args, m: {k: v * args[0] for k, v in g.items()},
                           "args": [scale]}
        m0 = {k: np.float32(v / np.float32(scale)) for k, v in m0.items()}
    F = fwi.FWI(d_obs, inpa, src, case["rec_loc"], shape, case["components"], case["chpr"],
                n_well_rec=case.get("n_well_rec", 0), param_functions=param_functions)
    evals_m, evals_rms = [], []
    inner = F.fprime

    def recorded(m0, freq):
        rms, grad = inner(m0, freq)
        evals_m.append(np.array(m0, np.float32))
        evals_rms.append(float(rms))
        return rms, grad
    F.fprime = recorded
    m_est, rms = F(m0, s["method"], iter=s["iter"], freqs=s["freqs"], n_params=s["n_params"], k_0=s["k_0"],
                   k_end=s["k_end"])
    out = {"m_" + k: np.asarray(v, np.float64) for k, v in m_est.items()}
    out["evals_rms"] = np.asarray(evals_rms)
    out["evals_m"] = np.stack(evals_m)
    np.savez_compressed(out_path, **out)


def _timelapse(case, inpa, src, shape, kw, b_obs, out_path):
    """PyFWI.tl_fwi.TimeLapse on the baseline (model_obs) and monitor
    (model_mon) data, both passed through prepare_residual as PyFWI's
    time-lapse example does; stores every model of the result dict
    (``<entry>_<param>``) and the misfit of every evaluation."""
    import numpy as np
    import PyFWI.tl_fwi as tl
    import PyFWI.wave_propagation as wave
    from PyFWI.processing import prepare_residual
    W_mon = wave.WavePropagator(inpa, src, case["rec_loc"], shape, chpr=0, **kw)
    m_obs = W_mon.forward_modeling({k: v.copy() for k, v in case["model_mon"].items()}, show=False)
    T = tl.TimeLapse(prepare_residual(b_obs), prepare_residual(m_obs), inpa, src, case["rec_loc"], shape,
                     components=case["components"], chpr=case["chpr"], n_well_rec=case.get("n_well_rec", 0))
    evals_rms = []
    for obj, name in ((T, "tl_fprime"), (T.inv_obj, "fprime")):
        inner = getattr(obj, name)

        def recorded(*a, _inner=inner):
            rms, grad = _inner(*a)
            evals_rms.append(float(rms))
            return rms, grad
        setattr(obj, name, recorded)
    s = case["tl"]
    inverted, _ = T({k: v.copy() for k, v in case["model_est"].items()}, iter=s["iter"], freqs=s["freqs"],
                    tl_method=s["tl_method"], n_params=s["n_params"], k_0=s["k_0"], k_end=s["k_end"])
    out = {"evals_rms": np.asarray(evals_rms)}
    for name, v in inverted.items():
        if isinstance(v, dict):
            for k, a in v.items():
                out["%s_%s" % (name, k)] = np.asarray(a, np.float64)
    np.savez_compressed(out_path, **out)


if __name__ == "__main__":
    main()
