"""The host logic of the inversion driver FWI (src/PyFWI/fwi.py:109-282),
without a GPU: the parameter blocks of ``__call__`` / ``lbfgs`` / ``cg``,
the float32 rounding of the model in ``fprime_single``, the user parameter
functions, and the device optimisers against SciPy's.

The propagator's misfit is replaced by a seeded quadratic in the model
vector, evaluated exactly as the reference's fprime is called (a float32
model vector in, the misfit and a float64 gradient vector out), so both the
device optimisers (pyfwi_b200.lbfgs / cg, here on CPU tensors) and SciPy's
(``inpa['optimizer'] = 'scipy'``, the reference's own calls) run through the
same driver code; they must visit the same models."""
import numpy as np
import pytest
import torch

import cases
from conftest import load_golden


def _fwi(optimizer, param_functions=None):
    from pyfwi_b200 import acquisition as acq
    from pyfwi_b200.fwi import FWI
    case = cases.tiny_dxr()
    inpa = dict(case["inpa"], cuda_device="cpu", optimizer=optimizer)
    src = acq.Source(case["src_loc"], inpa["dh"], inpa["dt"], case["src_type"])
    src.Ricker(case["fdom"])
    g = load_golden("tiny_dxr")
    d_obs = {k[6:]: v for k, v in g.items() if k.startswith("d_obs_")}
    F = FWI(d_obs, inpa, src, case["rec_loc"], case["model_est"]["vp"].shape, components=case["components"],
            chpr=case["chpr"], n_well_rec=case["n_well_rec"], param_functions=param_functions)
    return F, case


def _quadratic_misfit(F, case, seed=3):
    """A misfit with its minimum at the observed model: 0.5 sum w (m - t)^2
    over the (vp, vs, rho) vector, the gradient w (m - t); model vectors
    arrive as the driver passes them (numpy or torch, float32)."""
    n = F.nz * F.nx
    rng = np.random.default_rng(seed)
    t = np.concatenate([case["model_obs"][k].reshape(-1) for k in ("vp", "vs", "rho")]).astype(np.float64)
    w = rng.uniform(0.5, 2.0, 3 * n) * np.repeat([1e-4, 4e-4, 1e-4], n)
    calls = []

    def fprime(m0, freq):
        m = m0.cpu().numpy() if isinstance(m0, torch.Tensor) else np.asarray(m0)
        assert m.dtype == np.float32
        calls.append(m.copy())
        r = m.astype(np.float64) - t
        f, g = 0.5 * float(np.sum(w * r * r)), w * r
        return f, (torch.from_numpy(g) if isinstance(m0, torch.Tensor) else g)
    F.fprime = fprime
    return calls


def _run(optimizer, method, iters, n_params=1, k_0=1, k_end=4):
    F, case = _fwi(optimizer)
    calls = _quadratic_misfit(F, case)
    m, rms = F({k: v.copy() for k, v in case["model_est"].items()}, method, iter=iters, freqs=[0] * len(iters),
               n_params=n_params, k_0=k_0, k_end=k_end)
    return m, rms, calls, case


@pytest.mark.parametrize("method", ["lbfgs", "cg"])
@pytest.mark.parametrize("n_params,k_0,k_end", [(1, 1, 4), (2, 1, 4), (1, 2, 3)])
def test_device_and_scipy_optimisers_visit_the_same_models(method, n_params, k_0, k_end):
    m_d, rms_d, calls_d, case = _run("device", method, [3, 2], n_params, k_0, k_end)
    m_s, rms_s, calls_s, _ = _run("scipy", method, [3, 2], n_params, k_0, k_end)
    assert len(calls_d) == len(calls_s)
    for a, b in zip(calls_d, calls_s):
        assert np.array_equal(a, b)
    for k in m_d:
        assert np.abs(m_d[k] - m_s[k]).max() <= 1e-9 * np.abs(m_s[k]).max(), k
    # parameters outside [k_0, k_end) keep their starting values exactly
    n = case["model_est"]["vp"].size
    start = np.concatenate([case["model_est"][k].reshape(-1) for k in ("vp", "vs", "rho")])
    final = np.concatenate([m_d[k].reshape(-1) for k in ("vp", "vs", "rho")])
    for q in range(3):
        if not k_0 - 1 <= q < k_end - 1:
            assert np.array_equal(final[q * n:(q + 1) * n], start[q * n:(q + 1) * n]), q
        else:
            assert np.any(final[q * n:(q + 1) * n] != start[q * n:(q + 1) * n]), q
    assert len(rms_d) == len(rms_s) == 2


def test_models_reach_fprime_rounded_to_float32():
    """fprime_single rounds the whole model to float32 before the misfit
    (fwi.py:255), on the device path as on SciPy's."""
    _, _, calls, _ = _run("device", "lbfgs", [2])
    assert all(c.dtype == np.float32 for c in calls)


def test_parameter_block_bounds_are_checked():
    F, case = _fwi("device")
    _quadratic_misfit(F, case)
    with pytest.raises(Exception, match="can't be larger than k_end"):
        F({k: v.copy() for k, v in case["model_est"].items()}, "lbfgs", iter=[1], freqs=[0], n_params=2, k_0=3,
          k_end=4)


def test_unknown_optimizer_is_refused():
    with pytest.raises(ValueError, match="optimizer"):
        _fwi("adam")


def test_user_parameter_functions_see_numpy_on_the_device_path():
    """PyFWI's param_functions receive numpy dicts, as in the reference, also
    when the optimiser keeps its vectors on the device."""
    from pyfwi_b200 import fwi_tools as tools
    seen = []

    def to_dv(m, args):
        seen.append(type(m["vp"]))
        return {k: v * args[0] for k, v in m.items()}
    pf = {"dict2vec": tools.vel_dict2vec, "vec2dict": tools.vec2vel_dict, "model_to_dv": to_dv,
          "grad_from_dv": lambda g, args, m: {k: v * args[0] for k, v in g.items()}, "args": [2.0]}
    F, case = _fwi("device", param_functions=pf)
    # stand in for the propagator part of fprime, which calls the user
    # functions, to see what it is handed
    F._fprime = lambda m0, freq: (seen.append(type(m0)) or (0.0, np.zeros_like(np.asarray(m0, np.float64))))
    F.fprime(torch.zeros(3 * F.nz * F.nx, dtype=torch.float32), 0)
    assert seen and seen[0] is np.ndarray
