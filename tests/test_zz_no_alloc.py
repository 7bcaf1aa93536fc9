"""pyfwi_gradient_static: the gradient entry point for callers that cannot
allocate device memory (a host program with no CUDA allocator of its own,
or an application whose memory pool owns the whole device).  It runs on the
library's fixed device array instead of a caller workspace.

Checked through the C ABI against the regular path (caller workspace:
pyfwi_set_model, pyfwi_forward, pyfwi_l2_residual, pyfwi_gradient) on two
calls in a row, within the gradient tolerance of the parity tests.  This
file is collected last so a failure here comes after every other test."""
import ctypes

import numpy as np
import pytest

import cases
from conftest import load_golden, rel_l2
from helpers import product

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4
FIELDS = ["vx", "vz", "taux", "tauz", "tauxz"]


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _bind():
    from pyfwi_b200 import _native as N
    L = N.lib()
    L.pyfwi_gradient_static.restype = ctypes.c_int
    L.pyfwi_gradient_static.argtypes = [ctypes.c_void_p] * 6 + [ctypes.POINTER(ctypes.c_float), ctypes.c_int32,
                                                                 ctypes.POINTER(ctypes.c_void_p), ctypes.c_int32,
                                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return N, L


def test_static_scratch_gradient_matches_workspace_path():
    import torch
    from pyfwi_b200.engine import Plan

    N, L = _bind()
    case = cases.tiny_s8()
    g = load_golden("tiny_s8")
    W = product(case, segment=0, shot_batch=0)
    geom = W._geometry()
    dev = torch.device("cuda", 0)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)

    def opts():
        o = N.Options()
        o.checkpoint, o.snapshot, o.energy, o.tile = N.CKPT_EXACT, N.SNAP_FP32, 1, 0
        return o

    model = [torch.from_numpy(np.ascontiguousarray(case["model_est"][k])).to(dev) for k in ("vp", "vs", "rho")]
    damp = [torch.from_numpy(np.ascontiguousarray(W.dx_pml[0, :])).to(dev),
            torch.from_numpy(np.ascontiguousarray(W.dz_pml[:, 0])).to(dev)]
    obs = [torch.from_numpy(np.ascontiguousarray(g["d_obs_" + k])).to(dev) for k in FIELDS]
    src = np.ascontiguousarray(W._wavelet, np.float32)

    # regular path: caller-owned workspace
    A = Plan(geom, W.srcx, W.srcz, opts(), dev)
    A.set_model(*model, *damp)
    traces = A.forward(src)
    misfit_a = torch.zeros((), dtype=torch.float64, device=dev)
    scratch = torch.empty(N.REDUCE_SLOTS, dtype=torch.float64, device=dev)
    res = []
    for c in range(5):
        r = torch.empty_like(obs[c])
        N.check(L.pyfwi_l2_residual(_p(traces[c]), _p(obs[c]), _p(r), r.numel(), _p(scratch), _p(misfit_a),
                                    stream))
        res.append(r)
    grad_a = A.gradient(res, N.PARAM_LMD)
    torch.cuda.synchronize()

    # the static-scratch entry point, twice on the same plan
    B = Plan(geom, W.srcx, W.srcz, opts(), dev)
    observed = (ctypes.c_void_p * 5)(*[o.data_ptr() for o in obs])
    for call in range(2):
        grad_b = torch.full((3, int(W.nz), int(W.nx)), float("nan"), dtype=torch.float32, device=dev)
        misfit_b = torch.full((), float("nan"), dtype=torch.float64, device=dev)
        rc = L.pyfwi_gradient_static(B.handle, *[_p(t) for t in model], *[_p(t) for t in damp],
                                     src.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), int(src.shape[0]),
                                     observed, N.PARAM_LMD, _p(grad_b), _p(misfit_b), stream)
        assert rc == 0, L.pyfwi_last_error()
        torch.cuda.synchronize()
        for q in range(3):
            assert rel_l2(grad_b[q].cpu().numpy(), grad_a[q].cpu().numpy()) <= GRAD_TOL, (call, q)
        # the same reductions in the same order: the same bits
        assert float(misfit_b) == float(misfit_a), call


def test_static_scratch_rejects_oversized_surveys():
    import torch
    from pyfwi_b200.engine import Plan

    N, L = _bind()
    case = cases.c1()
    W = product(case)
    o = N.Options()
    o.checkpoint = N.CKPT_EXACT  # every step of 4 shots stored: far more than the array holds
    P = Plan(W._geometry(), W.srcx, W.srcz, o, torch.device("cuda", 0))
    z = ctypes.c_void_p(1)
    observed = (ctypes.c_void_p * 5)()
    rc = L.pyfwi_gradient_static(P.handle, z, z, z, z, z, None, 0, observed, 0, z, z, None)
    assert rc == N_E_WORKSPACE
    assert b"static array holds" in L.pyfwi_last_error()


N_E_WORKSPACE = -2
