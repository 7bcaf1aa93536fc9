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


class _Survey:
    """One case set up twice: the regular path (caller-owned workspace:
    pyfwi_set_model, pyfwi_forward, pyfwi_l2_residual per observed
    component, pyfwi_gradient) and a plan for the static-scratch entry
    point; `observed` lists the raw components in the misfit (the others
    are passed as NULL)."""

    def __init__(self, name, observed, energy):
        import torch
        from pyfwi_b200.engine import Plan
        N, L = _bind()
        self.N, self.L = N, L
        case = cases.by_name(name)
        g = load_golden(name)
        W = product(case, segment=0, shot_batch=0)
        geom = W._geometry()
        dev = torch.device("cuda", 0)
        self.stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)

        def opts():
            o = N.Options()
            o.checkpoint, o.snapshot, o.energy, o.tile = N.CKPT_EXACT, N.SNAP_FP32, energy, 0
            return o

        self.model = [torch.from_numpy(np.ascontiguousarray(case["model_est"][k])).to(dev)
                      for k in ("vp", "vs", "rho")]
        self.damp = [torch.from_numpy(np.ascontiguousarray(W.dx_pml[0, :])).to(dev),
                     torch.from_numpy(np.ascontiguousarray(W.dz_pml[:, 0])).to(dev)]
        self.obs = [torch.from_numpy(np.ascontiguousarray(g["d_obs_" + k])).to(dev) if k in observed else None
                    for k in FIELDS]
        self.src = np.ascontiguousarray(W._wavelet, np.float32)
        self.shape = (3, int(W.nz), int(W.nx))
        self.dev = dev

        # regular path
        A = Plan(geom, W.srcx, W.srcz, opts(), dev)
        A.set_model(*self.model, *self.damp)
        traces = A.forward(self.src)
        self.misfit = torch.zeros((), dtype=torch.float64, device=dev)
        scratch = torch.empty(N.REDUCE_SLOTS, dtype=torch.float64, device=dev)
        res = []
        for c in range(5):
            if self.obs[c] is None:
                res.append(None)
                continue
            r = torch.empty_like(self.obs[c])
            N.check(L.pyfwi_l2_residual(_p(traces[c]), _p(self.obs[c]), _p(r), r.numel(), _p(scratch),
                                        _p(self.misfit), self.stream))
            res.append(r)
        self.grad = A.gradient(res, N.PARAM_LMD)
        torch.cuda.synchronize()
        self.B = Plan(geom, W.srcx, W.srcz, opts(), dev)

    def static_call(self):
        """One pyfwi_gradient_static call; checks it against the regular path."""
        import torch
        observed = (ctypes.c_void_p * 5)(*[o.data_ptr() if o is not None else None for o in self.obs])
        grad = torch.full(self.shape, float("nan"), dtype=torch.float32, device=self.dev)
        misfit = torch.full((), float("nan"), dtype=torch.float64, device=self.dev)
        rc = self.L.pyfwi_gradient_static(self.B.handle, *[_p(t) for t in self.model], *[_p(t) for t in self.damp],
                                          self.src.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                          int(self.src.shape[0]), observed, self.N.PARAM_LMD, _p(grad), _p(misfit),
                                          self.stream)
        assert rc == 0, self.L.pyfwi_last_error()
        torch.cuda.synchronize()
        for q in range(3):
            assert rel_l2(grad[q].cpu().numpy(), self.grad[q].cpu().numpy()) <= GRAD_TOL, q
        # the same reductions in the same order: the same bits
        assert float(misfit) == float(self.misfit)


def test_static_scratch_gradient_matches_workspace_path():
    """Two calls in a row on one plan, every component observed."""
    s = _Survey("tiny_s8", FIELDS, energy=1)
    s.static_call()
    s.static_call()


def test_static_scratch_shared_between_plans():
    """The array is shared: a plan of another geometry (and shot count)
    uses it between two calls of the first, and some components are left
    out of the misfit (NULL observed pointers, so fewer residual planes)."""
    a = _Survey("tiny_s8", ["vx", "tauz"], energy=1)
    b = _Survey("tiny_dxr", ["vx", "vz"], energy=0)
    a.static_call()
    b.static_call()
    a.static_call()
    b.static_call()


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
