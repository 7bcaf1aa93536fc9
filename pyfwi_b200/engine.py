"""Device engine: a pyfwi_b200 plan, its workspace, and torch-tensor calls
into libpyfwi_b200.so.

torch provides device memory and the stream; every arithmetic step of the
propagator path runs in the library's kernels."""
import ctypes

import numpy as np
import torch

from . import _native as N


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def require_cuda(device):
    device = torch.device(device)
    if device.type != "cuda" or not torch.cuda.is_available():
        raise RuntimeError("pyfwi_b200 runs on a CUDA device only (got %s; CUDA available: %s)"
                           % (device, torch.cuda.is_available()))
    return device


class Plan:
    """One propagation plan (geometry + options) and its device workspace."""

    def __init__(self, geom, srcx, srcz, opts, device, chp=None):
        self.device = require_cuda(device)
        self.lib = N.lib()
        self.geom = geom
        self.opts = opts
        self._srcx = np.ascontiguousarray(srcx, np.int32)
        self._srcz = np.ascontiguousarray(srcz, np.int32)
        self._chp = None if chp is None else np.ascontiguousarray(chp, np.int32)
        if self._chp is not None:
            opts.nchp = int(self._chp.size)
            opts.chp = self._chp.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        h = ctypes.c_void_p()
        N.check(self.lib.pyfwi_plan_create(ctypes.byref(geom), self._srcx.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                           self._srcz.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                           ctypes.byref(opts), ctypes.byref(h)))
        self.handle = h
        size = ctypes.c_size_t()
        N.check(self.lib.pyfwi_workspace_size(h, ctypes.byref(size)))
        self.ws_bytes = size.value
        with torch.cuda.device(self.device):
            self._ws = torch.empty(self.ws_bytes + 256, dtype=torch.uint8, device=self.device)
        base = self._ws.data_ptr()
        self.ws = ctypes.c_void_p((base + 255) // 256 * 256)
        self.nz, self.nx, self.npml = geom.nz, geom.nx, geom.npml
        self.ns, self.nr, self.nt_ext = geom.ns, geom.nr, geom.nt_ext

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.pyfwi_plan_destroy(h)
            except Exception:
                pass
            self.handle = None

    @staticmethod
    def workspace_bytes(geom, opts, ns_src):
        """Workspace size a plan with these settings would need."""
        L = N.lib()
        srcx = np.zeros(geom.ns, np.int32)
        srcz = np.zeros(geom.ns, np.int32)
        h = ctypes.c_void_p()
        N.check(L.pyfwi_plan_create(ctypes.byref(geom), srcx.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                    srcz.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ctypes.byref(opts),
                                    ctypes.byref(h)))
        size = ctypes.c_size_t()
        N.check(L.pyfwi_workspace_size(h, ctypes.byref(size)))
        L.pyfwi_plan_destroy(h)
        return size.value

    def launches(self):
        c = ctypes.c_int64()
        N.check(self.lib.pyfwi_launch_count(self.handle, ctypes.byref(c)))
        return c.value

    def _flags(self):
        f = ctypes.c_int32()
        N.check(self.lib.pyfwi_plan_flags(self.handle, ctypes.byref(f)))
        return f.value

    @property
    def persist(self):
        """True when the plan runs its time loops as persistent kernels."""
        return bool(self._flags() & 1)

    @property
    def overlap(self):
        """True when the plan recomputes beside the adjoint on a second stream."""
        return bool(self._flags() & 2)

    @property
    def store_diffs(self):
        """True when the checkpoint segments hold the imaging's differences."""
        return bool(self._flags() & 4)

    def misfit_gradient(self, src_vals, observed, mean_stress, adjoint, param, traces=None):
        """pyfwi_misfit_gradient: observed / adjoint are lists of 5 device
        tensors [nt_ext, ns*nr] or None.  Returns (grad [3, nz, nx], misfit
        0-d float64 tensor, traces [5, nt_ext, ns*nr])."""
        sv = np.ascontiguousarray(src_vals, np.float32).reshape(-1, 4)
        if traces is None:
            traces = torch.empty((5, self.nt_ext, self.ns * self.nr), dtype=torch.float32, device=self.device)
        graph = bool(self.opts.graph)
        if graph:
            # the captured graph bakes in pointers: run on buffers the plan
            # keeps and copy in / out around the replay
            bufs = self.__dict__.setdefault("_mis_bufs", {})

            def keep(name, like):
                b = bufs.get(name)
                if b is None or b.shape != like.shape or b.dtype != like.dtype:
                    b = bufs[name] = torch.empty_like(like, memory_format=torch.contiguous_format)
                return b
            obs_in = [None if o is None else keep(("obs", q), o).copy_(o) for q, o in enumerate(observed)]
            adj_in = [None if a is None else keep(("adj", q), a) for q, a in enumerate(adjoint)]
            grad = keep("grad", torch.empty((3, self.nz, self.nx), dtype=torch.float32, device=self.device))
            misfit = keep("misfit", torch.empty((), dtype=torch.float64, device=self.device))
        else:
            obs_in, adj_in = observed, adjoint
            grad = torch.empty((3, self.nz, self.nx), dtype=torch.float32, device=self.device)
            misfit = torch.zeros((), dtype=torch.float64, device=self.device)
        N.check(self.lib.pyfwi_misfit_gradient(self.handle, self.ws, self.ws_bytes,
                                               sv.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), int(sv.shape[0]),
                                               _ptr_array(obs_in), int(bool(mean_stress)), _ptr_array(adj_in),
                                               int(param), _ptr(traces), _ptr(grad), _ptr(misfit),
                                               _stream(self.device)))
        self._keep = (observed, adjoint)
        if graph:
            for a, b in zip(adjoint, adj_in):
                if a is not None:
                    a.copy_(b)
            return grad.clone(), misfit.clone(), traces
        return grad, misfit, traces

    def check_device(self):
        """Synchronise the device stream and raise NativeError if a streaming
        kernel gave up waiting for a row copy, or a persistent kernel at a
        grid barrier, since the last check."""
        code = ctypes.c_int32()
        N.check(self.lib.pyfwi_device_error(self.handle, self.ws, self.ws_bytes, ctypes.byref(code),
                                            _stream(self.device)))

    def frame_check(self):
        """pyfwi_frame_check: nonzero cells in the zero frames of the
        workspace planes (0 unless a kernel wrote outside its domain)."""
        n = ctypes.c_int64()
        N.check(self.lib.pyfwi_frame_check(self.handle, self.ws, self.ws_bytes, ctypes.byref(n),
                                           _stream(self.device)))
        return n.value

    def checkpoint_states(self):
        """pyfwi_checkpoint_states: the states a reverse-mode plan stored at
        its checkpoint steps in the last forward call, a device tensor
        [ns, nchp, 5, nz+2npml, nx+2npml] (fields vx, vz, taux, tauz, tauxz)."""
        nchp = 0 if self._chp is None else int(self._chp.size)
        tnz, tnx = self.nz + 2 * self.npml, self.nx + 2 * self.npml
        out = torch.empty((self.ns, nchp, 5, tnz, tnx), dtype=torch.float32, device=self.device)
        N.check(self.lib.pyfwi_checkpoint_states(self.handle, self.ws, self.ws_bytes, _ptr(out),
                                                 _stream(self.device)))
        return out

    def wait_selftest(self, limit_ns):
        """pyfwi_wait_selftest: a bounded device wait that nothing ends gives
        up after limit_ns and sets the error word (read by check_device)."""
        N.check(self.lib.pyfwi_wait_selftest(self.handle, self.ws, self.ws_bytes, int(limit_ns),
                                             _stream(self.device)))

    def barrier_selftest(self, limit_ns):
        """pyfwi_barrier_selftest: the persistent kernels' grid barrier
        waiting for a CTA that does not exist gives up after limit_ns and sets
        the error word to 3 (read by check_device)."""
        N.check(self.lib.pyfwi_barrier_selftest(self.handle, self.ws, self.ws_bytes, int(limit_ns),
                                                _stream(self.device)))

    def profile(self, enable=True):
        """Bracket every step kernel with CUDA events (see profile_read)."""
        N.check(self.lib.pyfwi_profile_enable(self.handle, 1 if enable else 0))

    def profile_read(self, kind):
        """(launches, device ms, grid cells x shots) of kind 0 forward step,
        1 adjoint+imaging step, 2 reverse step since the last read."""
        n, ms, cells = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
        N.check(self.lib.pyfwi_profile_read(self.handle, int(kind), ctypes.byref(n), ctypes.byref(ms),
                                            ctypes.byref(cells)))
        return n.value, ms.value, cells.value

    def set_model(self, vp, vs, rho, damp_x, damp_z):
        args = [t.to(self.device, torch.float32).contiguous() for t in (vp, vs, rho, damp_x, damp_z)]
        N.check(self.lib.pyfwi_set_model(self.handle, self.ws, self.ws_bytes, *[_ptr(t) for t in args],
                                         _stream(self.device)))
        self._model_keep = args  # alive until the kernels ran

    def forward(self, src_vals, traces=None):
        """Run all shots; returns traces [5, nt_ext, ns*nr] (float32, device)."""
        sv = np.ascontiguousarray(src_vals, np.float32).reshape(-1, 4)
        if traces is None:
            traces = torch.empty((5, self.nt_ext, self.ns * self.nr), dtype=torch.float32, device=self.device)
        N.check(self.lib.pyfwi_forward(self.handle, self.ws, self.ws_bytes,
                                       sv.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), int(sv.shape[0]),
                                       _ptr(traces), _stream(self.device)))
        return traces

    def gradient(self, residual, param, grad=None, raw=None):
        """residual: list of 5 device tensors [nt_ext, ns*nr] or None.
        Returns grad [3, nz, nx] (float32, device).

        With graph replay on, the residual is copied into buffers the plan
        keeps, so every call presents the same pointers to the captured
        graph."""
        res = []
        for q, r in enumerate(residual):
            if r is None:
                res.append(None)
                continue
            r = r.to(self.device, torch.float32)
            if self.opts.graph:
                buf = self._res_bufs.get(q) if hasattr(self, "_res_bufs") else None
                if buf is None or buf.shape != r.shape:
                    if not hasattr(self, "_res_bufs"):
                        self._res_bufs = {}
                    buf = self._res_bufs[q] = torch.empty_like(r, memory_format=torch.contiguous_format)
                buf.copy_(r)
                r = buf
            res.append(r.contiguous())
        arr = (ctypes.c_void_p * 5)(*[(r.data_ptr() if r is not None else None) for r in res])
        if grad is None:
            if self.opts.graph:
                if getattr(self, "_grad_buf", None) is None:
                    self._grad_buf = torch.empty((3, self.nz, self.nx), dtype=torch.float32, device=self.device)
                grad = self._grad_buf
            else:
                grad = torch.empty((3, self.nz, self.nx), dtype=torch.float32, device=self.device)
        N.check(self.lib.pyfwi_gradient(self.handle, self.ws, self.ws_bytes, arr, int(param), _ptr(grad), _ptr(raw),
                                        _stream(self.device)))
        self._res_keep = res
        return grad.clone() if self.opts.graph else grad


def _ptr_array(ts):
    return (ctypes.c_void_p * 5)(*[(t.data_ptr() if t is not None else None) for t in ts])


def mean2(a, b):
    """(a + b) / 2 on the device (float32)."""
    a = a.contiguous()
    b = b.contiguous()
    out = torch.empty_like(a)
    N.check(N.lib().pyfwi_mean2(_ptr(a), _ptr(b), _ptr(out), a.numel(), _stream(a.device)))
    return out


def gaussian_weights(sigma, truncate=4.0):
    """Normalised Gaussian weights of scipy.ndimage.gaussian_filter1d
    (radius int(truncate * sigma + 0.5)), in double."""
    sigma = float(sigma)
    radius = int(truncate * sigma + 0.5)
    x = np.arange(-radius, radius + 1, dtype=np.float64)
    w = np.exp(-0.5 / (sigma * sigma) * x ** 2)
    return w / w.sum(), radius


def smooth(planes, sigma):
    """Gaussian smoothing of stacked (n, nz, nx) float32 device arrays with
    standard deviation `sigma` cells, returned as a new tensor; sigma <= 1e-15
    returns a copy (gaussian_filter leaves the array unchanged then)."""
    x = planes.contiguous()
    if float(sigma) <= 1e-15:
        return x.clone()
    w, radius = gaussian_weights(sigma)
    n, nz, nx = x.shape
    out = torch.empty_like(x)
    tmp = torch.empty_like(x)
    N.check(N.lib().pyfwi_smooth(_ptr(x), _ptr(out), _ptr(tmp), int(n), int(nz), int(nx),
                                 w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(radius), _stream(x.device)))
    return out


def l2_residual(dest, dobs):
    """L2 misfit of two dicts of device tensors: (rms as a 0-d float64 device
    tensor, residual dict)."""
    first = dest[[*dest][0]]
    dev = require_cuda(first.device)
    acc = torch.zeros((), dtype=torch.float64, device=dev)
    scratch = torch.empty(N.REDUCE_SLOTS, dtype=torch.float64, device=dev)
    res = {}
    for p in dest:
        e = dest[p].to(dev, torch.float32).contiguous()
        o = dobs[p].to(dev, torch.float32).contiguous()
        r = torch.empty_like(e)
        N.check(N.lib().pyfwi_l2_residual(_ptr(e), _ptr(o), _ptr(r), e.numel(), _ptr(scratch), _ptr(acc),
                                          _stream(dev)))
        res[p] = r
    return acc, res
