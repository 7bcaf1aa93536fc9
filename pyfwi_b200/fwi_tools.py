"""The part of PyFWI's fwi_tools the propagator path uses
(src/PyFWI/fwi_tools.py): finite-difference coefficients and stable time
step, model padding, the damping-layer profile, the L2 misfit, and the
model vector packing of the FWI driver."""
import numpy as np


class Fdm:
    """Staggered-grid coefficients of order 4 or 8 (fwi_tools.py:452-474) and
    the stable time step (fwi_tools.py:634-647)."""

    _COEF = {4: (9 / 8, -1 / 24, 0, 0), 8: (1715 / 1434, -114 / 1434, 14 / 1434, -1 / 1434)}
    _DH_N = {4: 4, 8: 3}

    def __init__(self, order):
        if order not in self._COEF:
            raise AssertionError("Order of the derivative has be either 4 or 8!")
        self._order = order
        self._c1, self._c2, self._c3, self._c4 = self._COEF[order]
        self.dh_n = self._DH_N[order]

    @property
    def order(self):
        return self._order

    c1 = property(lambda self: self._c1)
    c2 = property(lambda self: self._c2)
    c3 = property(lambda self: self._c3)
    c4 = property(lambda self: self._c4)

    def dt_computation(self, vp_max, dx, dz=None):
        if dz is None:
            dz = dx
        c_sum = np.abs(self._c1) + np.abs(self._c2) + np.abs(self._c3) + np.abs(self._c4)
        a = 1 / dx / dx * c_sum + 1 / dz / dz * c_sum
        return 2 / vp_max / np.sqrt(a * (1 + 4.0))


def expand_model(parameter, TNz, TNx, n_pml=10):
    """Pad a (nz, nx) property to (TNz, TNx) by edge replication
    (fwi_tools.py:776-811)."""
    nu = np.zeros((TNz, TNx)).astype(np.float32, order="C")
    nu[n_pml:TNz - n_pml, n_pml:TNx - n_pml] = parameter.astype(np.float32, order="C")
    nu[:n_pml, :] = nu[n_pml, :]
    nu[TNz - n_pml:, :] = nu[TNz - n_pml - 1, :]
    nu[:, TNx - n_pml:] = nu[:, TNx - n_pml - 1].reshape(-1, 1)
    nu[:, :n_pml] = nu[:, n_pml].reshape(-1, 1)
    return nu


def pml_delta_calculation(dh, n_pml=10, pml_r=1e-5):
    """Quadratic damping ramp d(r) = -(3 / 2L) (r / L)^2 log10(R), r = 0..npml-1
    cells, L = npml*dh (fwi_tools.py:1016-1063).  Same numpy operand types as
    the reference so the float32 values agree bit for bit."""
    delta1 = n_pml * dh
    r = (np.arange(n_pml) * dh)
    if delta1 != 0:
        return np.float32(-(3 / (2 * delta1)) * ((r / delta1) ** 2) * (np.log10(pml_r)))
    return np.array([])


def pml_counstruction(TNz, TNx, dh, n_pml=10, pml_r=1e-5, pml_dir=3):
    """Damping arrays (TNz, TNx) for x and z (fwi_tools.py:943-1013).
    pml_dir: 0 no x damping, 1 no z damping, 2 all sides, 3 no top."""
    dx_pml = np.zeros((TNz, TNx)).astype(np.float32, order="C")
    dz_pml = np.zeros((TNz, TNx)).astype(np.float32, order="C")
    a = pml_delta_calculation(dh, n_pml, pml_r)
    dx_pml[:, TNx - n_pml:] = a
    dx_pml[:, :n_pml] = np.flip(a, 0)
    a = pml_delta_calculation(dh, n_pml, pml_r)
    dz_pml[TNz - n_pml:, :] = a.reshape(-1, 1)
    dz_pml[:n_pml, :] = np.flip(a, 0).reshape(-1, 1)
    if pml_dir == 0:
        dx_pml = np.zeros(dx_pml.shape, np.float32)
    elif pml_dir == 1:
        dz_pml = np.zeros(dz_pml.shape, np.float32)
    elif pml_dir == 3:
        dz_pml[:n_pml, :] = np.zeros((len(a), dz_pml.shape[1]), dtype=np.float32)
    return dx_pml, dz_pml


class CostFunction:
    """Misfit functions (fwi_tools.py:1365-1422).  Only 'l2' is provided:
    rms = sum over components of 0.5 * |dest - dobs|^2, residual dest - dobs
    (float32).  numpy dicts or torch tensors (the tensor path runs on the
    device, accumulating in float64)."""

    def __init__(self, cost_function_type="l2"):
        if cost_function_type != "l2":
            raise NotImplementedError("only the 'l2' misfit is provided")
        self.cost_function_type = cost_function_type

    def __call__(self, dest, dobs):
        return self.l2(dest, dobs)

    @staticmethod
    def l2(dest, dobs):
        first = dest[[*dest][0]]
        if isinstance(first, np.ndarray):
            rms, res = 0, {}
            for p in dest:
                res[p] = np.float32(dest[p] - dobs[p])
                rms += 0.5 * (res[p].reshape(-1).T @ res[p].reshape(-1))
            return rms, res
        from .engine import l2_residual
        return l2_residual(dest, dobs)


LOWPASS_PADDING = 512  # zeros the reference appends to every trace before its FFT
_RESPONSES = {}


def lowpass_response(nt, highcut, fn, order=1):
    """The reference's zero-phase low-pass (lowpass / adj_lowpass,
    fwi_tools.py:1188-1258) as an nt x nt float32 matrix K, with
    lowpass(x)[t] = sum_s K[t][s] x[s] along time.

    The reference filters in the frequency domain: traces padded to
    n = nt + 512 samples, multiplied by h and conj(h) (h: freqz of
    butter(order, 2 highcut / fn) on the whole circle) and cut back to nt
    samples of the real inverse FFT.  That is a circular convolution with
    g = real(ifft(conj(h) h)), so K[t][s] = g[(t - s) mod n]; adj_lowpass
    applies the same product, and K is symmetric."""
    from scipy.signal import butter, freqz
    n = int(nt) + LOWPASS_PADDING
    b, a = butter(order, 2 * highcut / fn, btype="lowpass", output="ba")
    _, h = freqz(b, a, worN=n, whole=True)
    g = np.fft.ifft(np.conjugate(h) * h).real
    idx = (np.arange(nt)[:, None] - np.arange(nt)[None, :]) % n
    return np.ascontiguousarray(g[idx], np.float32)


def lowpass_spectrum(nt, highcut, fn, order=1):
    """The operator of lowpass_response applied by FFT: (nfft, filter) with
    nfft the smallest power of two >= 2 nt - 1 and filter the float32 array
    pyfwi_lowpass takes: the real spectrum of the response embedded in a
    circulant of nfft points (c[k] = c[nfft - k] = g[k] for k < nt, zero
    between), divided by nfft, followed by the twiddles exp(-2 pi i j / nfft),
    j < nfft / 2, as (cos, sin) pairs.  The product of a zero-padded trace's
    FFT with that spectrum, transformed back, is K x on the first nt
    samples."""
    from scipy.signal import butter, freqz
    nt = int(nt)
    n = nt + LOWPASS_PADDING
    b, a = butter(order, 2 * highcut / fn, btype="lowpass", output="ba")
    _, h = freqz(b, a, worN=n, whole=True)
    g = np.fft.ifft(np.conjugate(h) * h).real
    nfft = 1 << max(1, int(np.ceil(np.log2(2 * nt - 1))) if nt > 1 else 1)
    c = np.zeros(nfft)
    c[:nt] = g[:nt]
    c[nfft - nt + 1:] = g[1:nt][::-1]
    spec = np.fft.fft(c).real / nfft
    j = np.arange(nfft // 2)
    tw = np.stack([np.cos(2 * np.pi * j / nfft), -np.sin(2 * np.pi * j / nfft)], 1).reshape(-1)
    return nfft, np.ascontiguousarray(np.concatenate([spec, tw]), np.float32)


def _device_filter(nt, highcut, fn, order, device):
    import torch
    key = (int(nt), float(highcut), float(fn), int(order), str(device))
    if key not in _RESPONSES:
        nfft, f = lowpass_spectrum(nt, highcut, fn, order)
        _RESPONSES[key] = (nfft, torch.from_numpy(f).to(device))
    return _RESPONSES[key]


def _filter(x, highcut, fn, order, axis):
    """Filter (n_planes, nt, ncols) traces along axis 1 on the device
    (pyfwi_lowpass: FFT convolution with the response, one kernel launch);
    numpy in, numpy out (float64, as the reference)."""
    import torch
    from . import _native as N
    from .engine import _ptr, _stream
    if axis != 1:
        raise NotImplementedError("the traces are filtered along axis 1 (time), as the FWI driver does")
    as_numpy = isinstance(x, np.ndarray)
    t = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda() if as_numpy else x
    dev = t.device
    t = t.to(torch.float32).contiguous()
    shape = t.shape
    if t.ndim == 2:  # one plane
        t = t[None]
    t = t.reshape(t.shape[0], t.shape[1], -1)  # (planes, nt, traces): '3d' sections too
    out = torch.empty_like(t)
    nfft, filt = _device_filter(t.shape[1], highcut, fn, order, dev)
    N.check(N.lib().pyfwi_lowpass(_ptr(filt), nfft, _ptr(t), _ptr(out), int(t.shape[1]), int(t.shape[2]),
                                  int(t.shape[0]), _stream(dev)))
    out = out.reshape(shape)
    return out.cpu().numpy().astype(np.float64) if as_numpy else out


def lowpass(x1, highcut, fn, order=1, axis=1, show=False):
    """fwi_tools.py:1188-1222 on the device: the zero-phase Butterworth
    low-pass of traces (n_planes, nt, ncols) along time."""
    return _filter(x1, highcut, fn, order, axis)


def adj_lowpass(x, highcut, fn, order, axis=1):
    """fwi_tools.py:1225-1258: the adjoint of lowpass, the same operator."""
    return _filter(x, highcut, fn, order, axis)


def cost_seismic(d_pre0, d_obs0, fun, fn=None, freq=None, order=None, axis=None, sourc_weight=False, ns=None,
                 nr=None, params_oh=None):
    """Misfit and adjoint source of two data dicts (fwi_tools.py:1290-1345).
    With `freq` both data are low-passed (cost_preparation, :1153-1186), the
    L2 residual is formed, and the adjoint source is the low-passed residual
    (adj_cost_preparation, :1261-1273).  numpy or torch (device) dicts."""
    if sourc_weight or params_oh is not None:
        raise NotImplementedError("source weighting / parameter weights are not provided")
    if not freq:
        return fun(d_pre0, d_obs0)
    keys = [k for k in d_pre0]
    if not all(k in d_obs0 for k in keys):
        raise KeyError("the observed data miss components of the modelled data")
    f = lambda d: {k: v for k, v in zip(keys, lowpass(_stack(d, keys), freq, fn, order=order, axis=axis))}
    rms, res = fun(f(d_pre0), f(d_obs0))
    adj = adj_lowpass(_stack(res, keys), freq, fn, order=order, axis=axis)
    if isinstance(adj, np.ndarray):
        return rms, {k: adj[q].astype(np.float32) for q, k in enumerate(keys)}
    return rms, {k: adj[q] for q, k in enumerate(keys)}


def _stack(d, keys):
    first = d[keys[0]]
    if isinstance(first, np.ndarray):
        return np.stack([np.asarray(d[k], np.float64) for k in keys])
    import torch
    return torch.stack([d[k].to(torch.float32) for k in keys])


def vel_dict2vec(m0):
    """(vp, vs, rho) dict -> one float64 vector (fwi_tools.py:1066-1073);
    torch tensors give a tensor on their device."""
    import torch
    if isinstance(m0["vp"], torch.Tensor):
        return torch.cat([m0[k].reshape(-1).to(torch.float64) for k in ("vp", "vs", "rho")])
    nz, nx = m0[[*m0][0]].shape
    m = np.zeros((3 * nz * nx))
    m[:nz * nx] = m0["vp"].reshape(-1)
    m[nz * nx:2 * nz * nx] = m0["vs"].reshape(-1)
    m[2 * nz * nx:] = m0["rho"].reshape(-1)
    return m


def vec2vel_dict(m0, nz, nx):
    """Inverse of vel_dict2vec (fwi_tools.py:1076-1097)."""
    return {"vp": m0[:nz * nx].reshape(nz, nx), "vs": m0[nz * nx:2 * nz * nx].reshape(nz, nx),
            "rho": m0[2 * nz * nx:].reshape(nz, nx)}
