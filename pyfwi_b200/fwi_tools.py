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


def cost_seismic(d_pre0, d_obs0, fun, fn=None, freq=None, order=None, axis=None, sourc_weight=False, ns=None,
                 nr=None, params_oh=None):
    """Misfit and adjoint source of two data dicts (fwi_tools.py:1290-1345)
    for the unfiltered case (freq = None)."""
    if freq:
        raise NotImplementedError("band-limited misfit (freq) is not provided")
    if sourc_weight or params_oh is not None:
        raise NotImplementedError("source weighting / parameter weights are not provided")
    return fun(d_pre0, d_obs0)


def vel_dict2vec(m0):
    """(vp, vs, rho) dict -> one vector (fwi_tools.py:1066-1073)."""
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
