"""TEST INFRASTRUCTURE ONLY -- host driver of the CPU oracle.

This module is the checker for the CUDA product path.  Only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` may
import it; the product package never does.

It restates, in numpy plus the C kernels of ``oracle/elastic_oracle.c``, the
host side of PyFWI's propagator:

* ``WavePreparation.__init__`` set-up: time-step split, grid padding, source
  and receiver index constants, checkpoint schedule
  (PyFWI src/PyFWI/wave_propagation.py:18-144);
* the damping profile (src/PyFWI/fwi_tools.py:943-1063), model padding
  (fwi_tools.py:776-811) and material buffers (wave_propagation.py:570-591);
* ``forward_modeling`` (wave_propagation.py:859-887) and ``gradient``
  (wave_propagation.py:889-938), including ``gradient_reading``
  (wave_propagation.py:279-331), ``grad_lmd_to_vd`` (src/PyFWI/grad_switcher.py:331-383)
  and ``seismic_section`` (src/PyFWI/acquisition.py:313-333).

The numpy expressions that decide an index or a float32 rounding are written
with the same operand types as the reference so numpy's promotion rules give
the same bits.  Two precisions: ``'fp32'`` (reference semantics) and
``'fp64'`` (everything in double: the FP64 oracle).
"""
import ctypes
import os
import subprocess

import numpy as np
from scipy.ndimage import gaussian_filter

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")

_i32 = ctypes.c_int32
_f64 = ctypes.c_double


class OrcCfg(ctypes.Structure):
    """Mirror of ``orc_cfg`` in elastic_oracle.c."""
    _fields_ = [("Nz", _i32), ("Nx", _i32), ("sdo", _i32), ("npml", _i32),
                ("dt", _f64), ("dx", _f64), ("dz", _f64),
                ("c1", _f64), ("c2", _f64), ("c3", _f64), ("c4", _f64),
                ("nt", _i32), ("dt_scale", _i32), ("nt_ext", _i32),
                ("acq_type", _i32), ("Nr", _i32), ("n_main_rec", _i32),
                ("n_extera_rec", _i32), ("dxr", _i32),
                ("rec_top_left_const", _i32), ("rec_top_left_var", _i32),
                ("rec_top_right_const", _i32), ("rec_top_right_var", _i32),
                ("rec_surface_const", _i32), ("rec_surface_var", _i32)]


_LIBS = {}


def build():
    """Compile the oracle libraries (idempotent)."""
    subprocess.check_call(["make", "-s", "-C", HERE], stdout=subprocess.DEVNULL)


def lib(precision="fp32", img_round=None):
    """ctypes handle of liborc32.so / liborc64.so, building them if absent;
    img_round 'bf16' / 'fp24' (precision 'fp32' only): the build whose
    imaging rounds its five differences of the forward state to that format."""
    name = {"fp32": "liborc32.so", "fp64": "liborc64.so"}[precision]
    if img_round:
        if precision != "fp32" or img_round not in ("bf16", "fp24"):
            raise ValueError("img_round is 'bf16' or 'fp24' on the fp32 oracle")
        name = "liborc32_img%s.so" % img_round
    key = (precision, img_round or None)
    if key not in _LIBS:
        path = os.path.join(BUILD, name)
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        L.orc_forward_shot.restype = ctypes.c_int
        L.orc_forward_shot.argtypes = [ctypes.POINTER(OrcCfg), P, P, P, P, P, _i32, _i32, P, _i32, P, P, P, _i32]
        L.orc_gradient_shot.restype = ctypes.c_int
        L.orc_gradient_shot.argtypes = [ctypes.POINTER(OrcCfg), P, P, P, P, P, ctypes.POINTER(P), P, P, _i32,
                                        P, P, P, P, P, P]
        L.orc_step_forward.restype = None
        L.orc_step_forward.argtypes = [ctypes.POINTER(OrcCfg)] + [P] * 10 + [ctypes.c_int]
        L.orc_exact_gradient_shot.argtypes = [ctypes.POINTER(OrcCfg), P, P, P, P, P, _i32, _i32, P, _i32,
                                              ctypes.POINTER(P), P, P, P, P]
        _LIBS[key] = L
    return _LIBS[key]


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


# --------------------------------------------------------------------------
# host set-up, restated
# --------------------------------------------------------------------------
class Ricker:
    """Source object with the fields the propagator reads
    (src/PyFWI/acquisition.py:207-244): ``i``/``j`` grid indices,
    ``component`` mask, ``w`` wavelet and ``__call__``."""

    def __init__(self, src_loc, dh, dt, src_type=0):
        self.dh = dh
        self.i = np.int32(src_loc[:, 0] / self.dh)
        self.j = np.int32(src_loc[:, 1] / self.dh)
        self.dt = dt
        self.component = np.zeros(5, dtype=np.float32)
        if src_type == 0:
            self.component[2:4] = np.float32(1)
        elif src_type == 1:
            self.component[0] = np.float32(1)
        elif src_type == 2:
            self.component[1] = np.float32(1)

    def Ricker(self, fdom):
        self.t = np.arange(-1.0 / fdom, 1.0 / fdom + self.dt / 3, self.dt)
        self.w = np.float32((1.0 - 2.0 * (np.pi * fdom * self.t) ** 2) * np.exp(-(np.pi * fdom * self.t) ** 2))

    def __call__(self, ind):
        if ind < self.w.size:
            return self.w[ind] * self.component
        return np.float32(0.0) * self.component


def pml_delta(dh, n_pml, pml_r):
    """fwi_tools.py:1016-1063."""
    delta1 = n_pml * dh
    r = (np.arange(n_pml) * dh)
    if delta1 != 0:
        return np.float32(-(3 / (2 * delta1)) * ((r / delta1) ** 2) * (np.log10(pml_r)))
    return np.array([])


def pml_profiles(tnz, tnx, dh, n_pml, pml_r, pml_dir):
    """fwi_tools.py:943-1013: 2-D damping arrays (before the vp_max factor)."""
    dx_pml = np.zeros((tnz, tnx)).astype(np.float32, order="C")
    dz_pml = np.zeros((tnz, tnx)).astype(np.float32, order="C")
    a = pml_delta(dh, n_pml, pml_r)
    dx_pml[:, tnx - n_pml:] = a
    dx_pml[:, :n_pml] = np.flip(a, 0)
    a = pml_delta(dh, n_pml, pml_r)
    dz_pml[tnz - n_pml:, :] = a.reshape(-1, 1)
    dz_pml[:n_pml, :] = np.flip(a, 0).reshape(-1, 1)
    if pml_dir == 0:
        dx_pml = np.zeros(dx_pml.shape, np.float32)
    elif pml_dir == 1:
        dz_pml = np.zeros(dz_pml.shape, np.float32)
    elif pml_dir == 3:
        dz_pml[:n_pml, :] = np.zeros((len(a), dz_pml.shape[1]), dtype=np.float32)
    return dx_pml, dz_pml


def expand(param, tnz, tnx, n_pml, dtype=np.float32):
    """fwi_tools.py:776-811: edge-replicated padding (float32 as the
    reference; the FP64 oracle keeps double)."""
    nu = np.zeros((tnz, tnx)).astype(dtype, order="C")
    nu[n_pml:tnz - n_pml, n_pml:tnx - n_pml] = param.astype(dtype, order="C")
    nu[:n_pml, :] = nu[n_pml, :]
    nu[tnz - n_pml:, :] = nu[tnz - n_pml - 1, :]
    nu[:, tnx - n_pml:] = nu[:, tnx - n_pml - 1].reshape(-1, 1)
    nu[:, :n_pml] = nu[:, n_pml].reshape(-1, 1)
    return nu


def seismic_section(seismo, components=0, shape="3d"):
    """acquisition.py:313-333."""
    plan = {"1": ["taux"], "2": ["vx", "vz"], "3": ["taux", "tauz", "tauxz"],
            "4": ["vx", "vz", "taux", "tauz", "tauxz"]}
    data = {}
    if components != 0:
        for p in plan[str(components)]:
            data[p] = seismo[p]
    else:
        data["taux"] = (seismo["taux"] + seismo["tauz"]) / 2
        data["tauz"] = (seismo["taux"] + seismo["tauz"]) / 2
    if shape == "2d":
        (nt, nr, ns) = data[[*data][0]].shape
        for p in data:
            data[p] = np.reshape(data[p], (nt, nr * ns), "F")
    return data


def prepare_residual(res, s=1.):
    """src/PyFWI/processing.py:142-158."""
    data = {}
    shape = res[[*res][0]].shape
    for p in ["vx", "vz", "taux", "tauz", "tauxz"]:
        data[p] = s * res[p] if p in res else np.zeros(shape, np.float32)
    return data


def grad_lmd_to_vd(glam, gmu, grho, lam, mu, rho):
    """grad_switcher.py:331-383."""
    vp = np.sqrt((lam + 2 * mu) / rho)
    vs = np.sqrt(mu / rho)
    vs2 = vs ** 2
    vpvs = vp ** 2 - 2 * vs ** 2
    gvp = glam * 2 * vp * rho + gmu * 0 + grho * 0
    gvs = glam * (-4 * rho * vs) + gmu * 2 * vs * rho + grho * 0
    grho_out = glam * vpvs + gmu * vs2 + grho
    return gvp.astype(np.float32), gvs.astype(np.float32), grho_out.astype(np.float32)


FIELDS = ["vx", "vz", "taux", "tauz", "tauxz"]


def lowpass(x, highcut, fn, order, axis=1):
    """lowpass and adj_lowpass of fwi_tools.py:1188-1258 (the two apply the
    same product), in float64: traces (planes, nt, ncols) padded with 512
    zeros along time, FFT, times h and conj(h) (freqz of the Butterworth
    design on the whole circle), real inverse FFT, first nt samples."""
    from scipy.signal import butter, freqz
    assert axis == 1
    x = np.concatenate([np.asarray(x, np.float64), np.zeros((x.shape[0], 512, x.shape[2]))], axis=1)
    n = x.shape[1]
    X = np.fft.fft(x, n=n, axis=1)
    b, a = butter(order, 2 * highcut / fn, btype="lowpass", output="ba")
    _, h = freqz(b, a, worN=n, whole=True)
    X = np.conjugate(h)[None, :, None] * (h[None, :, None] * X)
    return np.fft.ifft(X, n=n, axis=1).real[:, :-512, :]


class OracleWavePropagator:
    """CPU oracle with the reference ``WavePropagator`` interface.

    ``precision='fp32'`` reproduces the reference's float32 semantics,
    ``'fp64'`` runs every array in double (the FP64 oracle).  ``img_round``
    ('bf16' or 'fp24', fp32 only) rounds the imaging's five differences of
    the forward state to that format (what a store of difference sets in it
    would give): a what-if for the error of such a store, not the reference.
    """

    def __init__(self, inpa, src, rec_loc, model_shape, components=0, n_well_rec=0, chpr=0,
                 precision="fp32", img_round=None):
        keys = [*inpa]
        self.precision = precision
        self.img_round = img_round
        self.real = np.float32 if precision == "fp32" else np.float64
        # wave_propagation.py:28-35
        self.dt_scale = np.ceil(inpa["dt"] / 0.0006)
        self.t = inpa["t"]
        self.dt_ext = inpa["dt"]
        self.dt = inpa["dt"] / self.dt_scale
        self.fn = 1.0 / 2.0 / 0.0006
        self.nt = int(1 + self.t // self.dt)
        self.nt_ext = int(1 + self.t // self.dt_ext)
        self.nx = np.int32(model_shape[1])
        self.nz = np.int32(model_shape[0])
        self.seismo_shape = inpa["seimogram_shape"] if "seimogram_shape" in keys else "2d"
        self.g_smooth = inpa["g_smooth"] if "g_smooth" in keys else 0
        if "npml" in keys:
            self.npml, pmlR, pml_dir = inpa["npml"], inpa["pmlR"], inpa["pml_dir"]
        else:
            self.npml, pmlR, pml_dir = 0, 0, 2
        self.sdo = np.int32(inpa["sdo"] / 2) if "sdo" in keys else 2
        rec_dis = inpa["rec_dis"] if "rec_dis" in keys else (rec_loc[1, :] - rec_loc[0, :]).max()
        self.acq_type = inpa["acq_type"] if "acq_type" in keys else 1
        self.energy_balancing = inpa["energy_balancing"] if "energy_balancing" in keys else False
        self.tnx = np.int32(self.nx + 2 * self.npml)
        self.tnz = np.int32(self.nz + 2 * self.npml)
        self.dh = np.float32(inpa["dh"])
        self.srcx = np.int32(src.i + self.npml)
        self.srcz = np.int32(src.j + self.npml)
        self.src = src
        self.ns = np.int32(src.i.size)
        self.dxr = np.int32(rec_dis / self.dh)
        chp = int(chpr * self.nt / 100)
        self.chp = np.linspace(0, self.nt - 1, chp, dtype=np.int32)
        if len(self.chp) < 2:
            self.chp = np.array([1, self.nt - 1])
        self.chp = self.chp.astype(np.int32)
        self.nchp = len(self.chp)
        self.rec_loc = rec_loc
        self.nr = rec_loc.shape[0]
        self.n_well_rec = n_well_rec
        self.n_surface_rec = self.nr - 2 * n_well_rec
        if n_well_rec == 0 and self.acq_type == 2:
            raise Exception(" Number of geophons in the wells is not defined")
        z = np.int32(0)
        self.rec_top_left_const = self.rec_top_left_var = z
        self.rec_top_right_const = self.rec_top_right_var = z
        self.rec_surface_const = self.rec_surface_var = z
        if self.acq_type == 0:
            self.rec_top_right_const = np.int32(rec_loc[0, 0] / self.dh + self.npml)
            self.rec_top_right_var = np.int32(rec_loc[0, 1] / self.dh + self.npml)
            self.src_cts = src.i[0]
        elif self.acq_type == 1:
            self.rec_surface_const = np.int32(rec_loc[0, 1] / self.dh + self.npml)
            self.rec_surface_var = np.int32(rec_loc[0, 0] / self.dh + self.npml)
            self.src_cts = src.j[0]
        elif self.acq_type == 2:
            a = np.int32(rec_loc[-self.n_well_rec, :] / self.dh + self.npml)
            self.rec_top_right_const, self.rec_top_right_var = np.copy(a[0]), np.copy(a[1])
            a = np.int32(rec_loc[self.n_well_rec, :] / self.dh + self.npml)
            self.rec_surface_const, self.rec_surface_var = np.copy(a[1]), np.copy(a[0])
            self.rec_top_left_const = np.int32(rec_loc[0, 0] / self.dh + self.npml)
            self.rec_top_left_var = np.int32(rec_loc[:, 1] / self.dh + self.npml)[0]
            self.src_cts = src.j[0]
        self.dx_pml, self.dz_pml = pml_profiles(self.tnz, self.tnx, self.dh, self.npml, pmlR, pml_dir)
        self.components = components
        # wave_propagation.py:423-490: stencil constants go through "%f"
        if self.sdo == 2:
            c = (9 / 8, -1 / 24, 0, 0)
        elif self.sdo == 4:
            c = (1715 / 1434, -114 / 1434, 14 / 1434, -1 / 1434)
        else:
            raise AssertionError("Order of the derivative has be either 4 or 8!")
        r6 = lambda x: float("%f" % x)
        self.cfg = OrcCfg(
            Nz=int(self.tnz), Nx=int(self.tnx), sdo=int(self.sdo), npml=int(self.npml),
            dt=r6(self.dt), dx=r6(self.dh), dz=r6(self.dh),
            c1=r6(c[0]), c2=r6(c[1]), c3=r6(c[2]), c4=r6(c[3]),
            nt=self.nt, dt_scale=int(self.dt_scale), nt_ext=self.nt_ext,
            acq_type=int(self.acq_type), Nr=int(self.nr), n_main_rec=int(self.n_surface_rec),
            n_extera_rec=int(self.n_well_rec), dxr=int(self.dxr),
            rec_top_left_const=int(self.rec_top_left_const), rec_top_left_var=int(self.rec_top_left_var),
            rec_top_right_const=int(self.rec_top_right_const), rec_top_right_var=int(self.rec_top_right_var),
            rec_surface_const=int(self.rec_surface_const), rec_surface_var=int(self.rec_surface_var))
        self.n_inj = int(np.ceil(self.nt / self.dt_scale))
        self.src_vals = np.zeros((self.n_inj, 4), np.float32)
        for k in range(self.n_inj):
            self.src_vals[k] = np.float32(self.src(k))[:4]

    # ---- materials ----------------------------------------------------
    def _materials(self, model0):
        model = dict(model0)
        for p in model:
            model[p] = expand(model[p], self.tnz, self.tnx, self.npml, self.real)
        v_max = model["vp"].max()
        vdx = self.dx_pml * v_max
        vdz = self.dz_pml * v_max
        if self.precision == "fp32":
            mu = model["rho"] * (model["vs"] ** 2)
            lam = model["rho"] * (model["vp"] ** 2) - 2 * mu
            rho = model["rho"]
            rho_b = 1 / model["rho"]
        else:
            m = {k: v.astype(np.float64) for k, v in model.items()}
            mu = m["rho"] * (m["vs"] ** 2)
            lam = m["rho"] * (m["vp"] ** 2) - 2 * mu
            rho = m["rho"]
            rho_b = 1 / m["rho"]
            vdx, vdz = vdx.astype(np.float64), vdz.astype(np.float64)
        R = self.real
        self.lam, self.mu, self.rho = lam.astype(R), mu.astype(R), rho.astype(R)
        self.vp, self.vs = model["vp"], model["vs"]
        self.rho_b = np.ascontiguousarray(rho_b, R)
        self.vdx = np.ascontiguousarray(vdx, R)
        self.vdz = np.ascontiguousarray(vdz, R)

    def _mats(self):
        return (_ptr(self.lam), _ptr(self.mu), _ptr(self.rho_b), _ptr(self.vdx), _ptr(self.vdz))

    def forward_shot(self, s, store=False):
        """Seismogram planes (5, nt_ext, nr) of shot s; with store=True also
        the checkpoint states (nchp, 5, tnz, tnx)."""
        L = lib(self.precision, self.img_round)
        seis = np.zeros((5, self.nt_ext, self.nr), self.real)
        W = np.zeros((self.nchp, 5, self.tnz, self.tnx), self.real) if store else None
        rc = L.orc_forward_shot(ctypes.byref(self.cfg), *self._mats(), int(self.srcx[s]), int(self.srcz[s]),
                                _ptr(self.src_vals), self.n_inj, _ptr(seis), _ptr(W), _ptr(self.chp), self.nchp)
        if rc != 0:
            raise MemoryError("oracle forward: allocation failed")
        return seis, W

    def forward_modeling(self, model0, show=False):
        self._materials(model0)
        self.seismogram = {f: np.zeros((self.nt_ext, self.nr, self.ns), self.real) for f in FIELDS}
        for s in range(self.ns):
            seis, _ = self.forward_shot(s)
            for k, f in enumerate(FIELDS):
                self.seismogram[f][:, :, s] = seis[k]
        if self.acq_type == 2:
            for p in self.seismogram:
                self.seismogram[p][:, :self.n_well_rec] = np.flip(self.seismogram[p][:, :self.n_well_rec], axis=1)
        return seismic_section(self.seismogram, self.components, shape=self.seismo_shape)

    def raw_gradient(self, res):
        """Six (tnz, tnx) accumulators (Gmu, Glam, Grho, and the three energy
        terms) summed over shots, from a prepared 2-D residual dict."""
        L = lib(self.precision, self.img_round)
        n = (int(self.tnz), int(self.tnx))
        G = [np.zeros(n, self.real) for _ in range(6)]
        for s in range(self.ns):
            _, W = self.forward_shot(s, store=True)
            planes = []
            for f in FIELDS:
                r = res[f][:, s * self.nr:(s + 1) * self.nr]
                planes.append(np.ascontiguousarray(r, self.real) if np.any(r) else None)
            arr = (ctypes.c_void_p * 5)(*[ctypes.c_void_p(p.ctypes.data) if p is not None else None for p in planes])
            rc = L.orc_gradient_shot(ctypes.byref(self.cfg), *self._mats(), arr, _ptr(W), _ptr(self.chp),
                                     self.nchp, *[_ptr(g) for g in G])
            if rc != 0:
                raise MemoryError("oracle gradient: allocation failed")
        return G

    def gradient(self, res, show=False, parameterization="dv"):
        if self.acq_type == 2:
            for p in self.seismogram:
                self.seismogram[p][:, :self.n_well_rec] = np.flip(self.seismogram[p][:, :self.n_well_rec], axis=1)
        res = prepare_residual(res, 1)
        Gmu, Glam, Grho, Pmu, Plam, Prho = self.raw_gradient(res)
        self.raw = dict(Gmu=Gmu, Glam=Glam, Grho=Grho, Pmu=Pmu, Plam=Plam, Prho=Prho)
        glam, gmu, grho0 = self._gradient_reading(Gmu, Glam, Grho, Pmu, Plam, Prho)
        npml, tnz, tnx = self.npml, self.tnz, self.tnx
        crop = lambda a: a[npml:tnz - npml, npml:tnx - npml]
        if parameterization == "dv":
            gvp, gvs, grho = grad_lmd_to_vd(glam, gmu, grho0, crop(self.lam), crop(self.mu), crop(self.rho))
            return {"vp": gaussian_filter(gvp, self.g_smooth), "vs": gaussian_filter(gvs, self.g_smooth),
                    "rho": gaussian_filter(grho, self.g_smooth)}
        return {"lam": gaussian_filter(glam, self.g_smooth), "mu": gaussian_filter(gmu, self.g_smooth),
                "rho": gaussian_filter(grho0, self.g_smooth)}

    # ---- exact discrete adjoint (no counterpart in the reference) -------
    def raw_traces(self, model0):
        """Raw receiver traces {field: (nt_ext, nr, ns)} of every shot, in
        recording order (before any section reshaping or well flip)."""
        self._materials(model0)
        out = {f: np.zeros((self.nt_ext, self.nr, self.ns), self.real) for f in FIELDS}
        for s in range(self.ns):
            seis, _ = self.forward_shot(s)
            for k, f in enumerate(FIELDS):
                out[f][:, :, s] = seis[k]
        return out

    def exact_gradient(self, model0, dtrace):
        """dJ/d(lam, mu, b) on the padded grid, summed over shots, for a
        misfit J of the raw traces with dJ/dtrace = dtrace ({field:
        (nt_ext, nr, ns)}, missing fields zero), the damping held fixed."""
        L = lib(self.precision, self.img_round)
        self._materials(model0)
        n = (int(self.tnz), int(self.tnx))
        G = [np.zeros(n, self.real) for _ in range(3)]
        every = np.arange(self.nt, dtype=np.int32)
        for s in range(self.ns):
            seis = np.zeros((5, self.nt_ext, self.nr), self.real)
            W = np.zeros((self.nt, 5, self.tnz, self.tnx), self.real)
            L.orc_forward_shot(ctypes.byref(self.cfg), *self._mats(), int(self.srcx[s]), int(self.srcz[s]),
                               _ptr(self.src_vals), self.n_inj, _ptr(seis), _ptr(W), _ptr(every), self.nt)
            planes = [np.ascontiguousarray(dtrace[f][:, :, s], self.real) if f in dtrace else None for f in FIELDS]
            arr = (ctypes.c_void_p * 5)(*[ctypes.c_void_p(p.ctypes.data) if p is not None else None for p in planes])
            rc = L.orc_exact_gradient_shot(ctypes.byref(self.cfg), *self._mats()[:5], int(self.srcx[s]),
                                           int(self.srcz[s]), _ptr(self.src_vals), self.n_inj, arr, _ptr(W),
                                           *[_ptr(g) for g in G])
            if rc != 0:
                raise MemoryError("oracle exact gradient: allocation failed")
        return G

    def model_gradient(self, model0, Glam, Gmu, Gb):
        """Chain rule from (lam, mu, b) on the padded grid to (vp, vs, rho) on
        the model grid: lam = rho vp^2 - 2 mu, mu = rho vs^2, b = 1/rho, and
        the edge-replicated padding folded back onto the edge cells."""
        R = np.float64
        vp, vs, rho = (expand(model0[k], self.tnz, self.tnx, self.npml, R) for k in ("vp", "vs", "rho"))
        Glam, Gmu, Gb = (np.asarray(g, R) for g in (Glam, Gmu, Gb))
        gp = {"vp": 2 * rho * vp * Glam,
              "vs": -4 * rho * vs * Glam + 2 * rho * vs * Gmu,
              "rho": (vp ** 2 - 2 * vs ** 2) * Glam + vs ** 2 * Gmu - Gb / rho ** 2}
        rows = np.clip(np.arange(self.tnz) - self.npml, 0, self.nz - 1)
        cols = np.clip(np.arange(self.tnx) - self.npml, 0, self.nx - 1)
        out = {}
        for k, g in gp.items():
            m = np.zeros((int(self.nz), int(self.nx)), R)
            np.add.at(m, (rows[:, None], cols[None, :]), g)
            out[k] = m
        return out

    def _gradient_reading(self, Gmu, Glam, Grho, Pmu, Plam, Prho):
        """wave_propagation.py:279-331."""
        R = self.real
        if not self.energy_balancing:
            Pmu = np.ones((self.tnz, self.tnx), R)
            Plam = np.ones((self.tnz, self.tnx), R)
            Prho = np.ones((self.tnz, self.tnx), R)
        sdo, npml, tnz, tnx = self.sdo, self.npml, self.tnz, self.tnx

        def factor_of(precond0):
            factor = np.zeros((self.nz, self.nx), R)
            denom = np.sqrt(np.copy(precond0))
            if self.acq_type == 0:
                denom = denom[npml + sdo:tnz - npml - sdo, npml + sdo + self.src_cts + 2:tnx - npml - sdo]
                factor[sdo:-sdo, sdo + self.src_cts + 2:-sdo] = 1 / denom
            else:
                denom = denom[npml + sdo + self.src_cts + 2:tnz - npml - sdo, npml + sdo:tnx - npml - sdo]
                factor[sdo + self.src_cts + 2:-sdo, sdo:-sdo] = 1 / denom
            return factor / np.abs(factor).max()

        crop = lambda a: a[npml:tnz - npml, npml:tnx - npml]
        grho = crop(Grho) * factor_of(Prho)
        gmu = crop(Gmu) * factor_of(Pmu)
        glam = crop(Glam) * factor_of(Plam)
        return glam, gmu, grho
