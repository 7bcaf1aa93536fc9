"""Acquisition helpers with PyFWI's interface (src/PyFWI/acquisition.py).

Geometry builders, the source object and the seismic-section formatter.
These run once per survey on the host (numpy), as in the reference."""
import numpy as np


def acq_parameters(ns, rec_dis, offsetx, depth, dh, sdo, acq_type):
    """Source and receiver locations for crosswell (0), surface (1) or both
    (2) acquisition (acquisition.py:5-59).  Returns
    (src_loc, rec_loc, n_surface_rec, n_well_rec)."""
    if rec_dis < dh:
        raise Exception("Receiver distance should be larger than spatial sampling")
    if acq_type == 0:
        src_loc, rec_loc = crosswell(ns, rec_dis, offsetx, depth, dh, sdo)
        n_surface_rec, n_well_rec = 0, rec_loc.shape[0]
    elif acq_type == 1:
        src_loc, rec_loc = surface_seismic(ns, rec_dis, offsetx, dh, sdo)
        n_surface_rec, n_well_rec = rec_loc.shape[0], 0
    elif acq_type == 2:
        src_loc, rec_loc = surface_seismic(ns, rec_dis, offsetx, dh, sdo)
        n_surface_rec = rec_loc.shape[0]
        _, well = crosswell(ns, rec_dis, offsetx, depth, dh, sdo)
        left_x = np.ones((well.shape), np.float32) @ (np.array([[rec_loc[0, 1]], [0]], np.float32))
        left = np.hstack((left_x, well[:, 1].reshape(-1, 1)))
        rec_loc = np.vstack((left, rec_loc, well))
        n_well_rec = well.shape[0]
    else:
        raise ValueError("acq_type must be 0, 1 or 2")
    return src_loc, rec_loc, n_surface_rec, n_well_rec


def crosswell(ns, rec_dis, offsetx, depth, dh, sdo):
    """Sources down the left side, receivers down the right (acquisition.py:62-124)."""
    rec_z = np.arange(2 * rec_dis, depth - (2 * rec_dis), rec_dis).reshape(-1, 1)
    nr = rec_z.size
    src_loc = np.empty((ns, 2), dtype=np.float32)
    src_loc[:, 0] = (sdo / 2 + 2) * dh
    src_loc[:, 1] = depth / 2 if ns == 1 else np.linspace(4 * dh, depth - 9 * dh, ns)
    rec_loc = np.hstack((np.ones((nr, 1)) * offsetx - (sdo / 2 + 2) * dh, rec_z))
    return src_loc.astype(np.float32), rec_loc.astype(np.float32)


def surface_seismic(ns, rec_dis, offsetx, dh, sdo):
    """Sources and receivers along the top (acquisition.py:127-185)."""
    rec_x = np.arange(2 * rec_dis, offsetx - 2 * rec_dis, rec_dis).reshape(-1, 1)
    nr = rec_x.size
    src_loc = np.empty((ns, 2), dtype=np.float32)
    src_loc[:, 1] = (sdo / 2 + 2) * dh
    src_loc[:, 0] = offsetx / 2 if ns == 1 else np.linspace(4 * dh, offsetx - 9 * dh, ns)
    rec_loc = np.hstack((rec_x, np.ones((nr, 1)) * (sdo / 2 + 2) * dh))
    return src_loc, rec_loc


class Source:
    """Point source (acquisition.py:188-257).

    ``i``/``j`` are the x/z grid indices of each shot, ``component`` the
    (vx, vz, taux, tauz, tauxz) weights: explosive (src_type 0) drives taux and
    tauz, 1 drives vx, 2 drives vz."""

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
        else:
            raise ValueError("src_type must be 0 (explosive), 1 (x) or 2 (z)")

    def __call__(self, ind=None):
        if ind < self.w.size:
            return self.w[ind] * self.component
        return np.float32(0.0) * self.component

    def Ricker(self, fdom):
        """Ricker wavelet of dominant frequency fdom, delayed by 1/fdom."""
        self.t = np.arange(-1.0 / fdom, 1.0 / fdom + self.dt / 3, self.dt)
        self.w = np.float32((1.0 - 2.0 * (np.pi * fdom * self.t) ** 2) * np.exp(-(np.pi * fdom * self.t) ** 2))

    def delta(self):
        """Unit spike."""
        self.w = np.float32(np.array([1]))


_PLAN = {"1": ["taux"], "2": ["vx", "vz"], "3": ["taux", "tauz", "tauxz"], "4": ["vx", "vz", "taux", "tauz", "tauxz"]}


def section_keys(components):
    """Output components of ``seismic_section`` for a components code."""
    return ["taux", "tauz"] if components == 0 else list(_PLAN[str(components)])


def seismic_section(seismo, components=0, shape="3d"):
    """Select components from (nt, nr, ns) traces; '2d' reshapes to
    (nt, nr*ns) with column s*nr + r (acquisition.py:313-333)."""
    data = {}
    if components != 0:
        for p in _PLAN[str(components)]:
            data[p] = seismo[p]
    else:
        data["taux"] = (seismo["taux"] + seismo["tauz"]) / 2
        data["tauz"] = (seismo["taux"] + seismo["tauz"]) / 2
    if shape == "2d":
        (nt, nr, ns) = data[[*data][0]].shape
        for p in data:
            data[p] = np.reshape(data[p], (nt, nr * ns), "F")
    return data
