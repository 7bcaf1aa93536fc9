"""Seeded survey cases shared by the golden-fixture script and the tests.

Each case is a dict: ``inpa`` (the reference's input-parameter dict),
``src_loc`` / ``rec_loc`` (metres, columns x then z), ``fdom``, ``src_type``,
``components``, ``chpr``, ``n_well_rec``, ``param`` ('dv' or 'lmd') and two
models ``model_obs`` / ``model_est`` of (nz, nx) float32 arrays.

``c1`` is the 100 x 100, 4-shot, 500-step survey with a circular anomaly; the
``tiny_*`` cases each exercise one corner of the reference's behaviour
(8th order, sub-stepped time, reverse-time reconstruction, crosswell and
two-well geometries, receiver spacing, directional sources, damping layouts).
"""
import numpy as np


def _t_for(nt, dt):
    # the reference takes nt = int(1 + t // dt); half a step of margin keeps
    # the float floor from dropping the last step
    return (nt - 1) * dt + dt / 2


def circle_model(nz, nx, vp, vs, rho, centre, radius, pert):
    """Homogeneous model plus a disc (cells with (z-zc)^2 + (x-xc)^2 < r^2)
    scaled by (1 + pert)."""
    zz, xx = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
    disc = (zz - centre[0]) ** 2 + (xx - centre[1]) ** 2 < radius ** 2
    m = {"vp": np.full((nz, nx), vp, np.float32), "vs": np.full((nz, nx), vs, np.float32),
         "rho": np.full((nz, nx), rho, np.float32)}
    for k in m:
        m[k][disc] *= np.float32(1 + pert)
    return m


def layered_model(nz, nx, seed, vp_lo=1500.0, vp_hi=2000.0, ratio=1.8):
    """Smooth random layered model: vp rises with depth plus a seeded bump."""
    rng = np.random.default_rng(seed)
    z = np.linspace(0, 1, nz)[:, None]
    x = np.linspace(0, 1, nx)[None, :]
    vp = vp_lo + (vp_hi - vp_lo) * z + 0 * x
    cz, cx, r = rng.uniform(0.3, 0.7), rng.uniform(0.3, 0.7), rng.uniform(0.1, 0.2)
    vp = vp * (1 + 0.05 * np.exp(-((z - cz) ** 2 + (x - cx) ** 2) / r ** 2))
    vp = vp.astype(np.float32)
    vs = (vp / ratio).astype(np.float32)
    rho = (310 * vp ** 0.25).astype(np.float32)
    return {"vp": vp, "vs": vs, "rho": rho}


def perturbed(model, seed, amp=0.05):
    rng = np.random.default_rng(seed)
    nz, nx = model["vp"].shape
    bump = np.zeros((nz, nx), np.float32)
    cz, cx = rng.integers(nz // 3, 2 * nz // 3), rng.integers(nx // 3, 2 * nx // 3)
    zz, xx = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
    bump[(zz - cz) ** 2 + (xx - cx) ** 2 < (min(nz, nx) // 5) ** 2] = amp
    return {k: (v * (1 + bump)).astype(np.float32) for k, v in model.items()}


def c1():
    """100 x 100 cells, dh = 1 m, 20-cell absorbing layer; vp = 2500, vs =
    vp / 1.73, rho = 2000 plus a radius-15 disc at +10 % for the observed
    data; four explosive 60 Hz Ricker shots and 100 receivers at z = 2 cells;
    dt = 0.2 ms, nt = 500; vx and vz recorded; every step checkpointed."""
    nz = nx = 100
    dh, dt = 1.0, 0.0002
    inpa = {"dt": dt, "t": _t_for(500, dt), "dh": dh, "npml": 20, "pmlR": 1e-5, "pml_dir": 2, "sdo": 4,
            "rec_dis": dh, "acq_type": 1}
    ns = 4
    src_loc = np.zeros((ns, 2), np.float32)
    src_loc[:, 0] = ((np.arange(ns) + 0.5) * nx / ns).astype(np.int32) * dh
    src_loc[:, 1] = 2 * dh
    rec_loc = np.zeros((nx, 2), np.float32)
    rec_loc[:, 0] = np.arange(nx) * dh
    rec_loc[:, 1] = 2 * dh
    vp = 2500.0
    bg = circle_model(nz, nx, vp, vp / 1.73, 2000.0, (50, 50), 15, 0.0)
    obs = circle_model(nz, nx, vp, vp / 1.73, 2000.0, (50, 50), 15, 0.10)
    return dict(name="c1", inpa=inpa, src_loc=src_loc, rec_loc=rec_loc, fdom=60.0, src_type=0, components=2,
                chpr=100, n_well_rec=0, param="dv", model_obs=obs, model_est=bg)


def _surface(nz, nx, dh, ns, rec_depth, src_depth, rec_step=1, rec_first=0, rec_last=None, src_x=None):
    rec_last = nx if rec_last is None else rec_last
    xs = np.arange(rec_first, rec_last, rec_step)
    rec_loc = np.stack([xs * dh, np.full(xs.size, rec_depth * dh)], 1).astype(np.float32)
    src_loc = np.zeros((ns, 2), np.float32)
    src_loc[:, 0] = (np.linspace(4, nx - 5, ns).astype(np.int32) if src_x is None else np.asarray(src_x)) * dh
    src_loc[:, 1] = src_depth * dh
    return src_loc, rec_loc


def tiny_s8():
    """8th-order stencil, all five components, energy-balanced 'lmd' gradient."""
    nz, nx, dh, dt = 30, 40, 2.0, 0.0004
    inpa = {"dt": dt, "t": _t_for(150, dt), "dh": dh, "npml": 6, "pmlR": 1e-5, "pml_dir": 2, "sdo": 8,
            "rec_dis": dh, "acq_type": 1, "energy_balancing": True}
    src_loc, rec_loc = _surface(nz, nx, dh, 2, rec_depth=3, src_depth=4, src_x=[10, 28])
    est = layered_model(nz, nx, 1)
    return dict(name="tiny_s8", inpa=inpa, src_loc=src_loc, rec_loc=rec_loc, fdom=80.0, src_type=0,
                components=4, chpr=100, n_well_rec=0, param="lmd", model_obs=perturbed(est, 2), model_est=est)


def tiny_dtscale():
    """dt = 1.1 ms: the propagator splits each sample into two steps."""
    nz, nx, dh, dt = 32, 36, 2.0, 0.0011
    inpa = {"dt": dt, "t": 0.13, "dh": dh, "npml": 5, "pmlR": 1e-5, "pml_dir": 2, "rec_dis": dh,
            "acq_type": 1}
    src_loc, rec_loc = _surface(nz, nx, dh, 2, rec_depth=2, src_depth=3, rec_first=1, rec_last=nx - 1)
    est = layered_model(nz, nx, 3, 1400.0, 1900.0)
    return dict(name="tiny_dtscale", inpa=inpa, src_loc=src_loc, rec_loc=rec_loc, fdom=40.0, src_type=0,
                components=0, chpr=100, n_well_rec=0, param="dv", model_obs=perturbed(est, 4), model_est=est)


def tiny_chpr():
    """10 % checkpoints: the backward pass reconstructs the rest in reverse time."""
    nz, nx, dh, dt = 28, 34, 2.0, 0.0004
    inpa = {"dt": dt, "t": _t_for(140, dt), "dh": dh, "npml": 5, "pmlR": 1e-5, "pml_dir": 3, "rec_dis": dh,
            "acq_type": 1}
    src_loc, rec_loc = _surface(nz, nx, dh, 3, rec_depth=2, src_depth=2)
    est = layered_model(nz, nx, 5)
    return dict(name="tiny_chpr", inpa=inpa, src_loc=src_loc, rec_loc=rec_loc, fdom=70.0, src_type=0,
                components=3, chpr=10, n_well_rec=0, param="dv", model_obs=perturbed(est, 6), model_est=est)


def tiny_crosswell():
    """Crosswell geometry (receivers down a column), no x damping, chpr = 0."""
    nz, nx, dh, dt = 36, 30, 2.0, 0.0004
    inpa = {"dt": dt, "t": _t_for(130, dt), "dh": dh, "npml": 5, "pmlR": 1e-5, "pml_dir": 0, "rec_dis": dh,
            "acq_type": 0, "sdo": 4}
    zs = np.arange(3, nz - 3)
    rec_loc = np.stack([np.full(zs.size, (nx - 4) * dh), zs * dh], 1).astype(np.float32)
    src_loc = np.array([[4 * dh, 10 * dh], [4 * dh, 24 * dh]], np.float32)
    est = layered_model(nz, nx, 7)
    return dict(name="tiny_crosswell", inpa=inpa, src_loc=src_loc, rec_loc=rec_loc, fdom=70.0, src_type=0,
                components=1, chpr=0, n_well_rec=0, param="dv", model_obs=perturbed(est, 8), model_est=est)


def tiny_dxr():
    """Receivers every second cell up to the right edge, no z damping, a
    directional (vx) source."""
    nz, nx, dh, dt = 30, 38, 2.0, 0.0004
    inpa = {"dt": dt, "t": _t_for(140, dt), "dh": dh, "npml": 4, "pmlR": 1e-5, "pml_dir": 1,
            "rec_dis": 2 * dh, "acq_type": 1}
    src_loc, rec_loc = _surface(nz, nx, dh, 2, rec_depth=3, src_depth=5, rec_step=2, rec_first=1)
    est = layered_model(nz, nx, 9)
    return dict(name="tiny_dxr", inpa=inpa, src_loc=src_loc, rec_loc=rec_loc, fdom=70.0, src_type=1,
                components=2, chpr=100, n_well_rec=0, param="dv", model_obs=perturbed(est, 10), model_est=est)


def tiny_both():
    """Surface line plus two wells (acq_type 2), all components."""
    nz, nx, dh, dt = 30, 34, 2.0, 0.0004
    inpa = {"dt": dt, "t": _t_for(120, dt), "dh": dh, "npml": 5, "pmlR": 1e-5, "pml_dir": 2, "rec_dis": dh,
            "acq_type": 2, "sdo": 4}
    # layout of acquisition.acq_parameters(acq_type=2): left well, surface line, right well
    zs = np.arange(4, nz - 4)
    left = np.stack([np.full(zs.size, 3 * dh), zs * dh], 1)
    xs = np.arange(4, nx - 4)
    surf = np.stack([xs * dh, np.full(xs.size, 3 * dh)], 1)
    right = np.stack([np.full(zs.size, (nx - 4) * dh), zs * dh], 1)
    rec_loc = np.vstack([left, surf, right]).astype(np.float32)
    src_loc = np.array([[12 * dh, 4 * dh], [22 * dh, 4 * dh]], np.float32)
    est = layered_model(nz, nx, 11)
    return dict(name="tiny_both", inpa=inpa, src_loc=src_loc, rec_loc=rec_loc, fdom=70.0, src_type=0,
                components=4, chpr=100, n_well_rec=int(zs.size), param="dv", model_obs=perturbed(est, 12),
                model_est=est)


def tiny_water():
    """A 6-cell water layer (vs = 0) over a layered solid, as in marine
    surveys: sources and receivers in the water, pressure recorded, 'dv'
    gradient."""
    nz, nx, dh, dt = 32, 40, 2.0, 0.0004
    inpa = {"dt": dt, "t": _t_for(150, dt), "dh": dh, "npml": 5, "pmlR": 1e-5, "pml_dir": 2, "sdo": 4,
            "rec_dis": dh, "acq_type": 1}
    src_loc, rec_loc = _surface(nz, nx, dh, 2, rec_depth=2, src_depth=3, src_x=[12, 27])
    est = layered_model(nz, nx, 13)
    obs = perturbed(est, 14)
    for m in (est, obs):
        m["vp"][:6] = 1500.0
        m["vs"][:6] = 0.0
        m["rho"][:6] = 1000.0
    return dict(name="tiny_water", inpa=inpa, src_loc=src_loc, rec_loc=rec_loc, fdom=70.0, src_type=0,
                components=0, chpr=100, n_well_rec=0, param="dv", model_obs=obs, model_est=est)


TINY = [tiny_s8, tiny_dtscale, tiny_chpr, tiny_crosswell, tiny_dxr, tiny_both, tiny_water]
ALL = [c1] + TINY  # cases with golden fixtures


def by_name(name):
    f = globals().get(name)
    if f is None or not callable(f) or not (name.startswith("c") or name.startswith("tiny_")):
        raise KeyError(name)
    return f()


def c2():
    """200 x 400 cells, dh = 5 m, 20-cell layer; two layers (vp 2000 / 3000,
    vs = vp / 1.8, Gardner rho = 310 vp^0.25) plus a Gaussian-smoothed random
    perturbation (3 % std, 10-cell correlation, seeded); 10 Ricker shots at
    10 Hz, 400 receivers, dt = 0.5 ms, nt = 2000; taux/tauz recorded."""
    from scipy.ndimage import gaussian_filter
    nz, nx, dh, dt = 200, 400, 5.0, 0.0005
    inpa = {"dt": dt, "t": _t_for(2000, dt), "dh": dh, "npml": 20, "pmlR": 1e-5, "pml_dir": 2, "sdo": 4,
            "rec_dis": dh, "acq_type": 1}
    vp = np.where(np.arange(nz)[:, None] < nz // 2, 2000.0, 3000.0) + 0 * np.arange(nx)[None, :]
    rng = np.random.default_rng(2024)
    pert = gaussian_filter(rng.standard_normal((nz, nx)), 10.0)
    pert *= 0.03 / pert.std()
    vp_obs = (vp * (1 + pert)).astype(np.float32)
    vp_est = gaussian_filter(vp, 5.0).astype(np.float32)

    def mk(v):
        return {"vp": v, "vs": (v / 1.8).astype(np.float32), "rho": (310 * v ** 0.25).astype(np.float32)}

    ns = 10
    src_loc = np.stack([np.linspace(20, nx - 21, ns).astype(np.int32) * dh, np.full(ns, 2 * dh)], 1).astype(np.float32)
    rec_loc = np.stack([np.arange(nx) * dh, np.full(nx, 2 * dh)], 1).astype(np.float32)
    return dict(name="c2", inpa=inpa, src_loc=src_loc, rec_loc=rec_loc, fdom=10.0, src_type=0, components=0,
                chpr=100, n_well_rec=0, param="dv", model_obs=mk(vp_obs), model_est=mk(vp_est))


def c3(ns=64):
    """500 x 1000 cells, dh = 5 m, 30-cell layer; vp rising 1800 -> 4000 m/s
    with depth, three dipping interfaces and a seeded lens (vs = vp / 1.8,
    Gardner rho); 64 shots at 8 Hz on a 15-cell pitch, 1000 receivers,
    dt = 0.5 ms, nt = 4000; every step available to the adjoint."""
    nz, nx, dh, dt = 500, 1000, 5.0, 0.0005
    inpa = {"dt": dt, "t": _t_for(4000, dt), "dh": dh, "npml": 30, "pmlR": 1e-5, "pml_dir": 2, "sdo": 4,
            "rec_dis": dh, "acq_type": 1}
    z = np.arange(nz)[:, None].astype(np.float64)
    x = np.arange(nx)[None, :].astype(np.float64)
    vp = 1800.0 + 2000.0 * z / (nz - 1) + 0 * x
    for k, (z0, slope, jump) in enumerate([(120, 0.08, 120.0), (260, -0.05, 150.0), (380, 0.03, -100.0)]):
        vp = vp + jump * (z > z0 + slope * (x - nx / 2))
    rng = np.random.default_rng(33)
    cz, cx = rng.uniform(180, 320), rng.uniform(350, 650)
    a, b = rng.uniform(30, 50), rng.uniform(80, 140)
    lens = ((z - cz) / a) ** 2 + ((x - cx) / b) ** 2 < 1
    vp = np.where(lens, vp * 0.92, vp)
    vp = np.clip(vp, 1800.0, 4000.0).astype(np.float32)
    model = {"vp": vp, "vs": (vp / 1.8).astype(np.float32), "rho": (310 * vp ** 0.25).astype(np.float32)}
    src_loc = np.stack([(20 + 15 * np.arange(ns)) * dh, np.full(ns, 2 * dh)], 1).astype(np.float32)
    rec_loc = np.stack([np.arange(nx) * dh, np.full(nx, 2 * dh)], 1).astype(np.float32)
    smooth = {k: v.copy() for k, v in model.items()}
    from scipy.ndimage import gaussian_filter
    smooth["vp"] = gaussian_filter(vp, 8.0).astype(np.float32)
    smooth["vs"] = (smooth["vp"] / 1.8).astype(np.float32)
    smooth["rho"] = (310 * smooth["vp"] ** 0.25).astype(np.float32)
    return dict(name="c3", inpa=inpa, src_loc=src_loc, rec_loc=rec_loc, fdom=8.0, src_type=0, components=0,
                chpr=100, n_well_rec=0, param="dv", model_obs=model, model_est=smooth)


def c4(n_models=32, seed=44):
    """The uneven batch: n_models seeded surveys, each a layered model (vp
    1500 -> 4500 m/s with depth, 2-4 dipping layers) with one anomaly (+-8 %
    disc), vs = vp / 1.8, Gardner rho; grid nz in [128, 512], nx in [128,
    1024], dh in [2, 10] m, 20-cell layer; dt = 0.5 dh / max(vp) (CFL 0.5;
    above 0.6 ms the propagator sub-steps); nt in [1000, 5000]; 4-16
    explosive shots at 2 cells depth and a receiver in every column at 2
    cells; f0 = min(vs) / (16 dh) clipped to [5, 30] Hz (at least 8 cells per
    wavelength at twice f0); vx and vz recorded, every step checkpointed.
    The estimate is the model smoothed (8-cell Gaussian)."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n_models):
        nz, nx = int(rng.integers(128, 513)), int(rng.integers(128, 1025))
        dh = float(rng.uniform(2.0, 10.0))
        z = np.arange(nz)[:, None] / (nz - 1)
        x = np.arange(nx)[None, :] / (nx - 1)
        vp = 1500.0 + 2200.0 * z + 0 * x
        for _ in range(int(rng.integers(2, 5))):
            z0, slope, jump = rng.uniform(0.15, 0.85), rng.uniform(-0.2, 0.2), rng.uniform(-150, 250)
            vp = vp + jump * (z > z0 + slope * (x - 0.5))
        cz, cx, r = rng.uniform(0.3, 0.7), rng.uniform(0.2, 0.8), rng.uniform(0.05, 0.15)
        disc = ((z - cz) * nz) ** 2 + ((x - cx) * nx) ** 2 < (r * min(nz, nx)) ** 2
        vp = np.clip(np.where(disc, vp * (1 + rng.choice([-0.08, 0.08])), vp), 1500.0, 4500.0).astype(np.float32)
        model = {"vp": vp, "vs": (vp / 1.8).astype(np.float32), "rho": (310 * vp ** 0.25).astype(np.float32)}
        est = {"vp": gaussian_filter(vp, 8.0).astype(np.float32)}
        est["vs"] = (est["vp"] / 1.8).astype(np.float32)
        est["rho"] = (310 * est["vp"] ** 0.25).astype(np.float32)
        dt = float(np.float32(0.5 * dh / float(vp.max())))
        nt = int(rng.integers(1000, 5001))
        ns = int(rng.integers(4, 17))
        f0 = float(np.clip(float(model["vs"].min()) / (16 * dh), 5.0, 30.0))
        inpa = {"dt": dt, "t": _t_for(nt, dt), "dh": dh, "npml": 20, "pmlR": 1e-5, "pml_dir": 2, "sdo": 4,
                "rec_dis": dh, "acq_type": 1}
        src_loc, rec_loc = _surface(nz, nx, dh, ns, rec_depth=2, src_depth=2)
        out.append(dict(name="c4_%02d" % q, inpa=inpa, src_loc=src_loc, rec_loc=rec_loc, fdom=f0, src_type=0,
                        components=2, chpr=100, n_well_rec=0, param="dv", model_obs=model, model_est=est))
    return out


def c5(ns=128, seed=55):
    """The thrust-belt survey: 1000 x 3000 cells, dh = 4 m, 40-cell layer;
    folded layers (vp 1500 -> 4500 m/s with depth, sinusoidal folds and two
    thrust offsets), vs = vp / 1.75 except a 40-cell water layer (vp 1500,
    vs 0, rho 1000), Gardner rho; ns explosive 6 Hz shots and 2000
    receivers (every 1.5 cells) at 2 cells depth in the water; dt = 0.4 ms,
    nt = 6000; pressure recorded.  The estimate is the model smoothed
    (20-cell Gaussian, water kept); ``model_mon`` is the model with vp -8 %
    in a 40 x 200-cell reservoir patch (the time-lapse monitor)."""
    from scipy.ndimage import gaussian_filter
    nz, nx, dh, dt = 1000, 3000, 4.0, 0.0004
    rng = np.random.default_rng(seed)
    z = np.arange(nz)[:, None].astype(np.float64)
    x = np.arange(nx)[None, :].astype(np.float64)
    fold = 60.0 * np.sin(2 * np.pi * x / rng.uniform(900, 1400)) * np.exp(-((z - 500) / 400) ** 2)
    depth = z + fold + 80.0 * (x > rng.uniform(900, 1300)) + 60.0 * (x > rng.uniform(1900, 2300))
    vp = 1800.0 + 2700.0 * np.clip((depth - 40) / (nz - 40), 0, 1)
    vp = vp + 150.0 * np.sign(np.sin(depth / rng.uniform(60, 90)))
    vp = np.clip(vp, 1500.0, 4500.0)
    vp[:40] = 1500.0
    vp = vp.astype(np.float32)
    vs = (vp / 1.75).astype(np.float32)
    vs[:40] = 0.0
    rho = (310 * vp ** 0.25).astype(np.float32)
    rho[:40] = 1000.0
    model = {"vp": vp, "vs": vs, "rho": rho}
    est = {"vp": gaussian_filter(vp, 20.0).astype(np.float32)}
    est["vp"][:40] = 1500.0
    est["vs"] = (est["vp"] / 1.75).astype(np.float32)
    est["vs"][:40] = 0.0
    est["rho"] = (310 * est["vp"] ** 0.25).astype(np.float32)
    est["rho"][:40] = 1000.0
    mon = {k: v.copy() for k, v in model.items()}
    mon["vp"][600:640, 1400:1600] *= np.float32(0.92)
    inpa = {"dt": dt, "t": _t_for(6000, dt), "dh": dh, "npml": 40, "pmlR": 1e-5, "pml_dir": 2, "sdo": 4,
            "rec_dis": 1.5 * dh, "acq_type": 1}
    src_loc = np.stack([np.linspace(40, nx - 41, ns).astype(np.int32) * dh, np.full(ns, 2 * dh)],
                       1).astype(np.float32)
    rec_loc = np.stack([np.arange(2000) * 1.5 * dh, np.full(2000, 2 * dh)], 1).astype(np.float32)
    return dict(name="c5", inpa=inpa, src_loc=src_loc, rec_loc=rec_loc, fdom=6.0, src_type=0, components=0,
                chpr=100, n_well_rec=0, param="dv", model_obs=model, model_est=est, model_mon=mon)


def fwi_lbfgs():
    """The inversion driver on tiny_dxr: FWI(...)(m0, 'lbfgs', iter=[2, 2],
    freqs=[60, 0], n_params=1, k_0=1, k_end=4), i.e. vp, then vs, then rho,
    two L-BFGS iterations each, first on data low-passed at 60 Hz, then on
    the full band."""
    case = tiny_dxr()
    case["name"] = "fwi_lbfgs"
    case["fwi"] = dict(method="lbfgs", iter=[2, 2], freqs=[60, 0], n_params=1, k_0=1, k_end=4)
    return case


def fwi_cg():
    """fwi_lbfgs with the conjugate-gradient method, inverting for the model
    in units of 2000 (m/s, kg/m^3) through PyFWI's param_functions (the
    model passed in and returned scaled, model_to_dv multiplying by 2000,
    grad_from_dv the gradient by 2000).  In physical units fmin_cg's first
    trial step (at most 1) moves this model by less than its float32
    rounding and the run takes no step; scaled, it moves a few m/s."""
    case = fwi_lbfgs()
    case["name"] = "fwi_cg"
    case["fwi"]["method"] = "cg"
    case["fwi"]["param_scale"] = 2000.0
    return case


def timelapse(method):
    """Time-lapse inversion on tiny_dxr: baseline = the case's observed
    model, monitor = baseline with vp -8 % in a 6 x 8-cell patch (a depleted
    reservoir), start = the case's estimate; TimeLapse(...)(m0, iter=[1],
    freqs=[60], tl_method=method, n_params=1, k_0=1, k_end=3): vp, then vs."""
    case = tiny_dxr()
    case["name"] = "tl_" + method
    mon = {k: v.copy() for k, v in case["model_obs"].items()}
    mon["vp"][14:20, 15:23] *= np.float32(0.92)
    case["model_mon"] = mon
    case["tl"] = dict(tl_method=method, iter=[1], freqs=[60], n_params=1, k_0=1, k_end=3)
    return case


TL_METHODS = ["pa", "cc", "dd", "sim", "wa", "cj", "cd", "cu"]


def _cut_record(case, nt):
    """The case with its record cut to nt trace samples (same dt)."""
    case = dict(case)
    case["inpa"] = dict(case["inpa"], t=_t_for(nt, case["inpa"]["dt"]))
    return case


def c2_parity():
    """The 200 x 400 survey exactly as configured (10 shots, nt = 2000):
    its fixture holds the reference's gradient on the whole survey."""
    case = c2()
    case["name"] = "c2_parity"
    return case


def c3_parity(nt=1200, shots=(20, 45)):
    """The 560 x 1060 padded grid of the 64-shot survey, two of its shots
    (x = 320 and 695 cells), the record cut to nt samples.  The product runs
    it with the 64-shot layout of the full survey: the two shots repeated 32
    times, all 64 in one launch, 157-step recompute segments."""
    case = c3(ns=64)
    case = _cut_record(case, nt)
    case["src_loc"] = case["src_loc"][list(shots)].copy()
    case["name"] = "c3_parity"
    return case


def c4_parity(n_samples=400, n_shots=2):
    """The largest sub-stepped model of the uneven batch (c4_08: 397 x 987
    cells, dh 9.26 m, dt 1.30 ms split into three internal steps), its first
    and last shots, the record cut to n_samples samples."""
    case = c4()[8]
    case = _cut_record(case, n_samples)
    idx = [0, len(case["src_loc"]) - 1][:n_shots]
    case["src_loc"] = case["src_loc"][idx].copy()
    case["name"] = "c4_parity"
    return case


def c5_parity(nz=300, nx=800, nt=1200):
    """The thrust-belt survey cropped to its top-left nz x nx cells (40-cell
    water layer with vs = 0 included, same 40-cell absorbing layer, dh, dt,
    6 Hz wavelet and receiver spacing), two shots, the record cut to nt
    samples."""
    case = c5(ns=128)
    case = _cut_record(case, nt)
    for key in ("model_obs", "model_est", "model_mon"):
        case[key] = {k: np.ascontiguousarray(v[:nz, :nx]) for k, v in case[key].items()}
    rec = case["rec_loc"]
    case["rec_loc"] = rec[rec[:, 0] < (nx - 1) * case["inpa"]["dh"]].copy()
    dh = case["inpa"]["dh"]
    case["src_loc"] = np.array([[200 * dh, 2 * dh], [560 * dh, 2 * dh]], np.float32)
    case["name"] = "c5_parity"
    return case


LARGE = [c2_parity, c3_parity, c4_parity, c5_parity]  # reference fixtures at the configured sizes
