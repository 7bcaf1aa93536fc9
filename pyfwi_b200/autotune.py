"""Step-kernel autotuner.

The library has several variants of the forward step and of the fused
adjoint+imaging step (``pyfwi_tile_count``): tile kernels with 16, 8 or 32
rows per tile, TMA-fed streaming kernels 128, 64 or 256 columns wide, and
16-row tile kernels whose adjoint CTAs carry 2 or 4 shots each (summing
their imaging in shared memory; their forward step is the first variant's),
tile kernels whose forward tile is staged by TMA box copies (their
adjoint is the cp.async tile kernel's), and the tile kernel whose adjoint
prefetches the tile's gradient accumulators into shared memory.
Which one is fastest depends on the grid, the number of shots per launch and
the absorbing layer, so ``tune`` times each on a short record of the survey at
hand and picks the fastest forward and the fastest adjoint variant
independently (``pyfwi_options.tile`` and ``adj_tile``).

Timing uses the library's own per-step CUDA events (``pyfwi_profile_*``) on a
plan of ``steps`` time steps and as many shots per launch as the survey's
plan will run (up to ``max_shots``).
Results are kept per process, keyed by device, half order, padded grid,
shots per launch and energy accumulation; set ``PYFWI_B200_TUNE_CACHE`` to a
JSON file path to keep them across processes.

The reference has one kernel shape (an OpenCL NDRange over the grid,
wave_propagation.py:625-856) and no tuner."""
import ctypes
import json
import os

import numpy as np
import torch

from . import _native as N
from .engine import Plan

_CACHE = {}


def _key(device, geom, shots, energy):
    name = torch.cuda.get_device_name(device)
    tnz, tnx = geom.nz + 2 * geom.npml, geom.nx + 2 * geom.npml
    return "%s|R%d|%dx%d|s%d|e%d" % (name, geom.half_order, tnz, tnx, shots, int(bool(energy)))


def _file_cache():
    path = os.environ.get("PYFWI_B200_TUNE_CACHE")
    if not path or not os.path.exists(path):
        return path, {}
    try:
        with open(path) as f:
            return path, json.load(f)
    except (OSError, ValueError):
        return path, {}


def _short_geometry(geom, steps, shots):
    g = N.Geometry.from_buffer_copy(geom)
    g.nt = int(steps)
    g.nt_ext = -(-int(steps) // int(geom.dt_scale))
    g.ns = int(shots)
    return g


def time_variant(geom, srcx, srcz, energy, shots, variant, device, steps=16):
    """(forward ms, adjoint ms) per launch of `variant` for `shots` shots
    per launch, measured on the second of two runs."""
    g = _short_geometry(geom, steps, shots)
    o = N.Options()
    o.checkpoint, o.segment, o.snapshot = N.CKPT_EXACT, 0, N.SNAP_FP32
    o.shot_batch, o.energy, o.tile = int(shots), int(bool(energy)), int(variant)
    P = Plan(g, np.asarray(srcx[:shots], np.int32), np.asarray(srcz[:shots], np.int32), o, device)
    tnz, tnx = g.nz + 2 * g.npml, g.nx + 2 * g.npml
    f = lambda v: torch.full((g.nz, g.nx), v, dtype=torch.float32, device=P.device)
    damp_x = torch.zeros(tnx, dtype=torch.float32)
    damp_z = torch.zeros(tnz, dtype=torch.float32)
    P.set_model(f(3000.0), f(1700.0), f(2200.0), damp_x, damp_z)
    src = np.zeros((g.nt_ext * int(g.dt_scale), 4), np.float32)
    src[0] = (0.0, 0.0, 1.0, 1.0)
    res = [torch.zeros((g.nt_ext, shots * g.nr), dtype=torch.float32, device=P.device) for _ in range(5)]
    P.profile(True)
    out = None
    for _ in range(2):
        P.forward(src)
        P.gradient(res, N.PARAM_LMD)
        P.check_device()
        nf, msf, _ = P.profile_read(0)
        na, msa, _ = P.profile_read(1)
        P.profile_read(2)
        out = (msf / max(nf, 1), msa / max(na, 1))
    P.profile(False)
    del P
    return out


def tune(geom, srcx, srcz, energy, shots_per_launch, device, steps=16, max_shots=64, variants=None):
    """(forward variant, adjoint variant, table) for plans of `geom` running
    `shots_per_launch` shots per launch.  table: {variant: (fwd ms, adj ms)}
    per launch of min(shots_per_launch, max_shots) shots (fewer if the short
    plans would not fit in a quarter of the free device memory)."""
    device = torch.device(device)
    tnz, tnx = geom.nz + 2 * geom.npml, geom.nx + 2 * geom.npml
    state = 5 * 4 * (tnz + 16) * (-(-(tnx + 16) // 32) * 32)
    free, _ = torch.cuda.mem_get_info(device)
    fit = max(1, int(0.25 * free) // ((steps + 6) * state))
    shots = int(max(1, min(shots_per_launch, max_shots, len(srcx), fit)))
    key = _key(device, geom, shots, energy)
    if key in _CACHE:
        return _CACHE[key]
    path, disk = _file_cache()
    if key in disk:
        v = disk[key]
        _CACHE[key] = (int(v[0]), int(v[1]), {int(k): tuple(t) for k, t in v[2].items()})
        return _CACHE[key]
    if variants is None:
        variants = range(N.lib().pyfwi_tile_count(int(geom.half_order)))
    table = {}
    for v in variants:
        table[int(v)] = time_variant(geom, srcx, srcz, energy, shots, v, device, steps)
    torch.cuda.empty_cache()
    fwd = min(table, key=lambda v: table[v][0])
    adj = min(table, key=lambda v: table[v][1])
    _CACHE[key] = (fwd, adj, table)
    if path:
        disk[key] = [fwd, adj, {str(k): list(t) for k, t in table.items()}]
        d = os.path.dirname(os.path.abspath(path))
        os.makedirs(d, exist_ok=True)
        tmp = path + ".tmp%d" % os.getpid()
        with open(tmp, "w") as f:
            json.dump(disk, f)
        os.replace(tmp, path)
    return _CACHE[key]
