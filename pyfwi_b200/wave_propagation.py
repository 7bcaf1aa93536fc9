"""Drop-in ``WavePropagator`` for PyFWI's elastic propagator
(src/PyFWI/wave_propagation.py).

Same constructor, ``forward_modeling`` and ``gradient`` as the reference and
the same set-up attributes (nt, nt_ext, dt, dt_scale, tnz, tnx, chp, srcx,
srcz, dxr, rec_* constants, dx_pml, dz_pml ...).  The per-step OpenCL loop
of the reference is replaced by one call into libpyfwi_b200.so per
``forward_modeling`` / ``gradient``; the checkpoints live in device memory.

Inputs may be numpy arrays (outputs are then numpy, as in the reference) or
torch tensors (outputs stay on the device).

Extra ``inpa`` keys (all optional): ``checkpoint`` ('exact' or 'reverse';
default: 'exact' when chpr == 100, else the reference's reverse-time scheme),
``segment`` (steps per recompute segment), ``shot_batch``, ``tile`` (step
kernel variant, 0..11 -- tile kernels of 16 / 8 / 32 rows, streaming kernels
of 128 / 64 / 256 columns, 16-row tile kernels whose adjoint CTAs carry 2 / 4
shots, tile kernels of 16 / 8 / 32 rows whose forward tile is staged by TMA
box copies, the 16-row tile kernels whose adjoint prefetches its gradient
accumulators -- or 'auto' to time them all on this survey first and
take the fastest forward and adjoint variant), ``adj_tile`` (adjoint step
variant when it differs from ``tile``), ``chunk`` (rows per CTA of the
streaming variants), ``graph`` (replay whole calls as CUDA graphs: True,
False, or 'auto', the default: on where a launch carries at most 8 M
cell-shots, where issuing launches from the host would cost a noticeable
share, and a call issues at most GRAPH_MAX_LAUNCHES launches; the library
runs longer calls directly either way), ``persist`` (run the time loops as persistent cooperative kernels,
many steps per launch with a grid barrier between steps, where the layout
stores every step in FP32 and the tile kernels run: True, False (the
default), or 'auto': on where a step carries at most 2 M cell-shots),
``overlap`` (exact checkpoints in FP32 with recompute segments: recompute
segment m - 1 on a second CUDA stream while the adjoint of segment m runs,
with two segment buffers), ``store`` ('differences', the default: in exact
mode with FP32 snapshots, the reference adjoint without energy terms and the
tile kernels 0..2, the forward steps that fill the checkpoint segments store
the five differences of each state that the imaging reads, and the adjoint
step reads them instead of differencing the state; 'states': store the
states),
``snapshot`` ('fp32'; 'bf16': the forward states the imaging reads are
stored in BF16 while the forward recurrence stays FP32, halving their memory
and their reads at the cost of rounding the imaged fields to 8 mantissa bits;
'fp24': the same with a byte plane widening BF16 to 15 mantissa bits, three
quarters of the FP32 store),
``adjoint`` ('reference': PyFWI's gradient, masked and normalised as
gradient_reading does; 'exact': the exact derivative of
J = 1/2 sum (section - observed)^2 of this library's discrete forward step on
the whole model grid, with ``res`` read as dJ/d(section), the absorbing
profiles held fixed; needs checkpoint 'exact'),
``cuda_device`` (torch device string).
"""
import warnings

import numpy as np
import torch

from . import _native as N
from . import acquisition as acq
from . import fwi_tools as tools
from .engine import Plan, mean2, smooth
from .processing import COMPONENTS

FIELDS = COMPONENTS
# step kernel variant when inpa has no 'tile': the 16-row tile kernels, or
# the 8-row ones for surveys of at most SMALL_SURVEY_CELLS cell-shots per step
# (twice the CTAs per step where a step is a few microseconds of latency:
# measured on B200, 100 x 100 + 20-cell layer, 4 shots: 8.1 against 11.9 ms
# per evaluation; 200 x 400 + 20, 10 shots: 108 against 113 ms)
DEFAULT_TILE, SMALL_TILE, SMALL_SURVEY_CELLS = 0, 1, 8_000_000
# inpa['overlap'] when absent: recompute segment m - 1 on a second stream
# beside the adjoint of segment m
OVERLAP_DEFAULT = False
# inpa['store'] when absent
STORE_DEFAULT = "differences"


def _slice_bounds(start, stop, n):
    """[lo, hi) of python slice(start, stop) on length n (empty -> (0, 0))."""
    lo, hi, _ = slice(int(start), int(stop)).indices(int(n))
    return (lo, hi) if hi > lo else (0, 0)


class WavePreparation:
    """Set-up of a survey (wave_propagation.py:16-246): time-step split, grid
    padding, index constants, checkpoint schedule and damping arrays, then a
    device plan for them."""

    def __init__(self, inpa, src, rec_loc, model_shape, components=0, n_well_rec=0, chpr=10):
        keys = [*inpa]
        # time axis (wave_propagation.py:28-35)
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
        # checkpoint schedule (wave_propagation.py:95-100)
        nchp = int(chpr * self.nt / 100)
        self.chp = np.linspace(0, self.nt - 1, nchp, dtype=np.int32)
        if len(self.chp) < 2:
            self.chp = np.array([1, self.nt - 1])
        self.nchp = len(self.chp)
        self.chpr = chpr
        self.rec_loc = rec_loc
        self.nr = rec_loc.shape[0]
        self.n_well_rec = n_well_rec
        self.n_surface_rec = self.nr - 2 * n_well_rec
        if n_well_rec == 0 and self.acq_type == 2:
            raise Exception(" Number of geophons in the wells is not defined")
        # receiver index constants (wave_propagation.py:116-144)
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
        else:
            raise ValueError("acq_type must be 0, 1 or 2")
        self.dx_pml, self.dz_pml = tools.pml_counstruction(self.tnz, self.tnx, self.dh, self.npml, pmlR, pml_dir)
        self.D = tools.Fdm(order=self.sdo * 2)
        self.components = components
        self.inpa = dict(inpa)
        self.device = torch.device(inpa.get("cuda_device", "cuda"))
        self._wavelet = self._source_values()
        self._plan = None  # built on first use (device memory is sized then)
        self._traces = None
        # cap in bytes on the device memory the layout may plan for (None:
        # what is free when the plan is built); SurveyBatch shares memory out
        self.memory_budget = None
        # False keeps the time loops one launch per step whatever
        # inpa['persist'] says (SurveyBatch runs surveys side by side, where
        # cooperative grids would compete for the SMs)
        self.persist_allowed = True

    @property
    def plan(self):
        if self._plan is None:
            self._build_plan(self.inpa)
        return self._plan

    @property
    def tile(self):
        """Forward step kernel variant of the plan (builds it)."""
        self.plan  # noqa: B018 (builds the plan)
        return self._tile

    @property
    def adj_tile(self):
        """Adjoint step kernel variant of the plan (builds it)."""
        self.plan  # noqa: B018 (builds the plan)
        return self._adj_tile

    # ---- geometry for the native plan --------------------------------------
    def _lines(self):
        """Receiver lines equivalent to the reference's receiver work items
        (elastic_surface.cl:30-39, elastic_crosswell.cl:95-102,
        elastic.cl:65-96): cell positions follow the reference's flat index
        (a column past the last one continues on the next row)."""
        tnz, tnx, dxr, nr = int(self.tnz), int(self.tnx), int(self.dxr), int(self.nr)
        if dxr < 1:
            raise ValueError("receiver spacing rec_dis / dh must be at least 1 cell")
        groups = []  # (slot0, [(row, col)], vz_from_vx)

        def row_group(row, col0, n_main, slot0):
            cells = []
            if 0 <= row < tnz:
                for j in range(0, tnx, dxr):
                    ir = j // dxr
                    if ir >= n_main:
                        break
                    flat = row * tnx + j + col0
                    cells.append(divmod(flat, tnx))
            return slot0, cells

        def col_group(col, row0, limit, slot0, vzx):
            cells = []
            if 0 <= col < tnx:
                for i in range(0, tnz, dxr):
                    ir = i // dxr
                    if ir >= limit or slot0 + ir >= nr:
                        break
                    cells.append((i + row0, col))
            return slot0, cells, vzx

        if self.acq_type == 1:
            s0, cells = row_group(int(self.rec_surface_const), int(self.rec_surface_var), int(self.n_surface_rec), 0)
            groups.append((s0, cells, 0))
        elif self.acq_type == 0:
            groups.append(col_group(int(self.rec_top_right_const), int(self.rec_top_right_var), nr, 0, 1))
        else:
            nw, nm = int(self.n_well_rec), int(self.n_surface_rec)
            groups.append(col_group(int(self.rec_top_left_const), int(self.rec_top_left_var), nw, 0, 0))
            s0, cells = row_group(int(self.rec_surface_const), int(self.rec_surface_var), nm, nw)
            groups.append((s0, cells, 0))
            groups.append(col_group(int(self.rec_top_right_const), int(self.rec_top_right_var), nr, nw + nm, 0))
        lines = []
        for slot0, cells, vzx in groups:
            # cells outside the grid are read out of bounds by the reference; drop them
            keep = [(k, rc) for k, rc in enumerate(cells) if 0 <= rc[0] < tnz and 0 <= rc[1] < tnx]
            if not keep:
                continue
            if keep[0][0] != 0 or any(k != q for q, (k, _) in enumerate(keep)):
                raise NotImplementedError("receiver line leaves the grid in its middle")
            rows = {rc[0] for _, rc in keep}
            if len(keep) == 1:
                lines.append((keep[0][1][0], keep[0][1][1], 0, 1, 1, slot0, vzx))
            elif len(rows) == 1:
                step = keep[1][1][1] - keep[0][1][1]
                if step <= 0 or any(keep[q][1][1] - keep[q - 1][1][1] != step for q in range(1, len(keep))):
                    raise NotImplementedError("surface receiver line wraps to the next grid row")
                lines.append((keep[0][1][0], keep[0][1][1], 0, step, len(keep), slot0, vzx))
            else:
                step = keep[1][1][0] - keep[0][1][0]
                lines.append((keep[0][1][0], keep[0][1][1], step, 0, len(keep), slot0, vzx))
        if not lines:
            lines.append((0, 0, 0, 1, 0, 0, 0))
        return lines

    def _mask_window(self):
        sdo, nz, nx = int(self.sdo), int(self.nz), int(self.nx)
        cts = int(self.src_cts)
        if self.acq_type == 0:
            r = _slice_bounds(sdo, -sdo, nz)
            c = _slice_bounds(sdo + cts + 2, -sdo, nx)
        else:
            r = _slice_bounds(sdo + cts + 2, -sdo, nz)
            c = _slice_bounds(sdo, -sdo, nx)
        return r + c

    def _geometry(self):
        g = N.Geometry()
        g.nz, g.nx, g.npml = int(self.nz), int(self.nx), int(self.npml)
        g.half_order = int(self.sdo)
        g.nt, g.nt_ext, g.dt_scale = int(self.nt), int(self.nt_ext), int(self.dt_scale)
        # the reference bakes dt, dh and c1..c4 into its kernels through "%f"
        # (wave_propagation.py:434-490)
        r6 = lambda x: float("%f" % x)
        g.dt = r6(self.dt)
        g.dh = r6(self.dh)
        for q, c in enumerate((self.D.c1, self.D.c2, self.D.c3, self.D.c4)):
            g.c[q] = r6(c)
        g.ns, g.nr = int(self.ns), int(self.nr)
        lines = self._lines()
        g.n_lines = len(lines)
        for q, (r0, c0, dr, dc, cnt, s0, vzx) in enumerate(lines):
            g.lines[q] = N.RecLine(r0, c0, dr, dc, cnt, s0, vzx)
        g.mask_row0, g.mask_row1, g.mask_col0, g.mask_col1 = self._mask_window()
        return g

    def _source_values(self):
        """(vx, vz, taux, tauz) amplitudes for each injection
        (wave_propagation.py:652-664)."""
        n_inj = int(np.ceil(self.nt / self.dt_scale))
        vals = np.zeros((n_inj, 4), np.float32)
        for k in range(n_inj):
            vals[k] = np.float32(self.src(k))[:4]
        return vals

    def _build_plan(self, inpa):
        exact_default = self.chpr == 100 or inpa.get("adjoint") == "exact"
        mode = inpa.get("checkpoint", "exact" if exact_default else "reverse")
        if mode not in ("exact", "reverse"):
            raise ValueError("inpa['checkpoint'] must be 'exact' or 'reverse'")
        self.checkpoint = mode
        geom = self._geometry()
        srcx = np.asarray(self.srcx, np.int32).reshape(-1)
        srcz = np.asarray(self.srcz, np.int32).reshape(-1)
        chp = np.asarray(self.chp, np.int32) if mode == "reverse" else None

        def opts(seg, batch):
            o = N.Options()
            o.checkpoint = N.CKPT_EXACT if mode == "exact" else N.CKPT_REVERSE
            o.segment = int(seg)
            o.snapshot = snapshot
            o.shot_batch = int(batch)
            # the exact gradient is not preconditioned: no energy terms
            o.energy = 1 if self.energy_balancing and self.adjoint != "exact" else 0
            o.tile, o.adj_tile = variants
            o.adjoint = N.ADJOINT_EXACT if self.adjoint == "exact" else N.ADJOINT_REFERENCE
            o.graph = int(self._graph_on(inpa.get("graph", "auto"), batch, seg))
            o.persist = int(self._persist_on(inpa.get("persist", False), batch))
            o.overlap = int(bool(inpa.get("overlap", OVERLAP_DEFAULT)))
            o.store_diffs = int(store == "differences")
            o.chunk = int(inpa.get("chunk", 0))
            if chp is not None:
                o.nchp = int(chp.size)
                o.chp = chp.ctypes.data_as(N.ctypes.POINTER(N.ctypes.c_int32))
            return o

        self.adjoint = inpa.get("adjoint", "reference")
        if self.adjoint not in ("reference", "exact"):
            raise ValueError("inpa['adjoint'] must be 'reference' or 'exact'")
        if self.adjoint == "exact" and mode != "exact":
            raise ValueError("inpa['adjoint'] = 'exact' needs checkpoint 'exact'")
        store = inpa.get("store", STORE_DEFAULT)
        if store not in ("differences", "states"):
            raise ValueError("inpa['store'] must be 'differences' or 'states'")
        snap = inpa.get("snapshot", "fp32")
        if snap not in ("fp32", "bf16", "fp24") or (snap != "fp32" and mode != "exact"):
            raise ValueError("inpa['snapshot'] must be 'fp32', 'bf16' or 'fp24' (the last two with checkpoint "
                             "'exact' only)")
        snapshot = {"fp32": N.SNAP_FP32, "bf16": N.SNAP_BF16, "fp24": N.SNAP_FP24}[snap]
        self.snapshot = snap
        small = int(self.tnz) * int(self.tnx) * int(self.ns) <= SMALL_SURVEY_CELLS
        tile = inpa.get("tile", SMALL_TILE if small else DEFAULT_TILE)
        adj_tile = inpa.get("adj_tile", None)
        variants = (0 if tile == "auto" else int(tile), 0 if adj_tile is None else int(adj_tile) + 1)
        seg = int(inpa.get("segment", 0))
        batch = int(inpa.get("shot_batch", 0))
        if mode == "exact" and ("segment" not in inpa or "shot_batch" not in inpa):
            seg, batch = self._auto_layout(geom, opts, seg, batch)
        if tile == "auto":
            from .autotune import tune
            fwd, adj, _ = tune(geom, srcx, srcz, self.energy_balancing, batch or int(self.ns), self.device)
            variants = (fwd, adj + 1)
        self._plan = Plan(geom, srcx, srcz, opts(seg, batch), self.device, chp=chp)
        self.segment, self.shot_batch = seg, batch
        self._tile, self._adj_tile = variants[0], (variants[1] - 1 if variants[1] else variants[0])

    # 'auto' replays captured graphs where a launch carries at most this many
    # cell-shots: there a step kernel runs for tens of microseconds or less and
    # issuing it from the host costs a noticeable share (measured on B200:
    # 100 x 100 + 20-cell layer, 4 shots: 1.9x; 200 x 400 + 20, 10 shots:
    # 1.08x); above it the kernels hide the issue cost and the copies into
    # the captured buffers are pure overhead
    GRAPH_AUTO_CELLS = 8_000_000
    # and where a gradient call issues at most this many launches (the
    # library's PYFWI_GRAPH_MAX_LAUNCHES: it runs longer calls directly)
    GRAPH_MAX_LAUNCHES = 600_000

    # 'auto' runs the time loops as persistent kernels (many steps per
    # cooperative launch, a grid barrier between steps) where a step carries
    # at most this many cell-shots.  Off by default: measured on B200 the
    # grid barrier costs more than the launches it saves (100 x 100 + 20,
    # 4 shots: 12.4 ms per evaluation persistent, 11.9 one launch per step,
    # 8.1 with 8-row tiles and graph replay; 200 x 400 + 20, 10 shots: 126
    # against 113 ms), because a step of a small grid is a few microseconds
    # of latency that a barrier does not shorten
    PERSIST_AUTO_CELLS = 2_000_000

    def _persist_on(self, persist, batch):
        if not self.persist_allowed:
            return False
        if persist == "auto":
            b = int(batch) if batch else int(self.ns)
            return int(self.tnz) * int(self.tnx) * b <= self.PERSIST_AUTO_CELLS
        if persist not in (True, False, 0, 1):
            raise ValueError("inpa['persist'] must be True, False or 'auto'")
        return bool(persist)

    def _graph_on(self, graph, batch, seg=0):
        if graph == "auto":
            b = int(batch) if batch else int(self.ns)
            nt, s = int(self.nt), int(seg) if seg and int(seg) < int(self.nt) else int(self.nt)
            m = -(-nt // s)
            launches = -(-int(self.ns) // b) * (2 * nt + (m - 1) * s + m + 16)
            return int(self.tnz) * int(self.tnx) * b <= self.GRAPH_AUTO_CELLS and launches <= self.GRAPH_MAX_LAUNCHES
        if graph not in (True, False, 0, 1):
            raise ValueError("inpa['graph'] must be True, False or 'auto'")
        return bool(graph)

    # Layout cost model, in units of one forward step of one cell of one shot:
    # an adjoint+imaging step costs about 1.9 of them; a forward step has a
    # fixed cost of about 4.6e5 and an adjoint step about 2.3e6 (B200, fitted
    # to 3 and 64 shots on 593,600 cells: forward 6 us + 7.7 us per shot,
    # adjoint 30 us + 14.4 us per shot).
    COST_ADJ, COST_FWD_STEP, COST_ADJ_STEP = 1.9, 4.6e5, 2.3e6

    def _auto_layout(self, geom, opts, seg, batch):
        """Shot batch and recompute segment of the exact checkpoint mode.

        Among the layouts whose workspace fits in free device memory, the one
        with the least modelled time for a misfit_gradient call: per group of
        b shots, nt forward steps plus (M - 1) * segment recomputed forward
        steps (M = ceil(nt / segment)) and nt adjoint steps, each step costing
        its cells x shots plus a fixed cost per step.  Storing every step of a
        few shots beats recomputing a large batch only where the grid is large
        enough to fill the GPU with a few shots."""
        free, _ = torch.cuda.mem_get_info(self.device)
        # blocks torch's caching allocator holds but does not use count as
        # free: it releases them when an allocation would otherwise fail
        free += torch.cuda.memory_reserved(self.device) - torch.cuda.memory_allocated(self.device)
        if self.memory_budget is not None:
            free = min(free, int(self.memory_budget / 0.9))
        traces = 5 * self.nt_ext * int(self.ns) * int(self.nr) * 4
        budget = int(0.9 * free) - 4 * traces - (256 << 20)
        nt, ns = int(self.nt), int(self.ns)
        cells = float(int(self.tnz) * int(self.tnx))
        memo = {}

        def fits(s, b):
            if (s, b) not in memo:
                memo[s, b] = Plan.workspace_bytes(geom, opts(s, b), ns) <= budget
            return memo[s, b]

        def largest_segment(b):
            if seg:
                return seg if fits(seg, b) else None
            if fits(nt, b):
                return nt
            # the store holds ceil(nt / s) + s states: growing for s >= sqrt(nt)
            lo = int(np.ceil(np.sqrt(nt)))
            if not fits(lo, b):
                return None
            hi = nt
            while hi - lo > 1:
                mid = (lo + hi) // 2
                lo, hi = (mid, hi) if fits(mid, b) else (lo, mid)
            # the same number of segments, evened out: fewer recomputed steps
            # ((M - 1) * s) in a smaller store
            return -(-nt // (-(-nt // lo)))

        def group_cost(s, b):
            m = -(-nt // s)
            fwd = nt + (m - 1) * s
            return fwd * (b * cells + self.COST_FWD_STEP) + nt * (b * cells * self.COST_ADJ + self.COST_ADJ_STEP)

        best = None
        for b in ([batch] if batch else range(ns, 0, -1)):
            s = largest_segment(b)
            if s is None:
                continue
            cost = (ns // b) * group_cost(s, b) + (group_cost(s, ns % b) if ns % b else 0.0)
            if best is None or cost < best[0]:
                best = (cost, s, b)
        if best is None:
            raise MemoryError("the survey does not fit in device memory (%.1f GB free)" % (free / 2 ** 30))
        return best[1], best[2]

    # ---- helpers ---------------------------------------------------------
    def _to_device(self, x):
        if isinstance(x, torch.Tensor):
            return x.to(self.device, torch.float32)
        return torch.from_numpy(np.ascontiguousarray(x, np.float32)).to(self.device, non_blocking=False)


class WavePropagator(WavePreparation):
    """Forward modelling and adjoint-state gradient (wave_propagation.py:594-938).

    Parameters as the reference: ``inpa`` dict, ``src`` (acquisition.Source
    with a wavelet), ``rec_loc`` (nr, 2) in metres, ``model_shape``,
    ``components`` (0: (taux+tauz)/2, 1: taux, 2: vx vz, 3: stresses, 4: all),
    ``n_well_rec``, ``chpr`` (checkpoint percentage)."""

    def __init__(self, inpa, src, rec_loc, model_shape, components=0, n_well_rec=0, chpr=0):
        WavePreparation.__init__(self, inpa=inpa, src=src, rec_loc=rec_loc, model_shape=model_shape,
                                 components=components, n_well_rec=n_well_rec, chpr=chpr)

    # ------------------------------------------------------------------
    def forward_modeling(self, model0, show=False):
        """Seismic section of the model dict {'vp', 'vs', 'rho'} ((nz, nx)
        arrays or tensors) in the shape set by inpa['seimogram_shape']."""
        if show:
            warnings.warn("show=True: live wavefield plotting is not available; ignored")
        as_numpy = not isinstance(model0["vp"], torch.Tensor)
        vp, vs, rho = (self._to_device(model0[k]) for k in ("vp", "vs", "rho"))
        self.plan.set_model(vp, vs, rho, *self._damping())
        self._traces = self.plan.forward(self._wavelet, self._traces)
        self._model_dev = tuple(t.clone() for t in (vp, vs, rho))  # for W: the caller may edit its tensors
        self._W, self._W_from_plan = None, self.checkpoint == "reverse"
        data = self._section(self._traces)
        self._check_device(as_numpy)
        if as_numpy:
            data = {k: v.cpu().numpy() for k, v in data.items()}
        return data

    def _damping(self):
        """The damping profiles per column and per row (the reference's 2-D
        dx_pml / dz_pml are separable), on the device, uploaded once."""
        if getattr(self, "_damp_dev", None) is None:
            self._damp_dev = tuple(torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(self.device)
                                   for a in (self.dx_pml[0, :], self.dz_pml[:, 0]))
        return self._damp_dev

    def _check_device(self, synchronous):
        """Raise if a streaming or persistent kernel stopped early.  Reading
        the error word synchronises, so it is done where the call synchronises
        anyway (host results) or where such a kernel may have run, never
        inside a CUDA-graph capture."""
        if torch.cuda.is_current_stream_capturing():
            return
        o = self.plan.opts
        if synchronous or 3 <= o.tile <= 5 or 4 <= o.adj_tile <= 6 or o.persist:
            self.plan.check_device()

    def _section(self, traces):
        """acquisition.seismic_section on device traces [5][nt_ext][ns*nr]."""
        nt, ns, nr = int(self.nt_ext), int(self.ns), int(self.nr)
        tr = traces
        if self.acq_type == 2 and self.n_well_rec:
            # wave_propagation.py:647-649: the left-well traces come out in reverse order
            nw = int(self.n_well_rec)
            idx = torch.arange(ns * nr, device=self.device).view(ns, nr)
            idx[:, :nw] = idx[:, :nw].flip(1)
            tr = traces.index_select(2, idx.reshape(-1))
        comp = {k: tr[q] for q, k in enumerate(FIELDS)}
        if self.components == 0:
            m = mean2(comp["taux"], comp["tauz"])
            data = {"taux": m, "tauz": mean2(comp["taux"], comp["tauz"])}
        else:
            data = {k: comp[k] for k in acq.section_keys(self.components)}
        if self.seismo_shape == "2d":
            return data
        return {k: v.view(nt, ns, nr).permute(0, 2, 1) for k, v in data.items()}

    @property
    def W(self):
        """The forward wavefields at the checkpoint steps ``chp``, as the
        reference keeps them (wave_propagation.py:150-156, filled at
        :710-727): {'vx', 'vz', 'taux', 'tauz', 'tauxz'}, each a float32
        array (tnz, tnx, ns, nchp) whose [:, :, s, k] is the state of shot s
        after internal step chp[k] of the last model run forward.  The
        reference copies them to the host on every forward run; here they are
        built on first access and kept until the next run: read from the
        plan's checkpoint store after forward_modeling in reverse mode, else
        from a forward run of a reverse-mode plan with the same checkpoint
        steps.  Zeros before any forward run, as in the reference."""
        if getattr(self, "_W", None) is not None:
            return self._W
        shape = (int(self.tnz), int(self.tnx), int(self.ns), int(self.nchp))
        if getattr(self, "_model_dev", None) is None:
            return {k: np.zeros(shape, np.float32) for k in FIELDS}
        if self._W_from_plan:
            states = self.plan.checkpoint_states()
        else:
            o = N.Options()
            o.checkpoint = N.CKPT_REVERSE
            o.tile, o.chunk = self.plan.opts.tile, self.plan.opts.chunk
            try:
                plan = Plan(self._geometry(), np.asarray(self.srcx, np.int32).reshape(-1),
                            np.asarray(self.srcz, np.int32).reshape(-1), o, self.device,
                            chp=np.asarray(self.chp, np.int32))
            except torch.cuda.OutOfMemoryError as e:
                raise MemoryError("W holds %d states of %d x %d cells per shot and field; they do not fit in "
                                  "device memory" % (int(self.nchp), int(self.tnz), int(self.tnx))) from e
            plan.set_model(*self._model_dev, *self._damping())
            plan.forward(self._wavelet)
            states = plan.checkpoint_states()
            del plan
        host = states.cpu().numpy()  # [ns, nchp, 5, tnz, tnx]
        del states
        self._W = {k: np.ascontiguousarray(host[:, :, q].transpose(2, 3, 0, 1)) for q, k in enumerate(FIELDS)}
        return self._W

    @property
    def seismogram(self):
        """Raw receiver traces of the last forward call, (nt_ext, nr, ns) per
        component (host copies)."""
        if self._traces is None:
            return None
        nt, ns, nr = int(self.nt_ext), int(self.ns), int(self.nr)
        return {k: self._traces[q].view(nt, ns, nr).permute(0, 2, 1).cpu().numpy() for q, k in enumerate(FIELDS)}

    # ------------------------------------------------------------------
    def gradient(self, res, show=False, parameterization="dv"):
        """Gradient of the misfit whose adjoint source is ``res`` (a dict of
        (nt_ext, nr*ns) arrays or tensors; missing components are zero).
        Returns {'vp','vs','rho'} ('dv') or {'lam','mu','rho'}."""
        if show:
            warnings.warn("show=True: live wavefield plotting is not available; ignored")
        as_numpy = not isinstance(res[[*res][0]], torch.Tensor)
        nt, nrs = int(self.nt_ext), int(self.nr) * int(self.ns)
        planes = []
        for k in FIELDS:
            if k not in res:
                planes.append(None)
                continue
            r = res[k]
            if r.ndim == 3:  # (nt, nr, ns) -> (nt, ns*nr)
                r = (np.transpose(r, (0, 2, 1)) if isinstance(r, np.ndarray) else r.permute(0, 2, 1))
            r = self._to_device(r).reshape(nt, nrs).contiguous()
            planes.append(r)
        if self.adjoint == "exact":
            planes = self._trace_adjoint(planes)
        param = N.PARAM_DV if parameterization == "dv" else N.PARAM_LMD
        g = self.plan.gradient(planes, param)
        if float(self.g_smooth) > 1e-15:  # gaussian_filter(., g_smooth) per parameter (:923-936)
            g = smooth(g, self.g_smooth)
        names = ("vp", "vs", "rho") if parameterization == "dv" else ("lam", "mu", "rho")
        out = {n: g[q] for q, n in enumerate(names)}
        self._check_device(as_numpy)
        if as_numpy:
            out = {k: v.cpu().numpy() for k, v in out.items()}
        return out

    def misfit_gradient(self, model0, d_obs, parameterization="dv"):
        """The misfit and gradient that FWI.fprime evaluates (fwi.py:229-252:
        forward_modeling, CostFunction('l2') on the section, gradient), in
        one library call that runs each shot group's forward pass, residual
        and adjoint in turn (pyfwi_misfit_gradient), so a layout of several
        shot groups models every group once.  d_obs: the observed section
        (the dict forward_modeling returns, '2d' or '3d', numpy or torch).
        Returns (rms, gradient dict); rms is a float for numpy input, else a
        0-d float64 device tensor."""
        if self.acq_type == 2 and self.n_well_rec:  # the section reorders traces: separate calls
            d_est = self.forward_modeling(model0)
            rms, res = tools.CostFunction("l2")(d_est, d_obs)
            return rms, self.gradient(res, parameterization=parameterization)
        as_numpy = not isinstance(model0["vp"], torch.Tensor)
        vp, vs, rho = (self._to_device(model0[k]) for k in ("vp", "vs", "rho"))
        self.plan.set_model(vp, vs, rho, *self._damping())
        self._model_dev = tuple(t.clone() for t in (vp, vs, rho))  # for W: the caller may edit its tensors
        self._W, self._W_from_plan = None, False
        nt, nrs = int(self.nt_ext), int(self.nr) * int(self.ns)
        obs = [None] * 5
        for k, v in d_obs.items():
            f = FIELDS.index(k)
            if v.ndim == 3:  # (nt, nr, ns) -> (nt, ns*nr)
                v = (np.transpose(v, (0, 2, 1)) if isinstance(v, np.ndarray) else v.permute(0, 2, 1))
            obs[f] = self._to_device(v).reshape(nt, nrs).contiguous()
        mean_stress = self.components == 0
        adj = [None] * 5
        for f in range(5):
            if obs[f] is not None or (mean_stress and f in (2, 3) and (obs[2] is not None or obs[3] is not None)):
                adj[f] = torch.empty((nt, nrs), dtype=torch.float32, device=self.device)
        param = N.PARAM_DV if parameterization == "dv" else N.PARAM_LMD
        g, rms, self._traces = self.plan.misfit_gradient(self._wavelet, obs, mean_stress, adj, param, self._traces)
        self._adjoint_source = {FIELDS[f]: adj[f] for f in range(5) if adj[f] is not None}
        if float(self.g_smooth) > 1e-15:
            g = smooth(g, self.g_smooth)
        names = ("vp", "vs", "rho") if parameterization == "dv" else ("lam", "mu", "rho")
        out = {n: g[q] for q, n in enumerate(names)}
        self._check_device(as_numpy)
        if as_numpy:
            return float(rms.item()), {k: v.cpu().numpy() for k, v in out.items()}
        return rms, out

    def _trace_adjoint(self, planes):
        """Exact adjoint: the section's dJ/d(section) per key -> dJ/d(raw
        trace) per field.  components 0 records (taux + tauz) / 2 under both
        keys, so each raw stress trace gets half the sum; acquisition 2 lists
        the left-well traces in reverse, a permutation undone here."""
        P = list(planes)
        if self.components == 0 and (P[2] is not None or P[3] is not None):
            tx = P[2] if P[2] is not None else torch.zeros_like(P[3])
            tz = P[3] if P[3] is not None else torch.zeros_like(P[2])
            P[2] = P[3] = mean2(tx, tz)
        if self.acq_type == 2 and self.n_well_rec:
            ns, nr, nw = int(self.ns), int(self.nr), int(self.n_well_rec)
            idx = torch.arange(ns * nr, device=self.device).view(ns, nr)
            idx[:, :nw] = idx[:, :nw].flip(1)
            P = [None if p is None else p.index_select(1, idx.reshape(-1)).contiguous() for p in P]
        return P

    def raw_gradient(self, res):
        """The six (tnz, tnx) accumulators (Gmu, Glam, Grho and the energy
        terms) before masking, for inspection and tests."""
        planes = [None if k not in res else self._to_device(res[k]).contiguous() for k in FIELDS]
        raw = torch.zeros((6, int(self.tnz), int(self.tnx)), dtype=torch.float32, device=self.device)
        self.plan.gradient(planes, N.PARAM_LMD, raw=raw)
        self._check_device(True)
        return raw
