"""Benchmark: FWI gradient evaluations of the 500 x 1000-cell, 64-shot,
4000-step elastic survey on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one misfit-and-gradient evaluation of all shots: forward
modelling, L2 residual against the observed data, adjoint-state gradient.  Throughput is
grid-cell updates per second: padded cells x internal time steps x shots,
counted once for the forward and once for the adjoint pass.

With N GPUs every rank evaluates its own 64-shot survey (weak scaling,
independent replicas: the propagator runs on one GPU and nothing is
exchanged on the data path); the step time is the maximum over ranks.
Rank 0 prints one JSON line.

--impl reference times the reference's own kernels (PyFWI's elastic.cl /
elastic_surface.cl compiled for the host CPU; oracle/ref_driver.py) in the
reference's loop order on a bounded sample of the same survey, with every
host thread.
"""
import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

METRIC = "FWI grad Gcell-updates/s & %HBM roofline, batched vs plain per-shot, grad err≤1e-4"
UNIT = "Gcell-updates/s"
WORKLOAD = "elastic FWI gradient, 500x1000 cells (+30-cell absorbing layer), 64 shots, 1000 receivers, nt=4000"

# algorithmic bytes per cell and shot-step (one FP32 read or write = 4 B)
BYTES_FWD = 52.0         # read vx vz txx tzz txz lam mu b, write 5 fields
BYTES_ADJ = 52.0         # adjoint propagation: same count
# imaging, per imaged cell: read 5 values of the forward state or of its
# difference set (4, 3 or 2 B each: FP32, 24-bit, BF16), read and write 3
# gradients (24 B); the forward steps that fill difference sets write 5
# values per imaged cell once per shot-step


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in self.rows for q in range(4) if r[3 + q].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm)}


def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


THRUST_BELT = ("elastic FWI gradient, thrust-belt survey: 1000x3000 cells (+40-cell absorbing layer, 40-cell "
               "water layer), %d of its 128 shots, 2000 receivers, nt=6000")


def survey(ns, nt=None, config="c3"):
    """The 500 x 1000-cell survey (config 'c3') or the 1000 x 3000 thrust-belt
    survey ('c5') with ns shots; nt shortens the record (small profiling
    cases only)."""
    import cases
    case = cases.c3(ns=ns) if config == "c3" else cases.c5(ns=ns)
    if nt:
        dt = case["inpa"]["dt"]
        case["inpa"]["t"] = (nt - 1) * dt + dt / 2
    return case


# --------------------------------------------------------------------------
# the reference arm and the CPU baseline
# --------------------------------------------------------------------------
def cpu_sample(case, seconds=15.0, max_steps=4000, detail=None):
    """Time the reference's kernels (or the oracle port when they are not
    built) on one shot over the first n steps, forward + backward; n is sized
    for about `seconds` of work.  Returns (Gcell-updates/s, kind, threads,
    description); `detail` (a dict), when given, receives the timed sample's
    seconds, steps and cell-updates."""
    import oracle as O
    import ref_driver
    inpa = case["inpa"]
    src = O.Ricker(case["src_loc"], inpa["dh"], inpa["dt"], case["src_type"])
    src.Ricker(case["fdom"])
    W = O.OracleWavePropagator(inpa, src, case["rec_loc"], case["model_est"]["vp"].shape,
                               components=case["components"], chpr=0)
    W._materials(case["model_est"])
    cells = int(W.tnz) * int(W.tnx)
    threads = len(os.sched_getaffinity(0))
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    if ref_driver.available(case["name"]):
        R = ref_driver.RefRunner(case["name"], W)
        probe = 16
        t = R.run_shot(0, probe)
        n = int(min(max_steps, int(W.nt), max(probe, seconds / (t / probe))))
        t = R.run_shot(0, n)
        kind = "reference"
        desc = ("PyFWI elastic.cl/elastic_surface.cl compiled for the host (OpenMP, %d threads), reference loop "
                "order, 1 shot x first %d of %d steps, forward + backward, every step stored" % (threads, n, W.nt))
    else:
        import ctypes
        L = O.lib("fp32")
        probe = 16

        def run(n):
            cfg = O.OrcCfg.from_buffer_copy(W.cfg)
            cfg.nt = n
            seis = np.zeros((5, W.nt_ext, W.nr), np.float32)
            store = np.zeros((n, 5, cells), np.float32)
            chp = np.arange(n, dtype=np.int32)
            G = [np.zeros(cells, np.float32) for _ in range(6)]
            res = (ctypes.c_void_p * 5)()
            t0 = time.perf_counter()
            L.orc_forward_shot(ctypes.byref(cfg), *W._mats(), int(W.srcx[0]), int(W.srcz[0]), O._ptr(W.src_vals),
                               W.n_inj, O._ptr(seis), O._ptr(store), O._ptr(chp), n)
            L.orc_gradient_shot(ctypes.byref(cfg), *W._mats(), res, O._ptr(store), O._ptr(chp), n,
                                *[O._ptr(g) for g in G])
            return time.perf_counter() - t0

        t = run(probe)
        n = int(min(max_steps, int(W.nt), max(probe, seconds / (t / probe))))
        t = run(n)
        kind = "port"
        desc = ("oracle restatement (C, OpenMP, %d threads), 1 shot x first %d of %d steps, forward + backward"
                % (threads, n, W.nt))
    if detail is not None:
        detail.update(seconds=t, steps=n, shots=1, cell_updates=2.0 * cells * n)
    return 2.0 * cells * n / t / 1e9, kind, threads, desc


def run_reference(args, world, rank):
    case = survey(1)
    if rank != 0:
        return
    for _ in range(args.warmup):
        cpu_sample(case, seconds=args.cpu_seconds / 3)
    vals, samples = [], []
    for _ in range(args.steps):
        detail = {}
        v, kind, cores, desc = cpu_sample(case, seconds=args.cpu_seconds, detail=detail)
        vals.append(v)
        samples.append(detail)
    value = statistics.median(vals)
    # cell-updates of one step of the workload (all shots, whole record,
    # forward + adjoint), from the survey itself
    full = survey(64)
    nz, nx = full["model_est"]["vp"].shape
    npml = full["inpa"]["npml"]
    nt = int(1 + full["inpa"]["t"] // full["inpa"]["dt"])
    cells = 2.0 * (nz + 2 * npml) * (nx + 2 * npml) * nt * len(full["src_loc"])
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            # a whole step of the workload on the host would take hours: this
            # is the step time the measured rate implies, not a timed step
            "ms_per_step": cells / (value * 1e9) * 1e3, "extrapolated": True,
            "timed_samples": samples,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample": desc, "cell_updates_per_step": cells},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------
def max_over_ranks(ms, world, dev):
    """The slowest rank's time: each rank's device-timed milliseconds, MAX
    over the process group (the only collective the bench issues)."""
    if world == 1:
        return float(ms)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def roofline(prof, ms, ncell, nint, ns, nt, steps, store, snapshot, hbm, peak_src, traffic_dir):
    """The roofline object of the JSON line from the profiled step kernels.

    prof[k] = (launches, device ms, cell-shots) of kernel kind k (0 forward,
    1 adjoint + imaging, 2 reverse) over the timed steps, ms the timed
    region.  Algorithmic bytes per cell-shot: BYTES_FWD / BYTES_ADJ, plus per
    imaged cell (nint per shot-step) 5 imaged values at their stored width
    and 3 gradients read and written; with difference sets the forward steps
    also write every shot-step's five values once.  traffic: the ncu DRAM
    bytes per cell-shot of a one-pass capture of the benchmark's launch shape
    (traffic_dir/traffic_<kernel>_c3[_differences].json, matching store and
    snapshot format), times this run's average launch; None without one."""
    # bytes per value of what the imaging reads: FP32 states or difference
    # sets, 24-bit (BF16 + byte) or BF16 snapshots
    vb = {"fp32": 4.0, "fp24": 3.0, "bf16": 2.0}[snapshot]
    q_bytes = 5 * vb * nint * int(ns) * int(nt) * steps if store == "differences" else 0.0
    names = {0: "fwd_step", 1: "adj_step", 2: "rev_step"}

    def kernel_roof(k):
        n_l, ms_k, cells_k = prof[k]
        if k == 1:
            alg = cells_k * BYTES_ADJ + (cells_k / ncell) * nint * (5 * vb + 24.0)
        else:
            alg = cells_k * BYTES_FWD + (q_bytes if k == 0 else 0.0)
        ach = alg / (ms_k * 1e-3) / 1e9 if ms_k > 0 else None
        return {"achieved": ach, "frac": ach / hbm if ach else None, "launches": n_l,
                "avg_launch_ms": ms_k / max(n_l, 1), "alg_bytes_per_launch": alg / max(n_l, 1)}

    def traffic_for(k):
        if traffic_dir is None:
            return None, None
        tp = os.path.join(traffic_dir, "traffic_%s_c3%s.json"
                          % (names[k], "_differences" if store == "differences" else ""))
        if not os.path.exists(tp):
            return None, None
        with open(tp) as f:
            tj = json.load(f)
        if tj.get("store", "states") != store or tj.get("snapshot", "fp32") != snapshot:
            return None, None
        return (tj["dram_bytes_per_cell_shot"] * prof[k][2] / max(prof[k][0], 1),
                {"ncu_capture": tj.get("capture"), "shots_per_launch": tj.get("shots_per_launch"),
                 "scaled_to": "cell-shots of this run's average launch"})

    per_kernel = {}
    for k in prof:
        if prof[k][0] > 0:
            per_kernel[names[k]] = kernel_roof(k)
            per_kernel[names[k]]["traffic"] = traffic_for(k)[0]
    dom = max(prof, key=lambda k: prof[k][1])  # dominant kernel: the most device time
    kr = per_kernel[names[dom]]
    traffic, traffic_src = traffic_for(dom)
    return {"bound": "hbm", "kernel": names[dom], "achieved": kr["achieved"], "peak": hbm, "unit": "GB/s",
            "frac": kr["frac"], "traffic": traffic, "traffic_source": traffic_src, "peak_source": peak_src,
            "launches": kr["launches"], "avg_launch_ms": kr["avg_launch_ms"],
            "alg_bytes_per_launch": kr["alg_bytes_per_launch"],
            "kernel_share": {names[k]: prof[k][1] / max(ms, 1e-9) for k in prof},
            "per_kernel": per_kernel}


def run_ours(args, world, rank, local):
    import torch
    import torch.distributed as dist
    from helpers import product

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    case = survey(args.shots, args.nt, args.config)
    extra = {"cuda_device": str(dev)}
    if args.segment:
        extra.update(segment=args.segment, shot_batch=args.shots)
    if args.tile is not None:
        extra["tile"] = args.tile if args.tile == "auto" else int(args.tile)
    if args.adj_tile is not None:
        extra["adj_tile"] = args.adj_tile
    if args.overlap is not None:
        extra["overlap"] = bool(args.overlap)
    if args.snapshot != "fp32":
        extra["snapshot"] = args.snapshot
    if args.store is not None:
        extra["store"] = args.store
    W = product(case, **extra)
    ncell = float(int(W.tnz) * int(W.tnx))
    nint = float((int(W.tnz) - 2 * (int(W.npml) + int(W.sdo)) + 1) * (int(W.tnx) - 2 * (int(W.npml) + int(W.sdo)) + 1))
    cell_updates = 2.0 * ncell * int(W.nt) * int(W.ns)  # forward + adjoint

    m_est = {k: torch.from_numpy(v).to(dev) for k, v in case["model_est"].items()}
    m_obs = {k: torch.from_numpy(v).to(dev) for k, v in case["model_obs"].items()}
    d_obs = {k: v.clone() for k, v in W.forward_modeling(m_obs).items()}

    def step(model, obs):
        # forward modelling, L2 misfit and gradient of every shot (FWI.fprime)
        rms, grad = W.misfit_gradient(model, obs, parameterization="dv")
        return torch.stack([grad["vp"], grad["vs"], grad["rho"]]), rms

    for _ in range(args.warmup):
        step(m_est, d_obs)
    torch.cuda.synchronize()

    sampler = ClockSampler(local) if rank == 0 else None
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
        time.sleep(0.3)
    W.plan.profile(True)
    launches0 = W.plan.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        g, rms = step(m_est, d_obs)
    e1.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches = W.plan.launches() - launches0
    clocks = sampler.stop() if sampler else None
    W.plan.profile(False)
    prof = {k: W.plan.profile_read(k) for k in (0, 1, 2)}
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, world, dev)
    value = world * cell_updates * args.steps / (ms_max * 1e-3) / 1e9

    # end to end through the public API from pinned host buffers
    host_model = {k: v.cpu().pin_memory() for k, v in m_est.items()}
    host_obs = {k: v.cpu().pin_memory() for k, v in d_obs.items()}
    h2d = sum(v.numel() * 4 for v in host_model.values()) + sum(v.numel() * 4 for v in host_obs.values())
    out_host = torch.empty((3, int(W.nz), int(W.nx)), dtype=torch.float32).pin_memory()
    rms_host = torch.empty((), dtype=torch.float64).pin_memory()
    d2h = out_host.numel() * 4 + 8
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record()
    for _ in range(args.steps):
        model = {k: v.to(dev, non_blocking=True) for k, v in host_model.items()}
        obs = {k: v.to(dev, non_blocking=True) for k, v in host_obs.items()}
        g, rms = step(model, obs)
        out_host.copy_(g, non_blocking=True)
        rms_host.copy_(rms, non_blocking=True)
    e3.record()
    torch.cuda.synchronize()
    e2e_value = world * cell_updates * args.steps / (max_over_ranks(e2.elapsed_time(e3), world, dev) * 1e-3) / 1e9

    if rank != 0:
        return
    misfit = float(rms.item())
    batched_shots_s = int(W.ns) * args.steps / (ms_max * 1e-3)
    shape = {"ns": int(W.ns), "nt": int(W.nt), "grid": [int(W.tnz), int(W.tnx)]}
    W_store_diffs, W_snapshot = W.plan.store_diffs, W.snapshot
    layout = {"checkpoint": W.checkpoint, "segment": W.segment, "shot_batch": W.shot_batch,
              "overlap": int(W.plan.opts.overlap), "snapshot": W.snapshot,
              "store": "differences" if W_store_diffs else "states",
              "kernels": {"forward": int(W.tile), "adjoint": int(W.adj_tile)}}
    plain = None
    if world == 1 and (args.plain_shots > 0 or args.inversion > 0 or args.uneven > 0 or args.configs):
        del step, W, d_obs, g, rms
        gc.collect()
        torch.cuda.empty_cache()
    if world == 1 and args.plain_shots > 0:
        plain = plain_form(args, dev, batched_shots_s)
    hbm, peak_src = peaks()
    roof = roofline(prof, ms, ncell, nint, shape["ns"], shape["nt"], args.steps,
                    "differences" if W_store_diffs else "states", W_snapshot, hbm, peak_src,
                    os.path.join(ROOT, "profiles") if args.config == "c3" else None)
    small = None
    if world == 1 and args.configs:
        gc.collect()
        torch.cuda.empty_cache()
        small = configs_run(args, dev)
    uneven = None
    if world == 1 and args.uneven > 0:
        gc.collect()
        torch.cuda.empty_cache()
        uneven = uneven_run(args, dev)
    inversion = None
    if world == 1 and args.inversion > 0:
        gc.collect()
        torch.cuda.empty_cache()
        inversion = {opt: inversion_run(args, case, dev, opt) for opt in args.optimizers.split(",")}
    cpu = None
    if world == 1 and not args.no_cpu:
        v, kind, cores, desc = cpu_sample(survey(1), seconds=args.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": desc}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD if args.config == "c3" else THRUST_BELT % shape["ns"],
                       "shots_per_gpu": shape["ns"], "nt": shape["nt"],
                       "grid": shape["grid"], **layout, "parallelism": "dp%d" % world,
                       "l2": "inputs larger than L2 (no flush)"},
            "roofline": roof, "cpu_baseline": cpu, "plain": plain,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches, "clocks": clocks,
            "misfit": misfit}
    if inversion:
        line["inversion"] = inversion
    if uneven:
        line["uneven_batch"] = uneven
    if small:
        line["configs"] = small
    print(json.dumps(line), flush=True)


def inversion_run(args, case, dev, optimizer):
    """`args.inversion` L-BFGS iterations of FWI on vp through the public
    driver (FWI.__call__, full band) with the optimiser on the device or
    SciPy's on the host: wall time per evaluation, and the wall time of the
    whole call outside the evaluations (the optimiser, the model and
    gradient vectors, the conversions at entry and exit)."""
    import torch
    from helpers import product
    from pyfwi_b200 import acquisition as acq
    from pyfwi_b200.fwi import FWI
    inpa = dict(case["inpa"], cuda_device=str(dev), optimizer=optimizer)
    src = acq.Source(case["src_loc"], inpa["dh"], inpa["dt"], case["src_type"])
    src.Ricker(case["fdom"])
    shape = case["model_est"]["vp"].shape
    kw = dict(components=case["components"], n_well_rec=case["n_well_rec"], chpr=case["chpr"])
    W = product(case, cuda_device=str(dev))
    d_obs = {k: v.clone() for k, v in W.forward_modeling(
        {k: torch.from_numpy(v).to(dev) for k, v in case["model_obs"].items()}).items()}
    del W
    gc.collect()
    F = FWI(d_obs, inpa, src, case["rec_loc"], shape, **kw)
    spent = [0.0, 0]
    inner = F.fprime

    def timed(m0, freq):
        t0 = time.perf_counter()
        out = inner(m0, freq)
        torch.cuda.synchronize()
        spent[0] += time.perf_counter() - t0
        spent[1] += 1
        return out
    F.fprime = timed
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    F({k: v.copy() for k, v in case["model_est"].items()}, "lbfgs", iter=[args.inversion], freqs=[0], n_params=1,
      k_0=1, k_end=2)
    total = time.perf_counter() - t0
    return {"iterations": args.inversion, "evaluations": spent[1], "s_per_evaluation": spent[0] / spent[1],
            "outside_evaluations_ms": (total - spent[0]) * 1e3, "parameters": int(np.prod(shape)),
            "layout": {"segment": F.segment, "shot_batch": F.shot_batch}}


def uneven_run(args, dev):
    """The uneven batch (`args.uneven` surveys of cases.c4): one misfit and
    gradient evaluation of every survey, (1) one survey after another, (2)
    together on per-survey streams (SurveyBatch), (3) as one CUDA graph
    (SurveyBatch(graph=True)), (4) one after another with plans that replay
    their own captured graphs (inpa['graph']); device time and
    Gcell-updates/s of each, after one untimed evaluation."""
    import cases
    import torch
    from helpers import product
    from pyfwi_b200.batch import SurveyBatch
    cs = cases.c4(args.uneven)
    props = [product(c, cuda_device=str(dev), graph=False) for c in cs]
    batch = SurveyBatch(props)  # shares the device memory out before any plan is built
    models, observed = [], []
    for W, c in zip(props, cs):
        m_obs = {k: torch.from_numpy(v).to(dev) for k, v in c["model_obs"].items()}
        observed.append({k: v.clone() for k, v in W.forward_modeling(m_obs).items()})
        models.append({k: torch.from_numpy(v).to(dev) for k, v in c["model_est"].items()})
    cells = sum(2.0 * int(W.tnz) * int(W.tnx) * int(W.nt) * int(W.ns) for W in props)

    def sequential():
        for W, m, o in zip(props, models, observed):
            W.misfit_gradient(m, o, parameterization="dv")

    graphed = SurveyBatch(props, graph=True)
    forms = {"sequential": sequential,
             "streams": lambda: batch.misfit_gradient(models, observed),
             "graph": lambda: graphed.misfit_gradient(models, observed)}
    out = {"surveys": len(props), "cell_updates": cells}

    def timed(name, fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out[name] = {"ms": ms, "value": cells / (ms * 1e-3) / 1e9, "unit": UNIT}
    for name, fn in forms.items():
        timed(name, fn)
    # (4) one survey after another again, each plan replaying its own
    # captured graph (inpa['graph'] = True)
    del forms, batch, graphed, props
    gc.collect()
    torch.cuda.empty_cache()
    props = [product(c, cuda_device=str(dev), graph=True) for c in cs]
    SurveyBatch(props)  # memory shares only

    def sequential_graphs():
        for W, m, o in zip(props, models, observed):
            W.misfit_gradient(m, o, parameterization="dv")
    timed("sequential_graph_plans", sequential_graphs)
    return out


def configs_run(args, dev):
    """The two smaller configurations (cases.c1: 100 x 100 cells, 4 shots,
    nt 500; cases.c2: 200 x 400 cells, 10 shots, nt 2000): one misfit and
    gradient evaluation of all shots on the device (CUDA events, 3 timed
    after 1 untimed) in four forms -- the plain form (one shot per launch
    sequence, every step one launch issued from the host), all shots per
    launch with launches issued from the host, the plan replaying its
    captured graph, and the persistent time loops -- and the reference's
    kernels on the host cores on one shot (bounded sample, as cpu_baseline);
    Gcell-updates/s and shots/s, and the best batched form's shots/s over the
    plain form's."""
    import cases
    import torch
    from helpers import product
    out = {}
    for name in ("c1", "c2"):
        case = cases.by_name(name)
        gpu = {}
        forms = (("plain", {"graph": False, "persist": False, "shot_batch": 1, "segment": 0, "store": "states"}),
                 ("launches", {"graph": False, "persist": False}), ("graph", {"graph": True, "persist": False}),
                 ("persistent", {"persist": True, "shot_batch": 0, "segment": 0}))
        for form, extra in forms:
            W = product(case, cuda_device=str(dev), **extra)
            obs = {k: v.clone() for k, v in W.forward_modeling(
                {k: torch.from_numpy(v).to(dev) for k, v in case["model_obs"].items()}).items()}
            model = {k: torch.from_numpy(v).to(dev) for k, v in case["model_est"].items()}
            per_shot = 2.0 * int(W.tnz) * int(W.tnx) * int(W.nt)
            W.misfit_gradient(model, obs)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            l0 = W.plan.launches()
            e0.record()
            for _ in range(3):
                W.misfit_gradient(model, obs)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / 3
            gpu[form] = {"ms_per_evaluation": ms, "value": per_shot * int(W.ns) / (ms * 1e-3) / 1e9, "unit": UNIT,
                         "shots_per_s": int(W.ns) / (ms * 1e-3),
                         "launches_per_evaluation": (W.plan.launches() - l0) / 3,
                         "layout": {"shot_batch": int(W.shot_batch), "segment": int(W.segment),
                                    "persist": int(W.plan.opts.persist), "graph": int(W.plan.opts.graph)}}
            del W, obs
        gpu["batched_over_plain"] = max(gpu[f]["shots_per_s"] for f in ("launches", "graph", "persistent")) / \
            gpu["plain"]["shots_per_s"]
        cpu = None
        if not args.no_cpu:
            v, kind, cores, desc = cpu_sample(case, seconds=args.cpu_seconds / 3)
            cpu = {"value": v, "unit": UNIT, "shots_per_s": v * 1e9 / per_shot, "cores": cores, "kind": kind,
                   "sample": desc}
        out[name] = {"gpu": gpu, "cpu": cpu}
    return out


def plain_form(args, dev, batched_shots_s):
    """The plain form on the same survey: one shot per launch sequence
    (shot_batch 1) with every forward step stored in FP32 (segment = nt),
    each launch issued from the host (no graph replay), on the first
    `--plain-shots` shots.  One untimed evaluation, one timed."""
    import torch
    from helpers import product
    case = survey(args.plain_shots, args.nt)
    extra = {"cuda_device": str(dev), "segment": 0, "shot_batch": 1, "graph": False, "persist": False,
             "store": "states"}
    if args.tile is not None:
        extra["tile"] = args.tile if args.tile == "auto" else int(args.tile)
    if args.adj_tile is not None:
        extra["adj_tile"] = args.adj_tile
    W = product(case, **extra)
    m_est = {k: torch.from_numpy(v).to(dev) for k, v in case["model_est"].items()}
    m_obs = {k: torch.from_numpy(v).to(dev) for k, v in case["model_obs"].items()}
    d_obs = {k: v.clone() for k, v in W.forward_modeling(m_obs).items()}

    def step():
        return W.misfit_gradient(m_est, d_obs, parameterization="dv")

    step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    shots_s = int(W.ns) / (ms * 1e-3)
    cells = 2.0 * int(W.tnz) * int(W.tnx) * int(W.nt) * int(W.ns)
    out = {"shots": int(W.ns), "shot_batch": int(W.shot_batch), "segment": int(W.segment),
           "snapshots": "fp32, every step", "ms": ms, "shots_per_s": shots_s,
           "value": cells / (ms * 1e-3) / 1e9, "unit": UNIT, "batched_shots_per_s": batched_shots_s,
           "batched_over_plain": batched_shots_s / shots_s}
    del W, d_obs
    gc.collect()
    torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--shots", type=int, default=64)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--nt", type=int, default=None, help="shorter record (profiling cases)")
    ap.add_argument("--segment", type=int, default=0, help="steps per recompute segment (default: auto)")
    ap.add_argument("--tile", default=None, help="step kernel variant 0..5, or 'auto' (autotuner)")
    ap.add_argument("--adj-tile", type=int, default=None, help="adjoint step kernel variant when it differs")
    ap.add_argument("--snapshot", choices=["fp32", "fp24", "bf16"], default="fp32",
                    help="format of the imaged forward states (fp24: within the gradient bar at 3/4 of the store)")
    ap.add_argument("--store", choices=["differences", "states"], default=None,
                    help="what the checkpoint segments hold for the imaging (default: the library's)")
    ap.add_argument("--overlap", type=int, default=None,
                    help="1: recompute segments on a second stream beside the adjoint (default: the library's)")
    ap.add_argument("--plain-shots", type=int, default=2,
                    help="shots of the plain one-shot-per-launch form timed beside the batched one (0: skip)")
    ap.add_argument("--inversion", type=int, default=0,
                    help="also time this many L-BFGS iterations of FWI (device and host optimiser)")
    ap.add_argument("--optimizers", default="device,scipy",
                    help="with --inversion: the optimisers to time (device: FWI's L-BFGS on the GPU; scipy: on the host)")
    ap.add_argument("--uneven", type=int, default=0,
                    help="also time a batch of this many uneven-size surveys (sequential, streams, graph)")
    ap.add_argument("--config", choices=["c3", "c5"], default="c3",
                    help="survey of the timed evaluation: the 500 x 1000 one (default) or the thrust-belt one")
    ap.add_argument("--configs", action="store_true",
                    help="also time the 100 x 100 and 200 x 400 configurations (device and host reference)")
    args = ap.parse_args()
    if args.impl == "reference":
        # rank 0 alone times the host CPU; other ranks have nothing to do
        world = int(os.environ.get("WORLD_SIZE", "1"))
        run_reference(args, world, int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_setup(args)
    try:
        run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
