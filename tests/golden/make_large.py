"""Regenerate the reference fixtures of the configured survey sizes.

    python tests/golden/make_large.py [case ...]     (cases.LARGE by default)

The reference (PyFWI's unmodified ``WavePropagator`` with its own OpenCL C
kernels compiled for the CPU, oracle/run_reference.py) keeps every stored
step of every shot in one host array (wave_propagation.py:150-156), which
for these surveys would not fit in host memory with all shots at once.  So
each shot runs as a survey of its own -- shots are independent in the
reference: the shot loop is outermost (wave_propagation.py:639, :740) and
each shot starts from zero fields -- and the per-shot results are put
together: trace columns side by side in shot order (the '2d' section
layout, acquisition.py:313-333) and gradients summed (the mask of
gradient_reading is fixed and grad_lmd_to_vd is linear when
energy_balancing is off, as in these cases).

Stored per case, ``<name>.npz``:

* ``cols``: the trace columns kept (a fixed stride over all ns*nr columns;
  the full sections would take tens of MB) and ``d_obs_*``, ``d_est_*``,
  ``seis_*`` on those columns, all in the '2d' layout (for components 0
  one stress key: the reference fills 'taux' and 'tauz' with the same
  mean);
* ``grad_*``: the whole gradient, ``rms``: the L2 misfit of the whole survey;
* ``f64_d_obs_*``, ``f64_d_est_*``, ``f64_seis_*``: the FP64 oracle's
  sections and raw traces on the same columns (``--fp64`` adds them to
  existing fixtures);
* ``in_sha``: a digest of the case's inputs, so a test can tell that
  tests/cases.py still builds the survey the fixture was made from;
* the set-up values the reference computed (``setup_*``).

It needs the reference tree (/root/reference), so it runs only where that
exists; the fixtures it writes are what the tests read everywhere else.
"""
import os
import pickle
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import cases  # noqa: E402
from helpers import input_digest  # noqa: E402

# trace columns kept per case (about 2 MB of traces each)
KEEP_COLS = {"c2_parity": 64, "c3_parity": 200, "c4_parity": 160, "c5_parity": 100}


def column_stride(n_cols, keep):
    return max(1, n_cols // keep)


def run_shot(case, s):
    one = dict(case)
    one["src_loc"] = case["src_loc"][s:s + 1].copy()
    with tempfile.TemporaryDirectory() as tmp:
        cp, op = os.path.join(tmp, "case.pkl"), os.path.join(tmp, "out.npz")
        with open(cp, "wb") as f:
            pickle.dump(one, f)
        subprocess.check_call([sys.executable, os.path.join(ROOT, "oracle", "run_reference.py"), cp, op])
        with np.load(op) as d:
            return {k: d[k] for k in d.files}


def make(case):
    ns = len(case["src_loc"])
    per = []
    for s in range(ns):
        t0 = time.time()
        per.append(run_shot(case, s))
        print("%s shot %d/%d: %.0f s" % (case["name"], s + 1, ns, time.time() - t0), flush=True)
    first = per[0]
    out = {}
    nr = first[[k for k in first if k.startswith("d_est_")][0]].shape[1]
    n_cols = nr * ns
    stride = column_stride(n_cols, KEEP_COLS.get(case["name"], 100))
    cols = np.arange(0, n_cols, stride)
    out["cols"] = cols
    sec_keys = [k for k in first if k.startswith(("d_obs_", "d_est_", "seis_"))]
    if case["components"] == 0:
        sec_keys = [k for k in sec_keys if not k.endswith("_tauz") or k.startswith("seis_")]
    for k in sec_keys:
        # raw traces come as (nt, nr, 1) per shot: side by side they take the
        # '2d' layout, column s*nr + r, like the sections
        full = np.concatenate([p[k].reshape(p[k].shape[0], -1) for p in per], axis=1)
        out[k] = np.ascontiguousarray(full[:, cols])
    for k in first:
        if k.startswith("grad_"):
            out[k] = np.sum([p[k].astype(np.float64) for p in per], axis=0).astype(np.float32)
    out["rms"] = np.asarray(sum(float(p["rms"]) for p in per))
    for k in first:
        if k.startswith("setup_") and k not in ("setup_srcx", "setup_srcz", "setup_dx_pml", "setup_dz_pml"):
            out[k] = first[k]
    out["setup_srcx"] = np.concatenate([p["setup_srcx"] for p in per])
    out["setup_srcz"] = np.concatenate([p["setup_srcz"] for p in per])
    out["in_sha"] = np.asarray(input_digest(case))
    path = os.path.join(HERE, case["name"] + ".npz")
    np.savez_compressed(path, **out)
    print(case["name"], "written", os.path.getsize(path) // 1024, "KB", flush=True)


def add_fp64(case):
    """Add the FP64 oracle's sections and raw traces on the kept columns
    (``f64_d_obs_*``, ``f64_d_est_*``, ``f64_seis_*``) to an existing fixture: the exact-arithmetic answer the
    reference's own float32 rounding is measured against (its float32 error
    exceeds 1e-5 on traces next to a source over long records)."""
    import oracle as O
    path = os.path.join(HERE, case["name"] + ".npz")
    with np.load(path) as d:
        out = {k: d[k] for k in d.files}
    cols = out["cols"]
    inpa = case["inpa"]
    nr = None
    secs = {"obs": [], "est": []}
    raw = []
    for s in range(len(case["src_loc"])):
        src = O.Ricker(case["src_loc"][s:s + 1], inpa["dh"], inpa["dt"], case["src_type"])
        src.Ricker(case["fdom"])
        W = O.OracleWavePropagator(inpa, src, case["rec_loc"], case["model_est"]["vp"].shape,
                                   components=case["components"], n_well_rec=case["n_well_rec"], chpr=0,
                                   precision="fp64")
        for which in ("obs", "est"):
            secs[which].append(W.forward_modeling({k: v.copy() for k, v in case["model_" + which].items()}))
        raw.append({k: np.asarray(v).reshape(v.shape[0], -1) for k, v in W.seismogram.items()})
    for k in raw[0]:
        if "seis_" + k in out:
            full = np.concatenate([r[k] for r in raw], axis=1)
            out["f64_seis_" + k] = np.ascontiguousarray(full[:, cols], np.float32)
    for which in ("obs", "est"):
        for k in secs[which][0]:
            if "d_%s_%s" % (which, k) not in out:
                continue
            full = np.concatenate([np.asarray(d[k]) for d in secs[which]], axis=1)
            out["f64_d_%s_%s" % (which, k)] = np.ascontiguousarray(full[:, cols], np.float32)
    np.savez_compressed(path, **out)
    print(case["name"], "FP64 sections added", os.path.getsize(path) // 1024, "KB", flush=True)


if __name__ == "__main__":
    args = sys.argv[1:]
    fp64_only = "--fp64" in args
    names = [a for a in args if a != "--fp64"] or [f.__name__ for f in cases.LARGE]
    for n in names:
        if not fp64_only:
            make(cases.by_name(n))
        add_fp64(cases.by_name(n))
