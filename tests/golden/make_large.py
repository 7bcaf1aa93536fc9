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


if __name__ == "__main__":
    names = sys.argv[1:] or [f.__name__ for f in cases.LARGE]
    for n in names:
        make(cases.by_name(n))
