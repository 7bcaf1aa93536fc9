"""Regenerate the golden fixtures of tests/golden/ from the PyFWI reference.

    python tests/golden/make_golden.py [case ...]

For every case of tests/cases.py this runs the unmodified reference driver
(PyFWI's ``WavePropagator`` with its own OpenCL C kernels compiled for the
CPU, see oracle/run_reference.py) in a subprocess and stores, per case,
``<name>.npz`` with

* the inputs (both models, geometry, wavelet parameters),
* the observed and estimated seismic sections (``d_obs_*``, ``d_est_*``),
* the five raw receiver traces of the estimate (``seis_*``, tiny cases only),
* the L2 misfit and the gradient (``grad_*``),
* the set-up values the reference computed (``setup_*``).

It needs the reference tree (/root/reference), so it runs only where that
exists; the fixtures it writes are what the tests read everywhere else.
"""
import os
import pickle
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
import cases  # noqa: E402


def make(case):
    with tempfile.TemporaryDirectory() as tmp:
        cp, op = os.path.join(tmp, "case.pkl"), os.path.join(tmp, "out.npz")
        with open(cp, "wb") as f:
            pickle.dump(case, f)
        subprocess.check_call([sys.executable, os.path.join(ROOT, "oracle", "run_reference.py"), cp, op])
        out = dict(np.load(op))
    if case["name"] == "c1":
        # keep the large case small: the raw traces are not stored
        out = {k: v for k, v in out.items() if not k.startswith("seis_")}
    for k in ("vp", "vs", "rho"):
        out["in_obs_" + k] = case["model_obs"][k]
        out["in_est_" + k] = case["model_est"][k]
    out["in_src_loc"] = case["src_loc"]
    out["in_rec_loc"] = case["rec_loc"]
    np.savez_compressed(os.path.join(HERE, case["name"] + ".npz"), **out)
    print(case["name"], "written")


if __name__ == "__main__":
    names = sys.argv[1:] or [f.__name__ for f in cases.ALL]
    for n in names:
        make(cases.by_name(n))
