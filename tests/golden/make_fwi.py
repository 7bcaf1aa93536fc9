"""Regenerate tests/golden/fwi_lbfgs.npz, fwi_cg.npz and tl_<method>.npz
from the PyFWI reference.

    python tests/golden/make_fwi.py [name ...]

Runs the unmodified reference inversion drivers (``PyFWI.fwi.FWI`` and
``PyFWI.tl_fwi.TimeLapse`` with SciPy's L-BFGS-B, on PyFWI's own OpenCL C
kernels compiled for the CPU, see oracle/run_reference_fwi.py) on the
``fwi_lbfgs``, ``fwi_cg`` and ``timelapse(method)`` cases of tests/cases.py and stores
the resulting models and the misfit of every evaluation (for FWI also the
model of every evaluation).  Needs the reference tree, so it runs only
where that exists.
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
        subprocess.check_call([sys.executable, os.path.join(ROOT, "oracle", "run_reference_fwi.py"), cp, op],
                              stdout=subprocess.DEVNULL)
        out = dict(np.load(op))
    np.savez_compressed(os.path.join(HERE, case["name"] + ".npz"), **out)
    print(case["name"], "written:", len(out["evals_rms"]), "evaluations")


def all_cases():
    return [cases.fwi_lbfgs(), cases.fwi_cg()] + [cases.timelapse(m) for m in cases.TL_METHODS]


if __name__ == "__main__":
    wanted = set(sys.argv[1:])
    for c in all_cases():
        if not wanted or c["name"] in wanted:
            make(c)
