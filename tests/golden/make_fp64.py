"""Regenerate the FP64 fixtures of tests/golden/ (``<name>_fp64.npz``).

    python tests/golden/make_fp64.py [case ...]

For every case of tests/cases.py this runs the oracle in double precision
(oracle/elastic_oracle.c built with every array in double) through the whole
pipeline a user runs (observed data from the true model, modelled data from
the estimate, the L2 residual, the gradient) and keeps the modelled data and
the gradient.  The GPU tests state the
error of the CUDA path (FP32 arithmetic, FP32 or BF16 snapshots) against
these, next to the error of the reference's own float32 run.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.dirname(HERE), os.path.join(ROOT, "oracle")):
    sys.path.insert(0, p)
import cases  # noqa: E402
from helpers import oracle_run  # noqa: E402


def make(case):
    d_obs, d_est, grad, _ = oracle_run(case, precision="fp64")
    out = {}
    out.update({"d_est_" + k: np.asarray(v, np.float64) for k, v in d_est.items()})
    out.update({"grad_" + k: np.asarray(v, np.float64) for k, v in grad.items()})
    np.savez_compressed(os.path.join(HERE, case["name"] + "_fp64.npz"), **out)
    print(case["name"], "fp64 written")


if __name__ == "__main__":
    names = sys.argv[1:] or [f.__name__ for f in cases.ALL]
    for n in names:
        make(cases.by_name(n))
