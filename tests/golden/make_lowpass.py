"""Regenerate tests/golden/lowpass.npz from the PyFWI reference.

    python tests/golden/make_lowpass.py

Runs the reference's own lowpass and adj_lowpass (src/PyFWI/fwi_tools.py:
1188-1258, imported from the reference tree with the test-only stand-in
modules of oracle/standin) on seeded trace planes and stores inputs and
outputs.  The filter parameters are those of the FWI driver (order 3,
Nyquist constant 1 / (2 * 0.0006), fwi.py:239 and wave_propagation.py:32).
It needs the reference tree (/root/reference), so it runs only where that
exists; the fixture it writes is what the tests read everywhere else.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle", "standin"), "/root/reference/src"]

from PyFWI import fwi_tools  # noqa: E402

CASES = [(130, 17, 25.0), (300, 19, 8.0)]  # (nt, ncols, cutoff Hz)
FN = 1.0 / 2.0 / 0.0006


def main():
    rng = np.random.default_rng(5)
    out = {}
    for q, (nt, ncols, hc) in enumerate(CASES):
        x = rng.standard_normal((3, nt, ncols)).astype(np.float32)
        r = rng.standard_normal((3, nt, ncols)).astype(np.float32)
        out["x%d" % q] = x
        out["r%d" % q] = r
        out["hc%d" % q] = np.float64(hc)
        out["low%d" % q] = fwi_tools.lowpass(x, hc, FN, order=3, axis=1)
        out["adj%d" % q] = fwi_tools.adj_lowpass(r, hc, FN, order=3, axis=1)
    np.savez_compressed(os.path.join(HERE, "lowpass.npz"), **out)
    print("lowpass.npz written")


if __name__ == "__main__":
    main()
