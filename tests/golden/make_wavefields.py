"""Regenerate tests/golden/wavefields.npz from the PyFWI reference.

    python tests/golden/make_wavefields.py

Runs the unmodified reference ``WavePropagator.forward_modeling`` (its own
host loop and OpenCL C kernels compiled for the CPU by the test-only
stand-in modules of oracle/standin) on the estimated model of four cases of
tests/cases.py and stores a few checkpoints of the wavefields it keeps,
``W[f][:, :, :, k]`` (src/PyFWI/wave_propagation.py:150-156, filled at
:710-727):

* ``tiny_chpr`` (10 % checkpoints, the reverse-time scheme),
* ``tiny_dxr`` (chpr = 100: every step stored),
* ``tiny_dtscale`` (sub-stepping: checkpoints count internal steps), and
* ``tiny_water`` (a vs = 0 layer, 8th-order stencil),

a few checkpoints of each, as ``<case>_<field>`` arrays (tnz, tnx, ns,
len(ks)) with the checkpoint indices in ``<case>_ks`` and the reference's
checkpoint steps in ``<case>_chp``.  It needs the reference tree (/root/reference), so it runs
only where that exists; the fixture it writes is what the tests read
everywhere else.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle", "standin"), "/root/reference/src"]

import cases  # noqa: E402
import PyFWI.acquisition as acq  # noqa: E402
import PyFWI.wave_propagation as wave  # noqa: E402

# checkpoint indices kept per case (-1: the last)
KS = {"tiny_chpr": [0, 1, 6, 12, 13], "tiny_dxr": [0, 1, 37, 70, 139], "tiny_dtscale": [0, 1, 2, 50, -1],
      "tiny_water": [1, 60, -1]}
FIELDS = ("vx", "vz", "taux", "tauz", "tauxz")


def main():
    out = {}
    for name, ks in KS.items():
        case = cases.by_name(name)
        inpa = dict(case["inpa"])
        src = acq.Source(case["src_loc"], inpa["dh"], inpa["dt"], src_type=case.get("src_type", 0))
        src.Ricker(case["fdom"])
        W = wave.WavePropagator(inpa, src, case["rec_loc"], case["model_est"]["vp"].shape, chpr=case["chpr"],
                                components=case["components"], n_well_rec=case.get("n_well_rec", 0))
        W.forward_modeling({k: v.copy() for k, v in case["model_est"].items()}, show=False)
        ks = np.arange(W.nchp)[ks]
        out[name + "_ks"] = ks.astype(np.int32)
        out[name + "_chp"] = np.asarray(W.chp, np.int32)
        for f in FIELDS:
            out[name + "_" + f] = np.ascontiguousarray(W.W[f][:, :, :, ks])
    np.savez_compressed(os.path.join(HERE, "wavefields.npz"), **out)
    print("wavefields.npz written")


if __name__ == "__main__":
    main()
