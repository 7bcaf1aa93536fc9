"""The stored wavefields WavePropagator.W (src/PyFWI/wave_propagation.py:
150-156, filled at :710-727) without a GPU: the fp32 oracle's checkpoint
states reproduce the reference's own W bit for bit (fixture made by running
PyFWI's forward_modeling, tests/golden/make_wavefields.py), so the oracle
pins the GPU tests of the product's W."""
import numpy as np
import pytest

import cases
from conftest import load_golden

FIELDS = ("vx", "vz", "taux", "tauz", "tauxz")


@pytest.mark.parametrize("name", ["tiny_chpr", "tiny_dxr", "tiny_dtscale", "tiny_water"])
def test_oracle_states_are_the_references_W(name):
    import oracle as O
    g = load_golden("wavefields")
    case = cases.by_name(name)
    inpa = case["inpa"]
    src = O.Ricker(case["src_loc"], inpa["dh"], inpa["dt"], case["src_type"])
    src.Ricker(case["fdom"])
    W = O.OracleWavePropagator(inpa, src, case["rec_loc"], case["model_est"]["vp"].shape,
                               components=case["components"], n_well_rec=case["n_well_rec"], chpr=case["chpr"])
    assert np.array_equal(W.chp, g[name + "_chp"])
    W._materials({k: v.copy() for k, v in case["model_est"].items()})
    ks = g[name + "_ks"]
    for s in range(int(W.ns)):
        _, states = W.forward_shot(s, store=True)  # (nchp, 5, tnz, tnx)
        for q, f in enumerate(FIELDS):
            ref = g[name + "_" + f][:, :, s, :]  # (tnz, tnx, len(ks))
            assert np.array_equal(states[ks, q].transpose(1, 2, 0), ref), (s, f)
