"""The multiscale low-pass (lowpass / adj_lowpass, fwi_tools.py:1188-1258)
on the CPU: the oracle's restatement reproduces the reference's outputs
(tests/golden/lowpass.npz, make_lowpass.py), and the nt x nt response the
device applies (pyfwi_b200.fwi_tools.lowpass_response) is the same operator."""
import os

import numpy as np

from conftest import GOLDEN

FN = 1.0 / 2.0 / 0.0006


def _fixture():
    with np.load(os.path.join(GOLDEN, "lowpass.npz")) as d:
        return {k: d[k] for k in d.files}


def test_oracle_lowpass_matches_reference():
    import oracle as O
    f = _fixture()
    for q in range(2):
        hc = float(f["hc%d" % q])
        np.testing.assert_allclose(O.lowpass(f["x%d" % q], hc, FN, 3), f["low%d" % q], rtol=0,
                                   atol=1e-12 * np.abs(f["low%d" % q]).max())
        np.testing.assert_allclose(O.lowpass(f["r%d" % q], hc, FN, 3), f["adj%d" % q], rtol=0,
                                   atol=1e-12 * np.abs(f["adj%d" % q]).max())


def test_response_matrix_is_the_reference_filter():
    from pyfwi_b200.fwi_tools import lowpass_response
    f = _fixture()
    for q in range(2):
        x, hc = f["x%d" % q].astype(np.float64), float(f["hc%d" % q])
        K = lowpass_response(x.shape[1], hc, FN, 3).astype(np.float64)
        assert np.array_equal(K, K.T)
        y = np.einsum("ts,psc->ptc", K, x)
        ref = f["low%d" % q]
        assert np.linalg.norm(y - ref) <= 1e-6 * np.linalg.norm(ref)
