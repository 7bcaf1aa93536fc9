"""The multiscale low-pass (lowpass / adj_lowpass, fwi_tools.py:1188-1258)
on the CPU: the oracle's restatement reproduces the reference's outputs
(tests/golden/lowpass.npz, make_lowpass.py); the nt x nt response
(pyfwi_b200.fwi_tools.lowpass_response) is the same operator, and so is
the spectrum the device's FFT kernel applies (lowpass_spectrum), here
applied with numpy's FFT exactly as the kernel does: two traces per complex
signal, zero-padded to nfft, times the real spectrum, transformed back."""
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


def test_spectrum_is_the_reference_filter():
    from pyfwi_b200.fwi_tools import lowpass_spectrum
    f = _fixture()
    for q in range(2):
        x, hc = f["x%d" % q].astype(np.float64), float(f["hc%d" % q])
        planes, nt, ncols = x.shape
        nfft, filt = lowpass_spectrum(nt, hc, FN, 3)
        assert nfft >= 2 * nt - 1 and nfft & (nfft - 1) == 0 and filt.shape == (2 * nfft,)
        spec = filt[:nfft].astype(np.float64)
        tw = filt[nfft:].reshape(-1, 2)
        j = np.arange(nfft // 2)
        assert np.allclose(tw[:, 0], np.cos(2 * np.pi * j / nfft), atol=1e-7)
        assert np.allclose(tw[:, 1], -np.sin(2 * np.pi * j / nfft), atol=1e-7)
        xp = np.zeros((planes, nfft, ncols + ncols % 2))
        xp[:, :nt, :ncols] = x
        z = xp[..., 0::2] + 1j * xp[..., 1::2]  # traces 2p and 2p + 1 in one complex signal
        w = np.fft.ifft(np.fft.fft(z, axis=1) * spec[None, :, None], axis=1) * nfft
        y = np.empty_like(xp[:, :nt])
        y[..., 0::2], y[..., 1::2] = w.real[:, :nt], w.imag[:, :nt]
        ref = f["low%d" % q]
        assert np.linalg.norm(y[..., :ncols] - ref) <= 1e-6 * np.linalg.norm(ref)
