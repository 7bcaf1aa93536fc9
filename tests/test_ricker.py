"""The reference's own unit test (PyFWI test/test_ricker.py:16-22), applied
to the product's Source: the Ricker wavelet equals its closed form exactly."""
import numpy as np

from pyfwi_b200.acquisition import Source


def ricker(fdom, dt):
    src = Source(src_loc=np.array([[0, 0]]), dh=1.0, dt=dt)
    src.Ricker(fdom=fdom)
    return src.w


def test_ricker():
    fdom, dt = 20.0, 0.004
    w = ricker(fdom=fdom, dt=dt)
    t = np.arange(-1.0 / fdom, 1.0 / fdom + dt / 3, dt)
    assert np.all(w == np.float32((1.0 - 2.0 * (np.pi * fdom * t) ** 2) * np.exp(-(np.pi * fdom * t) ** 2)))


def test_source_call_and_components():
    src = Source(np.array([[10.0, 4.0]], np.float32), 2.0, 0.001, src_type=0)
    src.Ricker(30)
    assert np.array_equal(src.component, np.float32([0, 0, 1, 1, 0]))
    assert np.array_equal(src(3), src.w[3] * src.component)
    assert not np.any(src(src.w.size + 5))
    assert src.i[0] == 5 and src.j[0] == 2
