"""Gradient smoothing on the device (pyfwi_smooth) against
scipy.ndimage.gaussian_filter, which the reference applies to each gradient
(wave_propagation.py:923-936)."""
import numpy as np
import pytest
from scipy.ndimage import gaussian_filter

import cases
from conftest import rel_l2
from helpers import product

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,sigma", [((3, 40, 70), 1.0), ((3, 40, 70), 2.5), ((2, 5, 9), 3.0),
                                         ((1, 64, 33), 0.6), ((3, 100, 100), 7.0)])
def test_smooth_matches_gaussian_filter(shape, sigma):
    import torch
    from pyfwi_b200.engine import smooth
    rng = np.random.default_rng(7)
    x = rng.standard_normal(shape).astype(np.float32)
    y = smooth(torch.from_numpy(x).cuda(), sigma).cpu().numpy()
    for q in range(shape[0]):
        ref = gaussian_filter(x[q], sigma)
        assert ref.dtype == np.float32
        np.testing.assert_allclose(y[q], ref, rtol=0, atol=2e-7 * np.abs(ref).max())


def test_gradient_with_g_smooth():
    case = cases.tiny_s8()
    res = None
    out = {}
    for s in (0, 2.0):
        inpa = dict(case["inpa"], g_smooth=s)
        W = product(dict(case, inpa=inpa))
        d = W.forward_modeling(case["model_est"])
        if res is None:
            res = {k: 0.5 * v for k, v in d.items()}
        out[s] = W.gradient(res)
    for k, v in out[2.0].items():
        ref = gaussian_filter(out[0][k], 2.0)
        assert rel_l2(v, ref) < 1e-6, k
