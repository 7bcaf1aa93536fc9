"""The product's host set-up (time axis, index constants, checkpoint list,
damping arrays, receiver lines, gradient window) against the values the
reference computed for the same surveys (golden fixtures).  No GPU: the
device plan is only built on first use."""
import numpy as np
import pytest

import cases
from conftest import load_golden
from pyfwi_b200 import acquisition as acq
from pyfwi_b200.wave_propagation import WavePropagator

NAMES = ["c1"] + [f.__name__ for f in cases.TINY]


def product(case):
    inpa = case["inpa"]
    src = acq.Source(case["src_loc"], inpa["dh"], inpa["dt"], case["src_type"])
    src.Ricker(case["fdom"])
    return WavePropagator(inpa, src, case["rec_loc"], case["model_est"]["vp"].shape, components=case["components"],
                          n_well_rec=case["n_well_rec"], chpr=case["chpr"])


@pytest.mark.parametrize("name", NAMES)
def test_setup_matches_reference(name):
    g = load_golden(name)
    W = product(cases.by_name(name))
    assert np.array_equal(W.chp, g["setup_chp"])
    assert W.nt == int(g["setup_nt"]) and W.nt_ext == int(g["setup_nt_ext"])
    assert float(W.dt_scale) == float(g["setup_dt_scale"]) and W.dt == float(g["setup_dt"])
    assert np.array_equal(W.srcx, g["setup_srcx"]) and np.array_equal(W.srcz, g["setup_srcz"])
    assert int(W.dxr) == int(g["setup_dxr"]) and int(W.sdo) == int(g["setup_sdo"])
    for k in ("rec_top_left_const", "rec_top_left_var", "rec_top_right_const", "rec_top_right_var",
              "rec_surface_const", "rec_surface_var", "src_cts"):
        assert int(getattr(W, k)) == int(g["setup_" + k]), k
    assert np.array_equal(W.dx_pml, g["setup_dx_pml"]) and np.array_equal(W.dz_pml, g["setup_dz_pml"])
    assert np.array_equal(W.src.w, g["setup_wavelet"])


def test_damping_profiles_are_separable():
    for name in NAMES:
        W = product(cases.by_name(name))
        assert np.array_equal(W.dx_pml, np.broadcast_to(W.dx_pml[0, :], W.dx_pml.shape))
        assert np.array_equal(W.dz_pml, np.broadcast_to(W.dz_pml[:, :1], W.dz_pml.shape))


def test_receiver_lines_cover_every_reference_receiver():
    """Each line cell equals the cell the reference's receiver work item reads."""
    W = product(cases.c1())
    lines = W._lines()
    assert lines == [(22, 20, 0, 1, 100, 0, 0)]
    W = product(cases.tiny_dxr())
    (r0, c0, dr, dc, cnt, s0, vzx), = W._lines()
    assert (dr, dc, s0, vzx) == (0, 2, 0, 0)
    for k in range(cnt):
        j = k * int(W.dxr)
        assert divmod(int(W.rec_surface_const) * int(W.tnx) + j + int(W.rec_surface_var), int(W.tnx)) == (r0, c0 + 2 * k)
    W = product(cases.tiny_crosswell())
    (r0, c0, dr, dc, cnt, s0, vzx), = W._lines()
    assert (dr, dc, vzx) == (1, 0, 1) and c0 == int(W.rec_top_right_const) and cnt == int(W.nr)
    W = product(cases.tiny_both())
    L = W._lines()
    assert len(L) == 3 and [l[5] for l in L] == [0, int(W.n_well_rec), int(W.n_well_rec) + int(W.n_surface_rec)]


def test_gradient_window_matches_reference_slices():
    for name in NAMES:
        W = product(cases.by_name(name))
        r0, r1, c0, c1 = W._mask_window()
        f = np.zeros((int(W.nz), int(W.nx)))
        sdo, cts = int(W.sdo), int(W.src_cts)
        if W.acq_type == 0:
            f[sdo:-sdo, sdo + cts + 2:-sdo] = 1
        else:
            f[sdo + cts + 2:-sdo, sdo:-sdo] = 1
        g = np.zeros_like(f)
        g[r0:r1, c0:c1] = 1
        assert np.array_equal(f, g), name


def test_source_values_follow_wavelet():
    W = product(cases.tiny_dtscale())
    n_inj = int(np.ceil(W.nt / W.dt_scale))
    assert W._wavelet.shape == (n_inj, 4)
    for k in range(n_inj):
        assert np.array_equal(W._wavelet[k], np.float32(W.src(k))[:4])


def test_geometry_struct_rounds_constants_like_the_reference_macros():
    W = product(cases.tiny_s8())
    g = W._geometry()
    assert g.half_order == 4 and abs(g.c[0] - 1.195955) < 1e-7 and abs(g.c[3] + 0.000697) < 1e-9
    assert np.float32(g.dt) == np.float32(float("%f" % W.dt))


def test_gaussian_weights_follow_scipy():
    """The smoothing weights are scipy's gaussian_filter1d kernel: filtering
    a unit impulse with them reproduces scipy on the same impulse."""
    from scipy.ndimage import gaussian_filter1d
    from pyfwi_b200.engine import gaussian_weights
    for sigma in (0.5, 1.0, 2.7, 6.0):
        w, r = gaussian_weights(sigma)
        x = np.zeros(4 * r + 9)
        x[2 * r + 4] = 1.0
        np.testing.assert_allclose(gaussian_filter1d(x, sigma), np.convolve(x, w, mode="same"), rtol=0, atol=1e-15)


LARGE = [f.__name__ for f in cases.LARGE]


@pytest.mark.parametrize("name", LARGE)
def test_setup_matches_reference_at_configured_sizes(name):
    """The same set-up values on the surveys of the configured sizes (the
    sub-stepped one included), and the fixture was made from the inputs
    tests/cases.py builds."""
    from helpers import input_digest
    g = load_golden(name)
    case = cases.by_name(name)
    assert input_digest(case) == str(g["in_sha"])
    W = product(case)
    assert np.array_equal(W.chp, g["setup_chp"])
    assert W.nt == int(g["setup_nt"]) and W.nt_ext == int(g["setup_nt_ext"])
    assert float(W.dt_scale) == float(g["setup_dt_scale"]) and W.dt == float(g["setup_dt"])
    assert np.array_equal(W.srcx, g["setup_srcx"]) and np.array_equal(W.srcz, g["setup_srcz"])
    assert int(W.dxr) == int(g["setup_dxr"]) and int(W.sdo) == int(g["setup_sdo"])
    for k in ("rec_top_left_const", "rec_top_left_var", "rec_top_right_const", "rec_top_right_var",
              "rec_surface_const", "rec_surface_var", "src_cts"):
        assert int(getattr(W, k)) == int(g["setup_" + k]), k
    assert np.array_equal(W.src.w, g["setup_wavelet"])
