"""The CPU oracle against the reference's own outputs (golden fixtures made
by running PyFWI's WavePropagator and its kernels, tests/golden/make_golden.py).

The oracle restates the reference arithmetic operation for operation, so the
fp32 oracle must reproduce the fixtures bit for bit."""
import os

import numpy as np
import pytest

import cases
from conftest import GOLDEN, load_golden, rel_l2
from helpers import oracle_run

TINY = [f.__name__ for f in cases.TINY]


def _obs_from_golden(g):
    return {k[len("d_obs_"):]: g[k] for k in g if k.startswith("d_obs_")}


@pytest.mark.parametrize("name", TINY)
def test_oracle_bit_exact_tiny(name):
    g = load_golden(name)
    case = cases.by_name(name)
    for k in ("vp", "vs", "rho"):
        assert np.array_equal(case["model_est"][k], g["in_est_" + k]), "case inputs drifted from the fixture"
    d_obs, d_est, grad, W = oracle_run(case)
    for k, v in d_obs.items():
        assert np.array_equal(v, g["d_obs_" + k]), k
    for k, v in d_est.items():
        assert np.array_equal(v, g["d_est_" + k]), k
    for k, v in W.seismogram.items():
        assert np.array_equal(v, g["seis_" + k]), k
    for k, v in grad.items():
        assert np.array_equal(v, g["grad_" + k]), k


def test_oracle_setup_matches_reference():
    for name in ["c1"] + TINY:
        g = load_golden(name)
        _, _, _, W = oracle_run(cases.by_name(name), gradient=False)
        assert np.array_equal(W.chp, g["setup_chp"])
        assert W.nt == int(g["setup_nt"]) and W.nt_ext == int(g["setup_nt_ext"])
        assert float(W.dt_scale) == float(g["setup_dt_scale"])
        assert np.array_equal(W.srcx, g["setup_srcx"]) and np.array_equal(W.srcz, g["setup_srcz"])
        assert int(W.dxr) == int(g["setup_dxr"])
        assert np.array_equal(W.dx_pml, g["setup_dx_pml"]) and np.array_equal(W.dz_pml, g["setup_dz_pml"])
        for k in ("rec_top_left_const", "rec_top_left_var", "rec_top_right_const", "rec_top_right_var",
                  "rec_surface_const", "rec_surface_var"):
            assert int(getattr(W, k)) == int(g["setup_" + k]), (name, k)


def test_oracle_bit_exact_c1():
    """Config 1 (100 x 100, 4 shots, 500 steps): forward and gradient."""
    g = load_golden("c1")
    d_obs, d_est, grad, _ = oracle_run(cases.by_name("c1"), d_obs=_obs_from_golden(g))
    for k, v in d_est.items():
        assert np.array_equal(v, g["d_est_" + k]), k
    for k, v in grad.items():
        assert np.array_equal(v, g["grad_" + k]), k


def test_fp64_oracle_close_to_reference():
    """The FP64 oracle differs from the reference's float32 run only by
    rounding: this bounds what float32 arithmetic can reach."""
    g = load_golden("tiny_s8")
    _, d_est, grad, _ = oracle_run(cases.by_name("tiny_s8"), precision="fp64")
    for k, v in d_est.items():
        assert rel_l2(v, g["d_est_" + k]) < 1e-5, k
    for k, v in grad.items():
        assert rel_l2(v, g["grad_" + k]) < 1e-3, k


def test_fp64_fixtures_reproduce():
    """The committed FP64 fixtures are what the FP64 oracle computes now."""
    case = cases.by_name("tiny_dxr")
    f = np.load(os.path.join(GOLDEN, "tiny_dxr_fp64.npz"))
    _, d_est, grad, _ = oracle_run(case, precision="fp64")
    for k, v in d_est.items():
        assert np.array_equal(np.asarray(v, np.float64), f["d_est_" + k]), k
    for k, v in grad.items():
        assert np.array_equal(np.asarray(v, np.float64), f["grad_" + k]), k
