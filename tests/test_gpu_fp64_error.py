"""Error of the CUDA path against the FP64 oracle (tests/golden/*_fp64.npz),
stated next to the error of the reference's own float32 run on the same
inputs.

Both runs do float32 arithmetic, so both sit at some distance from the FP64
result; the CUDA path (FMA, coefficients divided by dh once) may not be
further from it than a small multiple of the reference's distance.  With
BF16 snapshots the imaging reads forward fields rounded to 8 mantissa bits;
the seismograms are unaffected (the forward recurrence stays FP32) and the
gradient error is bounded separately."""
import os

import numpy as np
import pytest

import cases
from conftest import GOLDEN, load_golden, rel_l2
from helpers import l2_residual_np, product

pytestmark = pytest.mark.gpu

NAMES = ["c1"] + [f.__name__ for f in cases.TINY]
BF16_GRAD_TOL = 1e-2
FP24_GRAD_TOL = 1e-4  # the gradient bar of the configurations, against FP64


def _fp64(name):
    with np.load(os.path.join(GOLDEN, name + "_fp64.npz")) as d:
        return {k: d[k] for k in d.files}


def _run(case, **extra):
    W = product(case, **extra)
    d_obs = W.forward_modeling(case["model_obs"])
    d_est = W.forward_modeling(case["model_est"])
    res = l2_residual_np(d_est, d_obs)
    grad = W.gradient({k: v for k, v in res.items() if np.any(v)}, parameterization=case["param"])
    return d_est, grad


def _err(out, ref, prefix):
    return max(rel_l2(v, ref[prefix + k]) for k, v in out.items())


@pytest.mark.parametrize("name", NAMES)
def test_fp32_path_error_against_fp64(name):
    case = cases.by_name(name)
    f64, g32 = _fp64(name), load_golden(name)
    d_est, grad = _run(case)
    ours = (_err(d_est, f64, "d_est_"), _err(grad, f64, "grad_"))
    ref = (max(rel_l2(g32["d_est_" + k], f64["d_est_" + k]) for k in d_est),
           max(rel_l2(g32["grad_" + k], f64["grad_" + k]) for k in grad))
    print("\n%s vs FP64: seismograms ours %.2e reference %.2e | gradient ours %.2e reference %.2e"
          % (name, ours[0], ref[0], ours[1], ref[1]))
    assert ours[0] <= max(4 * ref[0], 1e-6), (ours, ref)
    assert ours[1] <= max(4 * ref[1], 1e-5), (ours, ref)


@pytest.mark.parametrize("name", [n for n in NAMES if cases.by_name(n)["chpr"] == 100])
def test_bf16_snapshot_error_against_fp64(name):
    case = cases.by_name(name)
    f64 = _fp64(name)
    d32, g32 = _run(case, checkpoint="exact")
    d16, g16 = _run(case, checkpoint="exact", snapshot="bf16")
    for k in d32:  # the forward recurrence is FP32 either way
        assert np.array_equal(d16[k], d32[k]), k
    e32, e16 = _err(g32, f64, "grad_"), _err(g16, f64, "grad_")
    print("\n%s gradient vs FP64: fp32 snapshots %.2e, bf16 snapshots %.2e" % (name, e32, e16))
    assert e16 <= BF16_GRAD_TOL, e16


@pytest.mark.parametrize("name", [n for n in NAMES if cases.by_name(n)["chpr"] == 100])
def test_fp24_snapshot_error_against_fp64(name):
    """24-bit snapshots (BF16 plus a byte: 15 mantissa bits) keep the
    gradient within 1e-4 of the FP64 oracle on three quarters of the FP32
    store; seismograms are bit-identical to FP32 snapshots."""
    case = cases.by_name(name)
    f64 = _fp64(name)
    d32, g32 = _run(case, checkpoint="exact")
    d24, g24 = _run(case, checkpoint="exact", snapshot="fp24")
    for k in d32:
        assert np.array_equal(d24[k], d32[k]), k
    e32, e24 = _err(g32, f64, "grad_"), _err(g24, f64, "grad_")
    print("\n%s gradient vs FP64: fp32 snapshots %.2e, fp24 snapshots %.2e" % (name, e32, e24))
    assert e24 <= FP24_GRAD_TOL, e24


def test_fp24_snapshots_on_the_200x400_survey():
    """The torch-check configuration (10 shots, nt 2000): the gradient with
    24-bit snapshots against the FP32-snapshot gradient and against the
    reference's own gradient, both within 1e-4 (the FP32-snapshot gradient
    is ~1e-5 from FP64 on every smaller case)."""
    case = cases.c2_parity()
    ref = load_golden("c2_parity")
    _, g32 = _run(case, checkpoint="exact")
    _, g24 = _run(case, checkpoint="exact", snapshot="fp24")
    e_32 = max(rel_l2(g24[k], g32[k]) for k in g24)
    e_ref = max(rel_l2(g24[k], ref["grad_" + k]) for k in g24)
    print("\nc2 fp24 snapshots: %.2e from fp32 snapshots, %.2e from the reference" % (e_32, e_ref))
    assert e_32 <= FP24_GRAD_TOL and e_ref <= FP24_GRAD_TOL, (e_32, e_ref)


def test_bf16_snapshots_with_segments_and_batches():
    """BF16 snapshots with recomputed segments and several shot groups give
    the same bits as one segment holding every step."""
    import torch
    case = cases.tiny_s8()
    g = load_golden("tiny_s8")
    res = l2_residual_np({k[6:]: v for k, v in g.items() if k.startswith("d_est_")},
                         {k[6:]: v for k, v in g.items() if k.startswith("d_obs_")})
    out = []
    for seg, batch in ((0, 0), (7, 0), (9, 1)):
        W = product(case, snapshot="bf16", segment=seg, shot_batch=batch)
        W.forward_modeling(case["model_est"])
        out.append(W.gradient(res, parameterization="lmd"))
        torch.cuda.synchronize()
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k
        assert rel_l2(out[2][k], out[0][k]) < 1e-6, k
