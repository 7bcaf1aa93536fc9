"""The persistent time loops (inpa['persist']): small surveys run many steps
per cooperative launch with a grid barrier between steps, through the same
tile code as the per-step kernels.

* Bits: the persistent and the per-step forms give the same seismograms,
  raw traces and gradients bit for bit -- several shot groups, sub-stepped
  time, wells plus a surface line, a water layer, and records longer than
  one launch's chunk of steps; with the 8th-order stencil and energy terms
  the gradients agree to float32 rounding.
* Reference: the 100 x 100 survey and the 200 x 400 survey (10 shots,
  2000 steps: four forward launches) against the reference's fixtures, with
  the persistent form on.
* Failure path, without a GPU fault: the barrier's bounded wait made to run
  out on purpose (pyfwi_barrier_selftest: a barrier that waits for a CTA
  that does not exist, the limit cut to 20 ms) sets the error word to 3; the
  next persistent call stops at its first barrier and raises; once the word
  is read the plan gives the clean results again."""
import time

import numpy as np
import pytest

import cases
from conftest import load_golden, rel_l2
from helpers import l2_residual_np, product, section_error

pytestmark = pytest.mark.gpu

SEIS_TOL = 1e-5
GRAD_TOL = 1e-4


def _evaluate(case, shot_batch=0, **extra):
    """Every step stored (one segment: the layout the persistent loops run)."""
    W = product(case, segment=0, shot_batch=shot_batch, **extra)
    d_obs = W.forward_modeling(case["model_obs"])
    d_est = W.forward_modeling(case["model_est"])
    raw = W.seismogram
    res = l2_residual_np(d_est, d_obs)
    grad = W.gradient({k: v for k, v in res.items() if np.any(v)}, parameterization=case["param"])
    return W, d_obs, d_est, raw, grad


@pytest.mark.parametrize("name,batch", [("c1", 0), ("c1", 3), ("tiny_dtscale", 0), ("tiny_s8", 1),
                                        ("tiny_both", 0), ("tiny_water", 0), ("tiny_dxr", 0)])
def test_persistent_loops_give_the_step_kernels_bits(name, batch):
    case = cases.by_name(name)
    Wp, *out_p = _evaluate(case, persist=True, shot_batch=batch)
    Ws, *out_s = _evaluate(case, persist=False, shot_batch=batch, store="states")  # the step kernels' states path
    assert Wp.plan.opts.persist == 1 and Ws.plan.opts.persist == 0
    energy = case["inpa"].get("energy_balancing", False)
    for q, (a, b) in enumerate(zip(out_p, out_s)):
        for k in a:
            if energy and q == 3:  # the energy terms' sums are grouped otherwise by the compiler: float32 rounding
                assert rel_l2(a[k], b[k]) < 1e-6, (name, k)
            else:
                assert np.array_equal(a[k], b[k]), (name, k)
    # the persistent form issued far fewer launches
    assert Wp.plan.launches() * 10 < Ws.plan.launches(), (Wp.plan.launches(), Ws.plan.launches())


def test_persistent_loops_on_the_200x400_survey():
    """2000 steps: the forward pass takes four launches of up to 512 steps."""
    case = cases.c2_parity()
    g = load_golden("c2_parity")
    Wp, d_obs, d_est, raw, grad = _evaluate(case, persist=True)
    _, d_obs_s, d_est_s, _, grad_s = _evaluate(case, persist=False, store="states")
    for k in d_est:
        assert np.array_equal(d_est[k], d_est_s[k]) and np.array_equal(d_obs[k], d_obs_s[k]), k
        if "d_est_" + k in g:
            ok, why = section_error(d_est[k][:, g["cols"]], g["d_est_" + k], g.get("f64_d_est_" + k), SEIS_TOL)
            assert ok, (k, why)
    for k in grad:
        assert np.array_equal(grad[k], grad_s[k]), k
        assert rel_l2(grad[k], g["grad_" + k]) < GRAD_TOL, k


def test_persistent_survey_matches_reference():
    """The 100 x 100 survey with the persistent loops ('auto' persists it)
    against the reference's fixture, on the reference's own residual."""
    case = cases.c1()
    g = load_golden("c1")
    W = product(case, persist="auto")
    assert W.plan.opts.persist == 1
    d_est = W.forward_modeling(case["model_est"])
    for k, v in d_est.items():
        assert rel_l2(v, g["d_est_" + k]) < SEIS_TOL, k
    res = l2_residual_np({k[6:]: v for k, v in g.items() if k.startswith("d_est_")},
                         {k[6:]: v for k, v in g.items() if k.startswith("d_obs_")})
    grad = W.gradient({k: v for k, v in res.items() if np.any(v)}, parameterization=case["param"])
    for k, v in grad.items():
        assert rel_l2(v, g["grad_" + k]) < GRAD_TOL, k


def test_barrier_wait_gives_up_and_the_context_stays_usable():
    import torch
    from pyfwi_b200._native import NativeError
    case = cases.tiny_dxr()
    g = load_golden("tiny_dxr")
    W = product(case, persist=True, segment=0, shot_batch=0)
    clean = W.forward_modeling(case["model_est"])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    W.plan.barrier_selftest(20_000_000)
    torch.cuda.synchronize()
    assert time.perf_counter() - t0 >= 0.02
    with pytest.raises(NativeError, match="device error word 3"):
        W.plan.check_device()
    # set it again: the next persistent call stops at its first barrier and raises
    W.plan.barrier_selftest(20_000_000)
    with pytest.raises(NativeError, match="device error word 3"):
        W.forward_modeling(case["model_est"])
    again = W.forward_modeling(case["model_est"])
    for k in clean:
        assert np.array_equal(again[k], clean[k]), k
        assert rel_l2(again[k], g["d_est_" + k]) < SEIS_TOL, k
    W.plan.check_device()
    for bad in (0, 999, 10 ** 11):
        with pytest.raises(NativeError, match="limit_ns"):
            W.plan.barrier_selftest(bad)
