"""Failure detection without a GPU fault.

Every device-side wait in the library is bounded: a streaming kernel that
does not see its row copy arrive gives up after one second of the GPU's
global timer, sets the workspace's error word and stops; later streaming
kernels see the word and stop at once; the host reads and clears the word
(pyfwi_device_error) and raises.  Here the wait is made to run out on
purpose (pyfwi_wait_selftest: an mbarrier nothing arrives at, the limit cut
to 20 ms) and the tests check the status the host reads and that the context
stays usable.  The other failures are injected from the host: a NaN model,
a memory budget no layout fits, a source outside the grid."""
import time

import numpy as np
import pytest

import cases
from conftest import load_golden, rel_l2
from helpers import product

pytestmark = pytest.mark.gpu

SEIS_TOL = 1e-5


def test_bounded_wait_gives_up_and_the_context_stays_usable():
    import torch
    from pyfwi_b200._native import NativeError
    case = cases.tiny_s8()
    g = load_golden("tiny_s8")
    W = product(case, tile=3)  # streaming kernels: they read the error word
    clean = W.forward_modeling(case["model_est"])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    W.plan.wait_selftest(20_000_000)
    torch.cuda.synchronize()
    assert time.perf_counter() - t0 >= 0.02
    # the next call's streaming kernels stop at once; the call reports it
    with pytest.raises(NativeError, match="device error word 1"):
        W.forward_modeling(case["model_est"])
    # reading the word cleared it: the context and the plan work on
    again = W.forward_modeling(case["model_est"])
    for k in clean:
        assert np.array_equal(again[k], clean[k]), k
        assert rel_l2(again[k], g["d_est_" + k]) < SEIS_TOL, k
    W.plan.check_device()


def test_wait_selftest_rejects_a_limit_out_of_range():
    from pyfwi_b200._native import NativeError
    W = product(cases.tiny_s8(), tile=3)
    W.forward_modeling(cases.tiny_s8()["model_est"])
    for bad in (0, 999, 10 ** 11):
        with pytest.raises(NativeError, match="limit_ns"):
            W.plan.wait_selftest(bad)
    W.plan.check_device()


@pytest.mark.parametrize("tile", [0, 3])
def test_nan_model_propagates_without_fault(tile):
    """A NaN cell spreads through the wavefield like any value; the next
    call on a clean model gives the clean traces again."""
    case = cases.tiny_dxr()
    g = load_golden("tiny_dxr")
    W = product(case, tile=tile)
    bad = {k: v.copy() for k, v in case["model_est"].items()}
    bad["vp"][15, 19] = np.nan
    d = W.forward_modeling(bad)
    assert any(np.isnan(v).any() for v in d.values())
    d = W.forward_modeling(case["model_est"])
    for k, v in d.items():
        assert np.isfinite(v).all() and rel_l2(v, g["d_est_" + k]) < SEIS_TOL, k


def test_layout_beyond_the_memory_budget_is_refused():
    case = cases.tiny_dxr()
    W = product(case)
    W.memory_budget = 1 << 20  # 1 MiB: not even the trace buffers fit
    with pytest.raises(MemoryError, match="does not fit"):
        W.forward_modeling(case["model_est"])
    W.memory_budget = None
    d = W.forward_modeling(case["model_est"])
    g = load_golden("tiny_dxr")
    for k, v in d.items():
        assert rel_l2(v, g["d_est_" + k]) < SEIS_TOL, k


def test_source_outside_the_grid_is_refused():
    from pyfwi_b200._native import NativeError
    case = cases.tiny_dxr()
    case["src_loc"] = case["src_loc"].copy()
    case["src_loc"][1, 0] = 10_000.0  # metres: far right of the 38-cell grid
    with pytest.raises((NativeError, ValueError, IndexError)):
        product(case).forward_modeling(case["model_est"])
