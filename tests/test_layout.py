"""The checkpoint layout chooser (WavePreparation._auto_layout) without a
GPU: the device memory query is replaced by fixed numbers and the layout
options are built as the propagator builds them.  For each configuration
the chosen shot batch and recompute segment must fit the memory, and the
choice must match the cost model: on the 64-shot 500 x 1000 survey with a
B200's free memory, all shots in one group with a segment of about
sqrt(2 * free / state) (the box chose 157 with its own free memory); on the
1000 x 3000 thrust-belt survey (128 shots, nt 6000), groups small enough
that the store fits, still large enough to fill the GPU."""
import numpy as np
import pytest
import torch

import cases
from helpers import product

GB = 1 << 30


@pytest.fixture
def free_memory(monkeypatch):
    def set_free(nbytes):
        monkeypatch.setattr(torch.cuda, "mem_get_info", lambda d=None: (int(nbytes), int(180 * GB)))
        monkeypatch.setattr(torch.cuda, "memory_reserved", lambda d=None: 0)
        monkeypatch.setattr(torch.cuda, "memory_allocated", lambda d=None: 0)
    return set_free


def _opts():
    from pyfwi_b200 import _native as N

    def opts(seg, batch):
        o = N.Options()
        o.checkpoint = N.CKPT_EXACT
        o.segment, o.shot_batch = int(seg), int(batch)
        o.snapshot = N.SNAP_FP32
        o.adjoint = N.ADJOINT_REFERENCE
        return o
    return opts


def _layout(case):
    from pyfwi_b200.engine import Plan
    W = product(case, cuda_device="cpu")
    geom, opts = W._geometry(), _opts()
    seg, batch = W._auto_layout(geom, opts, 0, 0)
    return W, seg, batch, Plan.workspace_bytes(geom, opts(seg, batch), int(W.ns))


def test_c3_keeps_all_shots_in_one_group(free_memory):
    free_memory(176 * GB)
    W, seg, batch, ws = _layout(cases.c3())
    assert batch == 64
    assert 140 <= seg <= 170, seg
    assert ws <= 0.9 * 176 * GB
    # the store holds ceil(nt / seg) restart states + seg states of 64 shots
    state = 20.0 * int(W.tnz) * int(W.tnx) * 64
    assert (-(-int(W.nt) // seg) + seg) * state <= ws
    # segments evened out: no shorter segment count would recompute fewer steps
    nt = int(W.nt)
    m = -(-nt // seg)
    assert seg == -(-nt // m), (seg, m)


def test_thrust_belt_survey_fits_and_fills_the_gpu(free_memory):
    free_memory(176 * GB)
    W, seg, batch, ws = _layout(cases.c5())
    assert ws <= 0.9 * 176 * GB
    assert int(W.tnz) * int(W.tnx) * batch >= 8_000_000  # a step launch of thousands of CTAs
    assert seg >= int(np.ceil(np.sqrt(int(W.nt))))
    print("\nthrust-belt survey: %d shots per group, %d-step segments, %.1f GB workspace"
          % (batch, seg, ws / GB))


def test_survey_that_cannot_fit_is_refused(free_memory):
    free_memory(2 * GB)
    with pytest.raises(MemoryError, match="does not fit"):
        _layout(cases.c5())


def test_less_memory_gives_shorter_segments_or_smaller_groups(free_memory):
    out = []
    for g in (176, 90):
        free_memory(g * GB)
        _, seg, batch, _ = _layout(cases.c3())
        out.append((seg, batch))
    (s1, b1), (s2, b2) = out
    assert s2 * b2 <= s1 * b1


def test_graph_auto_stays_off_for_calls_of_many_launches(free_memory):
    """'auto' graph replay: small launches (at most 8 M cell-shots) and calls
    of at most GRAPH_MAX_LAUNCHES launches.  The thrust-belt survey in groups
    of 2 shots (what the layout takes with the observed data of an inversion
    resident) issues over a million launches per gradient: no graph.  The
    100 x 100 survey, one group: graph."""
    free_memory(155 * GB)
    W, seg, batch, _ = _layout(cases.c5())
    assert int(W.tnz) * int(W.tnx) * batch <= W.GRAPH_AUTO_CELLS
    assert not W._graph_on("auto", batch, seg)
    assert W._graph_on(True, batch, seg)  # an explicit request stands (the library runs it directly)
    W1 = product(cases.c1(), cuda_device="cpu")
    assert W1._graph_on("auto", 0, 0)
