"""Memory check of every kernel path (the GPU pool has no sanitizer).

Each plane of the workspace sits in a frame of zero cells that the stencils
read and no kernel writes (update domains stop short of it).  After forward
modelling and a gradient on every geometry and kernel variant,
pyfwi_frame_check counts the nonzero frame cells of every FP32 plane
(materials, work and adjoint states, gradient accumulators, checkpoint
store): a write outside a kernel's domain, or a NaN leaking there, shows as
a nonzero count."""
import numpy as np
import pytest
import torch

import cases
from conftest import load_golden
from helpers import l2_residual_np, product

pytestmark = pytest.mark.gpu

NAMES = ["c1"] + [f.__name__ for f in cases.TINY]


def _golden_section(g, prefix):
    return {k[len(prefix):]: g[k] for k in g if k.startswith(prefix)}


def _run(name, **extra):
    g = load_golden(name)
    case = cases.by_name(name)
    W = product(case, **extra)
    W.forward_modeling(case["model_est"])
    res = l2_residual_np(_golden_section(g, "d_est_"), _golden_section(g, "d_obs_"))
    W.gradient({k: v for k, v in res.items() if np.any(v)}, parameterization=case["param"])
    return W


@pytest.mark.parametrize("tile", [0, 3, 7, 8])
@pytest.mark.parametrize("name", NAMES)
def test_no_write_outside_the_domains(name, tile):
    W = _run(name, tile=tile)
    assert W.plan.frame_check() == 0


@pytest.mark.parametrize("extra", [{"tile": 1}, {"tile": 2}, {"tile": 4}, {"tile": 5}, {"tile": 6}, {"tile": 9}, {"tile": 11},
                                   {"tile": 10}, {"persist": True, "segment": 0, "shot_batch": 0},
                                   {"snapshot": "fp24", "segment": 7}, {"overlap": True, "segment": 7}, {"tile": 0, "adj_tile": 3},
                                   {"segment": 7, "shot_batch": 1}, {"snapshot": "bf16", "segment": 9},
                                   {"graph": True}, {"graph": False}])
def test_no_write_outside_the_domains_variants(extra):
    W = _run("tiny_s8", **extra)  # 8th order, energy terms, all components
    assert W.plan.frame_check() == 0


@pytest.mark.parametrize("name,extra", [("tiny_s8", {"energy_balancing": False, "segment": 7}),
                                        ("tiny_s8", {"energy_balancing": False, "tile": 2}),
                                        ("c1", {"store": "states"}), ("tiny_dtscale", {"segment": 11, "overlap": True}),
                                        ("tiny_dtscale", {"snapshot": "fp24", "segment": 11}),
                                        ("tiny_s8", {"energy_balancing": False, "snapshot": "fp24", "segment": 9}),
                                        ("tiny_dxr", {"segment": 9, "tile": 1, "graph": True})])
def test_no_write_outside_the_domains_stored_differences(name, extra):
    """Difference sets in the checkpoint segments (the default where they
    apply; the 8th-order stencil without energy terms, recompute segments,
    overlap, graph replay), and stored states where they would apply."""
    W = _run(name, **extra)
    assert W.plan.store_diffs == (extra.get("store", "differences") == "differences")
    assert W.plan.frame_check() == 0


@pytest.mark.parametrize("name", ["tiny_dxr", "tiny_dtscale"])
@pytest.mark.parametrize("snapshot", ["fp32", "bf16"])
def test_no_write_outside_the_domains_exact_adjoint(name, snapshot):
    case = cases.by_name(name)
    W = product(case, adjoint="exact", snapshot=snapshot, segment=7)
    d = W.forward_modeling(case["model_est"])
    W.gradient({k: 0.01 * v for k, v in d.items()}, parameterization="dv")
    assert W.plan.frame_check() == 0


def test_no_write_outside_the_domains_fused_misfit():
    case = cases.tiny_both()
    g = load_golden("tiny_both")
    W = product(case)
    obs = {k: torch.from_numpy(v).cuda() for k, v in _golden_section(g, "d_obs_").items()}
    W.misfit_gradient({k: torch.from_numpy(v).cuda() for k, v in case["model_est"].items()}, obs)
    assert W.plan.frame_check() == 0


def test_frame_check_sees_a_planted_value():
    """The check itself: a value written on purpose (through the workspace
    tensor) into the frame cell (row 0, column 0) of the first material
    plane is counted, and counts no more once removed.  That plane starts
    after the 256-byte header, the source cells (2 x ns int32, rounded up to
    256 bytes) and the reduction scratch (PYFWI_REDUCE_SLOTS doubles), on the
    next multiple of the workspace's row alignment (the row of pitch floats,
    or two rows when that is not a multiple of 256 bytes)."""
    from pyfwi_b200 import _native as N
    W = _run("tiny_dxr")
    plan = W.plan
    assert plan.frame_check() == 0
    ws = plan._ws
    base = (ws.data_ptr() + 255) // 256 * 256 - ws.data_ptr()
    pitch = -(-(int(W.tnx) + 16) // 32) * 32
    row = pitch * 4
    ra = row if row % 256 == 0 else 2 * row

    def up(x, a=256):
        return -(-x // a) * a
    o_mat = up(256 + up(2 * int(W.ns) * 4) + up(N.REDUCE_SLOTS * 8), ra)
    cell = ws[base + o_mat:base + o_mat + 4].view(torch.float32)
    assert float(cell[0]) == 0.0
    cell[0] = 1.0
    assert plan.frame_check() == 1
    cell[0] = 0.0
    assert plan.frame_check() == 0
