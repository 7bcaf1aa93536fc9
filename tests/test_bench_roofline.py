"""The benchmark's roofline accounting, on the CPU: algorithmic bytes per
launch of each step kernel (with difference sets the forward steps also
write every shot-step's five imaged values once; the imaging reads them at
their stored width), the dominant kernel, and the ncu traffic taken from the
committed one-pass captures only where store and snapshot format match."""
import os

import pytest

import bench

NCELL, NINT, NS, NT = 560.0 * 1060.0, 495509.0, 64, 4000
CELLS = NCELL * NS  # cell-shots of one 64-shot launch
PROFILES = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "profiles")


def _prof(n_fwd=7850, ms_fwd=3995.6, n_adj=3999, ms_adj=3319.0):
    return {0: (n_fwd, ms_fwd, n_fwd * CELLS), 1: (n_adj, ms_adj, n_adj * CELLS), 2: (0, 0.0, 0.0)}


def _roof(store="differences", snapshot="fp32", prof=None, traffic_dir=PROFILES):
    prof = prof or _prof()
    return bench.roofline(prof, 7360.0, NCELL, NINT, NS, NT, 1, store, snapshot, 6547.2, "measured", traffic_dir)


def test_adjoint_bytes_per_launch():
    r = _roof()
    adj = r["per_kernel"]["adj_step"]
    assert adj["alg_bytes_per_launch"] == pytest.approx(NS * (52 * NCELL + 44 * NINT))
    assert adj["avg_launch_ms"] == pytest.approx(3319.0 / 3999)
    assert adj["frac"] == pytest.approx(adj["achieved"] / 6547.2)
    # 24-bit values: 15 B of imaged values per imaged cell instead of 20
    r24 = _roof(snapshot="fp24")
    assert r24["per_kernel"]["adj_step"]["alg_bytes_per_launch"] == pytest.approx(NS * (52 * NCELL + 39 * NINT))


def test_forward_bytes_count_the_difference_sets_once_per_shot_step():
    diff = _roof()["per_kernel"]["fwd_step"]["alg_bytes_per_launch"]
    states = _roof(store="states")["per_kernel"]["fwd_step"]["alg_bytes_per_launch"]
    assert states == pytest.approx(52 * CELLS)
    assert diff * 7850 == pytest.approx(7850 * 52 * CELLS + 20 * NINT * NS * NT)


def test_dominant_kernel_and_shares():
    r = _roof()
    assert r["kernel"] == "fwd_step"
    assert r["kernel_share"]["fwd_step"] == pytest.approx(3995.6 / 7360.0)
    r = _roof(prof=_prof(ms_fwd=3000.0, ms_adj=4100.0))
    assert r["kernel"] == "adj_step" and r["achieved"] == r["per_kernel"]["adj_step"]["achieved"]


def test_traffic_only_from_a_matching_capture():
    r = _roof()
    assert r["traffic"] == pytest.approx(49.54 * CELLS, rel=1e-3)  # traffic_fwd_step_c3_differences.json
    assert r["traffic_source"]["shots_per_launch"] == 64
    assert r["per_kernel"]["adj_step"]["traffic"] == pytest.approx(79.82 * CELLS, rel=1e-3)
    assert _roof(store="states")["traffic"] == pytest.approx(40.95 * CELLS, rel=1e-3)
    assert _roof(snapshot="fp24")["traffic"] is None  # no capture of the 24-bit kernels
    assert _roof(traffic_dir=None)["traffic"] is None
