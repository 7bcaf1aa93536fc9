"""Parity of the CUDA path with the reference's own outputs (golden
fixtures: PyFWI's WavePropagator and kernels run on the CPU).

Tolerances (relative L2 per component): seismograms 1e-5, gradients 1e-4;
index work (which trace is which, where sources and receivers sit) is
checked through the traces themselves."""
import numpy as np
import pytest

import cases
from conftest import load_golden, rel_l2
from helpers import l2_residual_np, product

pytestmark = pytest.mark.gpu

SEIS_TOL = 1e-5
GRAD_TOL = 1e-4
NAMES = ["c1"] + [f.__name__ for f in cases.TINY]


def _golden_section(g, prefix):
    return {k[len(prefix):]: g[k] for k in g if k.startswith(prefix)}


# tile kernel (64 x 16), the streaming kernels (128 / 64 / 256 columns), the
# tile kernels whose adjoint CTAs carry 2 / 4 shots, the TMA-staged tile
# forward (64 x 16), the adjoint with prefetched accumulators
VARIANTS = [0, 3, 4, 5, 6, 7, 8, 11]


@pytest.mark.parametrize("tile", VARIANTS)
@pytest.mark.parametrize("name", NAMES)
def test_forward_and_gradient_match_reference(name, tile):
    g = load_golden(name)
    case = cases.by_name(name)
    W = product(case, tile=tile)
    d_obs = W.forward_modeling(case["model_obs"])
    for k, v in d_obs.items():
        assert v.dtype == np.float32 and v.shape == g["d_obs_" + k].shape
        assert rel_l2(v, g["d_obs_" + k]) < SEIS_TOL, ("d_obs", k, rel_l2(v, g["d_obs_" + k]))
    d_est = W.forward_modeling(case["model_est"])
    for k, v in d_est.items():
        assert rel_l2(v, g["d_est_" + k]) < SEIS_TOL, ("d_est", k, rel_l2(v, g["d_est_" + k]))
    if "seis_vx" in g:
        raw = W.seismogram
        for k, v in raw.items():
            assert rel_l2(v, g["seis_" + k]) < SEIS_TOL, ("seis", k)
    # gradient on the reference's own residual (same inputs as the reference)
    res = l2_residual_np(_golden_section(g, "d_est_"), _golden_section(g, "d_obs_"))
    res = {k: v for k, v in res.items() if np.any(v)}
    grad = W.gradient(res, parameterization=case["param"])
    for k, v in grad.items():
        assert v.shape == g["grad_" + k].shape
        assert rel_l2(v, g["grad_" + k]) < GRAD_TOL, ("grad", k, rel_l2(v, g["grad_" + k]))


@pytest.mark.parametrize("name", ["c1", "tiny_s8", "tiny_chpr"])
def test_end_to_end_gradient_within_tolerance(name):
    """Residual from the product's own modelled data against the reference's
    observed data: the gradient an FWI iteration would use."""
    g = load_golden(name)
    case = cases.by_name(name)
    W = product(case)
    d_est = W.forward_modeling(case["model_est"])
    res = l2_residual_np(d_est, _golden_section(g, "d_obs_"))
    res = {k: v for k, v in res.items() if np.any(v)}
    grad = W.gradient(res, parameterization=case["param"])
    for k, v in grad.items():
        assert rel_l2(v, g["grad_" + k]) < GRAD_TOL, ("grad", k, rel_l2(v, g["grad_" + k]))


@pytest.mark.parametrize("name", ["tiny_dxr", "tiny_both"])
def test_three_d_section_shape(name):
    """inpa['seimogram_shape'] = '3d': sections come as (nt, nr, ns), the
    reference's array before its Fortran-order reshape to '2d'
    (acquisition.py:313-333)."""
    g = load_golden(name)
    case = cases.by_name(name)
    case["inpa"] = dict(case["inpa"], seimogram_shape="3d")
    W = product(case)
    d = W.forward_modeling(case["model_est"])
    for k, v in d.items():
        ref2 = g["d_est_" + k]
        nt, nrs = ref2.shape
        assert v.shape == (nt, int(W.nr), int(W.ns)), (k, v.shape)
        assert rel_l2(np.reshape(v, (nt, nrs), order="F"), ref2) < SEIS_TOL, k


@pytest.mark.parametrize("tile", VARIANTS + [1, 2])
def test_fluid_keeps_normal_stresses_equal(tile):
    """In the water layer (mu = 0) the reference's txx and tzz stay the same
    float at every step (its receivers there record identical traces); a
    rounding difference between them would have nothing to restore it and
    would grow into the velocities.  Every forward variant keeps them equal
    bit for bit, and the velocity traces near the sources stay within the
    seismogram tolerance."""
    g = load_golden("tiny_water")
    assert np.array_equal(g["seis_taux"], g["seis_tauz"])
    case = cases.tiny_water()
    W = product(case, tile=tile)
    W.forward_modeling(case["model_est"])
    raw = W.seismogram
    assert np.array_equal(raw["taux"], raw["tauz"])
    for k in ("vx", "vz"):
        assert rel_l2(raw[k], g["seis_" + k]) < SEIS_TOL, (k, rel_l2(raw[k], g["seis_" + k]))


def test_exact_checkpoint_segments_are_bit_identical():
    """Recomputing the forward in segments from restart states gives the
    same gradient bits as storing every step."""
    import torch
    case = cases.tiny_s8()
    g = load_golden("tiny_s8")
    res = l2_residual_np(_golden_section(g, "d_est_"), _golden_section(g, "d_obs_"))
    out = []
    for seg, batch in ((0, 0), (7, 0), (32, 1)):
        W = product(case, segment=seg, shot_batch=batch)
        W.forward_modeling(case["model_est"])
        out.append(W.gradient(res, parameterization="lmd"))
        torch.cuda.synchronize()
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k
        assert rel_l2(out[2][k], out[0][k]) < 1e-6, k


@pytest.mark.parametrize("name,seg,batch", [("tiny_s8", 7, 0), ("tiny_s8", 9, 1), ("c1", 50, 0), ("tiny_dtscale", 11, 0)])
def test_overlapped_recompute_gives_the_same_bits(name, seg, batch):
    """inpa['overlap']: the recompute of each segment runs on a second stream
    beside the adjoint of the segment after it (two segment buffers); the
    seismograms and gradients are the one-stream schedule's bit for bit."""
    import torch
    case = cases.by_name(name)
    g = load_golden(name)
    res = l2_residual_np(_golden_section(g, "d_est_"), _golden_section(g, "d_obs_"))
    res = {k: v for k, v in res.items() if np.any(v)}
    out = []
    for overlap in (False, True):
        W = product(case, segment=seg, shot_batch=batch, overlap=overlap)
        d = W.forward_modeling(case["model_est"])
        out.append((d, W.gradient(res, parameterization=case["param"])))
        torch.cuda.synchronize()
        assert W.plan.opts.overlap == int(overlap)
    for a, b in zip(out[0], out[1]):
        for k in a:
            assert np.array_equal(a[k], b[k]), (name, k)
    for k, v in out[1][1].items():
        assert rel_l2(v, g["grad_" + k]) < GRAD_TOL, k


def _c1_tile_corner_sources():
    """C1 with its four sources where the stencils of the cells next to them
    cross the 64 x 16 tile boundaries (padded cells (31, 63), (32, 64),
    (31, 65), (33, 62))."""
    case = cases.c1()
    dh = case["inpa"]["dh"]
    case["src_loc"] = np.array([[43, 11], [44, 12], [45, 11], [42, 13]], np.float32) * dh
    case["name"] = "c1_corners"
    return case


@pytest.mark.parametrize("name,seg,batch,extra", [
    ("c1", 0, 0, {}), ("c1", 50, 0, {}), ("c1", 37, 1, {"overlap": True}), ("c1_corners", 0, 0, {}),
    ("c1_corners", 64, 2, {}), ("tiny_dtscale", 11, 0, {}), ("tiny_both", 13, 0, {}), ("tiny_water", 0, 0, {}),
    ("tiny_dxr", 9, 0, {}), ("tiny_crosswell", 10, 0, {"checkpoint": "exact"}),
    ("tiny_s8", 7, 0, {"energy_balancing": False}), ("tiny_s8", 0, 0, {"energy_balancing": False, "tile": 1}),
    ("c1", 0, 0, {"tile": 2})])
def test_stored_differences_match_stored_states(name, seg, batch, extra):
    """inpa['store'] = 'differences': the forward steps that fill the
    checkpoint segments store the five differences of each state the imaging
    reads (the stress ones of a state written by the step that reads it, with
    the source of that step taken out), and the adjoint step reads them.  The
    seismograms are those of storing states bit for bit, the gradients agree to
    float32 rounding (the same operations in the same order), and where the
    case has golden fixtures they stay within the gradient bar."""
    import torch
    case = _c1_tile_corner_sources() if name == "c1_corners" else cases.by_name(name)
    W0 = product(case, segment=seg, shot_batch=batch, store="states", **extra)
    d_obs = W0.forward_modeling(case["model_obs"])
    d_est = W0.forward_modeling(case["model_est"])
    res = l2_residual_np(d_est, d_obs)
    res = {k: v for k, v in res.items() if np.any(v)}
    out = []
    for store in ("states", "differences"):
        W = product(case, segment=seg, shot_batch=batch, store=store, **extra)
        d = W.forward_modeling(case["model_est"])
        out.append((d, W.gradient(res, parameterization=case["param"])))
        torch.cuda.synchronize()
        assert W.plan.store_diffs == (store == "differences"), store
    for k in out[0][0]:
        assert np.array_equal(out[0][0][k], out[1][0][k]), ("seismogram", k)
    for k, v in out[1][1].items():
        assert rel_l2(v, out[0][1][k]) < 1e-6, (k, rel_l2(v, out[0][1][k]))
    if name in cases.__dict__ and case["chpr"] == 100 and not extra:
        g = load_golden(name)
        res = l2_residual_np(_golden_section(g, "d_est_"), _golden_section(g, "d_obs_"))
        res = {k: v for k, v in res.items() if np.any(v)}
        W = product(case, segment=seg, shot_batch=batch)
        W.forward_modeling(case["model_est"])
        for k, v in W.gradient(res, parameterization=case["param"]).items():
            assert rel_l2(v, g["grad_" + k]) < GRAD_TOL, ("grad", k)


@pytest.mark.parametrize("name,seg,batch,extra", [
    ("c1", 0, 0, {}), ("c1", 50, 0, {}), ("c1_corners", 64, 2, {}), ("tiny_dtscale", 11, 0, {}),
    ("tiny_s8", 7, 0, {"energy_balancing": False})])
def test_24_bit_stored_differences(name, seg, batch, extra):
    """inpa['snapshot'] = 'fp24' with stored differences: the difference sets
    kept in 24 bits (a BF16 plane and a byte plane, three quarters of the FP32
    store).  Each value is rounded once, after the differencing, so the
    gradient stays within 1e-5 of the FP32 difference sets (rounding the
    states before differencing costs far more: test_gpu_fp64_error)."""
    import torch
    case = _c1_tile_corner_sources() if name == "c1_corners" else cases.by_name(name)
    W0 = product(case, segment=seg, shot_batch=batch, **extra)
    d_obs = W0.forward_modeling(case["model_obs"])
    d_est = W0.forward_modeling(case["model_est"])
    res = l2_residual_np(d_est, d_obs)
    res = {k: v for k, v in res.items() if np.any(v)}
    out = []
    for snapshot in ("fp32", "fp24"):
        W = product(case, segment=seg, shot_batch=batch, snapshot=snapshot, **extra)
        d = W.forward_modeling(case["model_est"])
        out.append((d, W.gradient(res, parameterization=case["param"])))
        torch.cuda.synchronize()
        assert W.plan.store_diffs
    for k in out[0][0]:
        assert np.array_equal(out[0][0][k], out[1][0][k]), ("seismogram", k)
    for k, v in out[1][1].items():
        assert rel_l2(v, out[0][1][k]) < 1e-5, (k, rel_l2(v, out[0][1][k]))


def test_tile_variants_agree():
    """Tile kernels of every height give identical bits (forward and
    gradient); streaming kernels (other FMA grouping) agree to float32
    rounding; the variants whose adjoint CTAs carry several shots run the
    forward of variant 0 (identical bits) and sum the shots' imaging in
    another order (float32 rounding); the TMA-staged tile kernels give the
    tile kernels' bits.  All with stored states (difference sets apply to
    the tile kernels 0..2 only: test_stored_differences_match_stored_states)."""
    case = cases.tiny_dxr()
    g = load_golden("tiny_dxr")
    res = l2_residual_np(_golden_section(g, "d_est_"), _golden_section(g, "d_obs_"))
    base = None
    for tile in range(12):
        W = product(case, tile=tile, store="states")
        d = W.forward_modeling(case["model_est"])
        gr = W.gradient(res, parameterization=case["param"])
        if base is None:
            base = (d, gr)
        for out, ref, is_grad in ((d, base[0], False), (gr, base[1], True)):
            for k in out:
                if tile < 3 or tile >= 8 or (tile >= 6 and not is_grad):
                    assert np.array_equal(out[k], ref[k]), (tile, k)
                else:
                    assert rel_l2(out[k], ref[k]) < 1e-6, (tile, k)


@pytest.mark.parametrize("chunk", [3, 8, 1000])
def test_streaming_row_chunks_agree(chunk):
    """Splitting the rows among CTAs does not change the result."""
    case = cases.tiny_s8()
    g = load_golden("tiny_s8")
    W = product(case, tile=3, chunk=chunk)
    d = W.forward_modeling(case["model_est"])
    for k, v in d.items():
        assert rel_l2(v, g["d_est_" + k]) < SEIS_TOL, k
    res = l2_residual_np(_golden_section(g, "d_est_"), _golden_section(g, "d_obs_"))
    grad = W.gradient(res, parameterization="lmd")
    for k, v in grad.items():
        assert rel_l2(v, g["grad_" + k]) < GRAD_TOL, k


@pytest.mark.parametrize("fwd,adj", [(0, 3), (3, 0), (4, 5)])
def test_mixed_forward_and_adjoint_variants(fwd, adj):
    """A forward variant and a different adjoint variant in one plan."""
    case = cases.tiny_s8()
    g = load_golden("tiny_s8")
    W = product(case, tile=fwd, adj_tile=adj)
    assert (W.tile, W.adj_tile) == (fwd, adj)
    d = W.forward_modeling(case["model_est"])
    for k, v in d.items():
        assert rel_l2(v, g["d_est_" + k]) < SEIS_TOL, k
    res = l2_residual_np(_golden_section(g, "d_est_"), _golden_section(g, "d_obs_"))
    grad = W.gradient(res, parameterization="lmd")
    for k, v in grad.items():
        assert rel_l2(v, g["grad_" + k]) < GRAD_TOL, k


def test_autotuned_variants():
    """tile='auto' times every variant on the survey and runs the fastest
    forward and adjoint kernels; the result still matches the reference."""
    from pyfwi_b200 import autotune
    case = cases.tiny_chpr()
    g = load_golden("tiny_chpr")
    from pyfwi_b200 import _native as N
    W = product(case, tile="auto")
    n = N.lib().pyfwi_tile_count(int(W.sdo))
    assert n == 12
    assert 0 <= W.tile < n and 0 <= W.adj_tile < n
    tables = [t for (_, _, t) in autotune._CACHE.values()]
    assert any(sorted(t) == list(range(n)) and all(a > 0 and b > 0 for a, b in t.values()) for t in tables)
    d = W.forward_modeling(case["model_est"])
    for k, v in d.items():
        assert rel_l2(v, g["d_est_" + k]) < SEIS_TOL, k
    res = l2_residual_np(_golden_section(g, "d_est_"), _golden_section(g, "d_obs_"))
    grad = W.gradient(res, parameterization=case["param"])
    for k, v in grad.items():
        assert rel_l2(v, g["grad_" + k]) < GRAD_TOL, k


def test_tensor_inputs_stay_on_device():
    import torch
    case = cases.tiny_dtscale()
    W = product(case)
    m = {k: torch.from_numpy(v).cuda() for k, v in case["model_est"].items()}
    d = W.forward_modeling(m)
    assert all(isinstance(v, torch.Tensor) and v.is_cuda for v in d.values())
    res = {k: v * 0.5 for k, v in d.items()}
    gr = W.gradient(res)
    assert all(isinstance(v, torch.Tensor) and v.is_cuda for v in gr.values())
    W2 = product(case)
    d2 = W2.forward_modeling(case["model_est"])
    for k in d:
        assert np.array_equal(d[k].cpu().numpy(), d2[k])


@pytest.mark.parametrize("name,extra", [("c1", {}), ("tiny_dtscale", {"segment": 0, "shot_batch": 1}),
                                        ("tiny_chpr", {}), ("tiny_s8", {"segment": 9, "shot_batch": 3}),
                                        ("tiny_s8", {"adjoint": "exact", "shot_batch": 2, "segment": 0})])
def test_misfit_gradient_matches_separate_calls(name, extra):
    """misfit_gradient (forward, residual and adjoint fused per shot group)
    gives the misfit and gradient of forward_modeling + CostFunction('l2') +
    gradient, also when the shots run in several groups."""
    import torch
    from pyfwi_b200 import fwi_tools
    case = cases.by_name(name)
    g = load_golden(name)
    obs = _golden_section(g, "d_obs_")
    W = product(case, **extra)
    d_est = W.forward_modeling(case["model_est"])
    rms_a, res = fwi_tools.CostFunction("l2")(d_est, obs)
    grad_a = W.gradient(res, parameterization=case["param"])
    W2 = product(case, **extra)
    rms_b, grad_b = W2.misfit_gradient(case["model_est"], obs, parameterization=case["param"])
    torch.cuda.synchronize()
    assert abs(rms_b - rms_a) <= 1e-6 * abs(rms_a), (rms_a, rms_b)
    for k in grad_a:
        assert rel_l2(grad_b[k], grad_a[k]) <= 1e-6, k
    if "adjoint" not in extra:
        for k in grad_b:
            assert rel_l2(grad_b[k], g["grad_" + k]) < GRAD_TOL, k
    # the modelled traces are those of forward_modeling
    for k, v in W2.seismogram.items():
        assert np.array_equal(v, W.seismogram[k]), k


@pytest.mark.parametrize("name", ["tiny_dtscale", "tiny_s8"])
def test_graph_replay_of_misfit_gradient(name):
    """misfit_gradient with inpa['graph'] = True (one captured graph per
    plan, replayed with the observed data and adjoint buffers copied
    through): the same misfit, gradient and adjoint source bits as direct
    launches, over changing models and observed data."""
    import torch
    case = cases.by_name(name)
    g = load_golden(name)
    obs = {k: torch.from_numpy(v).cuda() for k, v in _golden_section(g, "d_obs_").items()}
    scaled = {k: (v * np.float32(1.02)) for k, v in case["model_est"].items()}
    direct, replay = product(case), product(case, graph=True)
    for model, o in ((case["model_est"], obs), (scaled, obs), (case["model_est"], {k: 1.1 * v for k, v in obs.items()})):
        m = {k: torch.from_numpy(v).cuda() for k, v in model.items()}
        ra, ga = direct.misfit_gradient(m, o, parameterization=case["param"])
        rb, gb = replay.misfit_gradient(m, o, parameterization=case["param"])
        torch.cuda.synchronize()
        assert float(ra) == pytest.approx(float(rb), rel=1e-12)  # double atomics: summation order
        for k in ga:
            assert torch.equal(ga[k], gb[k]), k
        for k, v in direct._adjoint_source.items():
            assert torch.equal(v, replay._adjoint_source[k]), k


def test_graph_replay_matches_direct_launches():
    """inpa['graph'] = True captures each forward / gradient call as a CUDA
    graph on first use and replays it after: same bits as direct launches,
    also when the model changes between calls (set_model is not captured)."""
    import torch
    case = cases.tiny_dtscale()
    g = load_golden("tiny_dtscale")
    res = l2_residual_np(_golden_section(g, "d_est_"), _golden_section(g, "d_obs_"))
    scaled = {k: (v * np.float32(1.02)) for k, v in case["model_est"].items()}
    direct, replay = product(case), product(case, graph=True)
    for model in (case["model_est"], case["model_est"], scaled):
        a = direct.forward_modeling(model), direct.gradient(res, parameterization="dv")
        b = replay.forward_modeling(model), replay.gradient(res, parameterization="dv")
        torch.cuda.synchronize()
        for da, db in zip(a, b):
            for k in da:
                assert np.array_equal(da[k], db[k]), k
