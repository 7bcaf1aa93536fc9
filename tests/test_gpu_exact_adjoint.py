"""The exact adjoint on the GPU (inpa['adjoint'] = 'exact').

1. Against the FP64 oracle's exact gradient (oracle/elastic_oracle.c,
   orc_exact_gradient_shot, itself pinned to central finite differences by
   test_oracle_exact_adjoint.py) on every small case, within the gradient
   tolerance 1e-4 or 3x the float32 rounding of the same arithmetic.
2. Through the torch.autograd.Function (torchfwi.Fwi) on the 200 x 400-cell
   two-layer survey: <dJ/dm, d> against central finite differences of the
   misfit with eps = 1e-3 (relative) on 32 seeded random directions, with the
   reference's gradient's agreement stated beside it."""
import numpy as np
import pytest
from scipy.ndimage import gaussian_filter

import cases
from conftest import load_golden, rel_l2
from helpers import fp64_propagator, product

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4
FIELDS = ["vx", "vz", "taux", "tauz", "tauxz"]
SECTION = {0: ["taux", "tauz"], 1: ["taux"], 2: ["vx", "vz"], 3: ["taux", "tauz", "tauxz"], 4: FIELDS}


def _oracle_exact(case, precision):
    """Oracle: exact model gradient of J = 1/2 sum (section - observed)^2."""
    W = fp64_propagator(case, precision)
    m_obs = {k: v.astype(W.real) for k, v in case["model_obs"].items()}
    m_est = {k: v.astype(W.real) for k, v in case["model_est"].items()}
    obs, est = W.raw_traces(m_obs), W.raw_traces(m_est)
    comp = case["components"]
    if comp == 0:  # both section keys hold (taux + tauz) / 2
        r = ((est["taux"] + est["tauz"]) / 2 - (obs["taux"] + obs["tauz"]) / 2).astype(W.real)
        dtr = {"taux": r, "tauz": r}
    else:
        dtr = {k: est[k] - obs[k] for k in SECTION[comp]}
    return W.model_gradient(m_est, *W.exact_gradient(m_est, dtr))


@pytest.mark.parametrize("name", [f.__name__ for f in cases.TINY])
def test_exact_gradient_matches_fp64_oracle(name):
    """Within 1e-4 of the FP64 oracle, or within 3x the distance of the
    same arithmetic in float32 (the oracle's FP32 build) where rounding in
    float32 alone is larger than that (cancelling gradients)."""
    case = cases.by_name(name)
    W = product(case, adjoint="exact")
    d_obs = W.forward_modeling(case["model_obs"])
    d_est = W.forward_modeling(case["model_est"])
    grad = W.gradient({k: d_est[k] - d_obs[k] for k in d_est}, parameterization="dv")
    ref, ref32 = _oracle_exact(case, "fp64"), _oracle_exact(case, "fp32")
    for k in ("vp", "vs", "rho"):
        err, err32 = rel_l2(grad[k], ref[k]), rel_l2(ref32[k], ref[k])
        print("\n%s %s vs FP64: GPU %.2e, FP32 oracle %.2e" % (name, k, err, err32))
        assert err <= max(GRAD_TOL, 3 * err32), (k, err, err32)


@pytest.mark.parametrize("snapshot,bound", [("bf16", 1e-2), ("fp24", 1e-4)])
@pytest.mark.parametrize("name", ["tiny_dxr", "tiny_dtscale"])
def test_exact_adjoint_with_narrow_snapshots(name, snapshot, bound):
    """The exact adjoint reading BF16 or 24-bit snapshots (FP32 arithmetic;
    S_{t+1} and S_t rounded to 8 or 15 mantissa bits, a segment's FP32
    restart state rounded the same way as it is read): the same gradient
    bits for any recompute segment (the snapshots come from the same FP32
    chain), float32 rounding for another shot grouping, and within 1e-2
    (BF16) of the FP64 oracle's exact gradient; 24 bits within 1e-4, or
    within 3x the distance of the same arithmetic in float32 (the oracle's
    FP32 build) where float32 rounding alone is larger than that."""
    import torch
    case = cases.by_name(name)
    d_obs = product(case).forward_modeling(case["model_obs"])
    out = []
    for seg, batch in ((0, 0), (7, 0), (9, 1)):
        W = product(case, adjoint="exact", snapshot=snapshot, segment=seg, shot_batch=batch)
        d_est = W.forward_modeling(case["model_est"])
        out.append(W.gradient({k: d_est[k] - d_obs[k] for k in d_est}, parameterization="dv"))
        torch.cuda.synchronize()
    ref = _oracle_exact(case, "fp64")
    ref32 = _oracle_exact(case, "fp32") if snapshot == "fp24" else None
    for k in ("vp", "vs", "rho"):
        assert np.array_equal(out[0][k], out[1][k]), k
        assert rel_l2(out[2][k], out[0][k]) < 1e-6, k
        err = rel_l2(out[0][k], ref[k])
        floor = 3 * rel_l2(ref32[k], ref[k]) if ref32 is not None else 0.0
        print("\n%s %s exact adjoint with %s snapshots vs FP64: %.2e (float32 floor %.2e)" % (name, k, snapshot, err,
                                                                                             floor))
        assert err <= max(bound, floor), (k, err)


def _directions(shape, vp, n, eps, seed=2024):
    """n seeded smooth random directions for (vp, vs, rho), each scaled to a
    maximum of 1, zero wherever the perturbation could raise max(vp) (the
    absorbing profiles scale with it)."""
    rng = np.random.default_rng(seed)
    keep = vp * (1 + 3 * eps) < vp.max()
    out = []
    for _ in range(n):
        d = {}
        for k in ("vp", "vs", "rho"):
            f = gaussian_filter(rng.standard_normal(shape), 10.0)
            d[k] = (f / np.abs(f).max() * keep).astype(np.float32)
        out.append(d)
    return out


@pytest.mark.parametrize("snapshot", ["fp32", "fp24", "bf16"])
def test_autograd_gradient_matches_central_differences(snapshot):
    """With FP32 snapshots the median relative error is bounded by 3e-3 (the
    float32 modelling noise at eps = 1e-3); with BF16 snapshots (FP32
    arithmetic, the imaging reads forward states rounded to 8 mantissa bits)
    by 1e-2."""
    import torch
    from pyfwi_b200.torchfwi import Fwi
    case = cases.c2()
    eps, ndir = 1e-3, 32
    dev = torch.device("cuda", 0)
    W = product(case, adjoint="exact", snapshot=snapshot)
    m0 = {k: torch.from_numpy(v).to(dev) for k, v in case["model_est"].items()}
    obs = W.forward_modeling({k: torch.from_numpy(v).to(dev) for k, v in case["model_obs"].items()})
    obs = (obs["taux"].clone(), obs["tauz"].clone())

    def misfit(m):
        tx, tz = Fwi.apply(W, m["vp"], m["vs"], m["rho"])
        return 0.5 * ((tx.double() - obs[0].double()) ** 2).sum() + 0.5 * ((tz.double() - obs[1].double()) ** 2).sum()

    leaves = {k: v.clone().requires_grad_(True) for k, v in m0.items()}
    misfit(leaves).backward()
    grad = {k: v.grad.double() for k, v in leaves.items()}
    # the reference-mode gradient on the same residual: the reference's own
    # gradient of this survey (fixture from PyFWI's WavePropagator) to 1e-4
    Wr = product(case)
    d = Wr.forward_modeling(m0)
    gref = Wr.gradient({k: d[k] - o for k, o in zip(("taux", "tauz"), obs)})
    golden = load_golden("c2_parity")
    ref_err = {k: rel_l2(gref[k].cpu().numpy(), golden["grad_" + k]) for k in gref}
    assert max(ref_err.values()) < 1e-4, ref_err

    rel, rel_ref, err, scale = [], [], [], []
    with torch.no_grad():
        for d in _directions(case["model_est"]["vp"].shape, case["model_est"]["vp"], ndir, eps):
            dm = {k: eps * m0[k] * torch.from_numpy(d[k]).to(dev) for k in d}
            jp = float(misfit({k: m0[k] + dm[k] for k in m0}))
            jm = float(misfit({k: m0[k] - dm[k] for k in m0}))
            fd = (jp - jm) / 2
            pred = sum(float((grad[k] * dm[k].double()).sum()) for k in dm)
            pred_ref = sum(float((gref[k].double() * dm[k].double()).sum()) for k in dm)
            rel.append(abs(pred - fd) / abs(fd))
            rel_ref.append(abs(pred_ref - fd) / abs(fd))
            err.append(abs(pred - fd))
            scale.append(abs(fd))
    rel, rel_ref = np.array(rel), np.array(rel_ref)
    noise = np.array(err) / np.median(scale)
    print("\nFD check (%s snapshots), %d directions, eps %.0e: exact adjoint median %.2e max %.2e (max %.2e of "
          "the median |dJ|) | reference gradient median %.2e"
          % (snapshot, ndir, eps, np.median(rel), rel.max(), noise.max(), np.median(rel_ref)))
    # float32 modelling leaves ~1e-3 of the typical misfit difference as noise
    # at eps = 1e-3 (so directions nearly orthogonal to the gradient show a
    # larger relative error); a wrong adjoint is off by O(1): the reference's
    # gradient, not the derivative of this misfit, is ~100 % off here
    bound = 1e-2 if snapshot == "bf16" else 3e-3
    assert np.median(rel) < bound and noise.max() < 1e-2, (rel, noise)
