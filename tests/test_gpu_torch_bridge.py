"""torchfwi.Fwi with the reference's adjoint (torchfwi.py:32-91): the gradient
autograd returns for L = 1/2 |taux - obs_x|^2 + 1/2 |tauz - obs_z|^2 is the
reference's WavePropagator.gradient on that residual, within 1e-4 relative
L2 of the reference's own output.

* the 200 x 400, 10-shot, 2000-step survey (the configuration of the torch
  gradient check), '2d' sections;
* the sub-stepped tiny survey with '3d' sections (nt, nr, ns): the
  adjoints reach backward in that shape and are laid out as the reference's
  Fortran-order reshape (torchfwi.py:71-74) before the gradient."""
import numpy as np
import pytest

import cases
from conftest import load_golden, rel_l2
from helpers import product

pytestmark = pytest.mark.gpu
GRAD_TOL = 1e-4


def _autograd_gradient(W, model, obs):
    import torch
    from pyfwi_b200.torchfwi import Fwi
    leaves = {k: v.clone().requires_grad_(True) for k, v in model.items()}
    tx, tz = Fwi.apply(W, leaves["vp"], leaves["vs"], leaves["rho"])
    assert tx.shape == obs[0].shape and tz.shape == obs[1].shape
    loss = 0.5 * ((tx.double() - obs[0].double()) ** 2).sum() + 0.5 * ((tz.double() - obs[1].double()) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    return {k: v.grad.cpu().numpy() for k, v in leaves.items()}, float(loss)


def test_reference_adjoint_through_autograd_on_the_200x400_survey():
    import torch
    dev = torch.device("cuda", 0)
    case = cases.c2_parity()
    g = load_golden("c2_parity")
    W = product(case)
    obs = W.forward_modeling({k: torch.from_numpy(v).to(dev) for k, v in case["model_obs"].items()})
    obs = (obs["taux"].clone(), obs["tauz"].clone())
    model = {k: torch.from_numpy(v).to(dev) for k, v in case["model_est"].items()}
    grad, loss = _autograd_gradient(W, model, obs)
    errs = {k: rel_l2(grad[k], g["grad_" + k]) for k in grad}
    assert max(errs.values()) < GRAD_TOL, errs
    # the misfit of the reference (CostFunction l2 over both stress keys)
    assert abs(loss - float(g["rms"])) <= 1e-4 * float(g["rms"]), (loss, float(g["rms"]))


@pytest.mark.parametrize("shape", ["2d", "3d"])
def test_reference_adjoint_through_autograd_section_shapes(shape):
    import torch
    dev = torch.device("cuda", 0)
    case = cases.tiny_dtscale()
    assert case["components"] == 0
    g = load_golden("tiny_dtscale")
    case["inpa"] = dict(case["inpa"], seimogram_shape=shape)
    W = product(case)
    obs = []
    for k in ("taux", "tauz"):
        o = g["d_obs_" + k]
        if shape == "3d":  # the reference's '2d' section is the Fortran-order reshape of (nt, nr, ns)
            o = np.reshape(o, (o.shape[0], int(W.nr), int(W.ns)), order="F")
        obs.append(torch.from_numpy(np.ascontiguousarray(o)).to(dev))
    model = {k: torch.from_numpy(v).to(dev) for k, v in case["model_est"].items()}
    grad, _ = _autograd_gradient(W, model, tuple(obs))
    errs = {k: rel_l2(grad[k], g["grad_" + k]) for k in grad}
    assert max(errs.values()) < GRAD_TOL, errs
