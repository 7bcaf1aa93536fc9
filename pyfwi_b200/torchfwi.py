"""``Fwi``: PyFWI's torch.autograd.Function (src/PyFWI/torchfwi.py:7-91).

forward(W, vp, vs, rho) -> (taux, tauz) runs W.forward_modeling; backward
feeds the incoming gradients as the taux / tauz adjoint sources of
W.gradient and returns (None, dL/dvp, dL/dvs, dL/drho).  Tensors stay on
their device (the reference moves everything to the CPU)."""
import torch


class Fwi(torch.autograd.Function):
    @staticmethod
    def forward(ctx, W, vp, vs, rho):
        d = W.forward_modeling({"vp": vp.detach(), "vs": vs.detach(), "rho": rho.detach()}, show=False)
        ctx.WavePropagator = W
        ctx.out_device = vp.device
        return d["taux"].to(vp.device), d["tauz"].to(vp.device)

    @staticmethod
    def backward(ctx, adj_tx, adj_tz):
        W = ctx.WavePropagator
        if adj_tz.ndim == 3:  # (nt, nr, ns) -> (nt, nr*ns), column s*nr + r
            nt, nr, ns = adj_tx.shape
            adj_tx = adj_tx.permute(0, 2, 1).reshape(nt, nr * ns)
            adj_tz = adj_tz.permute(0, 2, 1).reshape(nt, nr * ns)
        g = W.gradient({"taux": adj_tx.detach(), "tauz": adj_tz.detach()}, False)
        dev = ctx.out_device
        return None, g["vp"].to(dev), g["vs"].to(dev), g["rho"].to(dev)
