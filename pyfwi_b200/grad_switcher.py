"""Chain rule between (lam, mu, rho) and (vp, vs, rho) gradients with PyFWI's
interface (src/PyFWI/grad_switcher.py:331-447).  On the device path the
conversion runs inside the gradient kernel; these host versions serve callers
that hold numpy gradients."""
import numpy as np


def grad_lmd_to_vd(glam, gmu, grho, lam, mu, rho):
    """d/d(vp, vs, rho) from d/d(lam, mu, rho), float32 as the reference."""
    vp = np.sqrt((lam + 2 * mu) / rho)
    vs = np.sqrt(mu / rho)
    vs2 = vs ** 2
    vpvs = vp ** 2 - 2 * vs ** 2
    gvp = glam * 2 * vp * rho + gmu * 0 + grho * 0
    gvs = glam * (-4 * rho * vs) + gmu * 2 * vs * rho + grho * 0
    grho_out = glam * vpvs + gmu * vs2 + grho
    return gvp.astype(np.float32), gvs.astype(np.float32), grho_out.astype(np.float32)


def grad_vd_to_lmd(gvp, gvs, grho, vp, vs, rho):
    """d/d(lam, mu, rho) from d/d(vp, vs, rho)."""
    glam = gvp / (2 * rho * vp) + gvs * 0 + grho * 0
    gmu = gvp / (rho * vp) + gvs / (2 * rho * vs) + grho * 0
    grho_out = gvp * (- vp / 2 / rho) + gvs * (- vs / 2 / rho) + grho
    return glam.astype(np.float32), gmu.astype(np.float32), grho_out.astype(np.float32)
