"""``prepare_residual`` with PyFWI's interface (src/PyFWI/processing.py:142-158)."""
import numpy as np

COMPONENTS = ["vx", "vz", "taux", "tauz", "tauxz"]


def prepare_residual(res, s=1.):
    """Scale every component by s and fill the missing ones with zeros.
    Works on numpy arrays and on torch tensors."""
    data = {}
    first = res[[*res][0]]
    for p in COMPONENTS:
        if p in res:
            data[p] = s * res[p]
        elif isinstance(first, np.ndarray):
            data[p] = np.zeros(first.shape, np.float32)
        else:
            import torch
            data[p] = torch.zeros(first.shape, dtype=torch.float32, device=first.device)
    return data
