"""Shots across ranks: one process per GPU, each modelling its own shots;
the gradient and the misfit are summed over ranks with one all-reduce per
evaluation (the only exchange step of an FWI gradient).

The reference runs all shots in one process (wave_propagation.py:639, :740);
shots are independent, so a rank-local gradient over a subset of shots plus
a sum over ranks equals the single-process gradient up to float32 summation
order."""
import numpy as np


def shard_shots(n_shots, rank, world):
    """Indices of the shots rank `rank` of `world` owns (contiguous blocks,
    sizes differing by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(int(n_shots), int(world))
    lo = rank * base + min(rank, extra)
    return np.arange(lo, lo + base + (1 if rank < extra else 0))


def shard_sources(src, rank, world):
    """A copy of an acquisition.Source keeping only this rank's shots."""
    import copy
    idx = shard_shots(src.i.size, rank, world)
    out = copy.copy(src)
    out.i = src.i[idx]
    out.j = src.j[idx]
    return out, idx


def allreduce_gradient(grad, rms=None, group=None):
    """Sum a gradient (dict of tensors, or one tensor) and optionally the
    misfit over the ranks of `group`, in place."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return grad, rms
    if isinstance(grad, dict):
        keys = list(grad)
        flat = torch.stack([grad[k] for k in keys])
        dist.all_reduce(flat, group=group)
        for q, k in enumerate(keys):
            grad[k].copy_(flat[q])
    else:
        dist.all_reduce(grad, group=group)
    if rms is not None:
        dist.all_reduce(rms, group=group)
    return grad, rms


def trace_columns(shots, nr):
    """Columns of the (nt, nr*ns) trace layout that belong to `shots`."""
    shots = np.asarray(shots)
    return (shots[:, None] * nr + np.arange(nr)[None, :]).reshape(-1)
