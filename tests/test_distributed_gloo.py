"""The multi-rank path on CPU: two gloo ranks each take half of the shots,
compute their gradient (with the CPU oracle standing in for the device),
and the all-reduce of pyfwi_b200.distributed gives the gradient of all
shots."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from pyfwi_b200.distributed import allreduce_gradient, shard_shots, trace_columns


def test_shard_shots_partition():
    for n in (1, 2, 7, 64):
        for w in (1, 2, 3, 8):
            parts = [shard_shots(n, r, w) for r in range(w)]
            assert np.array_equal(np.concatenate(parts), np.arange(n))
            assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1
    with pytest.raises(ValueError):
        shard_shots(4, 2, 2)


def test_trace_columns():
    assert list(trace_columns([1, 3], 2)) == [2, 3, 6, 7]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import cases
        from helpers import oracle_run
        import oracle as O
        case = cases.tiny_s8()
        d_obs, d_est, _, W = oracle_run(case, gradient=False)
        shots = shard_shots(int(W.ns), rank, world)
        # this rank's propagator sees only its shots
        W.srcx, W.srcz = W.srcx[shots], W.srcz[shots]
        W.ns = np.int32(len(shots))
        cols = trace_columns(shots, int(W.nr))
        pe, po = O.prepare_residual(d_est, 1), O.prepare_residual(d_obs, 1)
        res = {k: np.ascontiguousarray((pe[k] - po[k])[:, cols], np.float32) for k in O.FIELDS}
        G = W.raw_gradient(res)
        g = {str(q): torch.from_numpy(G[q]) for q in range(3)}
        rms = torch.tensor(float(sum(0.5 * np.sum(res[k].astype(np.float64) ** 2) for k in res)), dtype=torch.float64)
        allreduce_gradient(g, rms)
        if rank == 0:
            np.savez(os.path.join(out_dir, "dist.npz"), *[g[str(q)].numpy() for q in range(3)], rms=rms.numpy())
    finally:
        dist.destroy_process_group()


def test_two_ranks_sum_to_single_process_gradient(tmp_path):
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    import cases
    from helpers import oracle_run
    import oracle as O
    case = cases.tiny_s8()
    d_obs, d_est, _, W = oracle_run(case, gradient=False)
    pe, po = O.prepare_residual(d_est, 1), O.prepare_residual(d_obs, 1)
    res = {k: (pe[k] - po[k]).astype(np.float32) for k in O.FIELDS}
    G = W.raw_gradient(res)
    d = np.load(tmp_path / "dist.npz")
    for q in range(3):
        a, b = d["arr_%d" % q], G[q]
        assert np.linalg.norm(a - b) <= 1e-6 * np.linalg.norm(b)
    rms = sum(0.5 * np.sum(res[k].astype(np.float64) ** 2) for k in res)
    assert abs(float(d["rms"]) - rms) <= 1e-9 * rms
