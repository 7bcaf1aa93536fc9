"""The multi-rank path of bench.py on CPU: with N ranks every rank evaluates
its own survey (independent replicas, nothing exchanged on the data path);
the only collective is the MAX over ranks of the device-timed step, taken
here on two gloo ranks."""
import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, world, torch.device("cpu"))
        with open(os.path.join(out_dir, "rank%d" % rank), "w") as f:
            f.write(repr(ms))
    finally:
        dist.destroy_process_group()


def test_step_time_is_the_slowest_rank(tmp_path):
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    got = [float((tmp_path / ("rank%d" % r)).read_text()) for r in range(2)]
    assert got == [15.0, 15.0]


def test_one_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(3.5, 1, torch.device("cpu")) == 3.5
