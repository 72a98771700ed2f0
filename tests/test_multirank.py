"""The bench's multi-rank plumbing on CPU: two gloo ranks, each timing its own replica solve, agree
on the slowest rank's time and report the whole-job rate from it (what `bench.py --gpus N` does over
NCCL, one rank per GPU)."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, steps, times, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t_max = bench.max_over_ranks_of(times[rank], dist, "cpu")
        out[rank] = (t_max, bench.whole_job_rate(world, steps, t_max))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    world, steps = 2, 5
    times = [0.090, 0.125]          # seconds each rank measured for its own steps
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), steps, times, out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    for t_max, rate in res.values():
        assert t_max == max(times)
        assert rate == world * steps / max(times)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks_of(0.25) == 0.25
    assert bench.whole_job_rate(1, 4, 0.5) == 8.0
