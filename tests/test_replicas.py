"""The N > 1 path of bench.py (replicas, one per GPU) on CPU: two gloo ranks agree on the
slowest rank's time and report the whole job's rate."""
import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 100.0 * (rank + 1)                  # the second rank is the slower one
        m = bench.max_over_ranks(ms, dist, device="cpu")
        out[rank] = (m, bench.whole_job_rate(world, 5, m))
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    world, port = 2, _free_port()
    out = mp.get_context("spawn").Manager().dict()
    mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
    for r in range(world):
        m, rate = out[r]
        assert m == 200.0
        assert abs(rate - world * 5 / 0.2) < 1e-9


def test_single_rank_is_unchanged():
    assert bench.max_over_ranks(123.0, None) == 123.0
    assert bench.whole_job_rate(1, 4, 500.0) == 8.0
