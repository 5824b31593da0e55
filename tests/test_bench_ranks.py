"""The bench's multi-GPU aggregation on CPU: two gloo ranks stand in for two GPUs running independent replicas."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r "took" 100 + 10 r ms for 1000 (r + 1) ray-steps
        t, n = bench.max_time_sum_work(100.0 + 10.0 * rank, 1000 * (rank + 1), torch.device("cpu"), world)
        out[rank] = (t, n)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_replicas_report_slowest_time_and_total_work():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(90)
            assert p.exitcode == 0
        res = dict(out)
    # every rank sees the same whole-job figures: max time, summed work
    assert res[0] == res[1] == (110.0, 3000.0)


def test_single_rank_needs_no_process_group():
    import torch

    import bench
    assert bench.max_time_sum_work(5.0, 7, torch.device("cpu"), 1) == (5.0, 7.0)
