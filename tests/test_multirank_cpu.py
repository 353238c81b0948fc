"""Multi-rank host logic of bench.py on CPU: two gloo ranks on 127.0.0.1.

bench.py runs one replica per GPU (the path shards by views but this build runs
independent replicas; no data-path collective). Its only collectives are the
timing reduction (the job's time is the slowest rank's) and the barriers of the
reference arm, which runs on rank 0 while the other ranks wait.
"""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        per_rank_ms = [120.0, 80.0][rank]
        job_ms = bench.max_over_ranks(per_rank_ms, world, torch.device("cpu"))
        rate = bench.job_rate(1000.0, world, job_ms / 10)
        # Reference-arm protocol: rank 0 works, the others wait at one barrier; rank 0 matches it at the end.
        if rank != 0:
            dist.barrier()
            worked = False
        else:
            worked = True
            dist.barrier()
        out[rank] = (job_ms, rate, worked)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time_and_sum_the_work():
    port = _free_port()
    with mp.Manager() as manager:
        out = manager.dict()
        mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
        results = dict(out)
    assert results[0][0] == results[1][0] == 120.0
    # 1000 units per rank per step, 2 ranks, 12 ms per step -> 1.667e5 units/s for the job.
    assert results[0][1] == pytest.approx(2 * 1000.0 / 0.012)
    assert results[0][2] is True and results[1][2] is False


def test_single_rank_is_identity():
    import bench

    assert bench.max_over_ranks(42.0, 1, torch.device("cpu")) == 42.0
    assert bench.job_rate(10.0, 1, 1.0) == pytest.approx(1e4)
