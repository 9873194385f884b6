"""The multi-process path on CPU: two gloo ranks, as bench.py runs under torchrun on GPUs.
Each rank owns its own realisations (no data-path collective); the job's time is the max
over ranks and its rate the units of all ranks over that time."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from mhdarcy import parallel


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    r, w, dist = parallel.init("gloo", timeout_s=60)
    try:
        assert (r, w) == (rank, world)
        t = 1.0 + rank  # rank 1 is the slow one
        tmax = parallel.max_over_ranks(t, dist)
        units = 3 * (rank + 1)
        rate = parallel.whole_job_rate(units, tmax, dist)
        part = list(parallel.shard(10, rank, world))
        seed = parallel.case_seed(3, rank, 0)
        q.put((rank, tmax, rate, part, seed))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        rank, tmax, rate, part, seed = q.get(timeout=120)
        out[rank] = (tmax, rate, part, seed)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == 2.0  # max over ranks
    assert out[0][1] == out[1][1] == pytest.approx((3 + 6) / 2.0)  # all units over the slowest time
    assert sorted(out[0][2] + out[1][2]) == list(range(10))  # the shards cover the batch once
    assert out[0][3] != out[1][3]  # every rank solves different realisations


def test_single_process_helpers():
    assert parallel.max_over_ranks(2.5) == 2.5
    assert parallel.whole_job_rate(10, 2.0) == 5.0
    assert [len(parallel.shard(10, r, 3)) for r in range(3)] == [4, 3, 3]
    assert list(parallel.shard(3, 0, 1)) == [0, 1, 2]
