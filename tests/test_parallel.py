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


def _shard_worker(rank, world, port, q, n_inst):
    """One rank of a batch run: solves its contiguous share of the instances with the CPU
    oracle (assembly, Jacobi-PCG, back-substitution) and gathers every rank's results."""
    import sys
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import cases as OC
    import oracle as O
    O.set_threads(1)  # one thread per rank: the same summation order as the check below
    r, w, dist = parallel.init("gloo", timeout_s=60)
    try:
        mine = {}
        for i in parallel.shard(n_inst, r, w):
            P, *_ = OC.problem(3, seed=parallel.case_seed(3, 0, i), n=4 + 2 * (i % 2))
            S, b = O.schur2(P)
            x, it, res = O.pcg_jacobi(S, b, rtol=1e-12)
            sol = O.resolve(P, x)
            mine[i] = (it, float(abs(sol).sum()))
        every = [None] * w
        dist.all_gather_object(every, mine)
        if r == 0:
            merged = {}
            for part in every:
                merged.update(part)
            q.put(merged)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_batch_sharded_over_two_gloo_ranks():
    """A fixed batch of realisations split over two ranks (as bench.py --config 3 does on GPUs):
    every instance is solved exactly once, and the gathered results equal a single-process
    solve of the whole batch."""
    import cases as OC
    import oracle as O
    n_inst, world, port = 5, 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, q, n_inst)) for r in range(world)]
    for p in procs:
        p.start()
    merged = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(merged) == list(range(n_inst))
    threads = O.num_threads()
    O.set_threads(1)
    try:
        _check_batch(merged, n_inst)
    finally:
        O.set_threads(threads)


def _check_batch(merged, n_inst):
    import cases as OC
    import oracle as O
    for i in range(n_inst):
        P, *_ = OC.problem(3, seed=parallel.case_seed(3, 0, i), n=4 + 2 * (i % 2))
        S, b = O.schur2(P)
        x, it, res = O.pcg_jacobi(S, b, rtol=1e-12)
        assert merged[i][0] == it
        assert merged[i][1] == pytest.approx(float(abs(O.resolve(P, x)).sum()), rel=1e-12)
