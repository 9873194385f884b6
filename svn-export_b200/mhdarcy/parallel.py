"""One process per GPU for independent MH solves.

The MH Darcy path does not exchange data between GPUs here: every rank assembles and solves
its own systems (a single mesh per rank, or its share of a batch of realisations), so the only
collectives are the ones that time a run (a barrier and a max over ranks) -- no collective on
the data path.  Flow123d's own parallel scheme (an element partition with halo exchanges,
darcy_flow_mh.cc:1358-1382) is not built.

The helpers take an initialised torch.distributed process group (NCCL on GPUs, gloo on CPU
for tests) or None for a single process.
"""
import datetime
import os


def init(backend="nccl", timeout_s=300):
    """rank, world and the process group module (None for one process), from the
    torchrun environment (RANK, WORLD_SIZE, MASTER_ADDR/MASTER_PORT)."""
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if world <= 1:
        return rank, world, None
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, dist


def case_seed(config, rank, instance=0):
    """Seed of a rank's synthetic system: every rank solves different realisations."""
    return 1234 + config + 1000 * rank + instance


def shard(n_total, rank, world):
    """Contiguous block of [0, n_total) owned by a rank (sizes differ by at most one)."""
    base, extra = divmod(n_total, world)
    lo = rank * base + min(rank, extra)
    return range(lo, lo + base + (1 if rank < extra else 0))


def max_over_ranks(x, dist=None, device="cpu"):
    """Largest value of x over the ranks (the job's time is that of its slowest rank)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, dist=None, device="cpu"):
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def whole_job_rate(units_per_rank, seconds_max, dist=None, device="cpu"):
    """Units per second of the whole job: the units all ranks processed over the slowest
    rank's time."""
    total = sum_over_ranks(units_per_rank, dist, device)
    return total / seconds_max if seconds_max > 0 else 0.0
