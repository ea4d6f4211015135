"""One process per GPU for independent replicas (the Brownian-dynamics step
does not shard: replicas never interact, so there is no collective on the
data path).  The only collectives are the timing reduction and barriers.

    rank, world, local = ranks.init()          # torchrun env, nccl on GPUs
    seed = ranks.replica_seed(base, r, rank)    # disjoint RNG keys per rank
    mine = ranks.shard(n_total, rank, world)    # replicas of this rank (strong scaling)
    ms = ranks.max_over_ranks(ms)               # slowest rank's device time
"""
from __future__ import annotations

import datetime
import os

RANK_SEED_STRIDE = 100000  # replicas per rank never collide below this many


def init(backend: str | None = None, timeout_s: int = 120):
    """Rank, world size and local rank from the torchrun environment; joins
    the process group when world > 1 (nccl when CUDA is present, else gloo)."""
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and not dist.is_initialized():
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local


def replica_seed(base: int, replica: int, rank: int) -> int:
    """RNG key of replica `replica` on rank `rank` (weak scaling: every rank
    runs its own replicas, all keys distinct)."""
    if replica >= RANK_SEED_STRIDE:
        raise ValueError("more replicas per rank than the seed stride")
    return base + replica + RANK_SEED_STRIDE * rank


def shard(n_total: int, rank: int, world: int) -> range:
    """Contiguous block of replica indices owned by `rank` (strong scaling:
    n_total replicas split as evenly as possible, each exactly once)."""
    q, r = divmod(n_total, world)
    lo = rank * q + min(rank, r)
    return range(lo, lo + q + (1 if rank < r else 0))


def max_over_ranks(value: float) -> float:
    """Largest value over all ranks (the slowest rank's time); identity
    without a process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def finalize():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
