"""Multi-rank plumbing of the replicas-only path (bd_aging_b200/ranks.py) on
CPU with the gloo backend, world size 2: max-over-ranks timing, disjoint
replica seeds, replica shards that cover every replica exactly once."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from bd_aging_b200 import ranks


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    try:
        r, w, _ = ranks.init("gloo", timeout_s=60)
        slowest = ranks.max_over_ranks(10.0 + 5.0 * r)  # rank 1 is slower
        seeds = [ranks.replica_seed(7, k, r) for k in range(64)]
        mine = list(ranks.shard(257, r, w))
        ranks.barrier()
        q.put((r, w, slowest, seeds, mine))
    finally:
        ranks.finalize()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    assert all(o[2] == 15.0 for o in out)  # every rank sees the slowest rank's time
    assert not set(out[0][3]) & set(out[1][3])  # replica seeds never collide across ranks
    covered = out[0][4] + out[1][4]
    assert sorted(covered) == list(range(257)) and abs(len(out[0][4]) - len(out[1][4])) <= 1


def test_single_process_helpers():
    assert ranks.max_over_ranks(3.5) == 3.5
    assert list(ranks.shard(10, 0, 1)) == list(range(10))
    with pytest.raises(ValueError):
        ranks.replica_seed(0, ranks.RANK_SEED_STRIDE, 0)
