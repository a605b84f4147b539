"""N>1 host logic on CPU with gloo (world size 2): walker sharding covers every
walker exactly once and the timing reduction takes the max over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def test_shard_partitions_exactly():
    from gluedmd_b200.dist import shard
    for n in (1, 7, 64, 65):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                a, b = shard(n, r, world)
                seen.extend(range(a, b))
            assert seen == list(range(n))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from gluedmd_b200 import dist as D
    dist = D.init("gloo", timeout_s=60)
    a, b = D.shard(64, rank, world)
    # each rank "times" its own walkers; the job time is the slowest rank
    t = 1.0 + rank
    m = D.max_over_ranks(t)
    total = D.sum_over_ranks(b - a)
    dist.barrier()
    q.put((rank, a, b, m, total))
    dist.destroy_process_group()


def test_two_rank_gloo_max_and_shard():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert out[0][1:3] == (0, 32) and out[1][1:3] == (32, 64)
    assert all(o[3] == 2.0 for o in out)  # max over ranks
    assert all(o[4] == 64 for o in out)   # every walker on exactly one rank
