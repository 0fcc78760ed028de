"""The N>1 plumbing on CPU: two gloo ranks shard views without overlap and agree on the max time."""
import os

import pytest
import torch.multiprocessing as mp

from slimtracin_b200 import dist as D


def test_shard_covers_every_item_once():
    for n in (0, 1, 7, 64, 65):
        for world in (1, 2, 3, 8):
            got = [x for r in range(world) for x in D.shard(list(range(n)), r, world)]
            assert got == list(range(n))
            sizes = [len(D.shard(list(range(n)), r, world)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        views = list(range(64))
        mine = D.shard(views, rank, world)
        t = 10.0 + rank * 5.0 + len(mine) * 0.01
        out.put((rank, mine, D.max_over_ranks(t), D.sum_over_ranks(len(mine))))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    (r0, v0, m0, s0), (r1, v1, m1, s1) = res
    assert sorted(v0 + v1) == list(range(64)) and not set(v0) & set(v1)
    assert m0 == m1 == max(10.0 + 0 * 5 + len(v0) * 0.01, 10.0 + 5.0 + len(v1) * 0.01)
    assert s0 == s1 == 64
