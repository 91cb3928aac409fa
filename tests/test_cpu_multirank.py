"""The N>1 path on CPU: world-size-2 gloo ranks shard one query's units and
sum (count, checksum) with the same reduction the GPU ranks use."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from accmultiwayjoins_b200 import data
from accmultiwayjoins_b200.dist import M64, allreduce_result, shard_range, shard_relation


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # strong form: one chain query, probe rows sharded
        rels = data.chain_relations(4000, 1 << 9, 3, seed=3)
        mine = [shard_relation(rels[0], rank, world)] + rels[1:]
        cnt, chk = O.mhj(mine)
        tot = allreduce_result(cnt, chk)
        # weak form: an independent triangle instance per rank
        s, d = data.rmat(10, 6000, 0.57, 0.19, 0.19, seed=20 + rank)
        tcnt, tchk = O.triangle(s, d)
        ttot = allreduce_result(tcnt, tchk)
        q.put((rank, tot, ttot))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_sharding_matches_single_process(built):
    from oracle import oracle as O
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    outs = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = O.mhj(data.chain_relations(4000, 1 << 9, 3, seed=3))
    tw = [O.triangle(*data.rmat(10, 6000, 0.57, 0.19, 0.19, seed=20 + r)) for r in range(world)]
    twant = (sum(c for c, _ in tw) & M64, sum(h for _, h in tw) & M64)
    for _, tot, ttot in outs:
        assert tot == want
        assert ttot == twant


def test_shard_range_covers_everything():
    n = 1001
    spans = [shard_range(n, r, 7) for r in range(7)]
    assert spans[0][0] == 0 and spans[-1][1] == n
    assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
    with pytest.raises(ValueError):
        shard_range(10, 3, 3)
