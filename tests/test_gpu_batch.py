"""Batched AMHJ (amj_batch_*): every query of a heterogeneous mix gives the
same count and checksum in the batch as alone (one query per call) and as the
oracle, for each layout, block size, task size, with and without a captured
CUDA graph; a replayed graph reads changed relation contents; the autotuner
returns a grid point."""
import numpy as np
import pytest

from accmultiwayjoins_b200 import AmjError, Context, _lib as L, data
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def oracle_of(q):
    if q["qt"] == "TRI":
        s, d = q["rels"][0][0]
        return O.triangle(s, d)
    return O.mhj(q["rels"])


@pytest.fixture(scope="module")
def mix():
    qs = list(data.query_mix(48, seed=7, min_rows=1000, max_rows=60000, out_cap=1 << 20))
    return qs, [oracle_of(q) for q in qs]


def submit_all(ctx, b, qs):
    keep = []
    for q in qs:
        rels = [ctx.relation(c, a) for c, a in q["rels"]]
        keep.append(rels)
        b.submit(q["qt"], rels)
    return keep


@pytest.mark.parametrize("layout", ["bucket", "oa"])
@pytest.mark.parametrize("block_size,task_chunk,load_factor", [(256, 1024, 0.0), (128, 32, 0.5), (512, 256, 0.85)])
def test_batch_matches_oracle(mix, layout, block_size, task_chunk, load_factor):
    qs, want = mix
    with Context(0) as ctx:
        b = ctx.batch()
        submit_all(ctx, b, qs)
        r = b.run(layout=layout, block_size=block_size, task_chunk=task_chunk, load_factor=load_factor)
        assert list(zip(r.counts, r.checksums)) == want
        assert r.tasks_popped == r.tasks_pushed
        assert r.units > 0 and r.launches > 0 and not r.graph


def test_batch_equals_one_query_per_call(mix):
    qs, want = mix
    with Context(0) as ctx:
        b = ctx.batch()
        keep = submit_all(ctx, b, qs)
        r = b.run()
        for q, rels, c, k in zip(qs, keep, r.counts, r.checksums):
            alone = ctx.amhj(q["qt"], rels)
            assert (alone.count, alone.checksum) == (c, k)


def test_batch_graph_capture_and_replay_reads_new_contents():
    import torch
    qs0 = list(data.query_mix(24, seed=11, min_rows=1000, max_rows=30000, out_cap=1 << 20))
    qs1 = list(data.query_mix(24, seed=11, min_rows=1000, max_rows=30000, out_cap=1 << 20))
    # same shapes and sizes, new contents: regenerate every column with another seed
    for q in qs1:
        for cols, _ in q["rels"]:
            for i, c in enumerate(cols):
                cols[i] = data.uniform(c.shape[0], 0, max(int(c.max()) + 1, 2), 99, i) if c.shape[0] else c
    with Context(0) as ctx:
        tensors = [[torch.from_numpy(c.copy()).cuda() for c in cols] for q in qs0 for cols, _ in q["rels"]]
        b = ctx.batch()
        it = iter(tensors)
        for q in qs0:
            rels = [ctx.relation(next(it), a) for _, a in q["rels"]]
            b.submit(q["qt"], rels)
        first = b.run(use_graph=True)
        again = b.run(use_graph=True)
        assert first.graph and again.graph
        want0 = [oracle_of(q) for q in qs0]
        assert list(zip(first.counts, first.checksums)) == want0
        assert list(zip(again.counts, again.checksums)) == want0
        # overwrite the borrowed device columns in place and replay
        new_cols = [cols for q in qs1 for cols, _ in q["rels"]]
        for ts, cols in zip(tensors, new_cols):
            for t, c in zip(ts, cols):
                t.copy_(torch.from_numpy(c))
        torch.cuda.synchronize()
        third = b.run(use_graph=True)
        assert list(zip(third.counts, third.checksums)) == [oracle_of(q) for q in qs1]
        eager = b.run(use_graph=False)
        assert (eager.counts, eager.checksums) == (third.counts, third.checksums)


def test_batch_work_sharing_across_queries():
    """Two skewed chains whose level-1 buckets are large, next to small
    queries: small tasks are pushed and popped across query boundaries."""
    q = [([data.uniform(100, 0, 100, 1), data.uniform(100, 0, 100, 2)], [0, 1]),
         ([data.uniform(2000, 0, 100, 3), data.uniform(2000, 0, 4, 4)], [1, 2]),
         ([data.uniform(20000, 0, 4, 5), data.uniform(20000, 0, 1 << 20, 6)], [2, 3])]
    small = data.chain_relations(3000, 1 << 12, 3, seed=5)
    want = [O.mhj(q), O.mhj(small), O.mhj(q)]
    with Context(0) as ctx:
        b = ctx.batch()
        for rels in (q, small, q):
            b.submit("NORMAL", [ctx.relation(c, a) for c, a in rels])
        r = b.run(task_chunk=32)
        assert list(zip(r.counts, r.checksums)) == want
        assert r.tasks_pushed > 0 and r.tasks_popped == r.tasks_pushed


@pytest.mark.parametrize("layout", ["bucket", "oa"])
def test_batch_limits_and_empty_relations(layout):
    """A 7-relation chain (6 build tables, 8 attributes), a 5-relation star,
    an empty build relation, an empty probe relation and a one-row query, in
    one batch: equal to one call per query and to the oracle."""
    long_chain = data.chain_relations(3000, 3000, 7, seed=31)
    fact, dims = data.star_relations(5000, [300, 200, 100, 50], theta=1.2, seed=32)
    star = [fact] + dims
    empty_build = data.chain_relations(2000, 256, 3, seed=33)
    empty_build[1] = ([np.zeros(0, np.int32), np.zeros(0, np.int32)], [1, 2])
    empty_probe = data.chain_relations(2000, 256, 3, seed=34)
    empty_probe[0] = ([np.zeros(0, np.int32), np.zeros(0, np.int32)], [0, 1])
    one = [([np.array([5], np.int32), np.array([7], np.int32)], [0, 1]),
           ([np.array([7, 7], np.int32), np.array([1, 2], np.int32)], [1, 2])]
    queries = [long_chain, star, empty_build, empty_probe, one]
    with Context(0) as ctx:
        b = ctx.batch()
        rels = []
        for q in queries:
            r = [ctx.relation(c, a) for c, a in q]
            rels.append(r)
            b.submit("NORMAL", r)
        got = b.run(layout=layout, block_size=256)
        for q, r, c, k in zip(queries, rels, got.counts, got.checksums):
            alone = ctx.amhj("NORMAL", r)
            assert (alone.count, alone.checksum) == (c, k) == O.mhj(q)
        assert got.counts[2] == 0 and got.counts[3] == 0 and got.counts[4] == 2


def test_batch_tuner_picks_a_grid_point(mix):
    qs, want = mix
    with Context(0) as ctx:
        b = ctx.batch()
        submit_all(ctx, b, qs)
        best, ms = b.tune(sample_every=4, load_factors=(0.5, 0.85), block_sizes=(128, 256), task_chunks=(64, 1024))
        assert best.load_factor in (np.float32(0.5), np.float32(0.85))
        assert best.block_size in (128, 256) and best.task_chunk in (64, 1024)
        assert ms > 0
        r = b.run(opts=best)
        assert list(zip(r.counts, r.checksums)) == want


def test_batch_rejects_what_it_does_not_run():
    with Context(0) as ctx:
        b = ctx.batch()
        with pytest.raises(AmjError) as e:
            b.run()
        assert e.value.status == L.AMJ_EINVAL
        one = ctx.relation([data.uniform(10, 0, 5, 1)], [0])
        with pytest.raises(AmjError) as e:
            b.submit("NORMAL", [one])
        assert e.value.status == L.AMJ_EUNSUPPORTED
        rels = [ctx.relation(c, a) for c, a in data.chain_relations(100, 50, 2, seed=1)]
        assert b.submit("NORMAL", rels) == 0
        with pytest.raises(AmjError) as e:
            b.run(block_size=96)
        assert e.value.status == L.AMJ_EINVAL
        r = b.run()
        assert (r.counts[0], r.checksums[0]) == O.mhj(data.chain_relations(100, 50, 2, seed=1))
