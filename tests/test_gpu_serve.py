"""Request server (amj_server_*): continuous batching over resident relations.

Every request's count and checksum is the same in the served mix as alone
(one amj_amhj_execute per query) and as the oracle; batches overlap on the
device; admission holds requests back by device memory; a request too large
for the budget spills to the out-of-core lane (or is rejected without one);
host-resident relations are served through the out-of-core lane."""
import threading
import time

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
    qs = list(data.query_mix(40, seed=21, min_rows=1000, max_rows=50000, out_cap=1 << 20))
    return qs, [oracle_of(q) for q in qs]


def test_served_results_equal_alone_and_in_the_mix(mix):
    qs, want = mix
    with Context(0) as ctx:
        rels = [[ctx.relation(c, a) for c, a in q["rels"]] for q in qs]
        alone = []
        for q, r in zip(qs, rels):
            x = ctx.amhj(q["qt"], r)
            alone.append((x.count, x.checksum))
        assert alone == want
        srv = ctx.server(lanes=2, max_batch=4)
        # a burst: more requests than two lanes of four hold, so batches queue and overlap
        tickets = [srv.submit(q["qt"], r) for q, r in zip(qs, rels)]
        got = [srv.wait(t) for t in tickets]
        assert [(g.count, g.checksum) for g in got] == want
        st = srv.stats()
        assert st["completed"] == len(qs) and st["batches"] >= len(qs) // 4
        assert st["max_inflight_batches"] == 2
        assert all(g.path == "batch" and 1 <= g.batch_size <= 4 for g in got)
        assert max(g.queue_ms for g in got) > 0.0
        srv.close()


def test_poisson_arrivals_are_served_by_continuous_batching(mix):
    qs, want = mix
    rng = np.random.Generator(np.random.PCG64(5))
    with Context(0) as ctx:
        rels = [[ctx.relation(c, a) for c, a in q["rels"]] for q in qs]
        srv = ctx.server(lanes=3, max_batch=64)
        order = rng.integers(0, len(qs), 300)
        gaps = rng.exponential(1.0 / 200.0, 300)       # 200 requests / s
        tickets = []

        def producer():
            t = time.perf_counter()
            for i, g in zip(order, gaps):
                t += g
                while time.perf_counter() < t:
                    time.sleep(0.0002)
                tickets.append((int(i), srv.submit(qs[i]["qt"], rels[i])))

        th = threading.Thread(target=producer)
        th.start()
        th.join()
        res = [(i, srv.wait(t)) for i, t in tickets]
        for i, r in res:
            assert (r.count, r.checksum) == want[i]
        lat = sorted(r.latency_ms for _, r in res)
        assert lat[len(lat) // 2] > 0 and lat[-1] < 60_000
        assert srv.stats()["completed"] == 300
        srv.close()


def test_admission_waits_for_memory_and_spills_what_never_fits():
    small = [data.chain_relations(20000, 1 << 14, 3, seed=s) for s in (1, 4, 7, 10)]
    big = data.chain_relations(400000, 1 << 18, 3, seed=13)
    with Context(0, ooc_slice_rows=50000) as ctx:
        srels = [[ctx.relation(c, a) for c, a in q] for q in small]
        brels = [ctx.relation(c, a) for c, a in big]
        # budget: room for about two small requests at a time, not for the big one
        srv = ctx.server(lanes=2, max_batch=8, mem_budget=6_000_000, ooc_lane=True, ooc_mem=64 << 20)
        ts = [srv.submit("NORMAL", r) for r in srels] + [srv.submit("NORMAL", brels)]
        got = [srv.wait(t) for t in ts]
        for q, g in zip(small, got[:4]):
            assert (g.count, g.checksum) == O.mhj(q) and g.path == "batch"
        assert (got[4].count, got[4].checksum) == O.mhj(big)
        assert got[4].path == "ooc" and got[4].spilled
        st = srv.stats()
        assert st["spilled"] == 1 and st["ooc_runs"] == 1 and st["batches"] >= 2
        assert st["peak_reserved_bytes"] <= st["budget_bytes"]
        srv.close()
        # without an out-of-core lane the big request is rejected
        srv = ctx.server(lanes=1, mem_budget=6_000_000, ooc_lane=False)
        t = srv.submit("NORMAL", brels)
        with pytest.raises(AmjError) as e:
            srv.wait(t)
        assert e.value.status == L.AMJ_EREJECT and "budget" in str(e.value)
        assert srv.stats()["rejected"] == 1
        srv.close()


def test_host_resident_relations_go_through_the_ooc_lane_beside_batches(mix):
    qs, want = mix
    chain = data.chain_relations(200000, 1 << 16, 4, seed=3)
    with Context(0, ooc_slice_rows=30000) as ctx:
        probe = ctx.relation(chain[0][0], chain[0][1], streamed=True)   # stays in pinned host memory
        builds = [ctx.relation(c, a) for c, a in chain[1:]]
        rels = [[ctx.relation(c, a) for c, a in q["rels"]] for q in qs]
        srv = ctx.server(lanes=2, max_batch=8)
        t_ooc = srv.submit("NORMAL", [probe] + builds)
        ts = [srv.submit(q["qt"], r) for q, r in zip(qs, rels)]
        got = [srv.wait(t) for t in ts]
        g = srv.wait(t_ooc)
        assert [(x.count, x.checksum) for x in got] == want
        assert g.path == "ooc" and not g.spilled
        assert (g.count, g.checksum) == O.mhj(chain)
        srv.close()


def test_index_cache_keeps_indexes_across_requests(mix):
    qs, want = mix
    with Context(0) as ctx:
        rels = [[ctx.relation(c, a) for c, a in q["rels"]] for q in qs[:10]]
        srv = ctx.server(lanes=2, max_batch=4)
        for _ in range(3):
            ts = [srv.submit(q["qt"], r) for q, r in zip(qs[:10], rels)]
            assert [(g.count, g.checksum) for g in (srv.wait(t) for t in ts)] == want[:10]
        st = srv.stats()
        assert st["index_builds"] > 0 and st["index_hits"] >= 2 * st["index_builds"] and st["index_bytes"] > 0
        srv.close()
        # a relation created after another was released (possibly at its address) is indexed anew
        srv = ctx.server(lanes=1)
        q1 = data.chain_relations(5000, 1 << 10, 3, seed=1)
        r1 = [ctx.relation(c, a) for c, a in q1]
        g1 = srv.wait(srv.submit("NORMAL", r1))
        for r in r1:
            r.release()
        q2 = data.chain_relations(5000, 1 << 10, 3, seed=2)
        r2 = [ctx.relation(c, a) for c, a in q2]
        g2 = srv.wait(srv.submit("NORMAL", r2))
        assert (g1.count, g1.checksum) == O.mhj(q1) and (g2.count, g2.checksum) == O.mhj(q2)
        srv.close()
        # without the cache every request builds its own indexes: same results
        srv = ctx.server(lanes=2, max_batch=4, index_cache=False)
        ts = [srv.submit(q["qt"], r) for q, r in zip(qs[:10], rels)]
        assert [(g.count, g.checksum) for g in (srv.wait(t) for t in ts)] == want[:10]
        assert srv.stats()["index_builds"] == 0
        srv.close()


def test_server_rejects_bad_requests():
    with Context(0) as ctx:
        srv = ctx.server(lanes=1, ooc_lane=False)
        one = ctx.relation([data.uniform(10, 0, 5, 1)], [0])
        with pytest.raises(AmjError) as e:
            srv.submit("NORMAL", [one])
        assert e.value.status == L.AMJ_EUNSUPPORTED
        rels = [ctx.relation(c, a) for c, a in data.chain_relations(100, 50, 3, seed=1)]
        with pytest.raises(AmjError) as e:
            srv.submit("NORMAL", rels, ooc=True)
        assert e.value.status == L.AMJ_EUNSUPPORTED
        with pytest.raises(AmjError) as e:
            srv.wait(12345)
        assert e.value.status == L.AMJ_EINVAL
        srv.close()
