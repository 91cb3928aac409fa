"""Host-side pieces of the batched and served workloads, without a GPU: the
seeded query mix (shapes, sizes, domains, skew, output bound), and the
bench's percentile helper."""
import numpy as np

from accmultiwayjoins_b200 import data
from oracle import oracle as O


def test_query_mix_is_seeded_and_within_bounds():
    a = list(data.query_mix(24, seed=3, min_rows=1000, max_rows=20000, out_cap=1 << 22))
    b = list(data.query_mix(24, seed=3, min_rows=1000, max_rows=20000, out_cap=1 << 22))
    assert [q["shape"] for q in a] == [q["shape"] for q in b]
    for qa, qb in zip(a, b):
        for (ca, aa), (cb, ab) in zip(qa["rels"], qb["rels"]):
            assert aa == ab and all(np.array_equal(x, y) for x, y in zip(ca, cb))
    shapes = {q["shape"] for q in a}
    assert shapes <= {"chain", "star", "triangle"} and len(shapes) == 3
    for q in a:
        if q["shape"] == "triangle":
            (s, d), at = q["rels"][0]
            assert at == [0, 1] and q["qt"] == "TRI" and np.all(s < d)
            continue
        assert 2 <= len(q["rels"]) <= 5
        for cols, at in q["rels"]:
            assert 1000 // 2 <= len(cols[0]) <= 20000 and all(c.dtype == np.int32 for c in cols)
        if q["theta"]:
            assert 0.5 <= q["theta"] <= 1.5
        if q["shape"] == "star":
            fact, dims = q["rels"][0], q["rels"][1:]
            for j, (cols, at) in enumerate(dims):
                assert np.array_equal(np.sort(cols[0]), np.arange(len(cols[0])))   # unique dimension keys
                assert fact[0][j].max() < len(cols[0])
            assert O.mhj(q["rels"])[0] == len(fact[0][0])                         # every foreign key matches


def test_query_mix_chains_keep_skew_on_the_build_side():
    qs = [q for q in data.query_mix(40, seed=11, min_rows=2000, max_rows=20000) if q["shape"] == "chain" and q["theta"]]
    assert qs
    for q in qs:
        for i, (cols, at) in enumerate(q["rels"]):
            assert at == [i, i + 1]
            if i:
                # the probe side (column 1 of the relation before) is uniform, the
                # build side (column 0 here) Zipf: its most frequent key is far above the mean
                c0 = cols[0]
                top = np.bincount(c0 - c0.min()).max()
                assert top > 4 * len(c0) / max(1, len(np.unique(c0)))


def test_bench_percentiles():
    import bench
    xs = [5.0, 1.0, 3.0, 2.0, 4.0]
    assert bench.pct(xs, 50) == 3.0 and bench.pct(xs, 99) == 5.0 and bench.pct(xs, 0) == 1.0


def _lookup_bytes(build_keys, B, key):
    """B_probe's bytes of one lookup: bounds, the bucket's keys, 8 B a match."""
    bucket = build_keys[(build_keys & (B - 1)) == (key & (B - 1))]
    return 8 + 4 * len(bucket) + 8 * int(np.count_nonzero(bucket == key))


def test_bench_star_algorithmic_bytes_match_a_direct_count():
    """The star workload's B_probe (16 B a fact row; per dimension lookup the
    bucket bounds, 4 B a key scanned, 8 B a match; floorPow2(rows) buckets)
    against a row-by-row count."""
    import argparse
    import bench
    wl = bench.Star(argparse.Namespace(star_rows=1500), 0, gen=O.GENERATORS)
    fact_cols = wl.rels[0][0]
    want = 0
    for r in range(len(fact_cols[0])):
        want += 16
        for j, (cols, _) in enumerate(wl.rels[1:]):
            B = 1 << (len(cols[0]).bit_length() - 1)
            want += _lookup_bytes(cols[0], B, fact_cols[j][r])
    assert wl.algorithmic_bytes() == want
    assert wl.lookups_per_launch() == 4 * len(fact_cols[0])
    assert wl.h2d == sum(4 * len(c[0]) * len(c) for c, _ in wl.rels)


def test_bench_chain_algorithmic_bytes_match_a_direct_count():
    """The chain workload's B_probe (8 B a probe row; a level-0 lookup per
    probe row and a level-1 lookup per level-0 match, each the bucket
    bounds, 4 B a key scanned and 8 B a match) against a row-by-row count,
    on a small chain of the same shape."""
    import bench
    rng = np.random.Generator(np.random.PCG64(5))
    n = 3000
    wl = bench.Chain.__new__(bench.Chain)
    wl.rels = [([rng.integers(0, 1 << 18, n).astype(np.int32), rng.integers(0, 1500, n).astype(np.int32)], [0, 1]),
               ([rng.integers(0, 1500, n).astype(np.int32), rng.integers(0, 1500, n).astype(np.int32)], [1, 2]),
               ([rng.integers(0, 1500, n).astype(np.int32), rng.integers(0, 1 << 18, n).astype(np.int32)], [2, 3])]
    wl.B, wl.plan = 2048, "multiway"
    (p0, p1), (b0, b1), (c0, _) = wl.rels[0][0], wl.rels[1][0], wl.rels[2][0]
    want, lookups = 0, 0
    for r in range(n):
        want += 8 + _lookup_bytes(b0, wl.B, p1[r])
        lookups += 1
        for j in np.nonzero(b0 == p1[r])[0]:
            want += _lookup_bytes(c0, wl.B, b1[j])
            lookups += 1
    assert wl.algorithmic_bytes() == want
    assert wl.lookups_per_launch() == lookups
