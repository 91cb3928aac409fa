"""The CPU oracle pinned against the reference's MHJ-CPU, the committed
golden fixtures (outputs of MHJ-CPU run here) and brute force."""
import json
import os
from collections import defaultdict

import numpy as np
import pytest

from accmultiwayjoins_b200 import data
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden.json")
M64 = (1 << 64) - 1


def mix(z):
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def tuple_hash(vals):
    h = 0x9E3779B97F4A7C15
    for v in vals:
        h = mix(h ^ (int(v) & 0xFFFFFFFF))
    return h


def brute_join(relations):
    """Nested-loop natural join of small relations, in query order."""
    k = 1 + max(a for _, attrs in relations for a in attrs)
    rows = []
    cols0, attrs0 = relations[0]
    for i in range(len(cols0[0])):
        t = [None] * k
        for c, a in zip(cols0, attrs0):
            t[a] = int(c[i])
        rows.append(t)
    for cols, attrs in relations[1:]:
        new = []
        for t in rows:
            for i in range(len(cols[0])):
                ok = all(t[a] is None or t[a] == int(c[i]) for c, a in zip(cols, attrs))
                if ok:
                    u = list(t)
                    for c, a in zip(cols, attrs):
                        u[a] = int(c[i])
                    new.append(u)
        rows = new
    return len(rows), sum(tuple_hash(t) for t in rows) & M64, sorted(tuple(t) for t in rows)


def load_golden():
    with open(GOLDEN) as f:
        return json.load(f)


def make_case(case):
    kind = case["kind"]
    if kind == "chain":
        return data.chain_relations(case["n"], case["key_range"], case["nrels"], seed=case["seed"])
    if kind == "star":
        fact, dims = data.star_relations(case["fact_rows"], case["dims"], theta=case["theta"], seed=case["seed"])
        return [fact] + dims
    raise ValueError(kind)


# the CPU suite stays within minutes: cases whose oracle run takes longer
# (the full-size star and triangle) are checked by the GPU tests only
CPU_CASES = [c for c in load_golden()["cases"]
             if c.get("fact_rows", 0) <= 1_000_000 and c.get("edges", 0) <= 1_000_000]


@pytest.mark.parametrize("case", [c for c in CPU_CASES if c["kind"] in ("chain", "star")], ids=lambda c: c["name"])
def test_oracle_matches_golden(built, case):
    rels = make_case(case)
    cnt, chk = O.mhj(rels)
    assert cnt == case["count"]
    assert f"{chk:016x}" == case["checksum"]


@pytest.mark.parametrize("case", [c for c in CPU_CASES if c["kind"] in ("tri", "four")], ids=lambda c: c["name"])
def test_cyclic_restatements_match_reference_golden(built, case):
    """The triangle and 4-clique restatements against the reference's own
    multi-key probe (fixtures written by tests/golden/make_golden.py)."""
    s, d = O.gen_rmat(case["scale"], case["nedges"], *case["abc"], seed=case["seed"])
    assert s.shape[0] == case["edges"]
    got = O.triangle(s, d) if case["kind"] == "tri" else O.four_clique(s, d)
    assert got == (case["count"], int(case["checksum"], 16))


@pytest.mark.skipif(not O.ref_available(multi_key=True), reason="reference MHJ-CPU harness not built")
@pytest.mark.parametrize("abc", [(0.57, 0.19, 0.19), (0.6, 0.15, 0.15)])
def test_reference_multi_key_probe_answers_tri_and_four(built, abc):
    """The reference's multi-key probe on the TRI / FOUR patterns equals the
    restatements, on the relation as given and through the degree-ordered
    copy renamed back; the shipped single-key probe does not (it never
    compares the second attribute of C(0,2))."""
    s, d = O.gen_rmat(9, 6000, *abc, seed=31)
    tri, four = O.triangle(s, d), O.four_clique(s, d)
    assert O.mhj_reference(O.tri_relations(s, d), nthreads=4, multi_key=True)[:2] == tri
    assert O.mhj_reference(O.four_relations(s, d), nthreads=4, multi_key=True)[:2] == four
    s2, d2, rank_to_id = O.degree_ordered_copy(s, d)
    assert O.mhj_reference(O.tri_relations(s2, d2), nthreads=3, multi_key=True, relabel=rank_to_id)[:2] == tri
    assert O.mhj_reference(O.four_relations(s2, d2), nthreads=2, multi_key=True, relabel=rank_to_id)[:2] == four
    assert O.mhj_reference(O.tri_relations(s, d), nthreads=4)[0] > tri[0]
    # chains: the multi-key probe compares only the join key, as the shipped one
    rels = data.chain_relations(5000, 1 << 10, 3, seed=2, gen=O.GENERATORS)
    assert O.mhj_reference(rels, multi_key=True)[:2] == O.mhj_reference(rels)[:2]


@pytest.mark.skipif(not O.ref_available(multi_key=True), reason="reference MHJ-CPU harness not built")
def test_reference_multi_key_tuples_equal_restatement_tuples(built):
    s, d = O.gen_rmat(8, 1500, 0.57, 0.19, 0.19, seed=3)
    cnt, chk, _, cols = O.mhj_reference(O.tri_relations(s, d), nthreads=2, tuples=True, multi_key=True)
    ocnt, ochk, ocols = O.triangle(s, d, tuples=True)
    assert (cnt, chk) == (ocnt, ochk)
    a, b = np.stack(cols, 1), np.stack(ocols, 1)
    assert np.array_equal(a[np.lexsort(a.T[::-1])], b[np.lexsort(b.T[::-1])])


@pytest.mark.parametrize("gen", ["rmat", "chain", "star"])
def test_oracle_generators_equal_product_generators(built, gen):
    """The oracle's own input generators (used by the CPU arm of bench.py so
    that it never loads the product library) are bit-identical to the
    product's."""
    if gen == "rmat":
        for args in [(8, 2000, 0.57, 0.19, 0.19, 3), (14, 1 << 18, 0.6, 0.15, 0.15, 22), (1, 10, 0.3, 0.3, 0.3, 1)]:
            for x, y in zip(O.gen_rmat(*args), data.rmat(*args)):
                assert np.array_equal(x, y)
    elif gen == "chain":
        a = data.chain_relations(50000, 1 << 12, 4, seed=5, gen=O.GENERATORS)
        b = data.chain_relations(50000, 1 << 12, 4, seed=5)
        assert [at for _, at in a] == [at for _, at in b]
        for (ca, _), (cb, _) in zip(a, b):
            assert all(np.array_equal(x, y) for x, y in zip(ca, cb))
    else:
        (fa, ta), da = data.star_relations(40000, [1000, 200, 100, 10], theta=1.1, seed=3, gen=O.GENERATORS)
        (fb, tb), db = data.star_relations(40000, [1000, 200, 100, 10], theta=1.1, seed=3)
        assert ta == tb and all(np.array_equal(x, y) for x, y in zip(fa, fb))
        for (ca, aa), (cb, ab) in zip(da, db):
            assert aa == ab and all(np.array_equal(x, y) for x, y in zip(ca, cb))
    assert np.array_equal(O.gen_uniform(1000, -(1 << 31), 1 << 31, 9, 4), data.uniform(1000, -(1 << 31), 1 << 31, 9, 4))
    assert np.array_equal(O.gen_zipf(1000, 77, 0.7, 9, 2), data.zipf(1000, 77, 0.7, 9, 2))


@pytest.mark.skipif(not O.ref_available(), reason="reference MHJ-CPU harness not built (reference sources absent)")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_matches_reference_mhj_cpu(built, seed):
    rels = data.chain_relations(20000, 1 << 12, 3, seed=seed)
    ref_cnt, ref_chk, _ = O.mhj_reference(rels, nthreads=4)
    assert O.mhj(rels) == (ref_cnt, ref_chk)
    fact, dims = data.star_relations(30000, [2000, 500, 100, 10], seed=seed)
    rels = [fact] + dims
    ref_cnt, ref_chk, _ = O.mhj_reference(rels, nthreads=3)
    assert O.mhj(rels) == (ref_cnt, ref_chk)


@pytest.mark.skipif(not O.ref_available(), reason="reference MHJ-CPU harness not built (reference sources absent)")
def test_reference_tuples_equal_oracle_tuples(built):
    rels = data.chain_relations(3000, 1 << 9, 4, seed=5)
    cnt, chk, _, cols = O.mhj_reference(rels, nthreads=2, tuples=True)
    ocnt, ochk, ocols = O.mhj(rels, tuples=True)
    assert (cnt, chk) == (ocnt, ochk)
    a = np.stack(cols, 1)
    b = np.stack(ocols, 1)
    assert np.array_equal(a[np.lexsort(a.T[::-1])], b[np.lexsort(b.T[::-1])])


def test_oracle_matches_brute_force_small(built):
    rels = data.chain_relations(60, 12, 3, seed=9)
    cnt, chk, tuples = brute_join(rels)
    assert O.mhj(rels) == (cnt, chk)
    ocnt, ochk, ocols = O.mhj(rels, tuples=True)
    got = sorted(tuple(int(x) for x in r) for r in np.stack(ocols, 1))
    assert got == tuples


def test_oracle_negative_and_duplicate_keys(built):
    r1 = ([np.array([-5, -5, 7, 2**31 - 1], np.int32), np.array([-1, -1, 3, -2**31], np.int32)], [0, 1])
    r2 = ([np.array([-1, -1, -2**31, 3], np.int32), np.array([10, 11, 12, 13], np.int32)], [1, 2])
    rels = [r1, r2]
    cnt, chk, _ = brute_join(rels)
    assert O.mhj(rels) == (cnt, chk)


def test_triangle_and_four_restatements_agree_with_join_patterns(built):
    s, d = data.rmat(9, 5000, 0.57, 0.19, 0.19, seed=4)
    tri = O.triangle(s, d)
    assert tri == O.mhj([([s, d], [0, 1]), ([s, d], [1, 2]), ([s, d], [0, 2])])
    four = O.four_clique(s, d)
    pat = [(0, 1), (1, 2), (2, 3), (0, 3), (0, 2), (1, 3)]
    assert four == O.mhj([([s, d], list(p)) for p in pat])


def test_triangle_bag_semantics_with_duplicates(built):
    s = np.array([0, 0, 1, 0, 0], np.int32)
    d = np.array([1, 2, 2, 1, 2], np.int32)
    rels = [([s, d], [0, 1]), ([s, d], [1, 2]), ([s, d], [0, 2])]
    cnt, chk, _ = brute_join(rels)
    assert O.triangle(s, d) == (cnt, chk)


def test_trie_build_oracle_is_a_csr(built):
    s, d = data.rmat(10, 8000, 0.57, 0.19, 0.19, seed=2)
    d0, o0, d1 = O.trie_build(s, d)
    order = np.lexsort((d, s))
    assert np.array_equal(d1, d[order])
    assert np.array_equal(d0, np.unique(s))
    counts = np.bincount(np.searchsorted(d0, s), minlength=len(d0))
    assert np.array_equal(np.diff(o0.astype(np.int64)), counts)


def trie_levels_by_definition(cols):
    """Level l = last values of the distinct (l+1)-prefixes of the sorted rows;
    offsets of level l = first row-rank of each prefix's children in level l+1."""
    a = np.stack([np.asarray(c, np.int64) for c in cols], 1)
    a = a[np.lexsort(a.T[::-1])] if len(a) else a
    k = a.shape[1]
    data, off = [], []
    prefixes = []
    for l in range(k - 1):
        heads = np.ones(len(a), bool)
        if len(a):
            heads[1:] = np.any(a[1:, :l + 1] != a[:-1, :l + 1], axis=1)
        prefixes.append(heads)
        data.append(a[heads, l].astype(np.int32))
    data.append(a[:, k - 1].astype(np.int32))
    for l in range(k - 1):
        nxt = np.cumsum(prefixes[l + 1]) - 1 if l + 1 < k - 1 else np.arange(len(a))
        starts = nxt[prefixes[l]].astype(np.uint64)
        end = prefixes[l + 1].sum() if l + 1 < k - 1 else len(a)
        off.append(np.append(starts, np.uint64(end)))
    return data, off


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5])
def test_trie_build_n_oracle_by_definition(built, k):
    rng = np.random.Generator(np.random.PCG64(k))
    n = 3000
    cols = [rng.integers(-4, 4, n).astype(np.int32) for _ in range(k)]
    cols[0][::7] = -(1 << 31)
    data, off = O.trie_build_n(cols)
    wd, wo = trie_levels_by_definition(cols)
    assert len(data) == k and len(off) == k - 1
    for a, b in zip(data, wd):
        assert np.array_equal(a, b)
    for a, b in zip(off, wo):
        assert np.array_equal(a, b)
    if k == 2:
        d0, o0, d1 = O.trie_build(cols[0], cols[1])
        assert np.array_equal(d0, data[0]) and np.array_equal(o0, off[0]) and np.array_equal(d1, data[1])


def test_trie_build_n_oracle_small_example(built):
    c = [np.array(x, np.int32) for x in ([3, 1, 2, 3, 2, 3], [5, 2, 4, 5, 9, 1], [1, 8, 8, 0, 7, 2])]
    data, off = O.trie_build_n(c)
    assert [list(d) for d in data] == [[1, 2, 3], [2, 4, 9, 1, 5], [8, 8, 7, 2, 0, 1]]
    assert [list(o) for o in off] == [[0, 1, 3, 5], [0, 1, 2, 3, 4, 6]]


def test_bucket_build_oracle(built):
    keys = data.uniform(5000, -1000, 1000, seed=3)
    hk, idx, bp = O.bucket_build(keys, 1024)
    assert bp[0] == 0 and bp[-1] == 5000
    for b in range(1024):
        seg = idx[bp[b]:bp[b + 1]]
        assert np.all(np.diff(seg.astype(np.int64)) > 0)
        assert np.all((keys[seg].astype(np.int64) & 1023) == b)
    assert np.array_equal(hk, keys[idx])


def test_checksum_definition_matches_python(built):
    cols = [data.uniform(100, -50, 50, seed=1, stream=s) for s in range(3)]
    want = sum(tuple_hash(t) for t in zip(*cols)) & M64
    assert data.checksum(cols) == want
