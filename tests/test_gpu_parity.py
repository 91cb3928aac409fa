"""Parity of the CUDA path (through the C ABI) with the CPU oracle: counts,
checksums and, at small sizes, sorted tuples; edge cases; every switch of
exec-AMHJ / exec-LFTJ; full-size property checks."""
import ctypes as C
import json
import os
import subprocess

import numpy as np
import pytest

from accmultiwayjoins_b200 import AmjError, Context, _lib as L, data
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "golden.json")


def sorted_rows(cols):
    a = np.stack([np.asarray(c, np.int64) for c in cols], 1)
    if a.shape[0] == 0:
        return a
    return a[np.lexsort(a.T[::-1])]


def rels_on(ctx, rels):
    return [ctx.relation(c, a) for c, a in rels]


# ------------------------------------------------------------ building blocks

@pytest.mark.parametrize("n,B,lo,hi", [(0, 1, 0, 1), (1, 1, 5, 6), (1000, 512, 0, 1000), (1 << 20, 1 << 19, 0, 1 << 18),
                                       (3_000_000, 1 << 21, -(1 << 30), 1 << 30), (100000, 1 << 16, 7, 8)])
def test_bucket_build_matches_oracle(ctx, n, B, lo, hi):
    import torch
    keys = data.uniform(n, lo, hi, seed=5) if n else np.zeros(0, np.int32)
    dk = torch.from_numpy(keys).cuda() if n else torch.zeros(1, dtype=torch.int32, device="cuda")
    hk = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    idx = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    bp = torch.empty(B + 1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    L.check(L.load().amj_bucket_build(ctx.handle, dk.data_ptr(), n, B, hk.data_ptr(), idx.data_ptr(), bp.data_ptr()))
    ohk, oidx, obp = O.bucket_build(keys, B)
    assert np.array_equal(bp.cpu().numpy().view(np.uint32), obp)
    assert np.array_equal(hk.cpu().numpy()[:n], ohk)
    assert np.array_equal(idx.cpu().numpy()[:n].view(np.uint32), oidx)


def trie_arrays(ctx, s, d):
    import torch
    lib = L.load()
    ds, dd = torch.from_numpy(s).cuda(), torch.from_numpy(d).cuda()
    h = C.c_void_p()
    L.check(lib.amj_trie_build(ctx.handle, ds.data_ptr(), dd.data_ptr(), len(s), C.byref(h)))
    l0, l1 = C.c_uint64(), C.c_uint64()
    L.check(lib.amj_trie_view(h, C.byref(l0), C.byref(l1), None, None, None))
    a0 = np.empty(max(l0.value, 1), np.int32)
    ao = np.empty(l0.value + 1, np.uint64)
    a1 = np.empty(max(l1.value, 1), np.int32)
    L.check(lib.amj_trie_download(h, a0.ctypes.data_as(C.POINTER(C.c_int32)),
                                  ao.ctypes.data_as(C.POINTER(C.c_uint64)), a1.ctypes.data_as(C.POINTER(C.c_int32))))
    return h, a0[:l0.value], ao, a1[:l1.value]


@pytest.mark.parametrize("case", ["small", "1M", "dups_negative"])
def test_trie_build_matches_oracle(ctx, case):
    if case == "small":
        s, d = data.rmat(8, 2000, 0.57, 0.19, 0.19, 3)
    elif case == "1M":
        s, d = data.rmat(16, 1 << 20, 0.57, 0.19, 0.19, 3)
    else:
        s = data.uniform(50000, -(1 << 31), 1 << 31, seed=1)
        s[::3] = s[0]
        d = data.uniform(50000, -40, 40, seed=2)
    h, a0, ao, a1 = trie_arrays(ctx, s, d)
    L.load().amj_trie_release(h)
    o0, oo, o1 = O.trie_build(s, d)
    assert np.array_equal(a0, o0) and np.array_equal(ao, oo) and np.array_equal(a1, o1)


def test_trie_tr_file_round_trip(ctx, tmp_path):
    lib = L.load()
    s, d = data.rmat(10, 8000, 0.57, 0.19, 0.19, 4)
    h, a0, ao, a1 = trie_arrays(ctx, s, d)
    p = str(tmp_path / "t.tr").encode()
    L.check(lib.amj_trie_save(h, p, 0, 1))
    h2 = C.c_void_p()
    x0, x1 = C.c_uint32(), C.c_uint32()
    L.check(lib.amj_trie_load(ctx.handle, p, C.byref(h2), C.byref(x0), C.byref(x1)))
    assert (x0.value, x1.value) == (0, 1)
    l0, l1 = C.c_uint64(), C.c_uint64()
    L.check(lib.amj_trie_view(h2, C.byref(l0), C.byref(l1), None, None, None))
    b0 = np.empty(l0.value, np.int32)
    bo = np.empty(l0.value + 1, np.uint64)
    b1 = np.empty(l1.value, np.int32)
    L.check(lib.amj_trie_download(h2, b0.ctypes.data_as(C.POINTER(C.c_int32)),
                                  bo.ctypes.data_as(C.POINTER(C.c_uint64)), b1.ctypes.data_as(C.POINTER(C.c_int32))))
    assert np.array_equal(a0, b0) and np.array_equal(ao, bo) and np.array_equal(a1, b1)
    lib.amj_trie_release(h)
    lib.amj_trie_release(h2)


def test_edgelist_to_tr_equals_trie_of_the_edges(ctx, tmp_path):
    """amj_edgelist_to_tr (the reference's edgelist_to_csr,
    LFTJ-GPU/edgelist_to_csr.cu) writes the .tr file of the trie the
    oracle builds from the same edges; repeated rows stay in level 1."""
    s, d = data.rmat(11, 20000, 0.57, 0.19, 0.19, 5)
    s = np.concatenate([s, s[:100]])
    d = np.concatenate([d, d[:100]])
    txt = tmp_path / "g.txt"
    with open(txt, "w") as f:
        f.write("# comment\n")
        for u, v in zip(s, d):
            f.write(f"{u}\t{v}\n")
    out = tmp_path / "g.tr"
    assert ctx.edgelist_to_tr(str(txt), str(out)) == len(s)
    d0, o0, d1 = O.trie_build(s, d)
    raw = open(out, "rb").read()
    na = np.frombuffer(raw[:4], np.uint32)[0]
    lens = np.frombuffer(raw[4:20], np.uint64)
    assert na == 2 and lens.tolist() == [len(d0), len(d1)]
    body = raw[28:]
    f0 = np.frombuffer(body[:4 * len(d0)], np.int32)
    f1 = np.frombuffer(body[4 * len(d0):4 * (len(d0) + len(d1))], np.int32)
    fo = np.frombuffer(body[4 * (len(d0) + len(d1)):], np.uint64)
    assert np.array_equal(f0, d0) and np.array_equal(f1, d1) and np.array_equal(fo, o0)
    # the swapped list is the reverse relation
    out2 = tmp_path / "r.tr"
    ctx.edgelist_to_tr(str(txt), str(out2), swap=True)
    r0, _, r1 = O.trie_build(d, s)
    raw2 = open(out2, "rb").read()[28:]
    assert np.array_equal(np.frombuffer(raw2[:4 * len(r0)], np.int32), r0)


def trie_n_levels(h):
    lib = L.load()
    lv = C.c_int()
    lens = (C.c_uint64 * 8)()
    L.check(lib.amj_trie_info(h, C.byref(lv), lens))
    data, off = [], []
    for l in range(lv.value):
        d = np.empty(max(lens[l], 1), np.int32)
        o = np.empty(lens[l] + 1, np.uint64)
        last = l + 1 == lv.value
        L.check(lib.amj_trie_download_level(h, l, d.ctypes.data_as(C.POINTER(C.c_int32)),
                                            None if last else o.ctypes.data_as(C.POINTER(C.c_uint64))))
        data.append(d[:lens[l]])
        if not last:
            off.append(o)
    return data, off


def trie_n_build(ctx, cols):
    import torch
    dc = [torch.from_numpy(np.ascontiguousarray(c, np.int32)).cuda() for c in cols]
    n = len(cols[0])
    ptrs = (C.c_void_p * len(cols))(*[c.data_ptr() if n else None for c in dc])
    h = C.c_void_p()
    L.check(L.load().amj_trie_build_n(ctx.handle, ptrs, len(cols), n, C.byref(h)))
    return h


@pytest.mark.parametrize("k,n,case", [(1, 1000, "narrow"), (2, 1 << 20, "rmat"), (3, 200000, "narrow"),
                                      (3, 2_000_000, "wide"), (4, 100000, "const"), (5, 300000, "narrow"),
                                      (3, 0, "empty"), (4, 1, "one"), (8, 5000, "narrow")])
def test_trie_build_n_matches_oracle(ctx, k, n, case):
    rng = np.random.Generator(np.random.PCG64(k * 7 + n))
    if case == "rmat":
        cols = list(data.rmat(16, n, 0.57, 0.19, 0.19, 3))
    elif case == "wide":
        cols = [rng.integers(-(1 << 31), 1 << 31, n, dtype=np.int64).astype(np.int32) for _ in range(k)]
        cols[1][::2] = cols[1][0]
    else:
        cols = [rng.integers(-3, 6, n).astype(np.int32) for _ in range(k)]
        if case == "const":
            cols[2][:] = 77
            cols[0][:] = -(1 << 31)
    h = trie_n_build(ctx, cols)
    got_d, got_o = trie_n_levels(h)
    L.load().amj_trie_release(h)
    want_d, want_o = O.trie_build_n(cols)
    assert len(got_d) == k and len(got_o) == k - 1
    for a, b in zip(got_d, want_d):
        assert np.array_equal(a, b)
    for a, b in zip(got_o, want_o):
        assert np.array_equal(a, b)


def test_trie_n_tr_file_round_trip_and_2_level_compatibility(ctx, tmp_path):
    lib = L.load()
    rng = np.random.Generator(np.random.PCG64(9))
    cols = [rng.integers(0, 50, 40000).astype(np.int32) for _ in range(4)]
    h = trie_n_build(ctx, cols)
    p = str(tmp_path / "t4.tr").encode()
    attrs = (C.c_uint32 * 4)(3, 0, 2, 1)
    L.check(lib.amj_trie_save_n(h, p, attrs))
    h2, got_attrs, lv = C.c_void_p(), (C.c_uint32 * 8)(), C.c_int()
    L.check(lib.amj_trie_load_n(ctx.handle, p, C.byref(h2), got_attrs, C.byref(lv)))
    assert lv.value == 4 and list(got_attrs)[:4] == [3, 0, 2, 1]
    a, b = trie_n_levels(h), trie_n_levels(h2)
    assert all(np.array_equal(x, y) for x, y in zip(a[0] + a[1], b[0] + b[1]))
    # 2-level calls refuse a 4-level trie
    with pytest.raises(AmjError):
        L.check(lib.amj_trie_save(h, p, 0, 1))
    lib.amj_trie_release(h)
    lib.amj_trie_release(h2)
    # a 2-level trie written by either writer is the same file, and both readers read it
    s, d = data.rmat(10, 8000, 0.57, 0.19, 0.19, 4)
    h2l, _, _, _ = trie_arrays(ctx, s, d)
    hn = trie_n_build(ctx, [s, d])
    p1, p2 = str(tmp_path / "a.tr").encode(), str(tmp_path / "b.tr").encode()
    L.check(lib.amj_trie_save(h2l, p1, 5, 6))
    L.check(lib.amj_trie_save_n(hn, p2, (C.c_uint32 * 2)(5, 6)))
    assert open(p1, "rb").read() == open(p2, "rb").read()
    h3 = C.c_void_p()
    L.check(lib.amj_trie_load_n(ctx.handle, p1, C.byref(h3), None, None))
    a, b = trie_n_levels(h2l), trie_n_levels(h3)
    assert all(np.array_equal(x, y) for x, y in zip(a[0] + a[1], b[0] + b[1]))
    # the 2-level download of an N-level trie with two levels
    l0, l1 = C.c_uint64(), C.c_uint64()
    L.check(lib.amj_trie_view(hn, C.byref(l0), C.byref(l1), None, None, None))
    o0, oo, o1 = O.trie_build(s, d)
    assert (l0.value, l1.value) == (len(o0), len(o1))
    for x in (h2l, hn, h3):
        lib.amj_trie_release(x)


# ------------------------------------------------------------------- AMHJ

SWITCHES = [dict(ws=0, dro=0, fib=0), dict(ws=1, dro=0, fib=0), dict(ws=0, dro=1, fib=0), dict(ws=1, dro=1, fib=0),
            dict(ws=1, dro=0, fib=1)]


@pytest.mark.parametrize("layout", ["bucket", "oa", "cuckoo"])
@pytest.mark.parametrize("sw", SWITCHES, ids=lambda s: "ws{ws}dro{dro}fib{fib}".format(**s))
@pytest.mark.parametrize("materialize", [False, True])
def test_amhj_chain_all_switches(layout, sw, materialize):
    with Context(0, layout=layout) as ctx:
        rels = data.chain_relations(20000, 1 << 12, 3, seed=11)
        got = ctx.amhj("NORMAL", rels_on(ctx, rels), materialize=materialize, **sw)
        cnt, chk, cols = O.mhj(rels, tuples=True)
        assert (got.count, got.checksum) == (cnt, chk)
        if materialize:
            assert np.array_equal(sorted_rows(got.columns), sorted_rows(cols))
            assert data.checksum(got.columns) == chk


@pytest.mark.parametrize("case", [c for c in json.load(open(GOLDEN))["cases"] if c["kind"] in ("chain", "star")],
                         ids=lambda c: c["name"])
def test_amhj_golden(ctx, case):
    if case["kind"] == "chain":
        rels = data.chain_relations(case["n"], case["key_range"], case["nrels"], seed=case["seed"])
    else:
        fact, dims = data.star_relations(case["fact_rows"], case["dims"], theta=case["theta"], seed=case["seed"])
        rels = [fact] + dims
    for ws in (0, 1):
        got = ctx.amhj("NORMAL", rels_on(ctx, rels), ws=ws)
        assert got.count == case["count"]
        assert f"{got.checksum:016x}" == case["checksum"]


@pytest.mark.parametrize("layout", ["bucket", "oa", "cuckoo"])
def test_amhj_star(layout):
    with Context(0, layout=layout) as ctx:
        fact, dims = data.star_relations(200000, [20000, 4000, 2000, 200], theta=1.1, seed=8)
        rels = [fact] + dims
        for sw in SWITCHES:
            got = ctx.amhj("NORMAL", rels_on(ctx, rels), **sw)
            assert (got.count, got.checksum) == O.mhj(rels)


@pytest.mark.parametrize("shape", ["chain4", "star", "tri", "four"])
def test_amhj_baseline_plans_match_oracle(ctx, shape):
    """The comparators of the reference's baselines: one thread per probe
    row (MHJ-GPU/Joins/MHJ.cuh) and a pairwise plan with materialised
    intermediates (MHJ-GPU/exec_PW.cu) give the operator's result."""
    if shape == "chain4":
        rels = data.chain_relations(30000, 1 << 12, 4, seed=12)
    elif shape == "star":
        fact, dims = data.star_relations(50000, [5000, 1000, 500, 50], theta=1.1, seed=13)
        rels = [fact] + dims
    else:
        s, d = data.rmat(10, 8000, 0.57, 0.19, 0.19, seed=14)
        rels = [([s, d], [0, 1])]
    hs = [ctx.relation(c, a) for c, a in rels]
    qt = {"tri": "TRI", "four": "FOUR"}.get(shape, "NORMAL")
    want = O.mhj(rels) if qt == "NORMAL" else (O.triangle(*rels[0][0]) if qt == "TRI" else O.four_clique(*rels[0][0]))
    for dego in (True, False):
        t = ctx.amhj(qt, hs, plan="thread_per_row", degree_order=dego)
        assert (t.count, t.checksum) == want
    if qt == "NORMAL":
        p = ctx.amhj(qt, hs, plan="pairwise")
        assert (p.count, p.checksum) == want and p.stats["slices"] == len(rels) - 1
        m = ctx.amhj(qt, hs, plan="pairwise", materialize=True)
        assert data.checksum(m.columns) == want[1]
        assert np.array_equal(sorted_rows(m.columns), sorted_rows(O.mhj(rels, tuples=True)[2]))
    with pytest.raises(AmjError):
        ctx.amhj(qt, hs, plan="thread_per_row", materialize=True)


def test_amhj_out_of_core_many_parts_host_partitioning():
    """A device budget so small that a stage needs more than 256 parts: the
    rows are then partitioned by the scatter on the host cores instead of the
    device grouping (which serves up to 256 parts).  Equal to the oracle and
    to the same query under a budget that groups on the device."""
    rels = [([data.uniform(50_000, 0, 50_000, 71 + i, 0), data.uniform(50_000, 0, 50_000, 71 + i, 1)], [i, i + 1])
            for i in range(3)]
    want = O.mhj(rels)
    with Context(0, mem_budget=4 << 10) as ctx:
        host = [ctx.relation(c, a, streamed=True) for c, a in rels]
        got = ctx.amhj("NORMAL", host, ooc=1)
        assert (got.count, got.checksum) == want
        assert got.stats["slices"] > 2 * 256   # part joins
    with Context(0, mem_budget=256 << 10) as ctx:
        host = [ctx.relation(c, a, streamed=True) for c, a in rels]
        got = ctx.amhj("NORMAL", host, ooc=1, materialize=True)
        assert (got.count, got.checksum) == want
        assert data.checksum(got.columns) == want[1]


def test_amhj_star_flat_path_with_repeated_dimension_keys(ctx):
    """Star count queries take the flat kernel (one thread per fact row, all
    dimension lookups together).  Dimensions with repeated keys give rows a
    product of matches; rows whose product exceeds the flat kernel's bound
    (a key repeated in every dimension) are joined by the DFS kernel after it.
    Equal to the oracle, count mode and materialised."""
    rng = np.random.Generator(np.random.PCG64(17))
    n = 100_000
    fact = [rng.integers(0, 500, n).astype(np.int32) for _ in range(3)]
    fact[0][:2000] = 7
    fact[1][:2000] = 7
    fact[2][:2000] = 7
    dims = []
    for j in range(3):
        keys = rng.integers(0, 500, 3000).astype(np.int32)
        keys[:40] = 7                          # 40^3 = 64000 tuples per hub row
        dims.append(([keys, rng.integers(-1000, 1000, 3000).astype(np.int32)], [j, 3 + j]))
    rels = [(fact, [0, 1, 2])] + dims
    want = O.mhj(rels)
    hs = [ctx.relation(c, a) for c, a in rels]
    for ws in (0, 1):
        got = ctx.amhj("NORMAL", hs, ws=ws)
        assert (got.count, got.checksum) == want, ws
    m = ctx.amhj("NORMAL", hs, materialize=True)
    assert (m.count, m.checksum) == want


@pytest.mark.parametrize("ndims", [1, 2, 3, 4])
def test_amhj_star_canonical_and_general_attribute_numbering(ctx, ndims):
    """The flat star count path has two kernels: one for the canonical
    numbering F(0..d-1), D_j(j, d + j), whose values stay in registers, and
    the general one for any other numbering.  The same star under both
    numberings (and dimensions given in reverse order) equals the oracle,
    with unique dimension keys, repeated keys (products of 2-256) and absent
    keys (empty products)."""
    rng = np.random.Generator(np.random.PCG64(40 + ndims))
    n = 60_000
    fact = [rng.integers(0, 3000, n).astype(np.int32) for _ in range(ndims)]
    dims = []
    for j in range(ndims):
        if j % 2 == 0:
            keys = rng.permutation(3000).astype(np.int32)[:2500]         # unique, some absent
        else:
            keys = rng.integers(0, 3000, 7000).astype(np.int32)          # repeated, some absent
        dims.append([keys, rng.integers(-(1 << 31), 1 << 31, len(keys), dtype=np.int64).astype(np.int32)])
    canon = [(fact, list(range(ndims)))] + [(dims[j], [j, ndims + j]) for j in range(ndims)][::-1]
    other = [(fact, [2 * j + 1 for j in range(ndims)])] + [(dims[j], [2 * j + 1, 2 * j]) for j in range(ndims)]
    for rels in (canon, other):
        want = O.mhj(rels)
        assert want[0] > 0
        hs = [ctx.relation(c, a) for c, a in rels]
        for ws in (0, 1):
            got = ctx.amhj("NORMAL", hs, ws=ws)
            assert (got.count, got.checksum) == want, (rels[0][1], ws)
        got = ctx.amhj("NORMAL", hs, plan="frontier")
        assert (got.count, got.checksum) == want


@pytest.mark.parametrize("nlev", [1, 2, 3, 4])
def test_amhj_chain_flat_walk_and_listed_rows(ctx, nlev):
    """Count queries over a canonical chain R0(0, 1) R_d(d + 1, d + 2) take
    the flat walk (one thread per probe row, one bucket head a lookup).
    Buckets of one to three rows are read from the head, longer ones from
    the columns, and rows whose walk exceeds its budget (a hot key) are
    joined by the DFS kernel.  Equal to the oracle for ws 0 and 1, and equal
    under another attribute numbering, which the DFS kernel joins."""
    rng = np.random.Generator(np.random.PCG64(60 + nlev))
    n = 40_000
    rels = [([rng.integers(0, 5000, n).astype(np.int32), rng.integers(0, 4000, n).astype(np.int32)], [0, 1])]
    for d in range(nlev):
        keys = rng.integers(0, 4000, 6000 + 3000 * d).astype(np.int32)
        keys[:700] = 11                      # a hot key: its rows exceed the walk's budget
        pay = rng.integers(0, 4000, len(keys)).astype(np.int32)
        rels.append(([keys, pay], [d + 1, d + 2]))
    rels[0][0][1][:50] = 11
    want = O.mhj(rels)
    assert want[0] > 0
    hs = [ctx.relation(c, a) for c, a in rels]
    for ws in (0, 1):
        got = ctx.amhj("NORMAL", hs, ws=ws)
        assert (got.count, got.checksum) == want, ws
    got = ctx.amhj("NORMAL", hs, plan="frontier")        # the frontier-DFS kernel for every row
    assert (got.count, got.checksum) == want
    k = nlev + 2
    other = [(c, [k - 1 - x for x in a]) for c, a in rels]   # the same chain, attributes numbered from the end
    got = ctx.amhj("NORMAL", [ctx.relation(c, a) for c, a in other])
    assert (got.count, got.checksum) == O.mhj(other)


@pytest.mark.parametrize("qt", ["TRI", "FOUR"])
@pytest.mark.parametrize("reorder", [True, False])
@pytest.mark.parametrize("degree_order", [True, False])
@pytest.mark.parametrize("plan", ["multiway", "hash"])
def test_amhj_tri_four(ctx, qt, reorder, degree_order, plan):
    """Every switch, on the relation as given and on its degree-ordered copy
    (the default for an oriented relation), through the bitmap / triangle
    matrix levels (plan "multiway" on the degree-ranked copy) and with every
    level a hash lookup; tuples come out in increasing order either way."""
    s, d = data.rmat(10, 6000, 0.57, 0.19, 0.19, seed=21)
    e = ctx.relation([s, d], [0, 1])
    want = O.triangle(s, d) if qt == "TRI" else O.four_clique(s, d)
    for sw in SWITCHES:
        got = ctx.amhj(qt, [e], reorder=reorder, degree_order=degree_order, plan=plan, **sw)
        assert (got.count, got.checksum) == want, sw
    got = ctx.amhj(qt, [e], materialize=True, reorder=reorder, degree_order=degree_order, plan=plan)
    assert data.checksum(got.columns) == want[1]
    t = got.tuples()
    assert np.all(t[:, :-1] < t[:, 1:])


@pytest.mark.parametrize("qt", ["TRI", "FOUR"])
def test_amhj_tri_four_repeated_rows_keep_bag_semantics(ctx, qt):
    """The hash join counts a repeated edge once per copy (a bag), the trie
    paths join sets: an oriented relation with repeated rows takes the
    level-by-level hash plan, equal to the oracle's multi-way join of the
    attribute pattern, while ALFTJ gives the set result."""
    s, d = data.rmat(9, 3000, 0.6, 0.15, 0.15, seed=3)
    s2, d2 = np.concatenate([s, s[:300]]), np.concatenate([d, d[:300]])
    e = ctx.relation([s2, d2], [0, 1])
    pattern = O.tri_relations(s2, d2) if qt == "TRI" else O.four_relations(s2, d2)
    want = O.mhj(pattern)
    for sw in ({}, {"ws": 1}, {"ws": 1, "fib": 1}):
        got = ctx.amhj(qt, [e], **sw)
        assert (got.count, got.checksum) == want, sw
    sets = ctx.lftj([e], clique4=qt == "FOUR")
    assert sets.count < want[0]
    assert (sets.count, sets.checksum) == (O.triangle(s, d) if qt == "TRI" else O.four_clique(s, d))


def test_amhj_dro_residual_resume():
    """An estimate far too small forces breakpoints and the residual pass."""
    with Context(0, dro_headroom=0.01) as ctx:
        rels = data.chain_relations(50000, 1 << 12, 3, seed=12)
        for ws in (0, 1):
            got = ctx.amhj("NORMAL", rels_on(ctx, rels), ws=ws, dro=1, materialize=True)
            cnt, chk, cols = O.mhj(rels, tuples=True)
            assert (got.count, got.checksum) == (cnt, chk)
            assert got.stats["residual_units"] > 0 and got.stats["rows_written_residual"] > 0
            assert np.array_equal(sorted_rows(got.columns), sorted_rows(cols))


def test_amhj_work_sharing_on_skew():
    """Zipf keys make a few huge buckets (about 9M output tuples); small tasks
    force splits below level 0 and level-0 chunks balance the probe side."""
    with Context(0, task_chunk=32) as ctx:
        n = 20000
        r1 = ([data.uniform(n, 0, 1000, 1), data.zipf(n, 1000, 1.2, 2)], [0, 1])
        r2 = ([data.zipf(n, 1000, 1.2, 3), data.uniform(n, 0, 1 << 16, 4)], [1, 2])
        r3 = ([data.uniform(n, 0, 1 << 16, 5), data.uniform(n, 0, 1 << 20, 6)], [2, 3])
        rels = [r1, r2, r3]
        want = O.mhj(rels)
        for dro in (0, 1):
            got = ctx.amhj("NORMAL", rels_on(ctx, rels), ws=1, dro=dro, materialize=bool(dro))
            assert (got.count, got.checksum) == want
            assert got.stats["tasks_popped"] == got.stats["tasks_pushed"]
            if dro:
                assert data.checksum(got.columns) == want[1]
        # a chain whose level-1 buckets are large: the task queue is used
        q = [([data.uniform(100, 0, 100, 1), data.uniform(100, 0, 100, 2)], [0, 1]),
             ([data.uniform(2000, 0, 100, 3), data.uniform(2000, 0, 4, 4)], [1, 2]),
             ([data.uniform(20000, 0, 4, 5), data.uniform(20000, 0, 1 << 20, 6)], [2, 3])]
        got = ctx.amhj("NORMAL", rels_on(ctx, q), ws=1)
        assert (got.count, got.checksum) == O.mhj(q)
        assert got.stats["tasks_pushed"] > 0 and got.stats["tasks_popped"] == got.stats["tasks_pushed"]


def fib_chain(n, dom):
    """A 4-way chain whose middle join attribute (2) is Zipf-skewed on both
    sides: the partial tuples reaching R2 concentrate on a few keys, each with
    a large bucket, so their suffix tuples are worth caching."""
    r0 = ([data.uniform(n, 0, 5000, 1), data.uniform(n, 0, dom, 2)], [0, 1])
    r1 = ([data.uniform(n, 0, dom, 3), data.zipf(n, dom, 1.1, 4)], [1, 2])
    r2 = ([data.zipf(n, dom, 1.1, 5), data.uniform(n, 0, 4000, 6)], [2, 3])
    r3 = ([data.uniform(n, 0, 4000, 7), data.uniform(n, 0, 1 << 20, 8)], [3, 4])
    return [r0, r1, r2, r3]


def test_amhj_fib_caches_frequent_suffixes():
    """Frequent-item buffering: same count/checksum as fib=0 and the oracle,
    and the cache is used (850M tuples, most of them served from it)."""
    with Context(0) as ctx:
        rels = fib_chain(20000, 2000)
        want = O.mhj(rels)
        rs = rels_on(ctx, rels)
        off = ctx.amhj("NORMAL", rs, ws=1, fib=0)
        on = ctx.amhj("NORMAL", rs, ws=1, fib=1)
        assert (off.count, off.checksum) == want
        assert (on.count, on.checksum) == want
        assert on.stats["fib_keys"] > 0 and on.stats["fib_rows_cached"] > 0
        assert on.stats["fib_rows_served"] > want[0] // 4
        assert off.stats["fib_keys"] == 0


@pytest.mark.parametrize("layout", ["bucket", "oa", "cuckoo"])
def test_amhj_fib_materialized_and_other_layouts(layout):
    """Materialised tuples with the cache on; the open-addressing and cuckoo
    layouts run without a cache and still agree."""
    with Context(0, layout=layout) as ctx:
        rels = fib_chain(4000, 2000)
        cnt, chk, cols = O.mhj(rels, tuples=True)
        got = ctx.amhj("NORMAL", rels_on(ctx, rels), fib=1, materialize=True)
        assert (got.count, got.checksum) == (cnt, chk)
        assert np.array_equal(sorted_rows(got.columns), sorted_rows(cols))
        if layout == "bucket":
            assert got.stats["fib_rows_served"] > 0


def test_amhj_fib_star_and_out_of_core():
    """A star join with a shared key (every level keyed on attribute 0) is
    cacheable below level 1; the cache also serves every slice of an
    out-of-core run."""
    n = 5000
    rels = [([data.zipf(n, 3000, 0.8, 1), data.uniform(n, 0, 1 << 20, 2)], [0, 1]),
            ([data.uniform(3000, 0, 3000, 3), data.uniform(3000, 0, 1 << 20, 4)], [0, 2]),
            ([data.zipf(n, 3000, 0.8, 5), data.uniform(n, 0, 1 << 20, 6)], [0, 3]),
            ([data.zipf(n, 3000, 0.8, 7), data.uniform(n, 0, 1 << 20, 8)], [0, 4])]
    want = O.mhj(rels)
    with Context(0, ooc_slice_rows=4096) as ctx:
        rs = rels_on(ctx, rels)
        for ooc in (0, 1):
            got = ctx.amhj("NORMAL", rs, ooc=ooc, fib=1)
            assert (got.count, got.checksum) == want, ooc
            assert got.stats["fib_keys"] > 0


@pytest.mark.parametrize("streamed", [False, True])
@pytest.mark.parametrize("materialize", [False, True])
def test_amhj_out_of_core(streamed, materialize):
    with Context(0, ooc_slice_rows=3000) as ctx:
        rels = data.chain_relations(20000, 1 << 11, 3, seed=13)
        handles = [ctx.relation(rels[0][0], rels[0][1], streamed=streamed)] + rels_on(ctx, rels[1:])
        for sw in SWITCHES[:4]:
            got = ctx.amhj("NORMAL", handles, ooc=1, materialize=materialize, **sw)
            cnt, chk = O.mhj(rels)
            assert (got.count, got.checksum) == (cnt, chk)
            assert got.stats["slices"] == 7
            if materialize:
                assert data.checksum(got.columns) == chk


def test_amhj_out_of_core_streamed_large_slices():
    """Host-streamed probe whose staging buffers are fresh pool allocations
    (4M rows, 1M-row slices, pinned and pageable host columns): equal to the
    device-resident join."""
    import torch
    n = 1 << 22
    rels = [([data.uniform(n, 0, n, 31 + i, 0), data.uniform(n, 0, n, 31 + i, 1)], [i, i + 1]) for i in range(4)]
    with Context(0, ooc_slice_rows=1 << 20) as ctx:
        dev = [ctx.relation(c, a) for c, a in rels]
        want = ctx.amhj("NORMAL", dev)
        pinned = [torch.from_numpy(c).pin_memory() for c in rels[0][0]]
        for cols in (rels[0][0], [p.numpy() for p in pinned]):
            probe = ctx.relation(cols, rels[0][1], streamed=True)
            for ws in (0, 1):
                got = ctx.amhj("NORMAL", [probe] + dev[1:], ooc=1, ws=ws)
                assert (got.count, got.checksum) == (want.count, want.checksum)
                assert got.stats["slices"] == 4


@pytest.mark.parametrize("shape", ["chain4", "star4", "cyclic"])
def test_amhj_out_of_core_build_relations_in_host_memory(shape):
    """Build relations kept in host memory (streamed=True) with ooc=1: the
    join runs in stages, each intermediate and build relation hash-partitioned
    on the key into parts within the memory budget (far below the inputs
    here), joined part by part.  Equal to the device-resident join and to the
    oracle, for every switch."""
    if shape == "chain4":
        n = 200_000
        rels = [([data.uniform(n, 0, n, 51 + i, 0), data.uniform(n, 0, n, 51 + i, 1)], [i, i + 1]) for i in range(4)]
    elif shape == "star4":
        fact, dims = data.star_relations(150_000, [20000, 5000, 2000, 300], theta=1.1, seed=9)
        rels = [fact] + dims
    else:   # a cycle closed by the last relation: a compared attribute besides the key
        rels = [([data.uniform(30000, 0, 3000, 61 + i, 0), data.uniform(30000, 0, 3000, 61 + i, 1)], p)
                for i, p in enumerate([[0, 1], [1, 2], [2, 3], [3, 0]])]
    want = O.mhj(rels)
    with Context(0, mem_budget=512 << 10) as ctx:
        dev = [ctx.relation(c, a) for c, a in rels]
        assert (lambda r: (r.count, r.checksum))(ctx.amhj("NORMAL", dev)) == want
        host = [ctx.relation(c, a, streamed=True) for c, a in rels]
        for sw in ({}, {"ws": 1}, {"dro": 1}):
            got = ctx.amhj("NORMAL", host, ooc=1, **sw)
            assert (got.count, got.checksum) == want, sw
            assert got.stats["slices"] >= 4
        # the pinned blocks the stages keep, given back; then a device probe
        # with host builds, and the materialised tuples
        ctx.trim()
        got = ctx.amhj("NORMAL", [dev[0]] + host[1:], ooc=1, materialize=True)
        assert (got.count, got.checksum) == want
        assert data.checksum(got.columns) == want[1]
        if shape == "cyclic":
            cnt, chk, cols = O.mhj(rels, tuples=True)
            assert np.array_equal(sorted_rows(got.columns), sorted_rows(cols))
        with pytest.raises(AmjError):
            ctx.amhj("NORMAL", host, ooc=0)


def test_amhj_edge_cases(ctx):
    z = np.zeros(0, np.int32)
    one = ([np.array([3], np.int32), np.array([4], np.int32)], [0, 1])
    cases = [
        [([z, z], [0, 1]), ([z, z], [1, 2])],
        [one, ([z, z], [1, 2])],
        [([z, z], [0, 1]), one and ([np.array([4], np.int32), np.array([9], np.int32)], [1, 2])],
        [one, ([np.array([4, 4, 4], np.int32), np.array([7, 8, 9], np.int32)], [1, 2])],
        # every key equal: one bucket holds the whole relation
        [([np.full(3000, 5, np.int32), np.arange(3000, dtype=np.int32)], [0, 1]),
         ([np.arange(3000, dtype=np.int32) % 7, np.full(3000, -1, np.int32)], [1, 2])],
        # extreme values
        [([np.array([-2**31, 2**31 - 1, 0], np.int32), np.array([2**31 - 1, -2**31, -1], np.int32)], [0, 1]),
         ([np.array([2**31 - 1, -2**31, -1], np.int32), np.array([1, 2, 3], np.int32)], [1, 2])],
    ]
    for rels in cases:
        want = O.mhj(rels)
        for sw in SWITCHES:
            got = ctx.amhj("NORMAL", rels_on(ctx, rels), materialize=True, **sw)
            assert (got.count, got.checksum) == want, (rels, sw)


def test_amhj_single_relation(ctx):
    rels = [([data.uniform(100, 0, 10, 1), data.uniform(100, 0, 10, 2)], [0, 1])]
    got = ctx.amhj("NORMAL", rels_on(ctx, rels), materialize=True)
    assert (got.count, got.checksum) == O.mhj(rels)


def test_amhj_rejects_bad_queries(ctx):
    a = ctx.relation([np.arange(4, dtype=np.int32), np.arange(4, dtype=np.int32)], [0, 2])
    b = ctx.relation([np.arange(4, dtype=np.int32), np.arange(4, dtype=np.int32)], [3, 4])
    with pytest.raises(AmjError) as e:
        ctx.amhj("NORMAL", [a, b])
    assert e.value.status == L.AMJ_EINVAL
    c = ctx.relation([np.arange(4, dtype=np.int32), np.arange(4, dtype=np.int32)], [0, 1])
    d = ctx.relation([np.arange(4, dtype=np.int32), np.arange(4, dtype=np.int32)], [2, 3])
    with pytest.raises(AmjError) as e:
        ctx.amhj("NORMAL", [c, d])
    assert e.value.status == L.AMJ_EUNSUPPORTED


# ------------------------------------------------------------------- ALFTJ

@pytest.mark.parametrize("algo", ["DFS", "BFS"])
@pytest.mark.parametrize("ws", [0, 1])
@pytest.mark.parametrize("heavy", [0, 1, 8])
@pytest.mark.parametrize("rankbits", [0, 32])
def test_lftj_triangle_small(algo, ws, heavy, rankbits):
    """DFS ws=1 is the wedge kernel over the degree-ranked copy; rankbits 32
    sends nearly every lookup below the bitmap, to the binary search."""
    if rankbits and (algo == "BFS" or not ws):
        pytest.skip("the wedge kernel is the DFS ws=1 path")
    with Context(0, lftj_heavy_degree=heavy, lftj_rank_bits=rankbits) as ctx:
        for seed, scale, ne in [(1, 8, 1500), (2, 12, 50000)]:
            s, d = data.rmat(scale, ne, 0.57, 0.19, 0.19, seed)
            e = ctx.relation([s, d], [0, 1])
            got = ctx.lftj([e], algo=algo, ws=ws)
            assert (got.count, got.checksum) == O.triangle(s, d)
            if algo == "DFS" and ws:
                m = ctx.lftj([e], algo=algo, ws=ws, materialize=True)
                assert (m.count, m.checksum) == (got.count, got.checksum)
                assert data.checksum(m.columns) == got.checksum


@pytest.mark.parametrize("scale,ne,seed", [(8, 1500, 1), (12, 60000, 2), (14, 1 << 18, 22)])
def test_lftj_clique4_matches_oracle_and_amhj_four(ctx, scale, ne, seed):
    """The ALFTJ 4-clique equals the oracle and AMHJ FOUR on the same relation
    (skewed R-MAT, 0.6/0.15/0.15/0.1); the largest case has hub edges that
    take the warp-cooperative path."""
    s, d = data.rmat(scale, ne, 0.6, 0.15, 0.15, seed)
    e = ctx.relation([s, d], [0, 1])
    want = O.four_clique(s, d)
    got = ctx.lftj([e], algo="DFS", clique4=True)
    assert (got.count, got.checksum) == want
    four = ctx.amhj("FOUR", [e], ws=1)
    assert (four.count, four.checksum) == want


@pytest.mark.parametrize("algo", ["DFS", "BFS", "clique4"])
def test_lftj_degree_order_gives_the_same_bag(ctx, algo):
    """An oriented relation may be joined through its degree-ordered copy (the
    default for BFS and the 4-clique): same count, checksum and tuples.  A
    relation that is not oriented is always joined as given."""
    s, d = data.rmat(13, 100000, 0.57, 0.19, 0.19, 9)
    e = ctx.relation([s, d], [0, 1])
    c4 = algo == "clique4"
    run = dict(algo="DFS" if c4 else algo, clique4=c4)
    want = O.four_clique(s, d) if c4 else O.triangle(s, d)
    for dego in (None, True, False):
        r = ctx.lftj([e], degree_order=dego, **run)
        assert (r.count, r.checksum) == want, dego
    m1 = ctx.lftj([e], degree_order=True, materialize=True, **run)
    m0 = ctx.lftj([e], degree_order=False, materialize=True, **run)
    assert np.array_equal(sorted_rows(m1.columns), sorted_rows(m0.columns))
    if not c4:
        rev = ctx.relation([d, s], [0, 1])   # every edge v > u: not oriented
        r = ctx.lftj([rev], degree_order=True, **run)
        assert (r.count, r.checksum) == O.triangle(d, s)


def test_lftj_clique4_materialized_and_rejections(ctx):
    s, d = data.rmat(11, 20000, 0.6, 0.15, 0.15, 7)
    e = ctx.relation([s, d], [0, 1])
    got = ctx.lftj([e], algo="DFS", clique4=True, materialize=True)
    cnt, chk = O.four_clique(s, d)
    assert got.count == cnt and len(got.columns) == 4
    assert data.checksum(got.columns) == chk
    m = ctx.amhj("FOUR", [e], materialize=True)
    assert np.array_equal(sorted_rows(got.columns), sorted_rows(m.columns))
    with pytest.raises(AmjError):
        ctx.lftj([e], algo="BFS", clique4=True)
    ooc = ctx.lftj([e], algo="DFS", clique4=True, ooc=1)
    assert (ooc.count, ooc.checksum) == (cnt, chk)
    empty = ctx.relation([np.zeros(0, np.int32), np.zeros(0, np.int32)], [0, 1])
    r = ctx.lftj([empty], clique4=True)
    assert (r.count, r.checksum) == (0, 0)


@pytest.mark.parametrize("algo", ["DFS", "BFS"])
def test_lftj_materialized_tuples(ctx, algo):
    s, d = data.rmat(11, 20000, 0.57, 0.19, 0.19, 5)
    e = ctx.relation([s, d], [0, 1])
    cnt, chk, cols = O.triangle(s, d, tuples=True)
    for ws in (0, 1):
        got = ctx.lftj([e], algo=algo, ws=ws, materialize=True)
        assert (got.count, got.checksum) == (cnt, chk)
        assert np.array_equal(sorted_rows(got.columns), sorted_rows(cols))


def test_lftj_three_relations_and_cross_operator(ctx):
    s, d = data.rmat(11, 20000, 0.57, 0.19, 0.19, 6)
    want = O.triangle(s, d)
    # three relations (0,1), (2,1) given with swapped column order, (0,2)
    R = ctx.relation([s, d], [0, 1])
    S = ctx.relation([d, s], [2, 1])
    T = ctx.relation([s, d], [0, 2])
    for algo in ("DFS", "BFS"):
        got = ctx.lftj([S, T, R], algo=algo)
        assert (got.count, got.checksum) == want
    e = ctx.relation([s, d], [0, 1])
    amhj = ctx.amhj("TRI", [e], ws=1)
    dfs = ctx.lftj([e], algo="DFS")
    bfs = ctx.lftj([e], algo="BFS")
    assert (amhj.count, amhj.checksum) == (dfs.count, dfs.checksum) == (bfs.count, bfs.checksum) == want


def distinct_rel(n, dom, seed, attrs):
    """A 2-column relation of distinct tuples (the LFTJ set semantics)."""
    a = data.uniform(n, 0, dom, seed, 0)
    b = data.uniform(n, 0, dom, seed, 1)
    pairs = np.unique(np.stack([a, b], 1), axis=0)
    return ([np.ascontiguousarray(pairs[:, 0]), np.ascontiguousarray(pairs[:, 1])], attrs)


GENERIC_QUERIES = {
    "4-cycle": [(0, 1), (1, 2), (2, 3), (0, 3)],
    "path4": [(0, 1), (1, 2), (2, 3)],
    "4-clique": [(0, 1), (1, 2), (2, 3), (0, 3), (0, 2), (1, 3)],
    "5-cycle+chord": [(0, 1), (1, 2), (2, 3), (3, 4), (0, 4), (1, 3)],
    "swapped columns": [(1, 0), (2, 1), (0, 2), (3, 2)],
}


@pytest.mark.parametrize("name", list(GENERIC_QUERIES))
@pytest.mark.parametrize("algo", ["DFS", "BFS"])
def test_lftj_generic_queries_match_amhj_and_oracle(ctx, name, algo):
    """Queries beyond the triangle (the reference's LFTJ stops at 3
    attributes and 3 tables) run through the generic leapfrog join: equal to
    AMHJ on the same relations and to the oracle."""
    pats = GENERIC_QUERIES[name]
    dom = 300 if len(pats) <= 4 else 120
    rels = [distinct_rel(4000, dom, 40 + i, list(p)) for i, p in enumerate(pats)]
    hs = [ctx.relation(c, a) for c, a in rels]
    want = O.mhj(rels)
    got = ctx.lftj(hs, algo=algo)
    assert (got.count, got.checksum) == want
    assert got.num_attrs == 1 + max(max(p) for p in pats)
    amhj = ctx.amhj("NORMAL", hs)
    assert (amhj.count, amhj.checksum) == want


def distinct_rows(n, dom, seed, attrs):
    """A relation of distinct tuples with len(attrs) columns."""
    cols = [data.uniform(n, 0, dom, seed, s) for s in range(len(attrs))]
    rows = np.unique(np.stack(cols, 1), axis=0)
    return ([np.ascontiguousarray(rows[:, j]) for j in range(len(attrs))], attrs)


# binding orders in which every attribute shares a relation with an earlier one
ORDERS = {
    "4-cycle": [(0, 1, 2, 3), (3, 2, 1, 0), (2, 1, 0, 3), (1, 0, 3, 2)],
    "5-cycle+chord": [(4, 3, 2, 1, 0), (1, 3, 0, 2, 4), (2, 1, 3, 4, 0)],
    "path4": [(3, 2, 1, 0), (1, 2, 0, 3)],
}


@pytest.mark.parametrize("name", list(ORDERS))
def test_lftj_attribute_orders_give_the_same_result(ctx, name):
    """attr_order (the reference's OOCWrapper / ALFTJ argument,
    LFTJ-GPU/ALFTJ.cuh:1125-1196, always the identity in its driver): every
    binding order gives the same bag, hashed and written in attribute-id
    order."""
    pats = GENERIC_QUERIES[name]
    rels = [distinct_rel(3000, 150 if len(pats) > 4 else 250, 70 + i, list(p)) for i, p in enumerate(pats)]
    hs = [ctx.relation(c, a) for c, a in rels]
    want = O.mhj(rels)
    for order in ORDERS[name]:
        got = ctx.lftj(hs, attr_order=order)
        assert (got.count, got.checksum) == want, order
    m = ctx.lftj(hs, attr_order=ORDERS[name][-1], materialize=True)
    cnt, chk, cols = O.mhj(rels, tuples=True)
    assert np.array_equal(sorted_rows(m.columns), sorted_rows(cols))
    if name == "4-cycle":
        # attributes 1 and 3 share no relation: binding 3 second is a cross product
        with pytest.raises(AmjError) as e:
            ctx.lftj(hs, attr_order=(1, 3, 0, 2))
        assert e.value.status == L.AMJ_EUNSUPPORTED


@pytest.mark.parametrize("clique4", [False, True])
def test_lftj_self_join_in_other_orders(ctx, clique4):
    s, d = data.rmat(10, 9000, 0.57, 0.19, 0.19, 12)
    e = ctx.relation([s, d], [0, 1])
    want = O.four_clique(s, d) if clique4 else O.triangle(s, d)
    orders = [(3, 1, 0, 2), (1, 2, 3, 0)] if clique4 else [(2, 1, 0), (1, 0, 2), (0, 1, 2)]
    for order in orders:
        got = ctx.lftj([e], clique4=clique4, attr_order=order)
        assert (got.count, got.checksum) == want, order
    # three relations of the triangle pattern, a non-identity order
    hs = [ctx.relation([s, d], [0, 1]), ctx.relation([s, d], [1, 2]), ctx.relation([s, d], [0, 2])]
    if not clique4:
        assert (lambda r: (r.count, r.checksum))(ctx.lftj(hs, attr_order=(2, 0, 1))) == want
    with pytest.raises(AmjError):
        ctx.lftj([e], attr_order=(0, 0, 1))
    ooc = ctx.lftj([e], clique4=clique4, attr_order=(1, 0, 2, 3)[:4 if clique4 else 3], ooc=1)
    assert (ooc.count, ooc.checksum) == want


@pytest.mark.parametrize("order", [None, (2, 0, 1, 3), (3, 2, 1, 0)])
def test_lftj_relations_of_three_columns(ctx, order):
    """Tries of three columns (build_trieN) in the generic join: a ternary
    relation R(0,1,2) with binary S(1,3), T(2,3), a unary U(3), equal to the
    oracle's multi-way join (the reference's LFTJ takes 2 columns only)."""
    R = distinct_rows(20000, 40, 81, [0, 1, 2])
    S = distinct_rel(1500, 40, 82, [1, 3])
    T = distinct_rel(1500, 40, 83, [2, 3])
    U = ([np.unique(data.uniform(30, 0, 40, 84, 0))], [3])
    rels = [R, S, T, U]
    hs = [ctx.relation(c, a) for c, a in rels]
    want = O.mhj(rels)
    assert want[0] > 0
    got = ctx.lftj(hs, attr_order=order)
    assert (got.count, got.checksum) == want
    m = ctx.lftj(hs, attr_order=order, materialize=True)
    assert np.array_equal(sorted_rows(m.columns), sorted_rows(O.mhj(rels, tuples=True)[2]))
    # a 4-column relation against two binary ones
    Q = distinct_rows(8000, 12, 85, [0, 1, 2, 3])
    rels2 = [Q, distinct_rel(100, 12, 86, [0, 4]), distinct_rel(100, 12, 87, [3, 4])]
    got = ctx.lftj([ctx.relation(c, a) for c, a in rels2], attr_order=None if order is None else (4, 0, 1, 2, 3))
    assert (got.count, got.checksum) == O.mhj(rels2)


def test_lftj_generic_materialized_and_rejections(ctx):
    rels = [distinct_rel(3000, 200, 60 + i, list(p)) for i, p in enumerate(GENERIC_QUERIES["4-cycle"])]
    hs = [ctx.relation(c, a) for c, a in rels]
    got = ctx.lftj(hs, materialize=True)
    cnt, chk, cols = O.mhj(rels, tuples=True)
    assert got.count == cnt and data.checksum(got.columns) == chk
    assert np.array_equal(sorted_rows(got.columns), sorted_rows(cols))
    # attribute 2 shares no relation with an earlier attribute: a cross product
    bad = [ctx.relation(c, a) for c, a in [distinct_rel(100, 50, 1, [0, 1]), distinct_rel(100, 50, 2, [2, 3]),
                                            distinct_rel(100, 50, 3, [1, 3])]]
    with pytest.raises(AmjError) as e:
        ctx.lftj(bad)
    assert e.value.status == L.AMJ_EUNSUPPORTED
    ooc = ctx.lftj(hs, ooc=1)
    assert (ooc.count, ooc.checksum) == (cnt, chk)


@pytest.mark.parametrize("rankbits", [0, 32, 1000])
def test_lftj_wedge_kernel_bitmap_and_low_prefix(rankbits):
    """R-MAT scale 17: with the default bitmap nearly every value is a bit
    test; with 32 ranks, vertices b with more than 256 children below the
    bitmap search S(b) in device memory instead of shared memory."""
    s, d = data.rmat(17, 1 << 21, 0.57, 0.19, 0.19, 3)
    want = O.triangle(s, d)
    with Context(0, lftj_rank_bits=rankbits) as ctx:
        e = ctx.relation([s, d], [0, 1])
        got = ctx.lftj([e], algo="DFS", ws=1)
        assert (got.count, got.checksum) == want
        keep = ctx.lftj([e], algo="DFS", ws=1, degree_order=False)
        assert (keep.count, keep.checksum) == want
    s, d = data.rmat(10, 9000, 0.57, 0.19, 0.19, 4)
    cnt, chk, cols = O.triangle(s, d, tuples=True)
    with Context(0, lftj_rank_bits=rankbits, ooc_slice_rows=2000) as ctx:
        e = ctx.relation([s, d], [0, 1])
        for ooc in (0, 1):
            m = ctx.lftj([e], algo="DFS", ws=1, ooc=ooc, materialize=True)
            assert (m.count, m.checksum) == (cnt, chk)
            assert np.array_equal(sorted_rows(m.columns), sorted_rows(cols))


def tiny_graphs():
    k5 = [(u, v) for u in range(5) for v in range(u + 1, 5)]
    big = [(5, 1 << 30), (5, (1 << 31) - 2), (1 << 30, (1 << 31) - 2), (7, 9)]
    return {"K5": k5, "one triangle": [(0, 1), (0, 2), (1, 2)], "star": [(0, 1), (0, 2), (0, 3)],
            "one edge": [(3, 4)], "sparse huge ids": big,
            "two triangles on an edge": [(0, 1), (0, 2), (1, 2), (0, 3), (1, 3)]}


@pytest.mark.parametrize("name", list(tiny_graphs()))
def test_lftj_triangle_tiny_and_sparse_graphs(ctx, name):
    """Small graphs through every triangle path; ids up to 2^31 - 2 make the
    degree order step aside (its arrays are sized by the largest id), and the
    relation is joined in its own order."""
    edges = tiny_graphs()[name]
    s = np.array([u for u, _ in edges], np.int32)
    d = np.array([v for _, v in edges], np.int32)
    want = O.triangle(s, d)
    e = ctx.relation([s, d], [0, 1])
    for algo in ("DFS", "BFS"):
        for ws in (0, 1):
            got = ctx.lftj([e], algo=algo, ws=ws, materialize=True)
            assert (got.count, got.checksum) == want, (algo, ws)
            assert data.checksum(got.columns) == want[1]
    assert (lambda r: (r.count, r.checksum))(ctx.amhj("TRI", [e], ws=1)) == want


def test_lftj_joins_relations_as_sets(ctx):
    """A repeated row counts once in every ALFTJ path (the leapfrog triejoin
    is defined over sets; the reference joins deduplicated edge lists)."""
    s, d = data.rmat(12, 40000, 0.57, 0.19, 0.19, 8)
    rng = np.random.Generator(np.random.PCG64(8))
    rep = rng.integers(0, len(s), len(s) // 5)
    perm = rng.permutation(len(s) + len(rep))
    sd, dd = np.concatenate([s, s[rep]])[perm], np.concatenate([d, d[rep]])[perm]
    want = O.triangle(s, d)
    e = ctx.relation([sd, dd], [0, 1])
    for algo in ("DFS", "BFS"):
        for ws in (0, 1):
            got = ctx.lftj([e], algo=algo, ws=ws)
            assert (got.count, got.checksum) == want, (algo, ws)
    R = ctx.relation([sd, dd], [0, 1])
    S = ctx.relation([dd, sd], [2, 1])
    T = ctx.relation([s, d], [0, 2])
    got = ctx.lftj([R, S, T], algo="DFS")
    assert (got.count, got.checksum) == want
    c4 = ctx.lftj([e], clique4=True)
    assert (c4.count, c4.checksum) == O.four_clique(s, d)
    cyc = [(0, 1), (1, 2), (2, 3), (0, 3)]
    plain = ctx.lftj([ctx.relation([s, d], list(p)) for p in cyc])
    dup = ctx.lftj([ctx.relation([sd, dd], list(p)) for p in cyc])
    assert (dup.count, dup.checksum) == (plain.count, plain.checksum) and plain.count > 0


def test_ranked_trie_rows_past_the_warp_sort():
    """The degree-ranked copy's trie sorts each row on its own: a warp sorts
    rows of up to 1024 values, a block the longer ones.  A 1100-vertex clique
    gives its lowest-ranked vertex 1099 higher-ranked neighbours; joined with
    a sparse graph, the triangles and 4-cliques equal the oracle through the
    ALFTJ and AMHJ paths that use the copy."""
    s, d = data.rmat(12, 30000, 0.57, 0.19, 0.19, seed=31)
    k = np.arange(5000, 6100, dtype=np.int32)
    ci, cj = np.triu_indices(len(k), 1)
    s2 = np.concatenate([s, k[ci]]).astype(np.int32)
    d2 = np.concatenate([d, k[cj]]).astype(np.int32)
    want = O.triangle(s2, d2)
    with Context(0) as c:
        e = c.relation([s2, d2], [0, 1])
        for ws in (0, 1):
            got = c.lftj([e], algo="DFS", ws=ws, degree_order=True)
            assert (got.count, got.checksum) == want, ws
        got = c.lftj([e], algo="BFS", degree_order=True)
        assert (got.count, got.checksum) == want
        got = c.amhj("TRI", [e])
        assert (got.count, got.checksum) == want


def test_lftj_out_of_core_slices():
    """ooc=1 (the reference's OOCWrapper, LFTJ-GPU/ooc_wrapper.cuh): tries in
    pinned host memory, a memory budget split over the heading attributes,
    value-range slices of the tries joined combination by combination.  A
    budget far below the tries' size forces many slices; every shape gives
    the in-memory result and the oracle's."""
    s, d = data.rmat(11, 30000, 0.57, 0.19, 0.19, 7)
    want = O.triangle(s, d)
    four = O.four_clique(s, d)
    with Context(0, mem_budget=64 << 10) as ctx:
        e = ctx.relation([s, d], [0, 1])
        for algo in ("DFS", "BFS"):
            got = ctx.lftj([e], algo=algo, ooc=1, materialize=True)
            assert (got.count, got.checksum) == want
            assert data.checksum(got.columns) == want[1]
            assert got.stats["slices"] >= 4
        got = ctx.lftj([e], clique4=True, ooc=1)
        assert (got.count, got.checksum) == four and got.stats["slices"] >= 4
        got = ctx.lftj([e], ooc=1, attr_order=(2, 0, 1))
        assert (got.count, got.checksum) == want
        # three relations of the triangle, and a 4-cycle of distinct relations
        hs = [ctx.relation([s, d], [0, 1]), ctx.relation([s, d], [1, 2]), ctx.relation([s, d], [0, 2])]
        assert (lambda r: (r.count, r.checksum))(ctx.lftj(hs, ooc=1)) == want
    rels = [distinct_rel(3000, 200, 90 + i, list(p)) for i, p in enumerate(GENERIC_QUERIES["4-cycle"])]
    with Context(0, mem_budget=8 << 10) as ctx:
        got = ctx.lftj([ctx.relation(c, a) for c, a in rels], ooc=1)
        assert (got.count, got.checksum) == O.mhj(rels) and got.stats["slices"] >= 4


def test_lftj_out_of_core_host_resident_relation():
    """A relation kept in pinned host memory (streamed=True) never enters the
    device whole: its trie is built in value ranges of its first column that
    fit the budget, and the join runs on slices."""
    import torch
    s, d = data.rmat(13, 120000, 0.57, 0.19, 0.19, 8)
    want = O.triangle(s, d)
    with Context(0, mem_budget=256 << 10) as ctx:
        pinned = [torch.from_numpy(s).pin_memory(), torch.from_numpy(d).pin_memory()]
        e = ctx.relation([pinned[0].numpy(), pinned[1].numpy()], [0, 1], streamed=True)
        got = ctx.lftj([e], ooc=1)
        assert (got.count, got.checksum) == want
        assert got.stats["slices"] >= 4
        with pytest.raises(AmjError):
            ctx.lftj([e], ooc=0)


def test_lftj_rejects_two_relations_and_edge_cases(ctx):
    e = ctx.relation([np.array([0], np.int32), np.array([1], np.int32)], [0, 1])
    with pytest.raises(AmjError) as x:
        ctx.lftj([e, e], algo="DFS")
    assert x.value.status == L.AMJ_EINVAL
    empty = ctx.relation([np.zeros(0, np.int32), np.zeros(0, np.int32)], [0, 1])
    for algo in ("DFS", "BFS"):
        assert ctx.lftj([empty], algo=algo).count == 0
        assert ctx.lftj([e], algo=algo).count == 0


# ---------------------------------------------------------- full size

def test_c1_chain_full_size(ctx):
    rels = data.chain_relations(1_000_000, 1 << 18, 3, seed=1)
    want = O.mhj(rels)
    got = ctx.amhj("NORMAL", rels_on(ctx, rels))
    assert (got.count, got.checksum) == want
    got = ctx.amhj("NORMAL", rels_on(ctx, rels), ws=1, dro=1, materialize=True)
    assert (got.count, got.checksum) == want
    assert data.checksum(got.columns) == want[1]


def test_c2_triangle_full_size(ctx):
    s, d = data.rmat(20, 1 << 24, 0.57, 0.19, 0.19, 20)
    want = O.triangle(s, d)
    e = ctx.relation([s, d], [0, 1])
    for algo in ("DFS", "BFS"):
        got = ctx.lftj([e], algo=algo)
        assert (got.count, got.checksum) == want
    got = ctx.amhj("TRI", [e], ws=1)
    assert (got.count, got.checksum) == want


def test_c3a_four_clique_full_size(ctx):
    """The skewed 4-clique configuration (R-MAT scale 22, 2^26 generated
    edges, 0.6/0.15/0.15/0.1, seed 22) through the two fast paths: the
    triangle matrices and the list-intersection kernel over the
    degree-ordered copy give the same count and checksum (the reference's
    multi-key probe pins both paths on smaller graphs of the same
    generator, tests/test_gpu_golden_cyclic.py)."""
    s, d = data.rmat(22, 1 << 26, 0.6, 0.15, 0.15, 22)
    e = ctx.relation([s, d], [0, 1])
    m = ctx.lftj([e], clique4=True)
    lists = ctx.lftj([e], clique4=True, clique4_lists=True)
    assert (m.count, m.checksum) == (lists.count, lists.checksum)
    assert (m.count, m.checksum) == (94478795231, 0x56807E4A9FC45902)
    # the configured operator, AMHJ FOUR ws=1 fib=1 (its last three levels
    # through the triangle matrices)
    a = ctx.amhj("FOUR", [e], ws=1, fib=1)
    assert (a.count, a.checksum) == (m.count, m.checksum)
    e.release()


def test_amhj_four_matrix_plan_materialises_the_hash_plan_tuples(ctx):
    """AMHJ FOUR through the triangle matrices writes the same tuples (each
    sorted, from the degree-ordered copy) as the level-by-level hash plan,
    to host and device result columns."""
    s, d = data.rmat(11, 1 << 15, 0.57, 0.19, 0.19, seed=5)
    e = ctx.relation([s, d], [0, 1])
    a = ctx.amhj("FOUR", [e], ws=1, fib=1, materialize=True)
    b = ctx.amhj("FOUR", [e], ws=1, plan="hash", materialize=True)
    assert a.count > 1000 and (a.count, a.checksum) == (b.count, b.checksum)
    assert np.array_equal(sorted_rows(a.columns), sorted_rows(b.columns))
    assert data.checksum(a.columns) == a.checksum


# ----------------------------------------------------- failure detection

def test_bounded_wait_times_out_and_context_survives(ctx):
    lib = L.load()
    st = lib.amj_selftest_bounded_wait(ctx.handle, 200)
    assert st == L.AMJ_ETIMEOUT
    assert b"bounded wait" in lib.amj_last_error()
    rels = data.chain_relations(1000, 256, 3, seed=1)
    got = ctx.amhj("NORMAL", rels_on(ctx, rels))
    assert (got.count, got.checksum) == O.mhj(rels)


def test_work_sharing_queue_overflow_falls_back():
    """A one-slot task queue under direct output cannot hold the splits the
    residual replay relies on: the overflow is detected on the device and the
    direct output is redone without work sharing, still exact."""
    with Context(0, task_chunk=32, task_capacity=1, dro_headroom=0.5) as ctx:
        q = [([data.uniform(100, 0, 100, 1), data.uniform(100, 0, 100, 2)], [0, 1]),
             ([data.uniform(2000, 0, 100, 3), data.uniform(2000, 0, 4, 4)], [1, 2]),
             ([data.uniform(20000, 0, 4, 5), data.uniform(20000, 0, 1 << 20, 6)], [2, 3])]
        want = O.mhj(q)
        got = ctx.amhj("NORMAL", rels_on(ctx, q), ws=1, dro=1, materialize=True)
        assert (got.count, got.checksum) == want
        assert got.stats["fallbacks"] >= 1
        assert data.checksum(got.columns) == want[1]
        got = ctx.amhj("NORMAL", rels_on(ctx, q), ws=1)   # count mode keeps unsplit work local
        assert (got.count, got.checksum) == want


# ------------------------------------------------------------------- CLIs

def test_cli_exec_amhj_and_exec_lftj(tmp_path):
    rels = data.chain_relations(5000, 1 << 10, 3, seed=2)
    d = tmp_path / "chain"
    d.mkdir()
    # file names sort as r0, r1, r2 only by attribute: write them in query order with --order
    for i, (cols, attrs) in enumerate(rels):
        data.write_db(str(d / data.db_name(len(cols[0]), attrs)), cols)
    names = sorted(os.listdir(d))
    order = [names.index(data.db_name(len(c[0]), a)) for c, a in rels]
    pos = [order.index(i) for i in range(len(names))]
    exe = os.path.join(ROOT, "accmultiwayjoins_b200", "bin", "exec-AMHJ")
    r = subprocess.run([exe, "NORMAL", str(d), "0", "1", "0", "0", "--order", ",".join(map(str, pos))],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    cnt, chk = O.mhj(rels)
    assert out["count"] == cnt and out["checksum"] == f"{chk:016x}"
    s, dd = data.rmat(10, 8000, 0.57, 0.19, 0.19, 3)
    g = tmp_path / "graph"
    g.mkdir()
    data.write_db(str(g / data.db_name(len(s), [0, 1])), [s, dd])
    want = O.triangle(s, dd)
    for algo in ("0", "1"):
        exe = os.path.join(ROOT, "accmultiwayjoins_b200", "bin", "exec-LFTJ")
        r = subprocess.run([exe, str(g), algo, "0", "1"], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr
        out = json.loads(r.stdout.strip().splitlines()[-1])
        assert out["count"] == want[0] and out["checksum"] == f"{want[1]:016x}"
    exe = os.path.join(ROOT, "accmultiwayjoins_b200", "bin", "exec-AMHJ")
    r = subprocess.run([exe, "TRI", str(g / data.db_name(len(s), [0, 1])), "0", "1", "0", "0"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert json.loads(r.stdout.strip().splitlines()[-1])["count"] == want[0]


def test_tbl_tables_join_end_to_end(ctx, tmp_path):
    """Delimited tables (TPC-H .tbl shape: '|'-separated, text fields with
    spaces, a trailing '|') go through amj_tbl_to_db to .db relations and
    then through the multi-way joins: a star (a fact table and three
    dimensions) and a 3-table chain, both equal to the oracle."""
    rng = np.random.default_rng(31)

    def table(name, cols, text=True):
        n = len(cols[0])
        with open(tmp_path / name, "w") as f:
            for i in range(n):
                f.write("|".join(str(c[i]) for c in cols) + ("|note %d x|" % i if text else "|") + "\n")
        return str(tmp_path / name)

    n = 80_000
    fact = table("lineitem.tbl", [rng.integers(0, 20000, n), rng.integers(0, 2000, n), rng.integers(0, 100, n),
                                  rng.integers(1, 50, n)])
    part = table("part.tbl", [np.arange(2000), rng.integers(0, 25, 2000)])
    supp = table("supplier.tbl", [rng.integers(0, 100, 300), rng.integers(0, 25, 300)])   # repeated keys
    orders = table("orders.tbl", [np.arange(20000), rng.integers(0, 1500, 20000)], text=False)
    cust = table("customer.tbl", [np.arange(1500), rng.integers(0, 25, 1500)])
    out = str(tmp_path)
    star = [data.tbl_to_db(fact, [0, 1, 2], [0, 1, 2], out), data.tbl_to_db(part, [0, 1], [1, 3], out),
            data.tbl_to_db(supp, [0, 1], [2, 4], out), data.tbl_to_db(orders, [0, 1], [0, 5], out)]
    chain = [data.tbl_to_db(fact, [0, 3], [0, 1], out), data.tbl_to_db(orders, [0, 1], [0, 2], out),
             data.tbl_to_db(cust, [0, 1], [2, 3], out)]
    assert os.path.basename(star[0]) == f"{n}_0_1_2.db"
    for files in (star, chain):
        rels = [data.read_db(p) for p in files]
        want = O.mhj(rels)
        assert want[0] > 0
        got = ctx.amhj("NORMAL", rels_on(ctx, rels))
        assert (got.count, got.checksum) == want
        got = ctx.amhj("NORMAL", rels_on(ctx, rels), ws=1, dro=1, materialize=True)
        assert (got.count, got.checksum) == want and data.checksum(got.columns) == want[1]


def test_sharded_join_shares_sum_to_the_query(ctx):
    """The multi-GPU form (accmultiwayjoins_b200.dist.sharded_join): the
    probe relation's rows split over 4 ranks, the other relations whole;
    the ranks' (count, checksum) pairs, summed mod 2^64, equal the query's.
    Run here as 4 shares in turn on one GPU (no collective)."""
    from accmultiwayjoins_b200.dist import M64, sharded_join
    chain = data.chain_relations(200_000, 1 << 14, 3, seed=21)
    s, d = data.rmat(14, 1 << 18, 0.57, 0.19, 0.19, seed=20)
    tri = [([s, d], [0, 1]), ([s, d], [1, 2]), ([s, d], [0, 2])]
    for rels, op, want in ((chain, "amhj", O.mhj(chain)), (tri, "amhj", O.triangle(s, d)),
                           (tri, "lftj", O.triangle(s, d))):
        parts = [sharded_join(ctx, rels, r, 4, op=op, reduce=False) for r in range(4)]
        got = (sum(c for c, _ in parts) & M64, sum(h for _, h in parts) & M64)
        assert got == want, op
        assert all(c > 0 for c, _ in parts)
