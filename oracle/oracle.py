"""ctypes bindings of the CPU oracle (liborc.so) and of the reference's
MHJ-CPU harness (_ref/libmhjref.so as shipped, _ref/libmhjref_mk.so with the
reference's multi-key probe branch, MHJ-CPU/MHJ.cpp:64-90 and :205-245).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product (libamj.so and the
accmultiwayjoins_b200 package) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_PATH = os.path.join(HERE, "liborc.so")
REF_PATH = os.path.join(HERE, "_ref", "libmhjref.so")
REF_MK_PATH = os.path.join(HERE, "_ref", "libmhjref_mk.so")

_orc = None
_ref = None
_ref_mk = None


class orc_rel(C.Structure):
    _fields_ = [("n", C.c_uint64), ("ncols", C.c_int), ("attr", C.c_int * 8), ("col", C.POINTER(C.c_int32) * 8)]


def _i32p(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32)) if a is not None else None


def build():
    """Compile the oracle (and, when the reference sources exist, the MHJ-CPU harness)."""
    subprocess.run(["make", "-C", HERE], check=True, stdout=subprocess.DEVNULL)


def orc():
    global _orc
    if _orc is None:
        if not os.path.exists(ORC_PATH):
            build()
        lib = C.CDLL(ORC_PATH)
        P = C.POINTER
        lib.orc_bucket_build.argtypes = [P(C.c_int32), C.c_uint64, C.c_uint64, P(C.c_int32), P(C.c_uint32),
                                         P(C.c_uint32)]
        lib.orc_trie_build.argtypes = [P(C.c_int32), P(C.c_int32), C.c_uint64, P(C.c_int32), P(C.c_uint64),
                                       P(C.c_int32), P(C.c_uint64)]
        lib.orc_mhj.argtypes = [C.c_int, P(orc_rel), C.c_int, P(C.c_uint64), P(C.c_uint64), P(P(C.c_int32)),
                                C.c_uint64]
        lib.orc_triangle.argtypes = [P(C.c_int32), P(C.c_int32), C.c_uint64, C.c_int, P(C.c_uint64), P(C.c_uint64),
                                     P(P(C.c_int32)), C.c_uint64]
        lib.orc_four_clique.argtypes = [P(C.c_int32), P(C.c_int32), C.c_uint64, C.c_int, P(C.c_uint64),
                                        P(C.c_uint64)]
        lib.orc_gen_uniform_i32.argtypes = [P(C.c_int32), C.c_uint64, C.c_int64, C.c_int64, C.c_uint64,
                                            C.c_uint64]
        lib.orc_gen_permutation_i32.argtypes = [P(C.c_int32), C.c_uint64, C.c_uint64, C.c_uint64]
        lib.orc_gen_zipf_i32.argtypes = [P(C.c_int32), C.c_uint64, C.c_uint64, C.c_double, P(C.c_int32),
                                         C.c_uint64, C.c_uint64]
        lib.orc_gen_rmat.argtypes = [C.c_int, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                     P(C.c_int32), P(C.c_int32), P(C.c_uint64)]
        _orc = lib
    return _orc


def ref_available(multi_key: bool = False) -> bool:
    return os.path.exists(REF_MK_PATH if multi_key else REF_PATH)


def _ref_argtypes():
    P = C.POINTER
    return [C.c_int, P(C.c_uint64), P(C.c_int), P(C.c_uint32), P(P(C.c_int32)), C.c_int, P(C.c_uint64),
            P(C.c_uint64), P(P(C.c_int32)), C.c_uint64, P(C.c_int), P(C.c_double)]


def ref(multi_key: bool = False, relabel: bool = False):
    """The MHJ-CPU harness's entry point: mhjref_run (single-key, as shipped)
    or mhjref_run_mk (the reference's multi-key probe); with relabel, the
    variant that renames result values through a map and sorts each tuple."""
    global _ref, _ref_mk
    relabel_args = [C.POINTER(C.c_int32), C.c_uint64]
    if multi_key:
        if _ref_mk is None:
            lib = C.CDLL(REF_MK_PATH)
            lib.mhjref_run_mk.argtypes = _ref_argtypes()
            lib.mhjref_run_mk_relabel.argtypes = _ref_argtypes() + relabel_args
            _ref_mk = lib
        return _ref_mk.mhjref_run_mk_relabel if relabel else _ref_mk.mhjref_run_mk
    if _ref is None:
        lib = C.CDLL(REF_PATH)
        lib.mhjref_run.argtypes = _ref_argtypes()
        lib.mhjref_run_relabel.argtypes = _ref_argtypes() + relabel_args
        _ref = lib
    return _ref.mhjref_run_relabel if relabel else _ref.mhjref_run


def _tuple_buffers(k, cap):
    cols = [np.empty(max(cap, 1), np.int32) for _ in range(k)]
    arr = (C.POINTER(C.c_int32) * k)(*[_i32p(c) for c in cols])
    return cols, arr


def mhj(relations, nthreads=0, tuples=False, cap=None):
    """Multi-way hash join restatement.  relations: list of (cols, attrs),
    relations[0] probes.  Returns (count, checksum[, columns])."""
    lib = orc()
    rels = (orc_rel * len(relations))()
    keep = []
    k = 0
    for i, (cols, attrs) in enumerate(relations):
        cols = [np.ascontiguousarray(c, dtype=np.int32) for c in cols]
        keep.append(cols)
        rels[i].n = cols[0].shape[0]
        rels[i].ncols = len(cols)
        for c, (col, a) in enumerate(zip(cols, attrs)):
            rels[i].attr[c] = int(a)
            rels[i].col[c] = _i32p(col)
            k = max(k, int(a) + 1)
    cnt, chk = C.c_uint64(), C.c_uint64()
    tcols, tarr = (None, None)
    if tuples:
        if cap is None:
            rc = lib.orc_mhj(len(relations), rels, nthreads, C.byref(cnt), C.byref(chk), None, 0)
            assert rc == 0, rc
            cap = cnt.value
        tcols, tarr = _tuple_buffers(k, cap)
    rc = lib.orc_mhj(len(relations), rels, nthreads, C.byref(cnt), C.byref(chk), tarr, cap or 0)
    if rc != 0:
        raise ValueError(f"orc_mhj failed ({rc})")
    if tuples:
        return cnt.value, chk.value, [c[:min(cnt.value, cap)] for c in tcols]
    return cnt.value, chk.value


def triangle(src, dst, nthreads=0, tuples=False):
    lib = orc()
    src = np.ascontiguousarray(src, np.int32)
    dst = np.ascontiguousarray(dst, np.int32)
    cnt, chk = C.c_uint64(), C.c_uint64()
    if tuples:
        rc = lib.orc_triangle(_i32p(src), _i32p(dst), src.shape[0], nthreads, C.byref(cnt), C.byref(chk), None, 0)
        assert rc == 0
        cap = cnt.value
        tcols, tarr = _tuple_buffers(3, cap)
        rc = lib.orc_triangle(_i32p(src), _i32p(dst), src.shape[0], nthreads, C.byref(cnt), C.byref(chk), tarr, cap)
        assert rc == 0
        return cnt.value, chk.value, [c[:cap] for c in tcols]
    rc = lib.orc_triangle(_i32p(src), _i32p(dst), src.shape[0], nthreads, C.byref(cnt), C.byref(chk), None, 0)
    if rc != 0:
        raise ValueError(f"orc_triangle failed ({rc})")
    return cnt.value, chk.value


def four_clique(src, dst, nthreads=0):
    lib = orc()
    src = np.ascontiguousarray(src, np.int32)
    dst = np.ascontiguousarray(dst, np.int32)
    cnt, chk = C.c_uint64(), C.c_uint64()
    rc = lib.orc_four_clique(_i32p(src), _i32p(dst), src.shape[0], nthreads, C.byref(cnt), C.byref(chk))
    if rc != 0:
        raise ValueError(f"orc_four_clique failed ({rc})")
    return cnt.value, chk.value


def trie_build_n(cols):
    """N-level trie of the columns: (data per level, offsets per level but the last)."""
    lib = orc()
    cols = [np.ascontiguousarray(c, np.int32) for c in cols]
    k, n = len(cols), cols[0].shape[0]
    data = [np.empty(max(n, 1), np.int32) for _ in range(k)]
    off = [np.empty(n + 1, np.uint64) for _ in range(k - 1)] or [np.empty(1, np.uint64)]
    lens = (C.c_uint64 * k)()
    cp = (C.POINTER(C.c_int32) * k)(*[_i32p(c) for c in cols])
    dp = (C.POINTER(C.c_int32) * k)(*[_i32p(d) for d in data])
    op = (C.POINTER(C.c_uint64) * max(1, k - 1))(*[o.ctypes.data_as(C.POINTER(C.c_uint64)) for o in off])
    rc = lib.orc_trie_build_n(cp, k, n, dp, op, lens)
    if rc != 0:
        raise ValueError(f"orc_trie_build_n failed ({rc})")
    lens = [int(lens[i]) for i in range(k)]
    return [data[l][:lens[l]].copy() for l in range(k)], [off[l][:lens[l] + 1].copy() for l in range(k - 1)]


def trie_build(c0, c1):
    lib = orc()
    c0 = np.ascontiguousarray(c0, np.int32)
    c1 = np.ascontiguousarray(c1, np.int32)
    n = c0.shape[0]
    d0 = np.empty(max(n, 1), np.int32)
    o0 = np.empty(n + 1, np.uint64)
    d1 = np.empty(max(n, 1), np.int32)
    l0 = C.c_uint64()
    rc = lib.orc_trie_build(_i32p(c0), _i32p(c1), n, _i32p(d0), o0.ctypes.data_as(C.POINTER(C.c_uint64)),
                            _i32p(d1), C.byref(l0))
    assert rc == 0
    m = l0.value
    return d0[:m], o0[:m + 1], d1[:n]


def bucket_build(keys, buckets):
    lib = orc()
    keys = np.ascontiguousarray(keys, np.int32)
    n = keys.shape[0]
    hk = np.empty(max(n, 1), np.int32)
    idx = np.empty(max(n, 1), np.uint32)
    bp = np.empty(buckets + 1, np.uint32)
    rc = lib.orc_bucket_build(_i32p(keys), n, buckets, _i32p(hk), idx.ctypes.data_as(C.POINTER(C.c_uint32)),
                              bp.ctypes.data_as(C.POINTER(C.c_uint32)))
    assert rc == 0
    return hk[:n], idx[:n], bp


def mhj_reference(relations, nthreads=0, tuples=False, multi_key=False, relabel=None):
    """Run the reference's MHJ-CPU (TBJ) on relations in query order.
    multi_key=True runs its multi-key probe, which compares every bound
    attribute (the semantics of TRI and FOUR; equal to the single-key probe
    on chains and stars).  relabel (int32 array): result values are renamed
    through it and every tuple sorted before hashing (see
    degree_ordered_copy).  Returns (count, checksum, seconds[, columns])."""
    base = ref(multi_key, relabel is not None)
    if relabel is not None:
        lab = np.ascontiguousarray(relabel, np.int32)

        def run(*a):
            return base(*a, _i32p(lab), lab.shape[0])
    else:
        run = base
    nt = len(relations)
    if nt < 3:
        # a two-relation join (one build table) crashes TBJ as compiled here
        # (SIGSEGV in the host process)
        raise ValueError("the reference MHJ-CPU needs at least three relations")
    lens = (C.c_uint64 * nt)()
    ncols = (C.c_int * nt)()
    attrs = (C.c_uint32 * (8 * nt))()
    data = (C.POINTER(C.c_int32) * (8 * nt))()
    keep = []
    k = 0
    for i, (cols, at) in enumerate(relations):
        cols = [np.ascontiguousarray(c, dtype=np.int32) for c in cols]
        keep.append(cols)
        lens[i] = cols[0].shape[0]
        ncols[i] = len(cols)
        for c, (col, a) in enumerate(zip(cols, at)):
            attrs[i * 8 + c] = int(a)
            data[i * 8 + c] = _i32p(col)
            k = max(k, int(a) + 1)
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    cnt, chk, kk, secs = C.c_uint64(), C.c_uint64(), C.c_int(), C.c_double()
    tcols, tarr, cap = None, None, 0
    if tuples:
        rc = run(nt, lens, ncols, attrs, data, nthreads, C.byref(cnt), C.byref(chk), None, 0, C.byref(kk),
                 C.byref(secs))
        if rc != 0:
            raise ValueError(f"the MHJ-CPU harness failed ({rc})")
        cap = cnt.value
        tcols, tarr = _tuple_buffers(k, cap)
    rc = run(nt, lens, ncols, attrs, data, nthreads, C.byref(cnt), C.byref(chk), tarr, cap, C.byref(kk),
             C.byref(secs))
    if rc != 0:
        raise ValueError(f"the MHJ-CPU harness failed ({rc})")
    if tuples:
        return cnt.value, chk.value, secs.value, [c[:cap] for c in tcols]
    return cnt.value, chk.value, secs.value


# ---- seeded inputs, generated without the product library (orc_gen.cpp) ----

def gen_uniform(n, lo, hi, seed, stream=0):
    out = np.empty(n, np.int32)
    if orc().orc_gen_uniform_i32(_i32p(out), n, lo, hi, seed, stream) != 0:
        raise ValueError("orc_gen_uniform_i32: bad arguments")
    return out


def gen_permutation(n, seed, stream=0):
    out = np.empty(n, np.int32)
    if orc().orc_gen_permutation_i32(_i32p(out), n, seed, stream) != 0:
        raise ValueError("orc_gen_permutation_i32: bad arguments")
    return out


def gen_zipf(n, domain, theta, seed, stream=0, rank_to_key=None):
    out = np.empty(n, np.int32)
    rk = None if rank_to_key is None else np.ascontiguousarray(rank_to_key, np.int32)
    if orc().orc_gen_zipf_i32(_i32p(out), n, domain, theta, _i32p(rk), seed, stream) != 0:
        raise ValueError("orc_gen_zipf_i32: bad arguments")
    return out


def gen_rmat(scale, nedges, a, b, c, seed):
    """Cleaned R-MAT edge relation (src < dst, no duplicates, shuffled)."""
    src = np.empty(nedges, np.int32)
    dst = np.empty(nedges, np.int32)
    m = C.c_uint64()
    if orc().orc_gen_rmat(scale, nedges, a, b, c, seed, _i32p(src), _i32p(dst), C.byref(m)) != 0:
        raise ValueError("orc_gen_rmat: bad arguments")
    return src[:m.value].copy(), dst[:m.value].copy()


class GENERATORS:
    """The primitive generators in the form accmultiwayjoins_b200.data's
    workload builders take (their `gen` argument): chain_relations,
    star_relations and query_mix then run without loading libamj."""
    uniform = staticmethod(gen_uniform)
    permutation = staticmethod(gen_permutation)
    zipf = staticmethod(gen_zipf)
    rmat = staticmethod(gen_rmat)


def degree_ordered_copy(src, dst):
    """Rename the vertices of an edge relation by their rank in (degree, id)
    order and orient every edge from the lower to the higher rank.  Returns
    (src', dst', rank_to_id).  Triangles and 4-cliques are the same vertex
    sets in both graphs, and each is listed once under either orientation, so
    the cyclic queries over the copy, renamed back through rank_to_id with
    every tuple sorted, give the tuples of the queries over the relation
    oriented u < v."""
    src = np.asarray(src, np.int64)
    dst = np.asarray(dst, np.int64)
    n_v = int(max(src.max(initial=-1), dst.max(initial=-1))) + 1
    deg = np.bincount(src, minlength=n_v) + np.bincount(dst, minlength=n_v)
    order = np.lexsort((np.arange(n_v), deg))          # rank -> id, by (degree, id)
    rank = np.empty(n_v, np.int64)
    rank[order] = np.arange(n_v)
    rs, rd = rank[src], rank[dst]
    lo, hi = np.minimum(rs, rd), np.maximum(rs, rd)
    return lo.astype(np.int32), hi.astype(np.int32), order.astype(np.int32)


def tri_relations(src, dst):
    """The TRI attribute pattern over one edge relation, A(0,1) B(1,2) C(0,2)
    (MHJ-GPU/exec_AMHJ.cu:32-49)."""
    return [([src, dst], [0, 1]), ([src, dst], [1, 2]), ([src, dst], [0, 2])]


def four_relations(src, dst):
    """The FOUR attribute pattern over one edge relation, A(0,1) B(1,2) C(2,3)
    D(0,3) E(0,2) F(1,3) (MHJ-GPU/exec_AMHJ.cu:50-69)."""
    pats = [(0, 1), (1, 2), (2, 3), (0, 3), (0, 2), (1, 3)]
    return [([src, dst], list(p)) for p in pats]


def timed(fn, *args, **kw):
    t0 = time.perf_counter()
    out = fn(*args, **kw)
    return out, time.perf_counter() - t0
