"""ctypes bindings of the CPU oracle (liborc.so) and of the reference's
MHJ-CPU harness (_ref/libmhjref.so).

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

_orc = None
_ref = None


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
        _orc = lib
    return _orc


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref():
    global _ref
    if _ref is None:
        lib = C.CDLL(REF_PATH)
        P = C.POINTER
        lib.mhjref_run.argtypes = [C.c_int, P(C.c_uint64), P(C.c_int), P(C.c_uint32), P(P(C.c_int32)), C.c_int,
                                   P(C.c_uint64), P(C.c_uint64), P(P(C.c_int32)), C.c_uint64, P(C.c_int),
                                   P(C.c_double)]
        _ref = lib
    return _ref


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


def mhj_reference(relations, nthreads=0, tuples=False):
    """Run the reference's MHJ-CPU (TBJ) on relations in query order.
    Returns (count, checksum, seconds[, columns])."""
    lib = ref()
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
        rc = lib.mhjref_run(nt, lens, ncols, attrs, data, nthreads, C.byref(cnt), C.byref(chk), None, 0,
                            C.byref(kk), C.byref(secs))
        assert rc == 0, rc
        cap = cnt.value
        tcols, tarr = _tuple_buffers(k, cap)
    rc = lib.mhjref_run(nt, lens, ncols, attrs, data, nthreads, C.byref(cnt), C.byref(chk), tarr, cap,
                        C.byref(kk), C.byref(secs))
    if rc != 0:
        raise ValueError(f"mhjref_run failed ({rc})")
    if tuples:
        return cnt.value, chk.value, secs.value, [c[:cap] for c in tcols]
    return cnt.value, chk.value, secs.value


def timed(fn, *args, **kw):
    t0 = time.perf_counter()
    out = fn(*args, **kw)
    return out, time.perf_counter() - t0
