"""Seeded synthetic relations (through libamj's host generators) and .db I/O.

The workloads follow the reference's data shapes: uniform int32 key columns
(MHJ-GPU/uniform_writer_.cu:66), Zipf columns with a rank-to-key permutation
(MHJ-GPU/data_generator.cuh:110-187), and graph edge relations.  The
reference reads external graph files; here an R-MAT generator stands in for
them (self-loops dropped, edges oriented u<v, duplicates removed, shuffled).
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

from . import _lib as L


def _i32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def uniform(n: int, lo: int, hi: int, seed: int, stream: int = 0) -> np.ndarray:
    out = np.empty(n, np.int32)
    L.check(L.load().amj_gen_uniform_i32(_i32p(out), n, lo, hi, seed, stream), "gen_uniform")
    return out


def permutation(n: int, seed: int, stream: int = 0) -> np.ndarray:
    out = np.empty(n, np.int32)
    L.check(L.load().amj_gen_permutation_i32(_i32p(out), n, seed, stream), "gen_permutation")
    return out


def zipf(n: int, domain: int, theta: float, seed: int, stream: int = 0, rank_to_key=None) -> np.ndarray:
    out = np.empty(n, np.int32)
    rk = None
    if rank_to_key is not None:
        rk = np.ascontiguousarray(rank_to_key, dtype=np.int32)
        if rk.shape[0] < domain:
            raise ValueError("rank_to_key shorter than the domain")
    L.check(L.load().amj_gen_zipf_i32(_i32p(out), n, domain, theta, _i32p(rk) if rk is not None else None, seed,
                                      stream), "gen_zipf")
    return out


def rmat(scale: int, nedges: int, a: float, b: float, c: float, seed: int):
    """Cleaned R-MAT edge relation: (src, dst) int32 arrays with src < dst."""
    src = np.empty(nedges, np.int32)
    dst = np.empty(nedges, np.int32)
    m = C.c_uint64()
    L.check(L.load().amj_gen_rmat(scale, nedges, a, b, c, seed, _i32p(src), _i32p(dst), C.byref(m)), "gen_rmat")
    m = int(m.value)
    return src[:m].copy(), dst[:m].copy()


def chain_relations(n: int, key_range: int, nrels: int = 3, seed: int = 1):
    """The chain workload R1(0,1) R2(1,2) .. : nrels relations of n rows, two
    uniform int32 columns in [0, key_range), relation i seeded seed+i."""
    rels = []
    for i in range(nrels):
        s = seed + i
        rels.append(([uniform(n, 0, key_range, s, 0), uniform(n, 0, key_range, s, 1)], [i, i + 1]))
    return rels


def star_relations(fact_rows: int, dim_rows, theta: float = 1.1, seed: int = 3):
    """The star workload: fact F(0..d-1) of Zipf foreign keys and dimensions
    Dj(j, d+j) of (unique key, uniform payload)."""
    d = len(dim_rows)
    dims = []
    fact_cols = []
    for j, m in enumerate(dim_rows):
        keys = permutation(m, seed, 100 + j)
        payload = uniform(m, -(1 << 31), (1 << 31), seed, 200 + j)
        dims.append(([keys, payload], [j, d + j]))
        rank_to_key = permutation(m, seed, 300 + j)
        fact_cols.append(zipf(fact_rows, m, theta, seed, 400 + j, rank_to_key=rank_to_key))
    return (fact_cols, list(range(d))), dims


def db_name(n: int, attrs) -> str:
    return f"{n}_" + "_".join(str(a) for a in attrs) + ".db"


def write_db(path: str, cols) -> None:
    cols = [np.ascontiguousarray(c, dtype=np.int32) for c in cols]
    n = cols[0].shape[0]
    ptrs = (C.POINTER(C.c_int32) * len(cols))(*[_i32p(c) for c in cols])
    L.check(L.load().amj_db_write(path.encode(), n, len(cols), ptrs), "db_write")


def read_db(path: str):
    """Read a .db file; returns (columns, attrs) with the schema from its name."""
    lib = L.load()
    n = C.c_uint64()
    nc = C.c_int()
    attrs = (C.c_uint32 * L.AMJ_MAX_COLS)()
    L.check(lib.amj_db_parse_name(path.encode(), C.byref(n), C.byref(nc), attrs), "db_parse_name")
    cols = [np.empty(n.value, np.int32) for _ in range(nc.value)]
    ptrs = (C.POINTER(C.c_int32) * nc.value)(*[_i32p(c) for c in cols])
    L.check(lib.amj_db_read(path.encode(), n.value, nc.value, ptrs), "db_read")
    return cols, [int(attrs[i]) for i in range(nc.value)]


def checksum(cols) -> int:
    """Checksum of column-major tuples (the definition in include/amj_checksum.h)."""
    cols = [np.ascontiguousarray(c, dtype=np.int32) for c in cols]
    n = cols[0].shape[0] if cols else 0
    ptrs = (C.POINTER(C.c_int32) * max(1, len(cols)))(*[_i32p(c) for c in cols])
    out = C.c_uint64()
    L.check(L.load().amj_checksum_host(ptrs, len(cols), n, C.byref(out)), "checksum_host")
    return int(out.value)
