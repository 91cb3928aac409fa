"""Seeded synthetic relations (through libamj's host generators) and .db I/O.

The workloads follow the reference's data shapes: uniform int32 key columns
(MHJ-GPU/uniform_writer_.cu:66), Zipf columns with a rank-to-key permutation
(MHJ-GPU/data_generator.cuh:110-187), and graph edge relations.  The
reference reads external graph files; here an R-MAT generator stands in for
them (self-loops dropped, edges oriented u<v, duplicates removed, shuffled).

The workload builders (chain_relations, star_relations, query_mix) take an
optional `gen`: any object with the four primitive generators uniform,
permutation, zipf and rmat of this module's signatures.  By default they are
this module's own (libamj); a caller that must not load the library passes
another implementation of the same definitions.
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


class _Libamj:
    """The primitive generators of this module (libamj)."""

    @staticmethod
    def uniform(*a, **k):
        return uniform(*a, **k)

    @staticmethod
    def permutation(*a, **k):
        return permutation(*a, **k)

    @staticmethod
    def zipf(*a, **k):
        return zipf(*a, **k)

    @staticmethod
    def rmat(*a, **k):
        return rmat(*a, **k)


def chain_relations(n: int, key_range: int, nrels: int = 3, seed: int = 1, gen=None):
    """The chain workload R1(0,1) R2(1,2) .. : nrels relations of n rows, two
    uniform int32 columns in [0, key_range), relation i seeded seed+i."""
    g = gen or _Libamj
    rels = []
    for i in range(nrels):
        s = seed + i
        rels.append(([g.uniform(n, 0, key_range, s, 0), g.uniform(n, 0, key_range, s, 1)], [i, i + 1]))
    return rels


def star_relations(fact_rows: int, dim_rows, theta: float = 1.1, seed: int = 3, gen=None):
    """The star workload: fact F(0..d-1) of Zipf foreign keys and dimensions
    Dj(j, d+j) of (unique key, uniform payload)."""
    g = gen or _Libamj
    d = len(dim_rows)
    dims = []
    fact_cols = []
    for j, m in enumerate(dim_rows):
        keys = g.permutation(m, seed, 100 + j)
        payload = g.uniform(m, -(1 << 31), (1 << 31), seed, 200 + j)
        dims.append(([keys, payload], [j, d + j]))
        rank_to_key = g.permutation(m, seed, 300 + j)
        fact_cols.append(g.zipf(fact_rows, m, theta, seed, 400 + j, rank_to_key=rank_to_key))
    return (fact_cols, list(range(d))), dims


def _log_uniform(rng, lo: float, hi: float) -> float:
    return float(np.exp(rng.uniform(np.log(lo), np.log(hi))))


def query_mix(count: int, seed: int = 4, min_rows: int = 10_000, max_rows: int = 4_000_000, min_dom_bits: int = 12,
              max_dom_bits: int = 24, theta_range=(0.5, 1.5), out_cap: int = 1 << 24, gen=None):
    """The heterogeneous query mix of the batched workload, one query at a time.

    Each query is a chain or a star of 2-5 relations, or a triangle, drawn
    with numpy's PCG64 seeded `seed`.  Relation sizes are log-uniform in
    [min_rows, max_rows]; join-key domains log-uniform in
    [2^min_dom_bits, 2^max_dom_bits]; half the queries are uniform, half
    Zipf with theta uniform in theta_range.

    * chain R0(0,1) R1(1,2) ..: the build side of every join (column 0 of
      R1..) is Zipf in a Zipf query, the probe side uniform, so the expected
      output is n0 * prod(n_j / D_j) whatever the skew.  While that exceeds
      out_cap the domains are doubled (up to 2^max_dom_bits), then the largest
      relation halved.
    * star F(0..d-1) D_j(j, d+j): dimensions with unique keys (a permutation
      of [0, m_j)), foreign keys uniform or Zipf over [0, m_j): |OUT| = |F|.
    * triangle: the TRI query over a cleaned R-MAT edge relation
      (0.57, 0.19, 0.19) with E generated edges and scale log2(E / 8).

    Yields dicts with shape, qt, rels (list of (columns, attrs)) and theta."""
    g = gen or _Libamj
    rng = np.random.Generator(np.random.PCG64(seed))
    for q in range(count):
        shape = ("chain", "star", "triangle")[int(rng.integers(0, 3))]
        zipfian = bool(rng.integers(0, 2))
        theta = float(rng.uniform(*theta_range)) if zipfian else 0.0
        qseed = seed * 1_000_003 + q
        if shape == "triangle":
            e = int(_log_uniform(rng, min_rows, max_rows))
            scale = max(8, int(round(np.log2(max(e, 256) / 8))))
            s, d = g.rmat(scale, e, 0.57, 0.19, 0.19, qseed)
            yield dict(shape=shape, qt="TRI", rels=[([s, d], [0, 1])], theta=0.0)
            continue
        r = int(rng.integers(2, 6))
        sizes = [int(_log_uniform(rng, min_rows, max_rows)) for _ in range(r)]
        if shape == "star":
            d = r - 1
            fact_cols, dims = [], []
            for j in range(d):
                m = sizes[j + 1]
                keys = g.permutation(m, qseed, 100 + j)
                payload = g.uniform(m, 0, 1 << 30, qseed, 200 + j)
                dims.append(([keys, payload], [j, d + j]))
                if zipfian:
                    fact_cols.append(g.zipf(sizes[0], m, theta, qseed, 400 + j,
                                          rank_to_key=g.permutation(m, qseed, 300 + j)))
                else:
                    fact_cols.append(g.uniform(sizes[0], 0, m, qseed, 400 + j))
            yield dict(shape=shape, qt="NORMAL", rels=[(fact_cols, list(range(d)))] + dims, theta=theta)
            continue
        doms = [int(_log_uniform(rng, 1 << min_dom_bits, 1 << max_dom_bits)) for _ in range(r - 1)]

        def expected():
            e = float(sizes[0])
            for j in range(1, r):
                e *= sizes[j] / doms[j - 1]
            return e

        while expected() > out_cap:
            grow = [j for j in range(r - 1) if doms[j] < (1 << max_dom_bits)]
            if grow:
                for j in grow:
                    doms[j] = min(doms[j] * 2, 1 << max_dom_bits)
                continue
            big = int(np.argmax(sizes))
            if sizes[big] <= min_rows:
                break
            sizes[big] = max(min_rows, sizes[big] // 2)
        rels = []
        for i in range(r):
            if i == 0:
                c0 = g.uniform(sizes[i], 0, 1 << max_dom_bits, qseed, 10 * i)
            elif zipfian:
                c0 = g.zipf(sizes[i], doms[i - 1], theta, qseed, 10 * i,
                          rank_to_key=g.permutation(doms[i - 1], qseed, 10 * i + 2))
            else:
                c0 = g.uniform(sizes[i], 0, doms[i - 1], qseed, 10 * i)
            hi = doms[i] if i < r - 1 else (1 << max_dom_bits)
            c1 = g.uniform(sizes[i], 0, hi, qseed, 10 * i + 1)
            rels.append(([c0, c1], [i, i + 1]))
        yield dict(shape=shape, qt="NORMAL", rels=rels, theta=theta)


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


def read_edgelist(path: str, swap: bool = False):
    """The edges of a text edge list as (src, dst) int32 arrays
    (amj_edgelist_read: two integers a line separated by ' ', '|' or tab;
    '#' / '%' comment lines skipped)."""
    lib = L.load()
    n = C.c_uint64()
    L.check(lib.amj_edgelist_read(path.encode(), int(swap), None, None, 0, C.byref(n)), "edgelist_read")
    src = np.empty(n.value, np.int32)
    dst = np.empty(n.value, np.int32)
    if n.value:
        L.check(lib.amj_edgelist_read(path.encode(), int(swap), _i32p(src), _i32p(dst), n.value, C.byref(n)),
                "edgelist_read")
    return src, dst


def edgelist_to_db(text_path: str, db_path: str = None, swap: bool = False) -> int:
    """Convert a text edge list to a 2-column .db file (default name: the
    edge list's path + ".db", as the reference's converter names it);
    returns the number of edges."""
    rows = C.c_uint64()
    db_path = db_path or text_path + ".db"
    L.check(L.load().amj_edgelist_to_db(text_path.encode(), db_path.encode(), int(swap), C.byref(rows)),
            "edgelist_to_db")
    return int(rows.value)


def tbl_to_db(tbl_path: str, fields, attrs, out_dir: str = None) -> str:
    """Selected fields of a delimited table (a TPC-H .tbl file) as a .db
    relation named "<rows>_<attrs>...db" in out_dir; returns its path."""
    if len(fields) != len(attrs):
        raise ValueError("one attribute per field")
    n = len(fields)
    buf = C.create_string_buffer(4096)
    rows = C.c_uint64()
    L.check(L.load().amj_tbl_to_db(tbl_path.encode(), (C.c_uint32 * n)(*fields), (C.c_uint32 * n)(*attrs), n,
                                   out_dir.encode() if out_dir else None, buf, 4096, C.byref(rows)), "tbl_to_db")
    return buf.value.decode()


def checksum(cols) -> int:
    """Checksum of column-major tuples (the definition in include/amj_checksum.h)."""
    cols = [np.ascontiguousarray(c, dtype=np.int32) for c in cols]
    n = cols[0].shape[0] if cols else 0
    ptrs = (C.POINTER(C.c_int32) * max(1, len(cols)))(*[_i32p(c) for c in cols])
    out = C.c_uint64()
    L.check(L.load().amj_checksum_host(ptrs, len(cols), n, C.byref(out)), "checksum_host")
    return int(out.value)
