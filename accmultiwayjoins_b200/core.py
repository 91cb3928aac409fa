"""Python host interface of the join operators, mirroring the reference's
operator API for this path:

* ``Context.amhj(query_type, relations, ooc, ws, dro, fib)`` is
  ``exec-AMHJ <NORMAL|TRI|FOUR> <path> <ooc> <ws> <dro> <fib>``
  (MHJ-GPU/exec_AMHJ.cu:218-246) / ``OOC<..>::execute`` (MHJ-GPU/ooc.cuh:77-82);
* ``Context.lftj(relations, algo, ooc, ws)`` is
  ``exec-LFTJ <path> <0=BFS|1=DFS> <ooc> <ws>`` (LFTJ-GPU/exec_LFTJ.cu:261-268) /
  ``OOCWrapper::execute_with_{BFS,DFS}`` (LFTJ-GPU/ooc_wrapper.cuh:404-427);
* ``Context.batch()`` collects many AMHJ queries and runs them in one build
  pass and one persistent probe launch (no reference counterpart);
* ``Context.server()`` serves AMHJ requests over resident relations by
  continuous batching, with admission by device memory and an out-of-core
  lane (no reference counterpart).

Every call goes through libamj.so; nothing here computes a join.  Errors
raise ``AmjError`` carrying the C status instead of exiting the process as
the reference does (common-utils/cuda/cuda_base.cuh:43-57).
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib as L

_QUERY = {"NORMAL": L.AMJ_QUERY_NORMAL, "TRI": L.AMJ_QUERY_TRI, "FOUR": L.AMJ_QUERY_FOUR}
_ALGO = {"BFS": L.AMJ_LFTJ_BFS, "DFS": L.AMJ_LFTJ_DFS, 0: L.AMJ_LFTJ_BFS, 1: L.AMJ_LFTJ_DFS}
_LAYOUT = {"bucket": L.AMJ_LAYOUT_BUCKET, "oa": L.AMJ_LAYOUT_OPEN_ADDR, "open_addr": L.AMJ_LAYOUT_OPEN_ADDR,
           "cuckoo": L.AMJ_LAYOUT_CUCKOO}
STAT_NAMES = ["tasks_pushed", "tasks_popped", "residual_units", "rows_written_main", "rows_written_residual",
              "estimate", "fallbacks", "slices", "fib_keys", "fib_rows_cached", "fib_rows_served", "batch_queries"]


@dataclass
class Result:
    count: int
    checksum: int
    num_attrs: int
    build_ms: float
    probe_ms: float
    total_ms: float
    stats: dict
    kernel_ms: tuple = ()
    columns: Optional[list] = None  # k numpy int32 arrays (attribute order) when materialised

    def tuples(self) -> np.ndarray:
        """Materialised tuples as an (rows, k) array."""
        if self.columns is None:
            raise ValueError("result was not materialised")
        return np.stack(self.columns, axis=1) if self.columns else np.zeros((0, 0), np.int32)


class Relation:
    """A relation registered with a context.

    ``cols`` are int32 columns: numpy arrays (copied to the device, or kept on
    the host for out-of-core probing with ``streamed=True``) or CUDA tensors
    (borrowed, must stay alive; the Relation keeps a reference)."""

    def __init__(self, ctx: "Context", cols: Sequence, attrs: Sequence[int], streamed: bool = False):
        lib = L.load()
        self.ctx = ctx
        self._keep = []
        ncols = len(cols)
        if ncols == 0 or ncols != len(attrs):
            raise ValueError("need one attribute per column")
        ptrs = (C.POINTER(C.c_int32) * ncols)()
        n = None
        where = L.AMJ_MEM_HOST
        for i, col in enumerate(cols):
            if hasattr(col, "data_ptr") and hasattr(col, "is_cuda") and col.is_cuda:
                import torch
                if col.dtype != torch.int32 or not col.is_contiguous():
                    raise ValueError("device columns must be contiguous torch.int32")
                ptrs[i] = C.cast(C.c_void_p(col.data_ptr()), C.POINTER(C.c_int32))
                where = L.AMJ_MEM_DEVICE
                length = col.numel()
            else:
                arr = np.ascontiguousarray(np.asarray(col), dtype=np.int32)
                ptrs[i] = arr.ctypes.data_as(C.POINTER(C.c_int32))
                length = arr.shape[0]
                col = arr
                if streamed:
                    where = L.AMJ_MEM_HOST_STREAMED
            self._keep.append(col)
            if n is None:
                n = length
            elif n != length:
                raise ValueError("columns differ in length")
        attr_arr = (C.c_uint32 * ncols)(*[int(a) for a in attrs])
        handle = C.c_void_p()
        L.check(lib.amj_rel_create(ctx.handle, n, ncols, attr_arr, ptrs, where, C.byref(handle)), "rel_create")
        if where == L.AMJ_MEM_HOST:
            self._keep = []  # copied to the device
        self.handle = handle
        ctx._relations.add(self)
        self.n = int(n)
        self.attrs = [int(a) for a in attrs]
        self.where = where

    def release(self):
        """Free the relation; a relation must be released before its context
        (Context.close releases the ones still alive)."""
        if getattr(self, "handle", None):
            if getattr(self.ctx, "handle", None):
                L.load().amj_rel_release(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


@dataclass
class BatchRun:
    counts: list
    checksums: list
    build_ms: float
    probe_ms: float
    total_ms: float
    launches: int
    tasks_pushed: int
    tasks_popped: int
    units: int
    build_rows: int
    build_jobs: int
    graph: bool


class Batch:
    """Many AMHJ queries run together (amj_batch).  ``submit`` compiles a
    query exactly as ``Context.amhj`` would; ``run`` returns every query's
    count and checksum, which equal the one-query-per-call results."""

    def __init__(self, ctx: "Context"):
        self.ctx = ctx
        h = C.c_void_p()
        self.handle = None
        L.check(L.load().amj_batch_create(ctx.handle, C.byref(h)), "batch_create")
        self.handle = h
        self._rels = []   # keeps the relations alive while the batch may read them

    def submit(self, query_type, relations: Sequence[Relation], reorder: bool = True) -> int:
        qt = _QUERY[query_type] if isinstance(query_type, str) else int(query_type)
        arr = (C.c_void_p * len(relations))(*[r.handle for r in relations])
        qid = C.c_uint32()
        flags = 0 if reorder else L.AMJ_F_NO_REORDER
        L.check(L.load().amj_batch_submit(self.handle, qt, arr, len(relations), flags, C.byref(qid)), "batch_submit")
        self._rels.extend(relations)
        return int(qid.value)

    def __len__(self) -> int:
        n = C.c_uint32()
        L.check(L.load().amj_batch_size(self.handle, C.byref(n)), "batch_size")
        return int(n.value)

    @staticmethod
    def _opts(layout="bucket", load_factor=0.0, block_size=256, task_chunk=1024, use_graph=False, grid_blocks=0):
        o = L.amj_batch_opts()
        o.layout = _LAYOUT[layout] if isinstance(layout, str) else int(layout)
        o.load_factor = load_factor
        o.block_size = block_size
        o.task_chunk = task_chunk
        o.use_graph = 1 if use_graph else 0
        o.grid_blocks = grid_blocks
        return o

    def run(self, layout="bucket", load_factor=0.0, block_size=256, task_chunk=1024, use_graph=False,
            opts: Optional[L.amj_batch_opts] = None) -> BatchRun:
        n = len(self)
        counts = (C.c_uint64 * max(n, 1))()
        chks = (C.c_uint64 * max(n, 1))()
        st = L.amj_batch_stats()
        o = opts if opts is not None else self._opts(layout, load_factor, block_size, task_chunk, use_graph)
        L.check(L.load().amj_batch_run(self.handle, C.byref(o), counts, chks, C.byref(st)), "batch_run")
        return BatchRun(counts=[int(counts[i]) for i in range(n)], checksums=[int(chks[i]) for i in range(n)],
                        build_ms=st.build_ms, probe_ms=st.probe_ms, total_ms=st.total_ms, launches=int(st.launches),
                        tasks_pushed=int(st.tasks_pushed), tasks_popped=int(st.tasks_popped), units=int(st.units),
                        build_rows=int(st.build_rows), build_jobs=int(st.build_jobs), graph=bool(st.graph))

    def tune(self, sample_every: int = 1, reps: int = 1, layout="bucket", load_factors=(), block_sizes=(),
             task_chunks=(), use_graph=False):
        """Autotune load factor x block size x task chunk on a sample of the
        batch; returns (amj_batch_opts, best median ms on the sample)."""
        g = L.amj_batch_tune_grid()
        g.layout = _LAYOUT[layout] if isinstance(layout, str) else int(layout)
        g.n_load_factor, g.n_block_size, g.n_task_chunk = len(load_factors), len(block_sizes), len(task_chunks)
        for i, v in enumerate(load_factors):
            g.load_factor[i] = v
        for i, v in enumerate(block_sizes):
            g.block_size[i] = v
        for i, v in enumerate(task_chunks):
            g.task_chunk[i] = v
        best = L.amj_batch_opts()
        best.use_graph = 1 if use_graph else 0
        ms = C.c_double()
        L.check(L.load().amj_batch_tune(self.handle, C.byref(g), int(sample_every), int(reps), C.byref(best),
                                        C.byref(ms)), "batch_tune")
        return best, float(ms.value)

    def close(self):
        if getattr(self, "handle", None):
            L.load().amj_batch_destroy(self.handle)
            self.handle = None
            self._rels = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class ServeResult:
    ticket: int
    count: int
    checksum: int
    path: str            # "batch" or "ooc"
    spilled: bool
    batch_id: int
    batch_size: int
    queue_ms: float
    exec_ms: float
    latency_ms: float


class Server:
    """Request server (amj_server): submit() returns a ticket at once, wait()
    returns that request's result.  The relations of a request are kept alive
    here until its result has been waited for."""

    def __init__(self, ctx: "Context", lanes: int = 2, max_batch: int = 256, mem_budget: int = 0,
                 ooc_lane: bool = True, ooc_mem: int = 0, ooc_slice_rows: int = 0, index_cache: bool = True,
                 index_cache_bytes: int = 0, **batch_kw):
        o = L.amj_serve_opts()
        o.lanes, o.max_batch, o.mem_budget = lanes, max_batch, mem_budget
        o.batch = Batch._opts(**batch_kw)
        o.ooc_lane, o.ooc_mem, o.ooc_slice_rows = int(bool(ooc_lane)), ooc_mem, ooc_slice_rows
        o.index_cache_bytes, o.no_index_cache = index_cache_bytes, 0 if index_cache else 1
        h = C.c_void_p()
        self.handle = None
        L.check(L.load().amj_server_create(ctx.handle, C.byref(o), C.byref(h)), "server_create")
        self.handle = h
        self.ctx = ctx
        self._held = {}

    def submit(self, query_type, relations: Sequence[Relation], ooc: bool = False, reorder: bool = True) -> int:
        qt = _QUERY[query_type] if isinstance(query_type, str) else int(query_type)
        arr = (C.c_void_p * len(relations))(*[r.handle for r in relations])
        t = C.c_uint64()
        flags = 0 if reorder else L.AMJ_F_NO_REORDER
        L.check(L.load().amj_server_submit(self.handle, qt, arr, len(relations), flags, int(bool(ooc)), C.byref(t)),
                "server_submit")
        self._held[int(t.value)] = list(relations)
        return int(t.value)

    def wait(self, ticket: int, timeout_ms: int = 600_000) -> ServeResult:
        r = L.amj_serve_result()
        st = L.load().amj_server_wait(self.handle, ticket, timeout_ms, C.byref(r))
        if st != L.AMJ_ETIMEOUT:
            self._held.pop(ticket, None)
        L.check(st, "server_wait")
        return ServeResult(ticket=ticket, count=int(r.count), checksum=int(r.checksum),
                           path="ooc" if r.path == 1 else "batch", spilled=bool(r.spilled), batch_id=int(r.batch_id),
                           batch_size=int(r.batch_size), queue_ms=r.queue_ms, exec_ms=r.exec_ms,
                           latency_ms=r.latency_ms)

    def stats(self) -> dict:
        s = L.amj_serve_stats()
        L.check(L.load().amj_server_stats(self.handle, C.byref(s)), "server_stats")
        return {name: int(getattr(s, name)) for name, _ in L.amj_serve_stats._fields_}

    def close(self):
        if getattr(self, "handle", None):
            L.load().amj_server_destroy(self.handle)
            self.handle = None
            self._held = {}

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """One CUDA device and stream (amj_ctx)."""

    def __init__(self, device: int = 0, layout: str = "bucket", load_factor: float = 0.5, task_chunk: int = 1024,
                 spin_limit_ms: int = 5000, task_capacity: int = 1 << 22, ooc_slice_rows: int = 0,
                 mem_budget: int = 0, lftj_heavy_degree: int = 0, dro_headroom: float = 0.0, max_blocks: int = 0,
                 lftj_rank_bits: int = 0):
        lib = L.load()
        o = L.amj_opts()
        o.block_size = 256
        o.layout = _LAYOUT[layout]
        o.load_factor = load_factor
        o.task_chunk = task_chunk
        o.spin_limit_ms = spin_limit_ms
        o.task_capacity = task_capacity
        o.ooc_slice_rows = ooc_slice_rows
        o.mem_budget = mem_budget
        o.lftj_heavy_degree = lftj_heavy_degree
        o.dro_headroom = dro_headroom
        o.max_blocks = max_blocks
        o.lftj_rank_bits = lftj_rank_bits
        h = C.c_void_p()
        self.handle = None
        self._relations = weakref.WeakSet()
        self._batches = weakref.WeakSet()
        L.check(lib.amj_ctx_create(device, C.byref(o), C.byref(h)), "ctx_create")
        self.handle = h

    def relation(self, cols, attrs, streamed: bool = False) -> Relation:
        return Relation(self, cols, attrs, streamed=streamed)

    def _result(self, res: L.amj_result, materialize: bool) -> Result:
        cols = None
        if materialize:
            k = res.num_attrs
            rows = int(res.rows)
            cols = []
            for a in range(k):
                if rows:
                    cols.append(np.ctypeslib.as_array(res.cols[a], shape=(rows,)).copy())
                else:
                    cols.append(np.zeros(0, np.int32))
        out = Result(count=int(res.count), checksum=int(res.checksum), num_attrs=int(res.num_attrs),
                     build_ms=float(res.build_ms), probe_ms=float(res.probe_ms), total_ms=float(res.total_ms),
                     stats={STAT_NAMES[i]: int(res.stats[i]) for i in range(len(STAT_NAMES))},
                     kernel_ms=tuple(float(res.kernel_ms[i]) for i in range(4)), columns=cols)
        L.load().amj_result_release(C.byref(res))
        return out

    def amhj(self, query_type, relations: Sequence[Relation], ooc: int = 0, ws: int = 0, dro: int = 0,
             fib: int = 0, materialize: bool = False, reorder: bool = True, degree_order: bool = True,
             plan: str = "multiway") -> Result:
        """degree_order=False joins a TRI / FOUR edge relation as given, never its
        degree-ordered copy (the results are the same).  plan: "multiway" (the
        operator; TRI / FOUR over one oriented edge relation without repeated rows
        answer their pair-key levels from a bitmap of b's children / the triangle
        matrices of the degree-ranked copy), "hash" (the operator with every level
        a hash lookup), "frontier" (the operator with every plan joined by the
        frontier-DFS kernel, no flat star / chain kernel), or a baseline to
        compare it with: "thread_per_row" (one thread per probe row, count
        only) or "pairwise" (2-relation joins with materialised
        intermediates)."""
        lib = L.load()
        qt = _QUERY[query_type] if isinstance(query_type, str) else int(query_type)
        arr = (C.c_void_p * len(relations))(*[r.handle for r in relations])
        flags = (L.AMJ_F_MATERIALIZE | L.AMJ_F_HOST_RESULT) if materialize else 0
        if not reorder:
            flags |= L.AMJ_F_NO_REORDER
        if not degree_order:
            flags |= L.AMJ_F_KEEP_ORDER
        flags |= {"multiway": 0, "thread_per_row": L.AMJ_F_THREAD_PER_ROW, "pairwise": L.AMJ_F_PAIRWISE,
                  "hash": L.AMJ_F_HASH_PLAN, "frontier": L.AMJ_F_FRONTIER}[plan]
        res = L.amj_result()
        L.check(lib.amj_amhj_execute(self.handle, qt, arr, len(relations), int(ooc), int(ws), int(dro), int(fib),
                                     flags, C.byref(res)), "amhj_execute")
        return self._result(res, materialize)

    def lftj(self, relations: Sequence[Relation], algo="DFS", ooc: int = 0, ws: int = 1,
             materialize: bool = False, clique4: bool = False, degree_order=None, attr_order=None,
             clique4_lists: bool = False) -> Result:
        """clique4: one edge relation joined as the 4-clique (FOUR pattern) instead of the triangle.
        degree_order: None for the operator's choice, True / False to force joining (or not) the
        degree-ordered copy of an oriented self-joined relation (same results either way).
        attr_order: the order in which attributes are bound (a permutation of 0..k-1; the
        results are the same for every order).
        clique4_lists: the 4-clique by list intersections even where the triangle matrices fit."""
        lib = L.load()
        arr = (C.c_void_p * len(relations))(*[r.handle for r in relations])
        flags = (L.AMJ_F_MATERIALIZE | L.AMJ_F_HOST_RESULT) if materialize else 0
        if clique4:
            flags |= L.AMJ_F_CLIQUE4
            if clique4_lists:
                flags |= L.AMJ_F_CLIQUE4_LISTS
        if degree_order is True:
            flags |= L.AMJ_F_DEGREE_ORDER
        elif degree_order is False:
            flags |= L.AMJ_F_KEEP_ORDER
        res = L.amj_result()
        if attr_order is None:
            L.check(lib.amj_lftj_execute(self.handle, arr, len(relations), _ALGO[algo], int(ooc), int(ws), flags,
                                         C.byref(res)), "lftj_execute")
        else:
            order = (C.c_uint32 * len(attr_order))(*[int(a) for a in attr_order])
            L.check(lib.amj_lftj_execute_ordered(self.handle, arr, len(relations), _ALGO[algo], int(ooc), int(ws),
                                                 flags, order, len(attr_order), C.byref(res)), "lftj_execute_ordered")
        return self._result(res, materialize)

    def edgelist_to_tr(self, text_path: str, tr_path: str, swap: bool = False) -> int:
        """Convert a text edge list to a .tr trie file (built on this
        context's device); returns the number of edges."""
        rows = C.c_uint64()
        L.check(L.load().amj_edgelist_to_tr(self.handle, text_path.encode(), tr_path.encode(), int(swap),
                                            C.byref(rows)), "edgelist_to_tr")
        return int(rows.value)

    def batch(self) -> Batch:
        b = Batch(self)
        self._batches.add(b)
        return b

    def server(self, **kw) -> Server:
        srv = Server(self, **kw)
        self._batches.add(srv)
        return srv

    def trim(self):
        """Give back the pinned host blocks and matrix area kept for reuse."""
        L.check(L.load().amj_ctx_trim(self.handle), "ctx_trim")

    def sync(self):
        L.check(L.load().amj_ctx_sync(self.handle), "ctx_sync")

    def close(self):
        if getattr(self, "handle", None):
            for b in list(getattr(self, "_batches", ())):
                b.close()
            for r in list(self._relations):
                r.release()
            L.load().amj_ctx_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cuda_device_available() -> bool:
    """True when libamj can create a context on device 0."""
    lib = L.load()
    h = C.c_void_p()
    st = lib.amj_ctx_create(0, None, C.byref(h))
    if st == L.AMJ_OK:
        lib.amj_ctx_destroy(h)
        return True
    return False
