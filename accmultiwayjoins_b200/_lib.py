"""ctypes binding of libamj.so, the C ABI declared in include/amj.h.

The library is built in-tree (``make -C accmultiwayjoins_b200/csrc``) and
loaded from this directory.  Loading it needs no GPU; every call that needs
one returns a status code (AMJ_ECUDA) when none is present.  There is no CPU
fallback: a missing library raises at import of the operator modules.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libamj.so")

AMJ_MAX_ATTRS = 8
AMJ_MAX_BUILD_TABLES = 6
AMJ_MAX_COLS = 8

AMJ_OK = 0
AMJ_EINVAL = -1
AMJ_ENOMEM = -2
AMJ_EOVERFLOW = -3
AMJ_ETIMEOUT = -4
AMJ_ECUDA = -5
AMJ_EUNSUPPORTED = -6
AMJ_EIO = -7
AMJ_EREJECT = -8

STATUS_NAMES = {
    AMJ_OK: "AMJ_OK", AMJ_EINVAL: "AMJ_EINVAL", AMJ_ENOMEM: "AMJ_ENOMEM", AMJ_EOVERFLOW: "AMJ_EOVERFLOW",
    AMJ_ETIMEOUT: "AMJ_ETIMEOUT", AMJ_ECUDA: "AMJ_ECUDA", AMJ_EUNSUPPORTED: "AMJ_EUNSUPPORTED",
    AMJ_EIO: "AMJ_EIO", AMJ_EREJECT: "AMJ_EREJECT",
}

AMJ_QUERY_NORMAL, AMJ_QUERY_TRI, AMJ_QUERY_FOUR = 0, 1, 2
AMJ_LFTJ_BFS, AMJ_LFTJ_DFS = 0, 1
AMJ_LAYOUT_BUCKET, AMJ_LAYOUT_OPEN_ADDR, AMJ_LAYOUT_CUCKOO = 0, 1, 2
AMJ_F_MATERIALIZE, AMJ_F_HOST_RESULT, AMJ_F_NO_REORDER, AMJ_F_CLIQUE4 = 0x1, 0x2, 0x4, 0x8
AMJ_F_KEEP_ORDER, AMJ_F_DEGREE_ORDER, AMJ_F_CLIQUE4_LISTS = 0x10, 0x20, 0x40
AMJ_F_THREAD_PER_ROW, AMJ_F_PAIRWISE, AMJ_F_HASH_PLAN, AMJ_F_FRONTIER = 0x80, 0x100, 0x200, 0x400
AMJ_MEM_DEVICE, AMJ_MEM_HOST, AMJ_MEM_HOST_STREAMED = 0, 1, 2


class amj_opts(C.Structure):
    _fields_ = [
        ("block_size", C.c_int),
        ("layout", C.c_int),
        ("load_factor", C.c_float),
        ("task_chunk", C.c_int),
        ("spin_limit_ms", C.c_uint32),
        ("task_capacity", C.c_uint64),
        ("ooc_slice_rows", C.c_uint64),
        ("mem_budget", C.c_uint64),
        ("lftj_heavy_degree", C.c_uint32),
        ("dro_headroom", C.c_float),
        ("max_blocks", C.c_uint32),
        ("lftj_rank_bits", C.c_uint32),
    ]


class amj_result(C.Structure):
    _fields_ = [
        ("count", C.c_uint64),
        ("checksum", C.c_uint64),
        ("num_attrs", C.c_int32),
        ("on_host", C.c_int32),
        ("cols", C.POINTER(C.c_int32) * AMJ_MAX_ATTRS),
        ("rows", C.c_uint64),
        ("build_ms", C.c_double),
        ("probe_ms", C.c_double),
        ("total_ms", C.c_double),
        ("stats", C.c_uint64 * 12),
        ("kernel_ms", C.c_double * 4),
        ("priv", C.c_void_p),
    ]


class amj_batch_opts(C.Structure):
    _fields_ = [
        ("layout", C.c_int),
        ("load_factor", C.c_float),
        ("block_size", C.c_int),
        ("task_chunk", C.c_int),
        ("use_graph", C.c_int),
        ("grid_blocks", C.c_int),
    ]


class amj_batch_stats(C.Structure):
    _fields_ = [
        ("build_ms", C.c_double),
        ("probe_ms", C.c_double),
        ("total_ms", C.c_double),
        ("launches", C.c_uint64),
        ("tasks_pushed", C.c_uint64),
        ("tasks_popped", C.c_uint64),
        ("units", C.c_uint64),
        ("build_rows", C.c_uint64),
        ("build_jobs", C.c_uint64),
        ("graph", C.c_int32),
        ("pad", C.c_int32),
    ]


class amj_batch_tune_grid(C.Structure):
    _fields_ = [
        ("layout", C.c_int),
        ("n_load_factor", C.c_int),
        ("n_block_size", C.c_int),
        ("n_task_chunk", C.c_int),
        ("load_factor", C.c_float * 8),
        ("block_size", C.c_int * 8),
        ("task_chunk", C.c_int * 8),
    ]


class amj_serve_opts(C.Structure):
    _fields_ = [
        ("lanes", C.c_int),
        ("max_batch", C.c_uint32),
        ("mem_budget", C.c_uint64),
        ("batch", amj_batch_opts),
        ("ooc_lane", C.c_int),
        ("ooc_mem", C.c_uint64),
        ("ooc_slice_rows", C.c_uint64),
        ("index_cache_bytes", C.c_uint64),
        ("no_index_cache", C.c_int),
        ("pad", C.c_int),
    ]


class amj_serve_result(C.Structure):
    _fields_ = [
        ("count", C.c_uint64),
        ("checksum", C.c_uint64),
        ("status", C.c_int32),
        ("path", C.c_int32),
        ("spilled", C.c_int32),
        ("batch_id", C.c_uint32),
        ("batch_size", C.c_uint32),
        ("pad", C.c_int32),
        ("queue_ms", C.c_double),
        ("exec_ms", C.c_double),
        ("latency_ms", C.c_double),
    ]


class amj_serve_stats(C.Structure):
    _fields_ = [
        ("submitted", C.c_uint64),
        ("completed", C.c_uint64),
        ("rejected", C.c_uint64),
        ("spilled", C.c_uint64),
        ("batches", C.c_uint64),
        ("ooc_runs", C.c_uint64),
        ("budget_bytes", C.c_uint64),
        ("peak_reserved_bytes", C.c_uint64),
        ("launches", C.c_uint64),
        ("index_hits", C.c_uint64),
        ("index_builds", C.c_uint64),
        ("index_bytes", C.c_uint64),
        ("max_inflight_batches", C.c_uint32),
        ("lanes", C.c_uint32),
    ]


class AmjError(RuntimeError):
    """A libamj call returned a non-zero status."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_P = C.c_void_p
_I32P = C.POINTER(C.c_int32)
_U32P = C.POINTER(C.c_uint32)
_U64P = C.POINTER(C.c_uint64)

# name -> (restype, argtypes); every symbol declared in include/amj.h
SIGNATURES = {
    "amj_last_error": (C.c_char_p, []),
    "amj_version": (C.c_char_p, []),
    "amj_ctx_create": (C.c_int, [C.c_int, C.POINTER(amj_opts), C.POINTER(_P)]),
    "amj_ctx_destroy": (None, [_P]),
    "amj_ctx_set_stream": (C.c_int, [_P, _P]),
    "amj_ctx_sync": (C.c_int, [_P]),
    "amj_stat_name": (C.c_char_p, [C.c_int]),
    "amj_ctx_launch_count": (C.c_int, [_P, _U64P]),
    "amj_ctx_trim": (C.c_int, [_P]),
    "amj_rel_create": (C.c_int, [_P, C.c_uint64, C.c_int, _U32P, C.POINTER(_I32P), C.c_int, C.POINTER(_P)]),
    "amj_rel_release": (None, [_P]),
    "amj_rel_info": (C.c_int, [_P, _U64P, C.POINTER(C.c_int), _U32P]),
    "amj_amhj_execute": (C.c_int, [_P, C.c_int, C.POINTER(_P), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.c_int, C.POINTER(amj_result)]),
    "amj_lftj_execute": (C.c_int, [_P, C.POINTER(_P), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.POINTER(amj_result)]),
    "amj_lftj_execute_ordered": (C.c_int, [_P, C.POINTER(_P), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _U32P,
                                           C.c_int, C.POINTER(amj_result)]),
    "amj_result_release": (None, [C.POINTER(amj_result)]),
    "amj_batch_create": (C.c_int, [_P, C.POINTER(_P)]),
    "amj_batch_submit": (C.c_int, [_P, C.c_int, C.POINTER(_P), C.c_int, C.c_int, _U32P]),
    "amj_batch_size": (C.c_int, [_P, _U32P]),
    "amj_batch_run": (C.c_int, [_P, C.POINTER(amj_batch_opts), _U64P, _U64P, C.POINTER(amj_batch_stats)]),
    "amj_batch_tune": (C.c_int, [_P, C.POINTER(amj_batch_tune_grid), C.c_uint32, C.c_int, C.POINTER(amj_batch_opts),
                                 C.POINTER(C.c_double)]),
    "amj_batch_destroy": (C.c_int, [_P]),
    "amj_server_create": (C.c_int, [_P, C.POINTER(amj_serve_opts), C.POINTER(_P)]),
    "amj_server_submit": (C.c_int, [_P, C.c_int, C.POINTER(_P), C.c_int, C.c_int, C.c_int, _U64P]),
    "amj_server_wait": (C.c_int, [_P, C.c_uint64, C.c_uint32, C.POINTER(amj_serve_result)]),
    "amj_server_stats": (C.c_int, [_P, C.POINTER(amj_serve_stats)]),
    "amj_server_destroy": (C.c_int, [_P]),
    "amj_bucket_build": (C.c_int, [_P, _P, C.c_uint64, C.c_uint64, _P, _P, _P]),
    "amj_bucket_build_static": (C.c_int, [_P, C.c_uint64, C.c_uint64, _P, _P, _P, _P]),
    "amj_trie_build": (C.c_int, [_P, _P, _P, C.c_uint64, C.POINTER(_P)]),
    "amj_trie_view": (C.c_int, [_P, _U64P, _U64P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]),
    "amj_trie_download": (C.c_int, [_P, _I32P, _U64P, _I32P]),
    "amj_trie_save": (C.c_int, [_P, C.c_char_p, C.c_uint32, C.c_uint32]),
    "amj_trie_load": (C.c_int, [_P, C.c_char_p, C.POINTER(_P), _U32P, _U32P]),
    "amj_trie_release": (None, [_P]),
    "amj_trie_build_n": (C.c_int, [_P, C.POINTER(_P), C.c_int, C.c_uint64, C.POINTER(_P)]),
    "amj_trie_info": (C.c_int, [_P, C.POINTER(C.c_int), _U64P]),
    "amj_trie_download_level": (C.c_int, [_P, C.c_int, _I32P, _U64P]),
    "amj_trie_save_n": (C.c_int, [_P, C.c_char_p, _U32P]),
    "amj_trie_load_n": (C.c_int, [_P, C.c_char_p, C.POINTER(_P), _U32P, C.POINTER(C.c_int)]),
    "amj_selftest_bounded_wait": (C.c_int, [_P, C.c_uint32]),
    "amj_gen_uniform_i32": (C.c_int, [_I32P, C.c_uint64, C.c_int64, C.c_int64, C.c_uint64, C.c_uint64]),
    "amj_gen_permutation_i32": (C.c_int, [_I32P, C.c_uint64, C.c_uint64, C.c_uint64]),
    "amj_gen_zipf_i32": (C.c_int, [_I32P, C.c_uint64, C.c_uint64, C.c_double, _I32P, C.c_uint64, C.c_uint64]),
    "amj_gen_rmat": (C.c_int, [C.c_int, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_uint64, _I32P, _I32P,
                               _U64P]),
    "amj_db_write": (C.c_int, [C.c_char_p, C.c_uint64, C.c_int, C.POINTER(_I32P)]),
    "amj_db_read": (C.c_int, [C.c_char_p, C.c_uint64, C.c_int, C.POINTER(_I32P)]),
    "amj_db_parse_name": (C.c_int, [C.c_char_p, _U64P, C.POINTER(C.c_int), _U32P]),
    "amj_checksum_host": (C.c_int, [C.POINTER(_I32P), C.c_int, C.c_uint64, _U64P]),
    "amj_edgelist_read": (C.c_int, [C.c_char_p, C.c_int, _I32P, _I32P, C.c_uint64, _U64P]),
    "amj_edgelist_to_db": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, _U64P]),
    "amj_edgelist_to_tr": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_int, _U64P]),
    "amj_tbl_to_db": (C.c_int, [C.c_char_p, _U32P, _U32P, C.c_int, C.c_char_p, C.c_char_p, C.c_uint64, _U64P]),
}

_lib = None


def load() -> C.CDLL:
    """Load libamj.so once and attach the C signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libamj.so not found at {LIB_PATH}; build it with `make -C accmultiwayjoins_b200/csrc`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, what: str = "") -> None:
    if status != AMJ_OK:
        msg = load().amj_last_error().decode(errors="replace")
        raise AmjError(status, f"{what}: {msg}" if what else msg)
