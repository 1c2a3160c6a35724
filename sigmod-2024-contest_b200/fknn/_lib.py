"""ctypes binding of libfknn.so (the C ABI declared in include/fknn.h).

The shared library is built in-tree by ``make -C sigmod-2024-contest_b200``
(or ``__graft_entry__.build()``).  There is no fallback: if the library is
missing or fails to load, importing a search entry point raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_float, c_int, c_int8, c_size_t, c_uint32, c_uint64,
                    c_void_p)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfknn.so")

FKNN_OK = 0
FKNN_EINVAL = -1
FKNN_ENOMEM = -2
FKNN_ECUDA = -3
FKNN_ETIMEOUT = -4
FKNN_EUNSUPPORTED = -5
FKNN_ENODEV = -6

MODE_EXACT_FP32 = 0
MODE_BF16_RERANK = 1
MODE_FP8_RERANK = 2
SEARCH_GRAPH = 1  # fknn_search_opts.flags FKNN_SEARCH_GRAPH

# Graph search forms (include/fknn.h FKNN_GRAPH_*), numbered as the Searcher methods.
GRAPH_SEARCH = 0
GRAPH_FILTER = 1
GRAPH_FILTER_SUBTIME = 2
GRAPH_CATEGORY_RANGE = 3
GRAPH_RANGE_SUBTIME = 4
GRAPH_RANGE = 5

_ERRNAMES = {
    FKNN_EINVAL: "FKNN_EINVAL",
    FKNN_ENOMEM: "FKNN_ENOMEM",
    FKNN_ECUDA: "FKNN_ECUDA",
    FKNN_ETIMEOUT: "FKNN_ETIMEOUT",
    FKNN_EUNSUPPORTED: "FKNN_EUNSUPPORTED",
    FKNN_ENODEV: "FKNN_ENODEV",
}


class FknnError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERRNAMES.get(code, code)}: {msg}")
        self.code = code


class IndexOpts(Structure):
    _fields_ = [("device", c_int), ("build_bf16", c_int), ("build_fp8", c_int), ("hbm_budget", c_uint64)]


class Tuning(Structure):
    _fields_ = [("list_slack", c_uint32), ("items_per_sm", c_uint32), ("min_chunk_blocks", c_uint32),
                ("bound_refresh", c_uint32), ("pilot_stride", c_uint32)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class SearchOpts(Structure):
    _fields_ = [("mode", c_int), ("kprime", c_uint32), ("flags", c_uint32)]


class SearchStats(Structure):
    _fields_ = [
        ("pairs_screened", c_uint64),
        ("pairs_passing", c_uint64),
        ("pairs_contraction", c_uint64),
        ("n_tiles", c_uint32),
        ("n_work_items", c_uint32),
        ("n_small", c_uint32),
        ("n_overflow", c_uint32),
        ("n_boundary_f64", c_uint32),
        ("kernel_launches", c_uint32),
        ("ms_plan", c_float),
        ("ms_screen", c_float),
        ("ms_merge", c_float),
        ("ms_scan", c_float),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class ServerOpts(Structure):
    _fields_ = [("mode", c_int), ("kprime", c_uint32), ("k", c_uint32), ("max_batch", c_uint32),
                ("slots", c_uint32), ("max_wait_us", c_uint32), ("hbm_budget", c_uint64)]


class ServerStats(Structure):
    _fields_ = [
        ("submitted", c_uint64),
        ("completed", c_uint64),
        ("failed", c_uint64),
        ("batches", c_uint64),
        ("admission_waits", c_uint64),
        ("budget_trims", c_uint64),
        ("scratch_bytes", c_uint64),
        ("budget_bytes", c_uint64),
        ("max_batch_seen", c_uint32),
        ("mean_batch", c_float),
        ("p50_ms", c_float),
        ("p99_ms", c_float),
        ("max_ms", c_float),
        ("mean_ms", c_float),
        ("span_s", ctypes.c_double),
        ("qps", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class RouterSubgraph(Structure):
    _fields_ = [("key", ctypes.c_int32), ("start", c_uint32), ("count", c_uint32), ("graph_bytes", c_void_p),
                ("nbytes", c_size_t)]


class RouterDesc(Structure):
    _fields_ = [("vecs", c_void_p), ("labels", c_void_p), ("ts", c_void_p), ("n", c_uint64),
                ("sorted_base_ids", c_void_p), ("sorted_base_ids_by_full_time", c_void_p),
                ("categories", POINTER(RouterSubgraph)), ("ncategories", c_uint32),
                ("buckets", POINTER(RouterSubgraph)), ("nbuckets", c_uint32), ("maxc_size", c_uint32),
                ("minc_size", c_uint32), ("device", c_int)]


class RouterParams(Structure):
    _fields_ = [(f, c_uint32) for f in ("ef0_full", "ef1min", "ef1max", "ef3min", "ef3max", "ef2_full_large",
                                        "ef2_full_medium", "ef2_full_small", "ef2_medium_large",
                                        "ef2_medium_medium", "ef2_medium_small")] + \
               [("bf_thr", c_float), ("bf_thr3", c_float), ("bf_refine_k", c_uint32), ("graph_refine_k", c_uint32),
                ("sel_rows", c_uint32)]


class RouterStats(Structure):
    _fields_ = [(f, c_uint32) for f in ("n_bruteforce", "n_category", "n_type0", "n_type2", "n_graph_calls",
                                        "n_split_small", "n_split_medium", "n_split_full")] + \
        [(f, c_float) for f in ("ms_total", "ms_prepare", "ms_bruteforce", "ms_category", "ms_type0", "ms_type2",
                                "ms_final")]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


# Every entry point of include/fknn.h with its ctypes signature.
SIGNATURES = {
    "fknn_version": (c_int, []),
    "fknn_last_error": (c_char_p, []),
    "fknn_index_create": (c_int, [c_void_p, c_void_p, c_void_p, c_uint64, c_uint32, POINTER(IndexOpts),
                                  POINTER(c_void_p)]),
    "fknn_index_create_from_file": (c_int, [c_char_p, POINTER(IndexOpts), POINTER(c_void_p)]),
    "fknn_index_destroy": (c_int, [c_void_p]),
    "fknn_read_base_file": (c_int, [c_char_p, POINTER(c_uint64), c_void_p, c_void_p, c_void_p]),
    "fknn_read_query_file": (c_int, [c_char_p, POINTER(c_uint32), c_void_p, c_void_p]),
    "fknn_sorted_query_order": (c_int, [c_void_p, c_uint32, c_void_p]),
    "fknn_save_knn": (c_int, [c_char_p, c_void_p, c_uint32, c_uint32]),
    "fknn_read_groundtruth": (c_int, [c_char_p, c_uint32, POINTER(c_uint32), c_void_p]),
    "fknn_index_bytes": (c_int, [c_void_p, POINTER(c_uint64)]),
    "fknn_index_set_tuning": (c_int, [c_void_p, c_int, POINTER(Tuning)]),
    "fknn_index_get_tuning": (c_int, [c_void_p, c_int, POINTER(Tuning)]),
    "fknn_index_test_withhold_copy": (c_int, [c_void_p]),
    "fknn_search": (c_int, [c_void_p, c_void_p, c_void_p, c_uint32, c_uint32, c_int, c_void_p, c_void_p, c_void_p]),
    "fknn_search_ex": (c_int, [c_void_p, c_void_p, c_void_p, c_uint32, c_uint32, POINTER(SearchOpts), c_void_p,
                               c_void_p, c_void_p, POINTER(SearchStats)]),
    "fknn_count_matches": (c_int, [c_void_p, c_void_p, c_uint32, c_void_p, c_void_p]),
    "fknn_filter_rows": (c_int, [c_void_p, c_void_p, c_void_p, POINTER(c_uint64), c_void_p]),
    "fknn_filter_rows_batch": (c_int, [c_void_p, c_void_p, c_uint32, c_void_p, c_void_p, c_void_p]),
    "fknn_filter_rows_noalloc": (c_int, [c_void_p, c_void_p, c_uint64, c_void_p, c_void_p, POINTER(c_uint64),
                                         c_void_p]),
    "fknn_bruteforce_rows": (c_int, [c_void_p, c_uint32, c_void_p, c_uint32, c_void_p]),
    "fknn_sq8_sym_train": (c_int, [c_void_p, c_uint64, POINTER(c_float), c_void_p]),
    "fknn_sq8_sym_encode": (c_int, [c_void_p, c_uint64, c_float, c_void_p]),
    "fknn_sq8_bruteforce": (c_int, [c_size_t, c_size_t, c_void_p, c_size_t, c_void_p, c_float, c_size_t, c_void_p]),
    "fknn_sq8_bruteforce_subgraph": (c_int, [c_size_t, c_size_t, c_void_p, c_void_p, c_size_t, c_void_p, c_float,
                                             c_size_t, c_void_p]),
    "fknn_sq8_release_thread_scratch": (c_int, []),
    "fknn_rerank": (c_int, [c_void_p, c_void_p, c_uint32, c_void_p, c_uint32, c_uint32, c_void_p, c_void_p,
                            c_void_p]),
    "fknn_graph_create": (c_int, [c_void_p, c_size_t, c_void_p, c_int, POINTER(c_void_p)]),
    "fknn_graph_destroy": (c_int, [c_void_p]),
    "fknn_graph_info": (c_int, [c_void_p, POINTER(c_uint32), POINTER(c_uint32), POINTER(c_float)]),
    "fknn_graph_search": (c_int, [c_void_p, c_void_p, c_uint32, c_int, c_uint32, c_uint32, c_uint32, c_void_p,
                                  c_void_p, c_void_p, c_void_p, c_void_p]),
    "fknn_router_default_params": (c_int, [POINTER(RouterParams)]),
    "fknn_router_create": (c_int, [POINTER(RouterDesc), POINTER(c_void_p)]),
    "fknn_router_search": (c_int, [c_void_p, c_void_p, c_void_p, c_uint32, POINTER(RouterParams), c_void_p,
                                   POINTER(RouterStats)]),
    "fknn_router_destroy": (c_int, [c_void_p]),
    "fknn_server_create": (c_int, [c_void_p, POINTER(ServerOpts), POINTER(c_void_p)]),
    "fknn_server_now_ns": (ctypes.c_int64, []),
    "fknn_server_submit": (c_int, [c_void_p, c_void_p, c_void_p, c_uint32, c_void_p, c_void_p, c_void_p,
                                   POINTER(c_uint64)]),
    "fknn_server_wait": (c_int, [c_void_p, c_uint64, c_int]),
    "fknn_server_drain": (c_int, [c_void_p, c_int]),
    "fknn_server_get_stats": (c_int, [c_void_p, POINTER(ServerStats), c_int]),
    "fknn_server_destroy": (c_int, [c_void_p]),
}

_lib = None


def load() -> ctypes.CDLL:
    """Loads libfknn.so once; raises if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libfknn.so is not built ({LIB_PATH}); build it with "
                           f"`make -C {os.path.dirname(_HERE)}` or __graft_entry__.build()")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != FKNN_OK:
        msg = load().fknn_last_error()
        raise FknnError(rc, msg.decode() if msg else "")


def last_error() -> str:
    return load().fknn_last_error().decode()
