"""ctypes loader of the CPU checker.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker / the timed CPU baseline; the product
library never calls it.

  restatement : oracle/libfknn_oracle.so  (oracle/fknn_oracle.c)
  reference   : oracle/_ref/libref_exact.so, oracle/_ref/libref_sq8.so,
                oracle/_ref/libref_graph.so, the reference's own code compiled
                from its sources (oracle/Makefile)
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_float, c_int, c_int8, c_uint32, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libfknn_oracle.so")
REF_EXACT_SO = os.path.join(HERE, "_ref", "libref_exact.so")
REF_SQ8_SO = os.path.join(HERE, "_ref", "libref_sq8.so")
REF_GRAPH_SO = os.path.join(HERE, "_ref", "libref_graph.so")
DIM = 100

_o = None
_re = None
_rs = None
_rg = None


def build(ref: bool = False) -> None:
    """make -C oracle (and the reference objects when the sources are present)."""
    targets = ["all"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def lib() -> ctypes.CDLL:
    global _o
    if _o is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        L.oracle_normal_l2.restype = c_float
        L.oracle_normal_l2.argtypes = [c_void_p, c_void_p, c_uint32]
        L.oracle_exact_knn.restype = c_int
        L.oracle_exact_knn.argtypes = [c_void_p, c_void_p, c_void_p, c_uint32, c_void_p, c_void_p, c_uint32,
                                       c_uint32, c_void_p, c_void_p, c_int]
        L.oracle_exact_knn_f64.restype = c_int
        L.oracle_exact_knn_f64.argtypes = L.oracle_exact_knn.argtypes
        L.oracle_count_matches.restype = None
        L.oracle_count_matches.argtypes = [c_void_p, c_void_p, c_uint32, c_void_p, c_uint32, c_void_p]
        L.oracle_sq8_sym_alpha.restype = c_float
        L.oracle_sq8_sym_alpha.argtypes = [c_void_p, c_uint64]
        L.oracle_sq8_sym_encode.restype = None
        L.oracle_sq8_sym_encode.argtypes = [c_void_p, c_uint64, c_float, c_void_p]
        L.oracle_l2sqr_sq8_sym.restype = ctypes.c_int32
        L.oracle_l2sqr_sq8_sym.argtypes = [c_void_p, c_void_p]
        L.oracle_sq8_bruteforce.restype = c_int
        L.oracle_sq8_bruteforce.argtypes = [c_uint64, c_void_p, c_void_p, c_uint64, c_void_p, c_float, c_void_p]
        L.oracle_graph_search.restype = c_int
        L.oracle_graph_search.argtypes = [c_void_p, ctypes.c_size_t, c_void_p, c_float, c_void_p, c_uint32, c_int,
                                          c_uint32, c_uint32, c_uint32, c_void_p, c_void_p, c_void_p, c_void_p]
        _o = L
    return _o


def ref_exact() -> ctypes.CDLL | None:
    """The reference Bruteforce (utils.h:80) compiled from its sources, or None."""
    global _re
    if _re is None and os.path.exists(REF_EXACT_SO):
        L = ctypes.CDLL(REF_EXACT_SO)
        L.ref_exact_bruteforce.restype = c_int
        L.ref_exact_bruteforce.argtypes = [c_void_p, c_uint32, c_void_p, c_uint32, c_void_p, POINTER(c_double)]
        L.ref_normal_l2.restype = c_float
        L.ref_normal_l2.argtypes = [c_void_p, c_void_p, c_uint32]
        _re = L
    return _re


def ref_sq8() -> ctypes.CDLL | None:
    global _rs
    if _rs is None and os.path.exists(REF_SQ8_SO):
        L = ctypes.CDLL(REF_SQ8_SO)
        L.ref_l2sqr_sq8_sym.restype = c_int
        L.ref_l2sqr_sq8_sym.argtypes = [c_void_p, c_void_p]
        L.ref_sq8_sym_train.restype = None
        L.ref_sq8_sym_train.argtypes = [c_void_p, c_uint32, POINTER(c_float), c_void_p]
        L.ref_sq8_sym_encode.restype = None
        L.ref_sq8_sym_encode.argtypes = [c_void_p, c_float, c_void_p]
        L.ref_sq8_bruteforce.restype = None
        L.ref_sq8_bruteforce.argtypes = [c_uint64, c_void_p, c_uint64, c_void_p, c_float, c_void_p]
        L.ref_sq8_bruteforce_subgraph.restype = None
        L.ref_sq8_bruteforce_subgraph.argtypes = [c_uint64, c_void_p, c_void_p, c_uint64, c_void_p, c_float, c_void_p]
        _rs = L
    return _rs


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def exact_knn(vecs, labels, ts, qvecs, metas, k: int = 100, nthreads: int = 0, f64: bool = False):
    """Restated utils.h:80 over SoA columns -> (ids (nq,k) u32, dists (nq,k))."""
    vecs, labels, ts = _c(vecs, np.float32), _c(labels, np.float32), _c(ts, np.float32)
    qvecs, metas = _c(qvecs, np.float32), _c(metas, np.float32)
    nq = qvecs.shape[0]
    ids = np.empty((nq, k), dtype=np.uint32)
    dists = np.empty((nq, k), dtype=np.float64 if f64 else np.float32)
    nthreads = nthreads or os.cpu_count() or 1
    fn = lib().oracle_exact_knn_f64 if f64 else lib().oracle_exact_knn
    rc = fn(vecs.ctypes.data, labels.ctypes.data, ts.ctypes.data, vecs.shape[0], qvecs.ctypes.data,
            metas.ctypes.data, nq, k, ids.ctypes.data, dists.ctypes.data, nthreads)
    if rc != 0:
        raise ValueError(f"oracle_exact_knn failed ({rc})")
    return ids, dists


def count_matches(labels, ts, metas) -> np.ndarray:
    labels, ts, metas = _c(labels, np.float32), _c(ts, np.float32), _c(metas, np.float32)
    out = np.empty(metas.shape[0], dtype=np.uint32)
    lib().oracle_count_matches(labels.ctypes.data, ts.ctypes.data, labels.shape[0], metas.ctypes.data,
                               metas.shape[0], out.ctypes.data)
    return out


def _sortable(f: np.ndarray) -> np.ndarray:
    """Order-preserving uint32 image of float32 (-0 folded onto +0)."""
    u = (np.asarray(f, dtype=np.float32) + np.float32(0.0)).view(np.uint32).astype(np.uint64)
    return np.where(u & 0x80000000, (~u) & 0xFFFFFFFF, u | 0x80000000)


def filter_rows(labels, ts, meta4) -> np.ndarray:
    """Ids (increasing, uint32) of the rows passing one predicate (type, v,
    l, r) of utils.h:110-137: type 0 every row, 1 int32(label) == int32(v),
    2 l <= ts <= r, 3 both."""
    labels, ts = _c(labels, np.float32), _c(ts, np.float32)
    m = np.asarray(meta4, dtype=np.float32).reshape(4)
    t = int(np.uint32(m[0]))
    keep = np.ones(labels.shape[0], dtype=bool)
    if t in (1, 3):
        keep &= labels.astype(np.int32) == np.int32(m[1])
    if t in (2, 3):
        keep &= (ts >= m[2]) & (ts <= m[3])
    return np.nonzero(keep)[0].astype(np.uint32)


def count_matches_sorted(labels, ts, metas) -> np.ndarray:
    """The passing-row count of each predicate (type, v, l, r) of
    utils.h:98-137 -- type 0 all rows, 1 int32(label) == int32(v),
    2 l <= ts <= r, 3 both -- from binary searches on sorted columns
    (the counts equal count_matches'; this form costs O((N + Q) log N),
    so it serves N = 1e7 with Q = 1e6)."""
    labels, ts, metas = _c(labels, np.float32), _c(ts, np.float32), _c(metas, np.float32)
    n = labels.shape[0]
    lab = labels.astype(np.int32).astype(np.int64)
    t_sorted = np.sort(ts)
    key = ((lab + (1 << 31)).astype(np.uint64) << np.uint64(32)) | _sortable(ts)
    key.sort()
    typ = metas[:, 0].astype(np.int64)
    out = np.zeros(metas.shape[0], dtype=np.int64)
    out[typ == 0] = n
    m2 = typ == 2
    out[m2] = np.searchsorted(t_sorted, metas[m2, 3], "right") - np.searchsorted(t_sorted, metas[m2, 2], "left")
    m13 = (typ == 1) | (typ == 3)
    v = (metas[m13, 1].astype(np.int32).astype(np.int64) + (1 << 31)).astype(np.uint64) << np.uint64(32)
    t1 = typ[m13] == 1
    lo = np.where(t1, v, v | _sortable(metas[m13, 2]))
    hi = np.where(t1, v | np.uint64(0xFFFFFFFF), v | _sortable(metas[m13, 3]))
    out[m13] = np.searchsorted(key, hi, "right") - np.searchsorted(key, lo, "left")
    return np.maximum(out, 0).astype(np.uint32)


def sq8_sym_train(vecs):
    vecs = _c(vecs, np.float32)
    a = lib().oracle_sq8_sym_alpha(vecs.ctypes.data, vecs.size)
    codes = np.empty((vecs.shape[0], 112), dtype=np.int8)
    lib().oracle_sq8_sym_encode(vecs.ctypes.data, vecs.shape[0], c_float(a), codes.ctypes.data)
    return a, codes


def sq8_sym_encode(vecs, alpha):
    vecs = _c(vecs, np.float32).reshape(-1, DIM)
    codes = np.empty((vecs.shape[0], 112), dtype=np.int8)
    lib().oracle_sq8_sym_encode(vecs.ctypes.data, vecs.shape[0], c_float(alpha), codes.ctypes.data)
    return codes


def sq8_bruteforce(k, codes, alpha, query, with_dists=False):
    codes, query = _c(codes, np.int8), _c(query, np.int8)
    ids = np.empty(k, dtype=np.int32)
    d = np.empty(k, dtype=np.float32) if with_dists else None
    rc = lib().oracle_sq8_bruteforce(k, ids.ctypes.data, d.ctypes.data if with_dists else None, codes.shape[0],
                                     codes.ctypes.data, c_float(alpha), query.ctypes.data)
    if rc != 0:
        raise ValueError("oracle_sq8_bruteforce: need 1 <= k <= npoints")
    return (ids, d) if with_dists else ids


def ref_graph() -> ctypes.CDLL | None:
    """The reference HNSW::Build + Searcher compiled from its sources, or None."""
    global _rg
    if _rg is None and os.path.exists(REF_GRAPH_SO):
        L = ctypes.CDLL(REF_GRAPH_SO)
        L.ref_hnsw_build.restype = c_int
        L.ref_hnsw_build.argtypes = [c_void_p, c_void_p, c_int, c_int, c_int, ctypes.c_char_p]
        L.ref_graph_search.restype = c_int
        L.ref_graph_search.argtypes = [ctypes.c_char_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int, c_int,
                                       c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
        _rg = L
    return _rg


def _opt_ptr(a, dt, shape):
    if a is None:
        return None, None
    a = _c(a, dt).reshape(shape)
    return a, a.ctypes.data


def graph_search(graph_bytes, vecs, queries, mode: int, k: int, refine: int, bounds=None, id_bounds=None,
                 ef: int = 32, with_dists: bool = False):
    """Restated Searcher (searcher.hpp:162-569) over Graph::save bytes; the
    searcher's codes are trained on vecs (Searcher::SetData).  Returns ids
    (nq, refine) int32 [and dists]."""
    gb = np.frombuffer(bytes(graph_bytes), dtype=np.uint8)
    alpha, codes = sq8_sym_train(_c(vecs, np.float32).reshape(-1, DIM))
    qc = sq8_sym_encode(queries, alpha)
    nq = qc.shape[0]
    b, bp = _opt_ptr(bounds, np.float32, (nq, 2))
    ib, ibp = _opt_ptr(id_bounds, np.int32, (nq, 2))
    ids = np.empty((nq, refine), dtype=np.int32)
    d = np.empty((nq, refine), dtype=np.float32) if with_dists else None
    rc = lib().oracle_graph_search(gb.ctypes.data, gb.size, codes.ctypes.data, c_float(alpha), qc.ctypes.data, nq,
                                   mode, k, ef, refine, bp, ibp, ids.ctypes.data,
                                   d.ctypes.data if with_dists else None)
    if rc != 0:
        raise ValueError(f"oracle_graph_search failed ({rc})")
    return (ids, d) if with_dists else ids


def ref_hnsw_graph(vecs, ts, R: int, efc: int, path: str) -> bytes:
    """Graph::save bytes of the reference HNSW::Build (out-degree R = 2M)."""
    R_ = ref_graph()
    if R_ is None:
        raise RuntimeError("oracle/_ref/libref_graph.so is not built")
    vecs, ts = _c(vecs, np.float32), _c(ts, np.float32)
    rc = R_.ref_hnsw_build(vecs.ctypes.data, ts.ctypes.data, vecs.shape[0], R, efc, path.encode())
    if rc != 0:
        raise RuntimeError("ref_hnsw_build failed")
    with open(path, "rb") as f:
        return f.read()


def ref_graph_search(path: str, vecs, labels, ts, queries, mode: int, k: int, refine: int, bounds=None,
                     id_bounds=None, with_dists: bool = False, timing: list | None = None):
    """The reference Searcher itself over the graph saved at path.  timing:
    a list that receives the seconds of the query loop alone (graph load and
    SetData excluded)."""
    R_ = ref_graph()
    if R_ is None:
        raise RuntimeError("oracle/_ref/libref_graph.so is not built")
    vecs, labels, ts = _c(vecs, np.float32), _c(labels, np.float32), _c(ts, np.float32)
    q = _c(queries, np.float32).reshape(-1, DIM)
    nq = q.shape[0]
    b, bp = _opt_ptr(bounds, np.float32, (nq, 2))
    ib, ibp = _opt_ptr(id_bounds, np.int32, (nq, 2))
    ids = np.empty((nq, refine), dtype=np.int32)
    d = np.empty((nq, refine), dtype=np.float32) if with_dists else None
    secs = ctypes.c_double(0.0)
    rc = R_.ref_graph_search(path.encode(), vecs.ctypes.data, labels.ctypes.data, ts.ctypes.data, vecs.shape[0],
                             q.ctypes.data, nq, mode, k, refine, bp, ibp, ids.ctypes.data,
                             d.ctypes.data if with_dists else None, ctypes.byref(secs))
    if rc != 0:
        raise RuntimeError("ref_graph_search failed")
    if timing is not None:
        timing.append(secs.value)
    return (ids, d) if with_dists else ids


_rh = None


def ref_hybrid() -> ctypes.CDLL | None:
    """The reference's whole approximate pipeline (baseline.cpp around
    hybrid_graph.cpp) compiled from its sources, or None."""
    global _rh
    REF_HYBRID_SO = os.path.join(HERE, "_ref", "libref_hybrid.so")
    if _rh is None and os.path.exists(REF_HYBRID_SO):
        L = ctypes.CDLL(REF_HYBRID_SO)
        L.ref_hybrid_run.restype = c_int
        L.ref_hybrid_run.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, c_int, c_int, c_void_p,
                                     POINTER(c_double)]
        _rh = L
    return _rh


def ref_hybrid_run(base_path: str, query_path: str, out_dir: str, nq: int, M: int = 16, efc: int = 100):
    """Runs the reference pipeline on contest files; returns (ids (nq,100)
    u32 in query order, BatchSearch seconds).  The subgraphs, base orders
    and maps it used are left in out_dir (read_hybrid_dir)."""
    L = ref_hybrid()
    if L is None:
        raise RuntimeError("oracle/_ref/libref_hybrid.so is not built")
    ids = np.empty((nq, 100), dtype=np.uint32)
    sec = c_double()
    rc = L.ref_hybrid_run(base_path.encode(), query_path.encode(), out_dir.encode(), M, efc, ids.ctypes.data,
                          ctypes.byref(sec))
    if rc != 0:
        raise RuntimeError("ref_hybrid_run failed")
    return ids, sec.value


def read_hybrid_dir(out_dir: str, n: int) -> dict:
    """The inputs the reference pipeline's BatchSearch used, as ref_hybrid_run
    wrote them: the base orders, the category and time-bucket subgraphs
    (key, start, count, Graph::save bytes; buckets in the reference's
    visiting order) and the category size extremes."""
    o = np.fromfile(os.path.join(out_dir, "orders.bin"), dtype=np.uint32).reshape(3, n)
    cats, bks, maxc, minc = [], [], 0, 0
    for line in open(os.path.join(out_dir, "maps.txt")):
        f = line.split()
        if f[0] == "c":
            p = os.path.join(out_dir, f"c{f[1]}.hnsw")
            if os.path.exists(p):  # categories without a graph have no file
                cats.append((int(f[1]), int(f[2]), int(f[3]), open(p, "rb").read()))
        elif f[0] == "t":
            bks.append((int(f[1]), int(f[2]), int(f[3]), open(os.path.join(out_dir, f"t{f[1]}.hnsw"), "rb").read()))
        elif f[0] == "m":
            maxc, minc = int(f[2]), int(f[3])
    return {"sorted_base_ids": o[0], "sorted_base_ids_by_time": o[1], "sorted_base_ids_by_full_time": o[2],
            "categories": cats, "buckets": bks, "maxc_size": maxc, "minc_size": minc}
