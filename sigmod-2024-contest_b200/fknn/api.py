"""Host-side mirror of the reference's filtered-kNN entry points over the C ABI.

Reference interfaces mirrored (paths inside KevinZeng08/sigmod-2024-contest):
  Bruteforce(nodes, queries, gt)                      utils.h:80-158
  bruteforce(dim, k, closest_points, npoints, ...)    bruteforce.h:244-265
  bruteforce_subgraph(..., distances, ...)            bruteforce.h:267-289
  SQ8SymmetricQuantizer.train / encode                pyglass/glass/quant/sq8_sym_quant.hpp:32-74
  GraphSearcher: Graph::load + Searcher::SetData and the six Search* forms
                                                      pyglass/glass/graph.hpp:117-137,
                                                      pyglass/glass/searcher.hpp:94-101,162-569
plus the resident-index form (Index) that the batch path uses, and the
request loop (Server) that serves a stream of queries with continuous
batching (no reference counterpart: the reference is batch-only).

Arrays may be numpy (host) or torch tensors (host or CUDA); torch CUDA tensors
are passed to the library as device pointers and stay on the device.
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_float, c_uint32, c_uint64, c_void_p
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import (MODE_BF16_RERANK, MODE_EXACT_FP32, MODE_FP8_RERANK, SEARCH_GRAPH, IndexOpts, SearchOpts, SearchStats,
                   ServerOpts, ServerStats, Tuning, check, load)

DIM = 100
K = 100  # utils.h:88
SQ8_CODE = 112  # code_size = d aligned to 16 (sq8_sym_quant.hpp:27)


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(x, dtype) -> int:
    """Address of a contiguous array of the given numpy dtype (numpy or torch)."""
    if x is None:
        return None
    if _is_torch(x):
        import torch
        tdt = {np.float32: torch.float32, np.uint32: torch.int32, np.int32: torch.int32, np.int8: torch.int8,
               np.float64: torch.float64}[np.dtype(dtype).type]
        if x.dtype != tdt and not (tdt == torch.int32 and x.dtype == torch.uint32):
            raise TypeError(f"expected a {tdt} tensor, got {x.dtype}")
        if not x.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return x.data_ptr()
    if not isinstance(x, np.ndarray) or x.dtype != np.dtype(dtype) or not x.flags.c_contiguous:
        raise TypeError(f"expected a C-contiguous numpy array of {np.dtype(dtype)}")
    return x.ctypes.data


def _stream_of(*xs) -> Optional[int]:
    for x in xs:
        if x is not None and _is_torch(x) and x.is_cuda:
            import torch
            return torch.cuda.current_stream(x.device).cuda_stream
    return None


class Index:
    """Resident filtered-kNN index on one GPU (fknn_index_create).

    vecs: (n, 100) float32, labels: (n,) float32 category (read as int32),
    ts: (n,) float32 timestamp.  Row position is the id.
    """

    def __init__(self, vecs, labels, ts, device: int = 0, build_bf16: bool = False, build_fp8: bool = False,
                 hbm_budget: int = 0):
        lib = load()
        vecs = np.ascontiguousarray(vecs, dtype=np.float32)
        labels = np.ascontiguousarray(labels, dtype=np.float32)
        ts = np.ascontiguousarray(ts, dtype=np.float32)
        n = labels.shape[0]
        if vecs.shape != (n, DIM) or ts.shape != (n,):
            raise ValueError("vecs must be (n, 100), labels and ts (n,)")
        opts = IndexOpts(device, int(build_bf16), int(build_fp8), hbm_budget)
        h = c_void_p()
        check(lib.fknn_index_create(vecs.ctypes.data, labels.ctypes.data, ts.ctypes.data, n, DIM, byref(opts),
                                    byref(h)))
        self._h = h
        self.n = n
        self.device = device

    @classmethod
    def from_file(cls, path: str, device: int = 0, build_bf16: bool = False, build_fp8: bool = False,
                  hbm_budget: int = 0) -> "Index":
        """fknn_index_create_from_file: a resident index straight from a
        contest base file (rows streamed to the device and split there)."""
        lib = load()
        opts = IndexOpts(device, int(build_bf16), int(build_fp8), hbm_budget)
        h = c_void_p()
        check(lib.fknn_index_create_from_file(path.encode(), byref(opts), byref(h)))
        self = cls.__new__(cls)
        self._h = h
        self.device = device
        nb = c_uint64()
        check(lib.fknn_read_base_file(path.encode(), byref(nb), None, None, None))
        self.n = nb.value
        return self

    def close(self) -> None:
        if getattr(self, "_h", None):
            load().fknn_index_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def device_bytes(self) -> int:
        b = c_uint64()
        check(load().fknn_index_bytes(self._h, byref(b)))
        return b.value

    def search(self, qvecs, metas, k: int = K, mode: int = MODE_EXACT_FP32, ids=None, dists=None,
               kprime: int = 0, with_dists: bool = True, stream: Optional[int] = None, return_stats: bool = False,
               graph: bool = False):
        """Filtered top-k.  metas rows are (type, v, l, r) as in utils.h:98-101.

        Returns (ids, dists) as numpy arrays for host inputs, or the given /
        newly allocated torch CUDA tensors for device inputs.  graph=True
        (reduced-precision modes) plans on the device and replays a captured
        CUDA graph while nq, k, kprime, the tuning and the buffers repeat.
        """
        lib = load()
        dev = _is_torch(qvecs) and qvecs.is_cuda
        nq = qvecs.shape[0]
        if ids is None:
            if dev:
                import torch
                ids = torch.empty((nq, k), dtype=torch.int32, device=qvecs.device)
                dists = torch.empty((nq, k), dtype=torch.float32, device=qvecs.device) if with_dists else None
            else:
                qvecs = np.ascontiguousarray(qvecs, dtype=np.float32)
                metas = np.ascontiguousarray(metas, dtype=np.float32)
                ids = np.empty((nq, k), dtype=np.uint32)
                dists = np.empty((nq, k), dtype=np.float32) if with_dists else None
        if stream is None:
            stream = _stream_of(qvecs, metas, ids)
        opts = SearchOpts(mode, kprime, SEARCH_GRAPH if graph else 0)
        st = SearchStats()
        check(lib.fknn_search_ex(self._h, _ptr(qvecs, np.float32), _ptr(metas, np.float32), nq, k, byref(opts),
                                 _ptr(ids, np.uint32), _ptr(dists, np.float32) if dists is not None else None,
                                 stream, byref(st)))
        if return_stats:
            return ids, dists, st.as_dict()
        return ids, dists

    def set_tuning(self, mode: int, list_slack: int = 0, items_per_sm: int = 0, min_chunk_blocks: int = 0,
                   bound_refresh: int = 0, pilot_stride: int = None) -> None:
        """fknn_index_set_tuning: plan / kernel parameters of one mode
        (pilot_stride None keeps the current one)."""
        if pilot_stride is None:
            pilot_stride = self.get_tuning(mode)["pilot_stride"]
        check(load().fknn_index_set_tuning(self._h, mode, byref(Tuning(list_slack, items_per_sm, min_chunk_blocks,
                                                                        bound_refresh, pilot_stride))))

    def apply_tuning(self, mode: int, table: Optional[str] = None) -> int:
        """Sets the index to the autotuned entry of this device, base size
        and mode (fknn/autotune.py table), if there is one; returns its k'
        (0 when there is no entry or the mode is exact)."""
        from . import autotune
        e = autotune.lookup(self.n, mode, self.device, table)
        if not e:
            return 0
        t = e["tuning"]
        self.set_tuning(mode, t["list_slack"], t["items_per_sm"], t["min_chunk_blocks"], t["bound_refresh"],
                        t["pilot_stride"])
        return int(e.get("kprime", 0))

    def get_tuning(self, mode: int) -> dict:
        t = Tuning()
        check(load().fknn_index_get_tuning(self._h, mode, byref(t)))
        return t.as_dict()

    def rerank(self, qvecs, cand, k: int = K, with_dists: bool = True, stream: Optional[int] = None):
        """fknn_rerank: the k best of each query's candidate ids (nq, nc)
        by exact FP32 distance, ascending.  Host arrays in, numpy out; torch
        CUDA tensors in, torch CUDA tensors out."""
        dev = _is_torch(qvecs) and qvecs.is_cuda
        nq, nc = cand.shape
        if dev:
            import torch
            ids = torch.empty((nq, k), dtype=torch.int32, device=qvecs.device)
            dists = torch.empty((nq, k), dtype=torch.float32, device=qvecs.device) if with_dists else None
            if stream is None:
                stream = _stream_of(qvecs)
        else:
            qvecs = np.ascontiguousarray(qvecs, dtype=np.float32)
            cand = np.ascontiguousarray(cand).astype(np.uint32, copy=False)
            ids = np.empty((nq, k), dtype=np.uint32)
            dists = np.empty((nq, k), dtype=np.float32) if with_dists else None
        check(load().fknn_rerank(self._h, _ptr(qvecs, np.float32), nq, _ptr(cand, np.uint32), nc, k,
                                 _ptr(ids, np.uint32), _ptr(dists, np.float32) if dists is not None else None,
                                 stream))
        return ids, dists

    def count_matches(self, metas) -> np.ndarray:
        metas = np.ascontiguousarray(metas, dtype=np.float32)
        out = np.empty(metas.shape[0], dtype=np.uint32)
        check(load().fknn_count_matches(self._h, metas.ctypes.data, metas.shape[0], out.ctypes.data, None))
        return out

    def filter_rows_batch(self, metas, out=None, counts=None, stream: Optional[int] = None):
        """fknn_filter_rows_batch: the passing ids of each predicate row of
        metas ((np, 4) host floats), one pass over the columns per 16
        predicates.  out ((np, n) int32) and counts ((np,) int64) are torch
        CUDA tensors (allocated when None); returns them, asynchronously
        written on `stream` (default: torch's current stream)."""
        import torch
        m = np.ascontiguousarray(metas, dtype=np.float32).reshape(-1, 4)
        npred = m.shape[0]
        if out is None:
            out = torch.empty((npred, self.n), dtype=torch.int32, device=f"cuda:{self.device}")
        if counts is None:
            counts = torch.empty(npred, dtype=torch.int64, device=f"cuda:{self.device}")
        if stream is None:
            stream = torch.cuda.current_stream(self.device).cuda_stream
        check(load().fknn_filter_rows_batch(self._h, m.ctypes.data, npred, out.data_ptr(), counts.data_ptr(),
                                            stream))
        return out, counts

    def filter_rows(self, meta4) -> np.ndarray:
        """Ids of the rows passing one predicate (type, v, l, r), increasing."""
        m = np.ascontiguousarray(meta4, dtype=np.float32).reshape(4)
        out = np.empty(self.n, dtype=np.uint32)
        cnt = c_uint64()
        check(load().fknn_filter_rows(self._h, m.ctypes.data, out.ctypes.data, byref(cnt), None))
        return out[: cnt.value].copy()


class Router:
    """fknn_router: HybridGraph::BatchSearch's routing (hybrid_graph.cpp:
    147-503) on the GPU, over the reference's subgraphs and base orders.

    categories / buckets: lists of (key, start, count, Graph::save bytes);
    buckets in the order the reference visits them for type-0 queries."""

    def __init__(self, vecs, labels, ts, sorted_base_ids, sorted_base_ids_by_full_time, categories, buckets,
                 maxc_size: int, minc_size: int, device: int = 0):
        lib = load()
        self._keep = [np.ascontiguousarray(vecs, np.float32), np.ascontiguousarray(labels, np.float32),
                      np.ascontiguousarray(ts, np.float32), np.ascontiguousarray(sorted_base_ids, np.uint32),
                      np.ascontiguousarray(sorted_base_ids_by_full_time, np.uint32)]
        v, l, t, sb, sf = self._keep

        def subs(lst):
            arr = (_lib.RouterSubgraph * max(1, len(lst)))()
            for i, (key, start, count, gb) in enumerate(lst):
                buf = np.frombuffer(bytes(gb), dtype=np.uint8)
                self._keep.append(buf)
                arr[i] = _lib.RouterSubgraph(int(key), int(start), int(count), buf.ctypes.data, buf.size)
            return arr
        ca, ba = subs(categories), subs(buckets)
        d = _lib.RouterDesc(v.ctypes.data, l.ctypes.data, t.ctypes.data, v.shape[0], sb.ctypes.data, sf.ctypes.data,
                            ca, len(categories), ba, len(buckets), int(maxc_size), int(minc_size), device)
        h = c_void_p()
        check(lib.fknn_router_create(byref(d), byref(h)))
        self._h = h
        self._keep = None  # the router holds its own copies

    @staticmethod
    def default_params() -> "_lib.RouterParams":
        p = _lib.RouterParams()
        check(load().fknn_router_default_params(byref(p)))
        return p

    def search(self, qvecs, metas, params=None):
        """ids (nq, 100) uint32 and the per-route statistics."""
        q = np.ascontiguousarray(qvecs, np.float32)
        m = np.ascontiguousarray(metas, np.float32)
        ids = np.empty((q.shape[0], K), np.uint32)
        st = _lib.RouterStats()
        check(load().fknn_router_search(self._h, q.ctypes.data, m.ctypes.data, q.shape[0],
                                        byref(params) if params is not None else None, ids.ctypes.data, byref(st)))
        return ids, st.as_dict()

    def close(self) -> None:
        if getattr(self, "_h", None):
            load().fknn_router_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def read_base_file(path: str):
    """fknn_read_base_file (utils.h:257 ReadBase): (vecs (n,100), labels (n,), ts (n,)) float32."""
    lib = load()
    n = c_uint64()
    check(lib.fknn_read_base_file(path.encode(), byref(n), None, None, None))
    vecs = np.empty((n.value, DIM), np.float32)
    labels = np.empty(n.value, np.float32)
    ts = np.empty(n.value, np.float32)
    check(lib.fknn_read_base_file(path.encode(), byref(n), vecs.ctypes.data, labels.ctypes.data, ts.ctypes.data))
    return vecs, labels, ts


def read_query_file(path: str):
    """fknn_read_query_file (utils.h:550 ReadQuery): (qvecs (nq,100), metas (nq,4)) float32."""
    lib = load()
    nq = c_uint32()
    check(lib.fknn_read_query_file(path.encode(), byref(nq), None, None))
    q = np.empty((nq.value, DIM), np.float32)
    m = np.empty((nq.value, 4), np.float32)
    check(lib.fknn_read_query_file(path.encode(), byref(nq), q.ctypes.data, m.ctypes.data))
    return q, m


def sorted_query_order(metas) -> np.ndarray:
    """fknn_sorted_query_order: the query order of ReadSortedQuery (utils.h:513-533)."""
    m = np.ascontiguousarray(metas, dtype=np.float32).reshape(-1, 4)
    out = np.empty(m.shape[0], np.uint32)
    check(load().fknn_sorted_query_order(m.ctypes.data, m.shape[0], out.ctypes.data))
    return out


def save_knn(path: str, ids) -> None:
    """fknn_save_knn (io.h:22 SaveKNN): nq x k uint32, no header."""
    a = np.ascontiguousarray(ids, dtype=np.uint32)
    check(load().fknn_save_knn(path.encode(), a.ctypes.data, a.shape[0], a.shape[1]))


def read_groundtruth(path: str, k: int = K) -> np.ndarray:
    """fknn_read_groundtruth (utils.h:194 ReadGroundTruth): (nq, k) uint32."""
    lib = load()
    nq = c_uint32()
    check(lib.fknn_read_groundtruth(path.encode(), k, byref(nq), None))
    out = np.empty((nq.value, k), np.uint32)
    check(lib.fknn_read_groundtruth(path.encode(), k, byref(nq), out.ctypes.data))
    return out


def Bruteforce(nodes, queries, gt: Optional[list] = None):
    """utils.h:80 Bruteforce: nodes rows (label, ts, 100 dims), queries rows
    (type, v, l, r, 100 dims) -> gt[nq][100] ascending (distance, id).

    Unlike the reference, queries with fewer than 100 passing rows do not
    throw; their tail is UINT32_MAX.  Returns gt (filled in place when a list
    is given).
    """
    nodes_a = np.ascontiguousarray(np.asarray(nodes, dtype=np.float32))
    q_a = np.ascontiguousarray(np.asarray(queries, dtype=np.float32))
    if nodes_a.ndim != 2 or nodes_a.shape[1] != DIM + 2 or q_a.ndim != 2 or q_a.shape[1] != DIM + 4:
        raise ValueError("nodes must be (n, 102) and queries (nq, 104)")
    out = np.empty((q_a.shape[0], K), dtype=np.uint32)
    check(load().fknn_bruteforce_rows(nodes_a.ctypes.data, nodes_a.shape[0], q_a.ctypes.data, q_a.shape[0],
                                      out.ctypes.data))
    if gt is not None:
        gt.clear()
        gt.extend(list(map(int, r)) for r in out)
        return gt
    return out


class SQ8SymmetricQuantizer:
    """sq8_sym_quant.hpp: one global scale alpha = max|x|, int8 codes of 112 bytes."""

    def __init__(self, dim: int = DIM):
        if dim != DIM:
            raise ValueError("dim must be 100")
        self.d = dim
        self.code_size = SQ8_CODE
        self.alpha = 0.0
        self.codes: Optional[np.ndarray] = None

    def train(self, data, n: Optional[int] = None) -> None:
        data = np.ascontiguousarray(data, dtype=np.float32).reshape(-1, DIM)
        if n is not None:
            data = data[:n]
        codes = np.empty((data.shape[0], SQ8_CODE), dtype=np.int8)
        a = c_float()
        check(load().fknn_sq8_sym_train(data.ctypes.data, data.shape[0], byref(a), codes.ctypes.data))
        self.alpha = a.value
        self.codes = codes

    def encode(self, vecs) -> np.ndarray:
        v = np.ascontiguousarray(vecs, dtype=np.float32).reshape(-1, DIM)
        out = np.empty((v.shape[0], SQ8_CODE), dtype=np.int8)
        check(load().fknn_sq8_sym_encode(v.ctypes.data, v.shape[0], c_float(self.alpha), out.ctypes.data))
        return out


def bruteforce(dim: int, k: int, closest_points, npoints: int, codes_in, alpha: float, nqueries: int,
               queries_in) -> None:
    """bruteforce.h:244 with the same arguments; closest_points (nqueries*k
    int32) is filled in the reference's heap-array order."""
    check(load().fknn_sq8_bruteforce(dim, k, _ptr(closest_points, np.int32), npoints, _ptr(codes_in, np.int8),
                                     c_float(alpha), nqueries, _ptr(queries_in, np.int8)))


def bruteforce_subgraph(dim: int, k: int, closest_points, distances, npoints: int, codes_in, alpha: float,
                        nqueries: int, queries_in) -> None:
    """bruteforce.h:267: also distances[k] = heap distance * alpha * alpha."""
    check(load().fknn_sq8_bruteforce_subgraph(dim, k, _ptr(closest_points, np.int32), _ptr(distances, np.float32),
                                              npoints, _ptr(codes_in, np.int8), c_float(alpha), nqueries,
                                              _ptr(queries_in, np.int8)))


class GraphSearcher:
    """The pyglass Searcher over one saved graph (Graph::save bytes), batched.

    Method names and arguments follow searcher.hpp; each takes a batch of
    queries (nq x 100) and returns ids (nq x refine, int32) -- and distances
    for the *SubTime forms -- equal to the reference's on the same graph.
    ``k`` is the reference's pool argument (capacity max(k, ef)).
    """

    def __init__(self, graph_bytes, data, device: int = 0):
        lib = load()
        gb = np.frombuffer(bytes(graph_bytes), dtype=np.uint8) if not isinstance(graph_bytes, np.ndarray) \
            else np.ascontiguousarray(graph_bytes, dtype=np.uint8)
        if _is_torch(data) and data.is_cuda:
            d = data
        else:
            d = np.ascontiguousarray(data, dtype=np.float32).reshape(-1, DIM)
        h = c_void_p()
        check(lib.fknn_graph_create(gb.ctypes.data, gb.size, _ptr(d, np.float32), device, byref(h)))
        self._h = h
        self.ef = 32
        n, deg, a = c_uint32(), c_uint32(), c_float()
        check(lib.fknn_graph_info(self._h, byref(n), byref(deg), byref(a)))
        self.nb, self.degree, self.alpha = n.value, deg.value, a.value

    @classmethod
    def load(cls, path: str, data, device: int = 0) -> "GraphSearcher":
        with open(path, "rb") as f:
            return cls(f.read(), data, device)

    def close(self) -> None:
        if getattr(self, "_h", None):
            load().fknn_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def SetEf(self, ef: int) -> None:
        self.ef = int(ef)

    def _run(self, mode, q, k, refine, bounds=None, id_bounds=None, with_dists=False, stream=None):
        lib = load()
        dev = _is_torch(q) and q.is_cuda
        if dev:
            import torch
            nq = q.shape[0]
            ids = torch.empty((nq, refine), dtype=torch.int32, device=q.device)
            dists = torch.empty((nq, refine), dtype=torch.float32, device=q.device) if with_dists else None
            if stream is None:
                stream = _stream_of(q)
        else:
            q = np.ascontiguousarray(q, dtype=np.float32).reshape(-1, DIM)
            nq = q.shape[0]
            ids = np.empty((nq, refine), dtype=np.int32)
            dists = np.empty((nq, refine), dtype=np.float32) if with_dists else None
        if bounds is not None and not _is_torch(bounds):
            bounds = np.ascontiguousarray(bounds, dtype=np.float32).reshape(nq, 2)
        if id_bounds is not None and not _is_torch(id_bounds):
            id_bounds = np.ascontiguousarray(id_bounds, dtype=np.int32).reshape(nq, 2)
        check(lib.fknn_graph_search(self._h, _ptr(q, np.float32), nq, mode, k, self.ef, refine,
                                    _ptr(bounds, np.float32), _ptr(id_bounds, np.int32), _ptr(ids, np.int32),
                                    _ptr(dists, np.float32) if dists is not None else None, stream))
        return (ids, dists) if with_dists else ids

    def Search(self, q, k: int):
        """searcher.hpp:162: k ids per query."""
        return self._run(_lib.GRAPH_SEARCH, q, k, k)

    def SearchFilter(self, q, k: int, refine: int):
        """searcher.hpp:262 (the filter argument is unused by the reference)."""
        return self._run(_lib.GRAPH_FILTER, q, k, refine)

    def SearchFilterSubTime(self, q, k: int, refine: int):
        """searcher.hpp:377: (ids, dists)."""
        return self._run(_lib.GRAPH_FILTER_SUBTIME, q, k, refine, with_dists=True)

    def SearchCategoryRange(self, q, k: int, refine: int, query_bound, id_bound):
        """searcher.hpp:301: per query (l, r) and (s_id, e_id)."""
        return self._run(_lib.GRAPH_CATEGORY_RANGE, q, k, refine, query_bound, id_bound)

    def SearchRangeFilterSubTime(self, q, k: int, refine: int, query_bound, id_bound):
        """searcher.hpp:415: (ids, dists)."""
        return self._run(_lib.GRAPH_RANGE_SUBTIME, q, k, refine, query_bound, id_bound, with_dists=True)

    def SearchRangeFilter(self, q, k: int, refine: int, query_bound, id_bound):
        """searcher.hpp:493."""
        return self._run(_lib.GRAPH_RANGE, q, k, refine, query_bound, id_bound)


class Server:
    """Continuous-batching request loop over a resident Index (fknn_server_*).

    submit() enqueues one request per query row and returns at once; the
    results land in the arrays it returns, which stay owned by this object
    until wait()/drain() report them complete."""

    def __init__(self, index: "Index", mode: int = MODE_EXACT_FP32, kprime: int = 0, k: int = K,
                 max_batch: int = 4096, slots: int = 3, max_wait_us: int = 0, hbm_budget: int = 0):
        lib = load()
        self.k = k
        self._index = index  # keep the index alive
        o = ServerOpts(mode, kprime, k, max_batch, slots, max_wait_us, hbm_budget)
        h = c_void_p()
        check(lib.fknn_server_create(index._h, byref(o), byref(h)))
        self._h = h
        self._keep = []  # output arrays of requests in flight

    @staticmethod
    def now_ns() -> int:
        return load().fknn_server_now_ns()

    def submit(self, qvecs, metas, arrival_ns=None, with_dists: bool = True, ids=None, dists=None):
        """Returns (first_ticket, ids (n,k) uint32, dists (n,k) float32 or None)."""
        q = np.ascontiguousarray(qvecs, dtype=np.float32).reshape(-1, DIM)
        m = np.ascontiguousarray(metas, dtype=np.float32).reshape(-1, 4)
        n = q.shape[0]
        if ids is None:
            ids = np.empty((n, self.k), dtype=np.uint32)
        if dists is None and with_dists:
            dists = np.empty((n, self.k), dtype=np.float32)
        arr = None if arrival_ns is None else np.ascontiguousarray(arrival_ns, dtype=np.int64)
        t = c_uint64()
        check(load().fknn_server_submit(self._h, q.ctypes.data, m.ctypes.data, n,
                                        arr.ctypes.data if arr is not None else None, ids.ctypes.data,
                                        dists.ctypes.data if dists is not None else None, byref(t)))
        self._keep.append((ids, dists))
        return t.value, ids, dists

    def wait(self, ticket: int, timeout_ms: int = -1) -> None:
        check(load().fknn_server_wait(self._h, ticket, timeout_ms))

    def drain(self, timeout_ms: int = -1) -> None:
        check(load().fknn_server_drain(self._h, timeout_ms))
        self._keep = []

    def stats(self, reset: bool = False) -> dict:
        st = ServerStats()
        check(load().fknn_server_get_stats(self._h, byref(st), int(reset)))
        return st.as_dict()

    def close(self) -> None:
        if getattr(self, "_h", None):
            load().fknn_server_destroy(self._h)
            self._h = None
            self._keep = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
