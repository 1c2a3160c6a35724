"""Graph fixtures for the graph-search tests: the golden fixture's inputs
and Graph::save byte layouts (pyglass/glass/graph.hpp:101-115,
hnsw/HNSWInitializer.hpp:73-82) of seeded random graphs.  Test
infrastructure only."""
from __future__ import annotations

import numpy as np

from fknn import datagen

# (mode, k, refine) of the golden fixture's reference calls
GRAPH_CASES = [(0, 32, 32), (0, 100, 100), (1, 64, 40), (1, 300, 150), (2, 64, 40), (2, 300, 150), (3, 64, 40),
               (3, 300, 150), (4, 64, 40), (4, 300, 150), (5, 64, 40), (5, 300, 150)]


def id_bounds_for(ts_sorted, bounds):
    """[first, last) positions of each window in timestamp-sorted points,
    the first clamped to a point (as the callers' lower_bound results are)."""
    ib = np.stack([np.searchsorted(ts_sorted, bounds[:, 0], "left"),
                   np.searchsorted(ts_sorted, bounds[:, 1], "right")], 1)
    ib[:, 0] = np.minimum(ib[:, 0], len(ts_sorted) - 1)
    return ib.astype(np.int32)


def windows(nq, seed, lo_max=0.9, log_w=(-3, 0)):
    rng = np.random.default_rng(seed)
    lo = rng.uniform(0, lo_max, nq).astype(np.float32)
    w = (10 ** rng.uniform(log_w[0], log_w[1], nq)).astype(np.float32)
    return np.stack([lo, lo + w], 1).astype(np.float32)


def graph_inputs():
    """Inputs of graph_hnsw.npz: config-1 data in timestamp order (a
    time-sorted sub-index), queries, windows and the id ranges they cover."""
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=2000, nq=48)
    order = np.argsort(ts, kind="stable")
    vecs, labels, ts = vecs[order], labels[order], ts[order]
    bounds = windows(q.shape[0], 2024)
    return vecs, labels, ts, q, bounds, id_bounds_for(ts, bounds)


def save_bytes(adj, ets, eps=(), up_lists=None, upK=0, ep=-1) -> bytes:
    """Graph::save layout; up_lists[i] is node i's levels * upK ids."""
    n, K = adj.shape
    parts = [np.int32(len(eps)).tobytes(), np.asarray(eps, dtype=np.int32).tobytes(),
             np.array([n, K], dtype=np.int32).tobytes(), np.ascontiguousarray(adj, dtype=np.int32).tobytes(),
             np.ascontiguousarray(ets, dtype=np.float32).tobytes()]
    if up_lists is not None:
        parts.append(np.array([n, upK, ep], dtype=np.int32).tobytes())
        for lst in up_lists:
            lst = np.asarray(lst, dtype=np.int32)
            parts.append(np.int32(lst.size).tobytes())
            parts.append(lst.tobytes())
    return b"".join(parts)


def random_graph(n, K, ts, seed, with_layers=True, dup_frac=0.02, pad_frac=0.2):
    """A seeded random graph: each list a random prefix of random ids (some
    repeated), -1 padded; edge timestamps are the neighbours' timestamps
    (as HNSW::Build stores them); optional random upper layers."""
    rng = np.random.default_rng(seed)
    adj = rng.integers(0, n, size=(n, K), dtype=np.int64).astype(np.int32)
    dup = rng.random((n, K)) < dup_frac
    adj[:, 1:][dup[:, 1:]] = adj[:, :-1][dup[:, 1:]]
    lens = np.where(rng.random(n) < pad_frac, rng.integers(1, K + 1, n), K)
    adj[np.arange(K)[None, :] >= lens[:, None]] = -1
    ets = np.where(adj >= 0, ts[np.maximum(adj, 0)], 0.0).astype(np.float32)
    if not with_layers:
        eps = rng.choice(n, size=min(8, n), replace=False).astype(np.int32)
        return save_bytes(adj, ets, eps=eps)
    upK = 16
    lvl = np.minimum(rng.geometric(0.9, n) - 1, 3)  # mostly 0, a few 1..3
    ep = int(np.argmax(lvl))
    lists = []
    for i in range(n):
        L = int(lvl[i])
        cand = np.nonzero(lvl >= 1)[0]
        lst = []
        for level in range(1, L + 1):
            pool = np.nonzero(lvl >= level)[0]
            m = int(rng.integers(1, upK + 1))
            ids = rng.choice(pool, size=min(m, len(pool)), replace=False).astype(np.int32)
            row = np.full(upK, -1, np.int32)
            row[:len(ids)] = ids
            lst.append(row)
        lists.append(np.concatenate(lst) if lst else np.zeros(0, np.int32))
    return save_bytes(adj, ets, up_lists=lists, upK=upK, ep=ep)
