"""Seeded synthetic workloads with the contest's shapes, and the contest
binary formats.

The contest data files are not used; these generators stand in for them with
the distributions the workloads are specified by:
  base rows   : 100-d float32 from a mixture of 256 Gaussian clusters
                (centres N(0,1), per-row noise N(0, 0.3^2)); an int32 category
                from a truncated Zipf; a float32 timestamp ~ U[0,1].
  queries     : vectors from the same mixture; type 0..3; v from the same Zipf
                (types 1/3, else -1); a window [l, r] (types 2/3, else -1).

File formats (utils.h:257-276, io.h:22-62):
  base   : u32 N, then N x [label f32, ts f32, 100 x f32]
  queries: u32 Q, then Q x [type, v, l, r, 100 x f32]
  knn    : Q x 100 u32, no header (io.h:22-33)
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Tuple

import numpy as np

DIM = 100
N_CENTRES = 256
SIGMA = 0.3


@dataclass(frozen=True)
class Workload:
    name: str
    n: int
    nq: int
    zipf_s: float
    n_labels: int
    window: str  # "uniform" (width U[0.05,0.5]) or "loguniform" (width log-U[1e-4,1])
    balanced_types: bool  # exactly 25% per type instead of i.i.d. uniform


# The five configurations of the task, in order.
WORKLOADS = {
    1: Workload("plain-exact-n1e5-q1e4", 100_000, 10_000, 1.1, 1000, "uniform", False),
    2: Workload("exact-fp32-n1e6-q1e5", 1_000_000, 100_000, 1.1, 1000, "uniform", False),
    3: Workload("precision-n1e7-q1e6", 10_000_000, 1_000_000, 1.1, 1000, "uniform", False),
    4: Workload("uneven-selectivity-n1e7-q1e6", 10_000_000, 1_000_000, 1.5, 10_000, "loguniform", True),
    5: Workload("serving-n1e7", 10_000_000, 1_000_000, 1.5, 10_000, "loguniform", True),
}


def _zipf(rng: np.random.Generator, s: float, nmax: int, size: int) -> np.ndarray:
    """Zipf(s) truncated to 1..nmax by rejection, returned as 0..nmax-1."""
    out = rng.zipf(s, size=size)
    bad = out > nmax
    while bad.any():
        out[bad] = rng.zipf(s, size=int(bad.sum()))
        bad = out > nmax
    return (out - 1).astype(np.int64)


def centres(seed: int) -> np.ndarray:
    return np.random.default_rng(seed).standard_normal((N_CENTRES, DIM), dtype=np.float32)


def make_base(n: int, zipf_s: float, n_labels: int, seed: int, chunk: int = 1 << 20
              ) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Returns (vecs (n,100) f32, labels (n,) f32, ts (n,) f32)."""
    rng = np.random.default_rng(seed)
    C = centres(seed)
    vecs = np.empty((n, DIM), dtype=np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        c = rng.integers(0, N_CENTRES, size=e - s)
        noise = rng.standard_normal((e - s, DIM), dtype=np.float32)
        noise *= np.float32(SIGMA)
        noise += C[c]
        vecs[s:e] = noise
    labels = _zipf(rng, zipf_s, n_labels, n).astype(np.float32)
    ts = rng.random(n, dtype=np.float32)
    return vecs, labels, ts


def make_queries(nq: int, zipf_s: float, n_labels: int, window: str, balanced_types: bool, base_seed: int,
                 seed: int) -> Tuple[np.ndarray, np.ndarray]:
    """Returns (qvecs (nq,100) f32, metas (nq,4) f32 = type, v, l, r)."""
    rng = np.random.default_rng(seed)
    C = centres(base_seed)
    c = rng.integers(0, N_CENTRES, size=nq)
    q = rng.standard_normal((nq, DIM), dtype=np.float32)
    q *= np.float32(SIGMA)
    q += C[c]
    if balanced_types:
        types = np.arange(nq) % 4
        rng.shuffle(types)
    else:
        types = rng.integers(0, 4, size=nq)
    v = _zipf(rng, zipf_s, n_labels, nq).astype(np.float32)
    if window == "uniform":
        w = rng.uniform(0.05, 0.5, size=nq)
    else:
        w = np.exp(rng.uniform(np.log(1e-4), 0.0, size=nq))
    l = rng.random(nq) * (1.0 - w)
    r = l + w
    metas = np.empty((nq, 4), dtype=np.float32)
    metas[:, 0] = types
    metas[:, 1] = np.where((types == 1) | (types == 3), v, -1.0)
    metas[:, 2] = np.where(types >= 2, l, -1.0)
    metas[:, 3] = np.where(types >= 2, r, -1.0)
    return q, metas


def make_workload(cfg: int, n: int | None = None, nq: int | None = None):
    """Base and queries of configuration cfg (1..5), optionally resized.

    Seeds: base 1234 + cfg, queries 1235 + cfg.
    """
    w = WORKLOADS[cfg]
    n = w.n if n is None else n
    nq = w.nq if nq is None else nq
    bseed = 1234 + cfg
    vecs, labels, ts = make_base(n, w.zipf_s, w.n_labels, bseed)
    q, metas = make_queries(nq, w.zipf_s, w.n_labels, w.window, w.balanced_types, bseed, 1235 + cfg)
    return vecs, labels, ts, q, metas


# ---- contest binary formats ----

def to_rows(vecs: np.ndarray, labels: np.ndarray, ts: np.ndarray) -> np.ndarray:
    rows = np.empty((vecs.shape[0], DIM + 2), dtype=np.float32)
    rows[:, 0] = labels
    rows[:, 1] = ts
    rows[:, 2:] = vecs
    return rows


def to_query_rows(q: np.ndarray, metas: np.ndarray) -> np.ndarray:
    rows = np.empty((q.shape[0], DIM + 4), dtype=np.float32)
    rows[:, :4] = metas
    rows[:, 4:] = q
    return rows


def write_base(path: str, vecs, labels, ts) -> None:
    with open(path, "wb") as f:
        np.array([vecs.shape[0]], dtype=np.uint32).tofile(f)
        to_rows(vecs, labels, ts).tofile(f)


def read_base(path: str):
    """utils.h:257 ReadBase: returns (vecs, labels, ts)."""
    with open(path, "rb") as f:
        n = int(np.fromfile(f, dtype=np.uint32, count=1)[0])
        rows = np.fromfile(f, dtype=np.float32, count=n * (DIM + 2)).reshape(n, DIM + 2)
    return np.ascontiguousarray(rows[:, 2:]), rows[:, 0].copy(), rows[:, 1].copy()


def write_queries(path: str, q, metas) -> None:
    with open(path, "wb") as f:
        np.array([q.shape[0]], dtype=np.uint32).tofile(f)
        to_query_rows(q, metas).tofile(f)


def read_queries(path: str):
    """utils.h:550 ReadQuery: returns (qvecs, metas)."""
    with open(path, "rb") as f:
        nq = int(np.fromfile(f, dtype=np.uint32, count=1)[0])
        rows = np.fromfile(f, dtype=np.float32, count=nq * (DIM + 4)).reshape(nq, DIM + 4)
    return np.ascontiguousarray(rows[:, 4:]), np.ascontiguousarray(rows[:, :4])


def save_knn(path: str, knn: np.ndarray) -> None:
    """io.h:22 SaveKNN: Q x 100 u32, no header."""
    np.ascontiguousarray(knn, dtype=np.uint32).tofile(path)


def read_groundtruth(path: str, k: int = 100) -> np.ndarray:
    """utils.h:194 ReadGroundTruth: u32 N header, then N x k u32."""
    with open(path, "rb") as f:
        n = int(np.fromfile(f, dtype=np.uint32, count=1)[0])
        return np.fromfile(f, dtype=np.uint32, count=n * k).reshape(n, k)


def recall_at_k(knn: np.ndarray, gt: np.ndarray) -> float:
    """utils.h:224 GetKNNRecall: set recall over the k columns (padding ids
    UINT32_MAX count as matches only against padding)."""
    nq, k = gt.shape
    hits = 0
    for i in range(nq):
        hits += len(np.intersect1d(knn[i], gt[i], assume_unique=False))
    return hits / (nq * k)


def recall_matrix(knn: np.ndarray, gt: np.ndarray, pad: int = 0xFFFFFFFF) -> float:
    """Mean per-query recall of knn against gt (both (nq, k) uint32), padding
    ids excluded; queries whose gt holds no valid id are skipped."""
    knn = np.asarray(knn, dtype=np.uint64)
    gt = np.asarray(gt, dtype=np.uint64)
    nq, k = gt.shape
    rows = np.arange(nq, dtype=np.uint64)[:, None] << np.uint64(32)
    gv = gt != pad
    a = (knn + rows)[knn != pad]
    b = (gt + rows)[gv]
    hit = np.zeros(gt.shape, dtype=bool)
    hit[gv] = np.isin(b, a)
    nvalid = gv.sum(axis=1)
    m = nvalid > 0
    if not m.any():
        return 1.0
    return float(np.mean(hit.sum(axis=1)[m] / nvalid[m]))
