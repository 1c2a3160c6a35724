"""fknn_rerank against the oracle: exact FP32 distances with the reference
arithmetic (oracle_normal_l2 pinned to distance.h:62-72), repeats dropped,
ascending (distance, id), padding when fewer than k distinct ids."""
import ctypes

import numpy as np
import pytest

import fknn
import oracle
from fknn import datagen

pytestmark = pytest.mark.gpu


def _expected(vecs, q, cand, k):
    L = oracle.lib()
    ids = np.full((q.shape[0], k), 0xFFFFFFFF, np.uint32)
    d = np.full((q.shape[0], k), np.inf, np.float32)
    for i in range(q.shape[0]):
        u = sorted(set(int(c) for c in cand[i] if c != 0xFFFFFFFF))
        qi = np.ascontiguousarray(q[i])
        sc = sorted((L.oracle_normal_l2(vecs[c].ctypes.data, qi.ctypes.data, 100), c) for c in u)[:k]
        for j, (dd, c) in enumerate(sc):
            ids[i, j], d[i, j] = c, dd
    return ids, d


@pytest.mark.parametrize("nc,k", [(150, 100), (300, 100), (2048, 128), (40, 40)])
def test_rerank_matches_oracle(nc, k):
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=20000, nq=48)
    rng = np.random.default_rng(nc)
    cand = rng.integers(0, vecs.shape[0], size=(q.shape[0], nc)).astype(np.uint32)
    cand[:, 1::7] = cand[:, 0:1]                       # repeats
    cand[::5, -3:] = 0xFFFFFFFF                        # empty slots
    if nc == 40:
        cand[3, :] = cand[3, 0]                        # one distinct id: padding
    with fknn.Index(vecs, labels, ts) as idx:
        ids, d = idx.rerank(q, cand, k=k)
    eids, ed = _expected(vecs, q, cand, k)
    np.testing.assert_array_equal(ids, eids)
    np.testing.assert_array_equal(d, ed)


def test_rerank_rejects_foreign_ids():
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=5000, nq=4)
    cand = np.zeros((4, 10), np.uint32)
    cand[2, 5] = 5000  # not a row
    with fknn.Index(vecs, labels, ts) as idx:
        with pytest.raises(fknn.FknnError):
            idx.rerank(q, cand, k=5)
        ids, _ = idx.rerank(q, np.zeros((4, 10), np.uint32), k=5)  # still usable
        assert (ids[:, 0] == 0).all() and (ids[:, 1:] == 0xFFFFFFFF).all()
