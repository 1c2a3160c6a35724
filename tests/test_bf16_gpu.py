"""BF16 tensor-core screen + FP32 re-rank + FP64 boundary (FKNN_MODE_BF16_RERANK)
on the GPU: recall@100 against the FP64 oracle (bar: >= 0.99 at every k'),
returned distances equal to the reference FP32 distance of each returned id
(bit for bit), and argument checks."""
import numpy as np
import pytest

import fknn
import oracle
from fknn import datagen

pytestmark = pytest.mark.gpu
UMAX = 0xFFFFFFFF


@pytest.fixture(scope="module")
def c1():
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=80000, nq=600)
    idx = fknn.Index(vecs, labels, ts, build_bf16=True)
    o64, d64 = oracle.exact_knn(vecs, labels, ts, q, metas, f64=True)
    yield vecs, labels, ts, q, metas, idx, o64, d64
    idx.close()


@pytest.mark.parametrize("kprime", [100, 200, 400, 800, 1024])
def test_recall_vs_fp64_oracle(c1, kprime):
    vecs, labels, ts, q, metas, idx, o64, _ = c1
    ids, dists, st = idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=kprime, return_stats=True)
    r = datagen.recall_matrix(ids, o64)
    assert r >= 0.99, (kprime, r, st)
    # padding only where fewer than 100 rows pass
    counts = oracle.count_matches(labels, ts, metas)
    for i in np.nonzero(counts < 100)[0]:
        assert np.all(ids[i, counts[i]:] == UMAX)


def test_distances_are_reference_fp32(c1):
    vecs, labels, ts, q, metas, idx, _, _ = c1
    ids, dists = idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=400)
    L = oracle.lib()
    rng = np.random.default_rng(2)
    for i in rng.choice(q.shape[0], 80, replace=False):
        qq = np.ascontiguousarray(q[i])
        for j in range(100):
            if ids[i, j] == UMAX:
                assert np.isinf(dists[i, j])
                continue
            x = np.ascontiguousarray(vecs[ids[i, j]])
            ref = np.float32(L.oracle_normal_l2(x.ctypes.data, qq.ctypes.data, 100))
            assert ref.view(np.uint32) == dists[i, j].view(np.uint32)


def test_same_ids_as_exact_when_recall_is_full(c1):
    vecs, labels, ts, q, metas, idx, o64, _ = c1
    ids, _ = idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=800)
    eids, _ = idx.search(q, metas)
    same_set = [set(a) == set(b) for a, b in zip(ids, eids)]
    assert np.mean(same_set) >= 0.99


def test_uneven_selectivity_workload():
    vecs, labels, ts, q, metas = datagen.make_workload(4, n=120000, nq=500)
    with fknn.Index(vecs, labels, ts, build_bf16=True) as idx:
        ids, _ = idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=200)
    o64, _ = oracle.exact_knn(vecs, labels, ts, q, metas, f64=True)
    assert datagen.recall_matrix(ids, o64) >= 0.99


def test_argument_checks():
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=5000, nq=8)
    with fknn.Index(vecs, labels, ts) as idx:
        with pytest.raises(fknn.FknnError) as e:
            idx.search(q, metas, mode=fknn.MODE_BF16_RERANK)
        assert e.value.code == fknn.FKNN_EUNSUPPORTED
    with fknn.Index(vecs, labels, ts, build_bf16=True) as idx:
        for kp in (50, 1025):
            with pytest.raises(fknn.FknnError) as e:
                idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=kp)
            assert e.value.code == fknn.FKNN_EINVAL
        ids, _ = idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=100)
        assert ids.shape == (8, 100)
