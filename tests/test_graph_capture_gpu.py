"""The reduced-precision search planned on the device and replayed as a
captured CUDA graph (fknn_search_opts.flags = FKNN_SEARCH_GRAPH): recall
against the FP64 oracle, agreement with the host-planned search, returned
distances equal to the reference FP32 distance of each id, replay of the
cached graph, a new capture when the shape changes, and the bounded-wait
failure path through the graph."""
import ctypes
import time

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
    idx = fknn.Index(vecs, labels, ts, build_bf16=True, build_fp8=True)
    o64, _ = oracle.exact_knn(vecs, labels, ts, q, metas, f64=True)
    yield vecs, labels, ts, q, metas, idx, o64
    idx.close()


@pytest.mark.parametrize("kprime", [100, 400, 1024])
def test_recall_and_agreement_with_host_plan(c1, kprime):
    vecs, labels, ts, q, metas, idx, o64 = c1
    gids, gd, gst = idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=kprime, graph=True, return_stats=True)
    hids, hd, hst = idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=kprime, return_stats=True)
    assert datagen.recall_matrix(gids, o64) >= 0.99
    # equal-screening-distance candidates may arrive in another order
    assert np.mean(np.all(gids == hids, axis=1)) >= 0.99
    assert gst["n_small"] == hst["n_small"]
    assert gst["pairs_passing"] == hst["pairs_passing"]
    counts = oracle.count_matches(labels, ts, metas)
    for i in np.nonzero(counts < 100)[0]:
        assert np.all(gids[i, counts[i]:] == UMAX)


def test_distances_are_reference_fp32(c1):
    vecs, labels, ts, q, metas, idx, _ = c1
    ids, dists = idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=400, graph=True)
    L = oracle.lib()
    rng = np.random.default_rng(5)
    for i in rng.choice(q.shape[0], 60, replace=False):
        qq = np.ascontiguousarray(q[i])
        for j in range(100):
            if ids[i, j] == UMAX:
                assert np.isinf(dists[i, j])
                continue
            x = np.ascontiguousarray(vecs[ids[i, j]])
            ref = np.float32(L.oracle_normal_l2(x.ctypes.data, qq.ctypes.data, 100))
            assert ref.view(np.uint32) == dists[i, j].view(np.uint32)


def test_replay_and_recapture(c1):
    vecs, labels, ts, q, metas, idx, o64 = c1
    a, ad, sa = idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=200, graph=True, return_stats=True)
    b, bd, sb = idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=200, graph=True, return_stats=True)
    assert sa["kernel_launches"] == sb["kernel_launches"] > 0
    assert np.mean(np.all(a == b, axis=1)) >= 0.99
    # other queries, same shape: the cached graph reads the new inputs
    rng = np.random.default_rng(9)
    perm = rng.permutation(q.shape[0])
    c, _ = idx.search(q[perm], metas[perm], mode=fknn.MODE_BF16_RERANK, kprime=200, graph=True)
    assert np.mean(np.all(c == a[perm], axis=1)) >= 0.99
    # another nq: a new capture
    h = q.shape[0] // 2 + 7
    d, _ = idx.search(q[:h], metas[:h], mode=fknn.MODE_BF16_RERANK, kprime=200, graph=True)
    assert datagen.recall_matrix(d, o64[:h]) >= 0.99
    # and back
    e, _ = idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=200, graph=True)
    assert np.mean(np.all(e == a, axis=1)) >= 0.99


def test_device_inputs_and_stream(c1):
    torch = pytest.importorskip("torch")
    vecs, labels, ts, q, metas, idx, o64 = c1
    dq = torch.from_numpy(q).cuda()
    dm = torch.from_numpy(metas).cuda()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        ids, dists = idx.search(dq, dm, mode=fknn.MODE_BF16_RERANK, kprime=400, graph=True)
        ids2, _ = idx.search(dq, dm, mode=fknn.MODE_BF16_RERANK, kprime=400, graph=True)
    s.synchronize()
    got = ids.cpu().numpy().view(np.uint32)
    assert datagen.recall_matrix(got, o64) >= 0.99
    assert np.mean(np.all(got == ids2.cpu().numpy().view(np.uint32), axis=1)) >= 0.99


def test_fp8_graph(c1):
    vecs, labels, ts, q, metas, idx, o64 = c1
    g, _ = idx.search(q, metas, mode=fknn.MODE_FP8_RERANK, kprime=400, graph=True)
    h, _ = idx.search(q, metas, mode=fknn.MODE_FP8_RERANK, kprime=400)
    assert abs(datagen.recall_matrix(g, o64) - datagen.recall_matrix(h, o64)) <= 0.005
    assert np.mean(np.all(g == h, axis=1)) >= 0.98


def test_exact_mode_ignores_the_flag(c1):
    vecs, labels, ts, q, metas, idx, _ = c1
    a, ad = idx.search(q[:64], metas[:64], graph=True)
    b, bd = idx.search(q[:64], metas[:64])
    assert (a == b).all() and (ad.view(np.uint32) == bd.view(np.uint32)).all()


def test_unknown_flag_is_rejected(c1):
    vecs, labels, ts, q, metas, idx, _ = c1
    lib = fknn.load()
    opts = fknn._lib.SearchOpts(fknn.MODE_BF16_RERANK, 200, 2)
    qq = np.ascontiguousarray(q[:4])
    mm = np.ascontiguousarray(metas[:4])
    ids = np.empty((4, 100), np.uint32)
    rc = lib.fknn_search_ex(idx._h, qq.ctypes.data, mm.ctypes.data, 4, 100, ctypes.byref(opts),
                            ids.ctypes.data, None, None, None)
    assert rc == fknn.FKNN_EINVAL


def test_bounded_wait_through_the_graph():
    vecs, labels, ts, q, metas = datagen.make_workload(2, n=300_000, nq=3000)
    with fknn.Index(vecs, labels, ts, build_bf16=True) as idx:
        lib = fknn.load()
        want, wd = idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=200, graph=True)
        exact, _ = idx.search(q, metas)
        assert lib.fknn_index_test_withhold_copy(idx._h) == fknn.FKNN_OK
        ids = np.full_like(want, 0xFFFFFFFE)
        dd = np.zeros_like(wd)
        t0 = time.perf_counter()
        with pytest.raises(fknn.FknnError) as e:
            idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=200, ids=ids, dists=dd, graph=True)
        took = time.perf_counter() - t0
        assert e.value.code == fknn.FKNN_ETIMEOUT
        assert 0.5 < took < 60.0, took
        same = np.all(ids == want, axis=1)
        exact_rows = np.all(ids == exact, axis=1)
        assert (~(same | exact_rows)).sum() <= q.shape[0] // 100
        assert (ids != 0xFFFFFFFE).all()
        again, _ = idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=200, graph=True)
        assert (~np.all(again == want, axis=1)).sum() <= q.shape[0] // 100
