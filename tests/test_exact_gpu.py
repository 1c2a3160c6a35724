"""Exact FP32 path on the GPU (through the C ABI) against the reference's
ids (golden fixtures) and the oracle restatement: ids bit-exact, distances
bit-exact (the tolerance named for distances is 1e-5 relative; the kernel
reaches 0)."""
import os

import numpy as np
import pytest

import fknn
import oracle
from fknn import datagen

pytestmark = pytest.mark.gpu
UMAX = 0xFFFFFFFF


def run(vecs, labels, ts, q, metas, k=100, **kw):
    with fknn.Index(vecs, labels, ts) as idx:
        return idx.search(q, metas, k=k, **kw)


def assert_same_as_oracle(vecs, labels, ts, q, metas, k=100):
    with fknn.Index(vecs, labels, ts) as idx:
        ids, dists, st = idx.search(q, metas, k=k, return_stats=True)
    oids, odists = oracle.exact_knn(vecs, labels, ts, q, metas, k=k)
    bad = np.nonzero(np.any(ids != oids, axis=1))[0]
    assert len(bad) == 0, f"{len(bad)} queries differ, first {bad[:5]}"
    np.testing.assert_array_equal(dists.view(np.uint32), odists.view(np.uint32))
    # candidate lists only overflow into the exact scan on near-tie floods
    assert st["n_overflow"] <= max(2, q.shape[0] // 50), st
    return ids, dists


@pytest.mark.parametrize("name", ["exact_c1.npz", "exact_c4.npz"])
def test_ids_equal_reference_fixture(golden_dir, name):
    f = np.load(os.path.join(golden_dir, name))
    vecs, labels, ts, q, metas = datagen.make_workload(int(f["cfg"]), n=int(f["n"]), nq=int(f["nq"]))
    ids, dists = run(vecs, labels, ts, q, metas)
    sel = f["sel"]
    np.testing.assert_array_equal(ids[sel], f["gt"])
    # every query, including those with fewer than 100 passing rows
    oids, odists = oracle.exact_knn(vecs, labels, ts, q, metas)
    np.testing.assert_array_equal(ids, oids)
    np.testing.assert_allclose(dists, odists, rtol=1e-5)
    np.testing.assert_array_equal(dists.view(np.uint32), odists.view(np.uint32))


def test_ties_equal_reference_fixture(golden_dir):
    f = np.load(os.path.join(golden_dir, "exact_ties.npz"))
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=400, nq=30)
    v3, l3, t3 = np.repeat(vecs, 3, axis=0), np.repeat(labels, 3), np.repeat(ts, 3)
    q3 = np.concatenate([vecs[:20], q[:10]])
    m3 = np.zeros((30, 4), dtype=np.float32)
    ids, _ = run(v3, l3, t3, q3, m3)
    np.testing.assert_array_equal(ids, f["gt"])


def test_all_rows_identical_overflow_path():
    """Every distance ties: the candidate lists overflow and the exact scan
    answers, still ordered by id."""
    n = 20000
    vecs = np.tile(np.linspace(-1, 1, 100, dtype=np.float32), (n, 1))
    labels = np.zeros(n, np.float32)
    ts = np.linspace(0, 1, n, dtype=np.float32)
    q = np.zeros((6, 100), np.float32)
    metas = np.array([[0, -1, -1, -1], [1, 0, -1, -1], [2, -1, 0.2, 0.9], [3, 0, 0.5, 0.51], [2, -1, 0, 1],
                      [0, -1, -1, -1]], np.float32)
    ids, dists = run(vecs, labels, ts, q, metas)
    oids, odists = oracle.exact_knn(vecs, labels, ts, q, metas)
    np.testing.assert_array_equal(ids, oids)
    assert list(ids[0, :5]) == [0, 1, 2, 3, 4]


@pytest.mark.parametrize("cfg,n,nq", [(1, 60000, 400), (4, 60000, 400), (2, 200000, 300)])
def test_matches_oracle_all_query_types(cfg, n, nq):
    vecs, labels, ts, q, metas = datagen.make_workload(cfg, n=n, nq=nq)
    assert_same_as_oracle(vecs, labels, ts, q, metas)


@pytest.mark.parametrize("k", [1, 7, 64, 100, 128])
def test_k_values(k):
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=30000, nq=200)
    assert_same_as_oracle(vecs, labels, ts, q, metas, k=k)


def test_edge_predicates():
    vecs, labels, ts, q, _ = datagen.make_workload(1, n=20000, nq=12)
    ts[:50] = 0.0
    ts[50:60] = -0.0  # compares equal to +0
    labels[100:110] = 3.7  # truncates to 3 (utils.h:109)
    metas = np.array([
        [1, 123456, -1, -1],   # label absent: empty
        [2, -1, 0.9, 0.1],     # l > r: empty
        [2, -1, 2.0, 3.0],     # window past every timestamp
        [2, -1, 0.0, 0.0],     # only ts == 0 rows (incl. -0.0)
        [2, -1, -0.0, 0.0],
        [3, 0, 0.0, 1.0],      # whole label 0
        [1, 3, -1, -1],        # label 3 incl. the 3.7 rows
        [3, 3, 0.3, 0.30001],  # tiny window
        [0, -1, -1, -1],
        [1, 0, -1, -1],
        [2, -1, 0.25, 0.25000003],
        [3, 7, 0.1, 0.2],
    ], np.float32)
    ids, dists = assert_same_as_oracle(vecs, labels, ts, q, metas)
    assert np.all(ids[0] == UMAX) and np.all(ids[1] == UMAX) and np.all(ids[2] == UMAX)


def test_fewer_rows_than_k():
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=37, nq=20)
    ids, dists = assert_same_as_oracle(vecs, labels, ts, q, metas)
    assert np.all(ids[:, 37:] == UMAX)


def test_device_pointers_and_counts():
    torch = pytest.importorskip("torch")
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=50000, nq=300)
    with fknn.Index(vecs, labels, ts) as idx:
        dq = torch.from_numpy(q).cuda()
        dm = torch.from_numpy(metas).cuda()
        ids_d, dists_d = idx.search(dq, dm, k=100)
        assert ids_d.is_cuda
        ids_h, dists_h = idx.search(q, metas, k=100)
        np.testing.assert_array_equal(ids_d.cpu().numpy().view(np.uint32), ids_h)
        np.testing.assert_array_equal(dists_d.cpu().numpy(), dists_h)
        np.testing.assert_array_equal(idx.count_matches(metas), oracle.count_matches(labels, ts, metas))


def test_filter_rows_compaction():
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=100003, nq=16)
    with fknn.Index(vecs, labels, ts) as idx:
        for m in metas:
            got = idx.filter_rows(m)
            t = int(m[0])
            v = np.int32(m[1])
            keep = np.ones(len(ts), bool)
            if t in (1, 3):
                keep &= labels.astype(np.int32) == v
            if t in (2, 3):
                keep &= (ts >= m[2]) & (ts <= m[3])
            np.testing.assert_array_equal(got, np.nonzero(keep)[0].astype(np.uint32))


def test_filter_rows_many_tiles():
    """More tiles than one scan block holds (4.5M rows = 1,099 tiles of 4,096)."""
    n = 4_500_000
    rng = np.random.default_rng(3)
    labels = rng.integers(0, 50, n).astype(np.float32)
    ts = rng.random(n, dtype=np.float32)
    vecs = np.zeros((n, 100), np.float32)
    with fknn.Index(vecs, labels, ts) as idx:
        for m in (np.array([0, 0, 0, 0], np.float32), np.array([1, 7, 0, 0], np.float32),
                  np.array([2, 0, 0.25, 0.5], np.float32), np.array([3, 7, 0.1, 0.9], np.float32)):
            got = idx.filter_rows(m)
            t = int(m[0])
            keep = np.ones(n, bool)
            if t in (1, 3):
                keep &= labels.astype(np.int32) == np.int32(m[1])
            if t in (2, 3):
                keep &= (ts >= m[2]) & (ts <= m[3])
            np.testing.assert_array_equal(got, np.nonzero(keep)[0].astype(np.uint32))


@pytest.mark.parametrize("n", [100, 4096, 1_000_003])
def test_filter_rows_batch_matches_oracle(n):
    """fknn_filter_rows_batch: 21 predicates in one call (two passes of at
    most 16), every query type, an empty result, exact-boundary windows and
    a row count that is not a multiple of the chunk; ids and device counts
    equal the oracle's, and the single-predicate call agrees."""
    torch = pytest.importorskip("torch")
    vecs, labels, ts, q, metas = datagen.make_workload(4, n=n, nq=17)
    extra = np.array([[1, 99_999, -1, -1],          # category that no row has
                      [2, ts[n // 2], ts[n // 2], 0],  # a window of one timestamp
                      [3, labels[0], 0.0, 1.0],
                      [0, -1, -1, -1]], np.float32)
    extra[1, 3] = extra[1, 2]
    preds = np.concatenate([metas, extra])
    with fknn.Index(vecs, labels, ts) as idx:
        out, counts = idx.filter_rows_batch(preds)
        torch.cuda.synchronize()
        out_h, counts_h = out.cpu().numpy().view(np.uint32), counts.cpu().numpy()
        for p in range(preds.shape[0]):
            want = oracle.filter_rows(labels, ts, preds[p])
            assert counts_h[p] == len(want), p
            np.testing.assert_array_equal(out_h[p, :len(want)], want)
        np.testing.assert_array_equal(idx.filter_rows(preds[2]), oracle.filter_rows(labels, ts, preds[2]))
    assert counts_h[17] == 0 and counts_h[20] == n and counts_h[18] >= 1


def test_filter_rows_fractional_and_negative_labels():
    """The label test is int32(label) == int32(v) (utils.h:118): labels that
    are not integers, negative labels, zero, values truncating from either
    side, large magnitudes and fractional predicate values; the compaction
    evaluates it as a float interval, which must select the same rows."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(11)
    n = 300_001
    base = np.array([-3.7, -3.0, -2.999, -0.5, -0.0, 0.0, 0.5, 0.999, 1.0, 1.5, 2.0, 2.999999, 3.0, 7.25,
                     16777216.0, 16777218.0, -16777216.0, 1e9, -1e9, 2147483520.0], np.float32)
    labels = base[rng.integers(0, len(base), n)]
    ts = rng.random(n, dtype=np.float32)
    vecs = np.zeros((n, 100), np.float32)
    vals = [-4, -3, -2, -1, 0, 1, 2, 3, 7, 16777216, 16777217, 16777218, -16777216, 1000000000, -1000000000,
            2147483520, 2.5, -2.5, 0.9, -0.9]
    preds = np.array([[1, v, 0, 0] for v in vals] + [[3, v, 0.2, 0.7] for v in vals[:8]], np.float32)
    with fknn.Index(vecs, labels, ts) as idx:
        out, counts = idx.filter_rows_batch(preds)
        torch.cuda.synchronize()
        out_h, counts_h = out.cpu().numpy().view(np.uint32), counts.cpu().numpy()
    for p in range(preds.shape[0]):
        want = oracle.filter_rows(labels, ts, preds[p])
        assert counts_h[p] == len(want), (p, preds[p], counts_h[p], len(want))
        np.testing.assert_array_equal(out_h[p, :len(want)], want)


def test_invalid_queries_rejected():
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=5000, nq=4)
    with fknn.Index(vecs, labels, ts) as idx:
        bad = metas.copy()
        bad[0, 0] = 4
        with pytest.raises(fknn.FknnError) as e:
            idx.search(q, bad)
        assert e.value.code == fknn.FKNN_EINVAL
        q2 = q.copy()
        q2[1, 5] = np.nan
        with pytest.raises(fknn.FknnError):
            idx.search(q2, metas)
        with pytest.raises(fknn.FknnError):
            idx.search(q, metas, k=129)
        # the index is still usable after a rejected call
        ids, _ = idx.search(q, metas)
        np.testing.assert_array_equal(ids, oracle.exact_knn(vecs, labels, ts, q, metas)[0])
    v = vecs.copy()
    v[3, 3] = np.inf
    with pytest.raises(fknn.FknnError):
        fknn.Index(v, labels, ts)


def test_bruteforce_rows_dropin():
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=8000, nq=50)
    nodes = datagen.to_rows(vecs, labels, ts)
    queries = datagen.to_query_rows(q, metas)
    gt = fknn.Bruteforce(nodes, queries)
    np.testing.assert_array_equal(gt, oracle.exact_knn(vecs, labels, ts, q, metas)[0])
    lst = []
    fknn.Bruteforce(nodes.tolist()[:2000], queries.tolist()[:3], lst)
    assert len(lst) == 3 and len(lst[0]) == 100


def test_full_size_sampled_against_oracle():
    """Config 2 at full size (N=1e6, Q=1e5): every result sorted and
    self-consistent, a seeded sample of 400 queries bit-exact vs the oracle."""
    vecs, labels, ts, q, metas = datagen.make_workload(2)
    with fknn.Index(vecs, labels, ts) as idx:
        ids, dists, st = idx.search(q, metas, return_stats=True)
    assert st["n_overflow"] == 0
    valid = ids != UMAX
    assert np.all(np.isinf(dists[~valid]))
    assert np.all(dists[:, 1:] >= dists[:, :-1])  # ascending, +inf padding last
    rng = np.random.default_rng(11)
    sel = rng.choice(q.shape[0], 400, replace=False)
    oids, odists = oracle.exact_knn(vecs, labels, ts, q[sel], metas[sel])
    np.testing.assert_array_equal(ids[sel], oids)
    np.testing.assert_array_equal(dists[sel].view(np.uint32), odists.view(np.uint32))
