"""The contest's binary files through the C ABI (no GPU needed, except the
index built straight from a file): base and query readers, the
ReadSortedQuery order, SaveKNN and ReadGroundTruth, against files written
by the format restatement in fknn/datagen.py (utils.h:257-276, 550-566,
io.h:22-33, utils.h:194-221)."""
import os

import numpy as np
import pytest

import fknn
import oracle
from fknn import datagen


def test_base_and_query_files_round_trip(tmp_path):
    vecs, labels, ts, q, metas = datagen.make_workload(4, n=70_001, nq=333)
    bp, qp = str(tmp_path / "base.bin"), str(tmp_path / "q.bin")
    datagen.write_base(bp, vecs, labels, ts)
    datagen.write_queries(qp, q, metas)
    v2, l2, t2 = fknn.read_base_file(bp)
    np.testing.assert_array_equal(v2, vecs)
    np.testing.assert_array_equal(l2, labels)
    np.testing.assert_array_equal(t2, ts)
    q2, m2 = fknn.read_query_file(qp)
    np.testing.assert_array_equal(q2, q)
    np.testing.assert_array_equal(m2, metas)


def test_truncated_and_missing_files_are_rejected(tmp_path):
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=100, nq=10)
    bp = str(tmp_path / "base.bin")
    datagen.write_base(bp, vecs, labels, ts)
    with open(bp, "r+b") as f:
        f.truncate(os.path.getsize(bp) - 4)
    with pytest.raises(fknn.FknnError) as e:
        fknn.read_base_file(bp)
    assert e.value.code == fknn.FKNN_EINVAL
    with pytest.raises(fknn.FknnError):
        fknn.read_query_file(str(tmp_path / "missing.bin"))


def test_save_knn_and_read_groundtruth(tmp_path):
    rng = np.random.default_rng(4)
    ids = rng.integers(0, 2**32 - 1, size=(57, 100), dtype=np.uint64).astype(np.uint32)
    p = str(tmp_path / "out.bin")
    fknn.save_knn(p, ids)
    assert open(p, "rb").read() == ids.tobytes()  # io.h:22-33: rows only, no header
    gp = str(tmp_path / "gt.bin")
    with open(gp, "wb") as f:  # utils.h:170-192 SaveGroundTruth: u32 N, then the rows
        np.array([57], np.uint32).tofile(f)
        ids.tofile(f)
    np.testing.assert_array_equal(fknn.read_groundtruth(gp), ids)
    np.testing.assert_array_equal(fknn.read_groundtruth(gp), datagen.read_groundtruth(gp))


def sorted_order_restated(metas):
    """utils.h:513-533's comparator: (uint32 type, int32 v, l, r) ascending."""
    t = metas[:, 0].astype(np.uint32)
    v = metas[:, 1].astype(np.int32)
    return np.lexsort((metas[:, 3], metas[:, 2], v, t))  # stable, last key primary


@pytest.mark.parametrize("cfg", [1, 4])
def test_sorted_query_order(cfg):
    q, metas = datagen.make_workload(cfg, n=10, nq=5000)[3:]
    got = fknn.sorted_query_order(metas)
    np.testing.assert_array_equal(got, sorted_order_restated(metas))
    # the keys are nondecreasing in that order
    m = metas[got]
    assert np.all(np.diff(m[:, 0]) >= 0)


@pytest.mark.gpu
def test_index_from_file_equals_index_from_arrays(tmp_path):
    vecs, labels, ts, q, metas = datagen.make_workload(2, n=150_003, nq=400)
    bp = str(tmp_path / "base.bin")
    datagen.write_base(bp, vecs, labels, ts)
    with fknn.Index.from_file(bp, build_bf16=True) as a, fknn.Index(vecs, labels, ts, build_bf16=True) as b:
        assert a.n == b.n == vecs.shape[0]
        ia, da = a.search(q, metas)
        ib, db = b.search(q, metas)
        np.testing.assert_array_equal(ia, ib)
        np.testing.assert_array_equal(da, db)
        np.testing.assert_array_equal(ia, oracle.exact_knn(vecs, labels, ts, q, metas)[0])
        ba, _ = a.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=200)
        bb, _ = b.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=200)
        assert datagen.recall_matrix(ba, bb) > 0.999
