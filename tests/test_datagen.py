"""Synthetic workload generator and contest file formats."""
import numpy as np

from fknn import datagen


def test_deterministic_and_shaped():
    a = datagen.make_workload(1, n=2000, nq=100)
    b = datagen.make_workload(1, n=2000, nq=100)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    vecs, labels, ts, q, metas = a
    assert vecs.shape == (2000, 100) and q.shape == (100, 100) and metas.shape == (100, 4)
    assert vecs.dtype == np.float32 and metas.dtype == np.float32
    assert labels.min() >= 0 and labels.max() <= 999 and np.all(labels == np.round(labels))
    assert ts.min() >= 0 and ts.max() <= 1
    t = metas[:, 0]
    assert set(np.unique(t)) <= {0.0, 1.0, 2.0, 3.0}
    w = metas[t >= 2, 3] - metas[t >= 2, 2]
    assert w.min() >= 0.05 - 1e-6 and w.max() <= 0.5 + 1e-6
    assert np.all(metas[(t == 0) | (t == 2), 1] == -1)


def test_config4_balanced_types_and_loguniform_windows():
    _, labels, _, _, metas = datagen.make_workload(4, n=5000, nq=4000)
    assert np.all(np.bincount(metas[:, 0].astype(int)) == 1000)
    w = metas[metas[:, 0] >= 2, 3] - metas[metas[:, 0] >= 2, 2]
    assert w.min() >= 1e-4 * 0.999 and w.max() <= 1.0
    assert labels.max() <= 9999


def test_contest_file_round_trip(tmp_path):
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=500, nq=20)
    datagen.write_base(str(tmp_path / "b.bin"), vecs, labels, ts)
    datagen.write_queries(str(tmp_path / "q.bin"), q, metas)
    v2, l2, t2 = datagen.read_base(str(tmp_path / "b.bin"))
    q2, m2 = datagen.read_queries(str(tmp_path / "q.bin"))
    np.testing.assert_array_equal(v2, vecs)
    np.testing.assert_array_equal(l2, labels)
    np.testing.assert_array_equal(t2, ts)
    np.testing.assert_array_equal(q2, q)
    np.testing.assert_array_equal(m2, metas)
    assert (tmp_path / "b.bin").stat().st_size == 4 + 500 * 102 * 4
    knn = np.arange(2000, dtype=np.uint32).reshape(20, 100)
    datagen.save_knn(str(tmp_path / "o.bin"), knn)
    assert (tmp_path / "o.bin").stat().st_size == 20 * 100 * 4


def test_recall():
    gt = np.arange(300, dtype=np.uint32).reshape(3, 100)
    knn = gt.copy()
    knn[0, :10] = 1000
    assert abs(datagen.recall_at_k(knn, gt) - (290 / 300)) < 1e-12
