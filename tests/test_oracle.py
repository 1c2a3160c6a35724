"""The CPU oracle (oracle/fknn_oracle.c) pinned against the reference's own
outputs: golden fixtures made by the compiled reference
(tests/golden/make_golden.py) and, where the reference objects are built
(oracle/_ref), live comparisons."""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from fknn import datagen

# where the reference sources lie (only the recipes that compile or read them use this)
REF_ROOT = os.environ.get("REF_ROOT", "/root/reference")


def _digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("name", ["exact_c1.npz", "exact_c4.npz"])
def test_exact_matches_reference_fixture(golden_dir, name):
    f = np.load(os.path.join(golden_dir, name))
    vecs, labels, ts, q, metas = datagen.make_workload(int(f["cfg"]), n=int(f["n"]), nq=int(f["nq"]))
    assert _digest(vecs, labels, ts, q, metas) == str(f["sha_inputs"]), "generator output changed"
    counts = oracle.count_matches(labels, ts, metas)
    np.testing.assert_array_equal(counts, f["counts"])
    sel = f["sel"]
    ids, dists = oracle.exact_knn(vecs, labels, ts, q[sel], metas[sel])
    np.testing.assert_array_equal(ids, f["gt"])
    assert np.all(np.diff(dists, axis=1) >= 0)


@pytest.mark.parametrize("cfg", [1, 3, 4])
def test_count_matches_sorted_equals_scan(cfg):
    """The sorted-column count (used at N = 1e7) equals the row scan,
    including windows whose bounds fall exactly on row timestamps."""
    vecs, labels, ts, q, metas = datagen.make_workload(cfg, n=40_000, nq=4_000)
    hit = np.nonzero(metas[:, 0] >= 2)[0][:100]
    metas[hit, 2] = ts[hit]
    metas[hit[::2], 3] = ts[hit[::2]]
    np.testing.assert_array_equal(oracle.count_matches_sorted(labels, ts, metas),
                                  oracle.count_matches(labels, ts, metas))


def test_filter_rows_counts_equal_the_c_restatement():
    """oracle.filter_rows (the predicate as a column mask) passes exactly
    the rows oracle_count_matches counts, on every query type."""
    vecs, labels, ts, q, metas = datagen.make_workload(4, n=30_000, nq=400)
    counts = oracle.count_matches(labels, ts, metas)
    for i in range(metas.shape[0]):
        ids = oracle.filter_rows(labels, ts, metas[i])
        assert len(ids) == counts[i]
        assert np.all(np.diff(ids.astype(np.int64)) > 0)


def test_exact_ties_match_reference_fixture(golden_dir):
    f = np.load(os.path.join(golden_dir, "exact_ties.npz"))
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=400, nq=30)
    v3, l3, t3 = np.repeat(vecs, 3, axis=0), np.repeat(labels, 3), np.repeat(ts, 3)
    q3 = np.concatenate([vecs[:20], q[:10]])
    m3 = np.zeros((30, 4), dtype=np.float32)
    assert _digest(v3, l3, t3, q3, m3) == str(f["sha_inputs"])
    ids, dists = oracle.exact_knn(v3, l3, t3, q3, m3)
    np.testing.assert_array_equal(ids, f["gt"])
    # exact ties resolved by the smaller id
    assert list(ids[0, :3]) == [0, 1, 2] and dists[0, 0] == 0.0


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_ROOT, "dummy-data.bin")), reason="reference data absent")
def test_exact_matches_reference_on_dummy_data(golden_dir):
    f = np.load(os.path.join(golden_dir, "dummy_gt.npz"))
    dpath, qpath = os.path.join(REF_ROOT, "dummy-data.bin"), os.path.join(REF_ROOT, "dummy-queries.bin")
    assert hashlib.sha256(open(dpath, "rb").read()).hexdigest() == str(f["sha_data"])
    vecs, labels, ts = datagen.read_base(dpath)
    q, metas = datagen.read_queries(qpath)
    ids, _ = oracle.exact_knn(vecs, labels, ts, q, metas)
    np.testing.assert_array_equal(ids, f["gt"])


def test_padding_when_fewer_than_k_rows_pass():
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=3000, nq=200)
    counts = oracle.count_matches(labels, ts, metas)
    ids, dists = oracle.exact_knn(vecs, labels, ts, q, metas)
    short = np.nonzero(counts < 100)[0]
    assert len(short) > 0
    for i in short:
        c = int(counts[i])
        assert np.all(ids[i, c:] == 0xFFFFFFFF) and np.all(np.isinf(dists[i, c:]))
        assert np.all(ids[i, :c] != 0xFFFFFFFF)


def test_f64_oracle_orders_like_f32_on_well_separated_rows():
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=5000, nq=50)
    metas[:, 0] = 0  # every row passes, so no padding
    i32, _ = oracle.exact_knn(vecs, labels, ts, q, metas)
    i64, d64 = oracle.exact_knn(vecs, labels, ts, q, metas, f64=True)
    agree = np.mean([len(np.intersect1d(a, b)) / 100.0 for a, b in zip(i32, i64)])
    assert agree > 0.99
    assert d64.dtype == np.float64


def test_sq8_matches_reference_fixture(golden_dir):
    f = np.load(os.path.join(golden_dir, "sq8.npz"))
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=6000, nq=12)
    assert _digest(vecs, q) == str(f["sha_inputs"])
    alpha, codes = oracle.sq8_sym_train(vecs)
    assert np.float32(alpha) == f["alpha"]
    assert _digest(codes) == str(f["codes_sha"])
    qcodes = oracle.sq8_sym_encode(q, alpha)
    np.testing.assert_array_equal(qcodes, f["qcodes"])
    tie_codes = np.repeat(codes[:700], 4, axis=0)
    for j, (k, s, npnt, src) in enumerate(f["cases"]):
        slab = (codes if src == 0 else tie_codes)[s:s + npnt]
        for i in range(q.shape[0]):
            ids, d = oracle.sq8_bruteforce(int(k), slab, alpha, qcodes[i], with_dists=True)
            np.testing.assert_array_equal(ids, f[f"ids{j}"][i])
            np.testing.assert_array_equal(d, f[f"dists{j}"][i])


def test_sq8_known_answer(golden_dir):
    kat = json.load(open(os.path.join(golden_dir, "sq8_kat.json")))
    x = np.zeros(112, dtype=np.int8)
    y = np.zeros(112, dtype=np.int8)
    x[:32] = kat["a0"]
    y[:32] = kat["a1"]
    assert oracle.lib().oracle_l2sqr_sq8_sym(x.ctypes.data, y.ctypes.data) == kat["l2sqr_sq8_sym"] == 210929


@pytest.mark.skipif(oracle.ref_exact() is None, reason="reference objects not built (make -C oracle ref)")
def test_restatement_equals_live_reference():
    R = oracle.ref_exact()
    L = oracle.lib()
    rng = np.random.default_rng(7)
    a = rng.standard_normal((64, 100), dtype=np.float32) * 3
    b = rng.standard_normal((64, 100), dtype=np.float32)
    for i in range(64):
        x = R.ref_normal_l2(a[i].ctypes.data, b[i].ctypes.data, 100)
        y = L.oracle_normal_l2(a[i].ctypes.data, b[i].ctypes.data, 100)
        assert np.float32(x).view(np.uint32) == np.float32(y).view(np.uint32)
    vecs, labels, ts, q, metas = datagen.make_workload(4, n=8000, nq=120)
    counts = oracle.count_matches(labels, ts, metas)
    sel = np.nonzero(counts >= 100)[0]
    rows, qrows = datagen.to_rows(vecs, labels, ts), datagen.to_query_rows(q[sel], metas[sel])
    gt = np.empty((len(sel), 100), dtype=np.uint32)
    assert R.ref_exact_bruteforce(rows.ctypes.data, rows.shape[0], qrows.ctypes.data, len(sel), gt.ctypes.data,
                                  None) == 0
    ids, _ = oracle.exact_knn(vecs, labels, ts, q[sel], metas[sel])
    np.testing.assert_array_equal(ids, gt)


@pytest.mark.skipif(oracle.ref_sq8() is None, reason="reference objects not built (make -C oracle ref)")
def test_sq8_restatement_equals_live_reference():
    R = oracle.ref_sq8()
    rng = np.random.default_rng(3)
    codes = rng.integers(-127, 128, size=(3000, 112), dtype=np.int8)
    codes[:, 100:] = 0
    codes[1000:2000] = codes[:1000]  # duplicate distances
    for k in (1, 50, 140, 3000):
        qv = np.ascontiguousarray(codes[rng.integers(0, 3000)])
        ids = np.empty(k, dtype=np.int32)
        R.ref_sq8_bruteforce(k, ids.ctypes.data, 3000, codes.ctypes.data, ctypes.c_float(1.0), qv.ctypes.data)
        np.testing.assert_array_equal(oracle.sq8_bruteforce(k, codes, 1.0, qv), ids)


def _graph_fixture(golden_dir):
    from graph_util import graph_inputs
    f = np.load(os.path.join(golden_dir, "graph_hnsw.npz"))
    vecs, labels, ts, q, bounds, ib = graph_inputs()
    assert _digest(vecs, labels, ts, q) == str(f["sha_inputs"]), "generator output changed"
    np.testing.assert_array_equal(bounds, f["bounds"])
    np.testing.assert_array_equal(ib, f["id_bounds"])
    return f, vecs, labels, ts, q, bounds, ib


def test_graph_search_matches_reference_fixture(golden_dir):
    """Restated Searcher == the reference Searcher on a reference HNSW graph,
    all six search forms (searcher.hpp:162-569)."""
    f, vecs, labels, ts, q, bounds, ib = _graph_fixture(golden_dir)
    gb = f["graph"].tobytes()
    for j, (mode, k, refine) in enumerate(f["cases"]):
        wd = int(mode) in (2, 4)
        out = oracle.graph_search(gb, vecs, q, int(mode), int(k), int(refine), bounds, ib, with_dists=wd)
        ids = out[0] if wd else out
        np.testing.assert_array_equal(ids, f[f"ids{j}"], err_msg=f"case {j} mode {mode}")
        if wd:
            np.testing.assert_array_equal(out[1], f[f"dists{j}"], err_msg=f"case {j} mode {mode}")


def test_graph_search_rejects_bad_inputs():
    from graph_util import random_graph
    ts = np.sort(np.random.default_rng(1).random(500).astype(np.float32))
    gb = random_graph(500, 16, ts, seed=3)
    vecs = np.random.default_rng(2).standard_normal((500, 100)).astype(np.float32)
    with pytest.raises(ValueError):  # truncated bytes
        oracle.graph_search(gb[:-7], vecs, vecs[:2], 0, 10, 10)
    with pytest.raises(ValueError):  # a seed past the last point
        oracle.graph_search(gb, vecs, vecs[:1], 3, 10, 10, np.array([[0, 1]], np.float32),
                            np.array([[600, 700]], np.int32))


@pytest.mark.skipif(oracle.ref_graph() is None, reason="reference graph objects not built (oracle/_ref)")
def test_graph_restatement_equals_live_reference(tmp_path):
    """Seeded HNSW graphs of several sizes and degrees; the restated Searcher
    equals the reference Searcher call for call."""
    from graph_util import id_bounds_for, windows
    for (n, R, cfg) in [(3000, 16, 1), (12000, 32, 4)]:
        vecs, labels, ts, q, metas = datagen.make_workload(cfg, n=n, nq=40)
        order = np.argsort(ts, kind="stable")
        vecs, labels, ts = vecs[order], labels[order], ts[order]
        path = str(tmp_path / f"g{n}.bin")
        gb = oracle.ref_hnsw_graph(vecs, ts, R, 80, path)
        bounds = windows(q.shape[0], n, log_w=(-4, 0))
        ib = id_bounds_for(ts, bounds)
        for mode, k, refine in [(0, 50, 50), (1, 500, 150), (2, 120, 60), (3, 200, 150), (4, 200, 150),
                                (5, 33, 34)]:
            wd = mode in (2, 4)
            r = oracle.ref_graph_search(path, vecs, labels, ts, q, mode, k, refine, bounds, ib, with_dists=wd)
            o = oracle.graph_search(gb, vecs, q, mode, k, refine, bounds, ib, with_dists=wd)
            if wd:
                np.testing.assert_array_equal(o[0], r[0])
                np.testing.assert_array_equal(o[1], r[1])
            else:
                np.testing.assert_array_equal(o, r)
