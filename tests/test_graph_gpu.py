"""Graph beam search on the GPU (k_graph_search through fknn_graph_search)
against the reference Searcher's outputs (golden fixture) and the oracle
restatement (pinned to the reference by tests/test_oracle.py): ids and
distances equal, all six search forms."""
import os

import numpy as np
import pytest

import fknn
import oracle
from fknn import datagen
from graph_util import graph_inputs, id_bounds_for, random_graph, windows

pytestmark = pytest.mark.gpu

FORMS = {0: "Search", 1: "SearchFilter", 2: "SearchFilterSubTime", 3: "SearchCategoryRange",
         4: "SearchRangeFilterSubTime", 5: "SearchRangeFilter"}


def _run(gs, mode, q, k, refine, bounds, ib):
    if mode == 0:
        return gs.Search(q, k)
    if mode in (1, 2):
        return getattr(gs, FORMS[mode])(q, k, refine)
    return getattr(gs, FORMS[mode])(q, k, refine, bounds, ib)


def _check(gs, gb, vecs, q, mode, k, refine, bounds, ib, ef=32):
    gs.SetEf(ef)
    wd = mode in (2, 4)
    got = _run(gs, mode, q, k, refine, bounds, ib)
    exp = oracle.graph_search(gb, vecs, q, mode, k, refine, bounds, ib, ef=ef, with_dists=wd)
    if wd:
        np.testing.assert_array_equal(got[0], exp[0], err_msg=f"mode {mode} k {k} refine {refine}")
        np.testing.assert_array_equal(got[1], exp[1], err_msg=f"mode {mode} k {k} refine {refine}")
    else:
        np.testing.assert_array_equal(got, exp, err_msg=f"mode {mode} k {k} refine {refine}")


def test_matches_reference_fixture(golden_dir):
    f = np.load(os.path.join(golden_dir, "graph_hnsw.npz"))
    vecs, labels, ts, q, bounds, ib = graph_inputs()
    gb = f["graph"].tobytes()
    with fknn.GraphSearcher(gb, vecs) as gs:
        for j, (mode, k, refine) in enumerate(f["cases"]):
            mode, k, refine = int(mode), int(k), int(refine)
            got = _run(gs, mode, q, k, refine, bounds, ib)
            if mode in (2, 4):
                np.testing.assert_array_equal(got[0], f[f"ids{j}"], err_msg=f"case {j}")
                np.testing.assert_array_equal(got[1], f[f"dists{j}"], err_msg=f"case {j}")
            else:
                np.testing.assert_array_equal(got, f[f"ids{j}"], err_msg=f"case {j}")


@pytest.mark.parametrize("layers", [True, False])
def test_random_graph_all_forms(layers):
    """Random adjacency with repeats and -1 padding; with the HNSW upper
    layers and with the entry-point list instead."""
    n = 20000
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=n, nq=64)
    ts = np.sort(ts)
    gb = random_graph(n, 48, ts, seed=11 + layers, with_layers=layers)
    bounds = windows(q.shape[0], 5, log_w=(-4, 0))
    ib = id_bounds_for(ts, bounds)
    with fknn.GraphSearcher(gb, vecs) as gs:
        for mode in range(6):
            for k, refine, ef in [(40, 40, 32), (400, 150, 32), (20, 33, 32), (64, 65, 64)]:
                if mode == 0:
                    refine = k
                _check(gs, gb, vecs, q, mode, k, refine, bounds, ib, ef=ef)


def test_many_queries_reuse_warp_slots():
    """More queries than resident warps: each warp's visited bitmap is
    reused, so its lazily cleared blocks must not leak between queries."""
    n = 6000
    vecs, labels, ts, q, metas = datagen.make_workload(4, n=n, nq=9000)
    ts = np.sort(ts)
    gb = random_graph(n, 24, ts, seed=5)
    bounds = windows(q.shape[0], 6)
    ib = id_bounds_for(ts, bounds)
    with fknn.GraphSearcher(gb, vecs) as gs:
        for mode in (1, 3, 4):
            _check(gs, gb, vecs, q, mode, 32, 32, bounds, ib)


def test_device_tensors_in_and_out():
    torch = pytest.importorskip("torch")
    vecs, labels, ts, q, bounds, ib = graph_inputs()
    f = np.load(os.path.join(os.path.dirname(__file__), "golden", "graph_hnsw.npz"))
    gb = f["graph"].tobytes()
    with fknn.GraphSearcher(gb, torch.from_numpy(vecs).cuda()) as gs:
        qd = torch.from_numpy(q).cuda()
        ids, d = gs.SearchRangeFilterSubTime(qd, 300, 150, torch.from_numpy(bounds).cuda(),
                                             torch.from_numpy(ib).cuda())
        assert ids.is_cuda and d.is_cuda
        j = [tuple(c) for c in f["cases"].tolist()].index((4, 300, 150))
        np.testing.assert_array_equal(ids.cpu().numpy(), f[f"ids{j}"])
        np.testing.assert_array_equal(d.cpu().numpy(), f[f"dists{j}"])


def test_bad_inputs_fail_loudly_and_leave_the_handle_usable():
    vecs, labels, ts, q, bounds, ib = graph_inputs()
    f = np.load(os.path.join(os.path.dirname(__file__), "golden", "graph_hnsw.npz"))
    gb = f["graph"].tobytes()
    with pytest.raises(fknn.FknnError) as e:
        fknn.GraphSearcher(gb[:-5], vecs)
    assert e.value.code == fknn.FKNN_EINVAL
    with fknn.GraphSearcher(gb, vecs) as gs:
        bad = ib.copy()
        bad[3] = (1990, 2600)  # seeds 1990 + 61 i run past the last point
        with pytest.raises(fknn.FknnError) as e:
            gs.SearchCategoryRange(q, 64, 40, bounds, bad)
        assert e.value.code == fknn.FKNN_EINVAL
        with pytest.raises(fknn.FknnError):
            gs.SearchFilter(q, 64, 66)  # refine > max(k, ef) + 1
        got = gs.SearchCategoryRange(q, 64, 40, bounds, ib)
        j = [tuple(c) for c in f["cases"].tolist()].index((3, 64, 40))
        np.testing.assert_array_equal(got, f[f"ids{j}"])


@pytest.mark.skipif(oracle.ref_graph() is None, reason="reference graph objects not built (oracle/_ref)")
def test_reference_hnsw_graph_large_pool(tmp_path):
    """A reference-built HNSW graph (degree 56, the contest's M = 28) with
    the contest's pool sizes (ef 1800-2800 range)."""
    n = 60000
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=n, nq=48)
    order = np.argsort(ts, kind="stable")
    vecs, labels, ts = vecs[order], labels[order], ts[order]
    gb = oracle.ref_hnsw_graph(vecs, ts, 56, 200, str(tmp_path / "g.bin"))
    bounds = windows(q.shape[0], 8, log_w=(-3, 0))
    ib = id_bounds_for(ts, bounds)
    with fknn.GraphSearcher(gb, vecs) as gs:
        for mode in range(1, 6):
            _check(gs, gb, vecs, q, mode, 1800, 150, bounds, ib)


@pytest.mark.skipif(oracle.ref_graph() is None, reason="reference graph objects not built (oracle/_ref)")
def test_recall_after_fp32_rerank(tmp_path):
    """The graph path's quality: SearchFilter candidates (k = 1000,
    refine = 150) re-ranked in FP32 reach recall@100 >= 0.98 against the
    exact top-100."""
    n = 100000
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=n, nq=200)
    gb = oracle.ref_hnsw_graph(vecs, ts, 32, 100, str(tmp_path / "g.bin"))
    with fknn.GraphSearcher(gb, vecs) as gs:
        cand = gs.SearchFilter(q, 1000, 150)
    d = ((vecs[cand] - q[:, None, :]) ** 2).sum(-1)
    top = np.take_along_axis(cand, np.argsort(d, axis=1, kind="stable")[:, :100], 1)
    exact, _ = oracle.exact_knn(vecs, labels, ts, q, np.zeros((q.shape[0], 4), np.float32))
    rec = np.mean([len(np.intersect1d(top[i], exact[i])) / 100 for i in range(q.shape[0])])
    assert rec >= 0.98, rec
