"""fknn_router: the reference's BatchSearch routing (hybrid_graph.cpp:
147-503) on the GPU, run over the very subgraphs and base orders the
reference pipeline (compiled from its sources, oracle/_ref) built and used
on the same data.  Per query type its recall@100 against the exact ids must
be within 0.005 of the reference pipeline's own.

The uneven-selectivity generator at N = 1.2e6 puts 38 % of the rows in one
category, so with the reference's selectivity denominator (1e7 rows) every
route runs: the SQ8 brute force (most predicates), the largest category's
graph (its type-1 queries), the ten time-bucket graphs (type 0) and the
split of wide windows into FULL / MEDIUM / SMALL buckets (type 2)."""
import numpy as np
import pytest

import fknn
import oracle
from fknn import datagen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pipeline(tmp_path_factory):
    if oracle.ref_hybrid() is None:
        pytest.skip("the reference pipeline (oracle/_ref/libref_hybrid.so) is not built")
    d = str(tmp_path_factory.mktemp("hybrid"))
    vecs, labels, ts, q, metas = datagen.make_workload(4, n=1_200_000, nq=2000)
    datagen.write_base(d + "/base.bin", vecs, labels, ts)
    datagen.write_queries(d + "/queries.bin", q, metas)
    ref_ids, ref_s = oracle.ref_hybrid_run(d + "/base.bin", d + "/queries.bin", d, q.shape[0])
    h = oracle.read_hybrid_dir(d, vecs.shape[0])
    with fknn.Index(vecs, labels, ts) as idx:
        gt, _ = idx.search(q, metas)
    return vecs, labels, ts, q, metas, ref_ids, h, gt


def test_router_recall_matches_the_reference_pipeline(pipeline):
    vecs, labels, ts, q, metas, ref_ids, h, gt = pipeline
    with fknn.Router(vecs, labels, ts, h["sorted_base_ids"], h["sorted_base_ids_by_full_time"], h["categories"],
                     h["buckets"], h["maxc_size"], h["minc_size"]) as router:
        ids, st = router.search(q, metas)
        ids2, _ = router.search(q, metas)  # a second call on the same router
    # every route ran
    assert st["n_bruteforce"] > 0 and st["n_category"] > 0 and st["n_type0"] > 0 and st["n_type2"] > 0, st
    assert st["n_split_full"] + st["n_split_medium"] + st["n_split_small"] > 0, st
    for t in range(4):
        s = metas[:, 0] == t
        ours = datagen.recall_matrix(ids[s], gt[s])
        ref = datagen.recall_matrix(ref_ids[s], gt[s])
        assert abs(ours - ref) <= 0.005, (t, ours, ref)
    assert datagen.recall_matrix(ids2, ids) > 0.999


def test_router_rejects_bad_subgraphs(pipeline):
    vecs, labels, ts, q, metas, ref_ids, h, gt = pipeline
    cats = [(k, s, c + 1, b) for k, s, c, b in h["categories"][:1]]  # a count that does not match its graph
    with pytest.raises(fknn.FknnError):
        fknn.Router(vecs, labels, ts, h["sorted_base_ids"], h["sorted_base_ids_by_full_time"], cats, [],
                    h["maxc_size"], h["minc_size"])
