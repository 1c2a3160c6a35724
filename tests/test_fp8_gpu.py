"""FP8-e4m3 per-dimension-scaled screen (FKNN_MODE_FP8_RERANK): the analogue
of the per-dimension SQ8 codes (sq8_quant.hpp:30-63) on tcgen05
kind::f8f6f4, followed by the same FP32 re-rank and FP64 boundary as the
BF16 form.  Bar: recall@100 >= 0.99 against the FP64 oracle at k' >= 400 on
these sizes; returned distances are the reference FP32 distances."""
import numpy as np
import pytest

import fknn
import oracle
from fknn import datagen

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cfg,kprime", [(1, 400), (1, 800), (4, 400)])
def test_recall_vs_fp64_oracle(cfg, kprime):
    vecs, labels, ts, q, metas = datagen.make_workload(cfg, n=80000, nq=500)
    with fknn.Index(vecs, labels, ts, build_fp8=True) as idx:
        ids, dists = idx.search(q, metas, mode=fknn.MODE_FP8_RERANK, kprime=kprime)
    o64, _ = oracle.exact_knn(vecs, labels, ts, q, metas, f64=True)
    assert datagen.recall_matrix(ids, o64) >= 0.99
    L = oracle.lib()
    for i in range(0, 500, 37):
        qq = np.ascontiguousarray(q[i])
        for j in range(0, 100, 11):
            if ids[i, j] == 0xFFFFFFFF:
                continue
            x = np.ascontiguousarray(vecs[ids[i, j]])
            assert np.float32(L.oracle_normal_l2(x.ctypes.data, qq.ctypes.data, 100)) == dists[i, j]


def test_fp8_needs_its_codes():
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=3000, nq=4)
    with fknn.Index(vecs, labels, ts, build_bf16=True) as idx:
        with pytest.raises(fknn.FknnError) as e:
            idx.search(q, metas, mode=fknn.MODE_FP8_RERANK)
        assert e.value.code == fknn.FKNN_EUNSUPPORTED
