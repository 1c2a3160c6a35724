"""The request loop (fknn_server_*): continuous batching over a resident
index.  Each request's result is the same alone and in a mix with other
requests arriving while batches are on the device, and the same as a direct
fknn_search of that query."""
import threading
import time

import numpy as np
import pytest

import fknn
from fknn import datagen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def data():
    vecs, labels, ts, q, metas = datagen.make_workload(4, n=200_000, nq=3000)
    idx = fknn.Index(vecs, labels, ts, build_bf16=True)
    yield idx, q, metas
    idx.close()


@pytest.mark.parametrize("mode", [fknn.MODE_EXACT_FP32, fknn.MODE_BF16_RERANK])
def test_same_result_alone_and_in_the_mix(data, mode):
    idx, q, metas = data
    kp = 200 if mode == fknn.MODE_BF16_RERANK else 0
    direct_ids, direct_d = idx.search(q, metas, k=100, mode=mode, kprime=kp)
    probe = np.arange(0, q.shape[0], 15)  # 200 requests checked alone
    with fknn.Server(idx, mode=mode, kprime=kp, max_batch=512, slots=3) as srv:
        alone = {}
        for i in probe:
            t, ids, d = srv.submit(q[i:i + 1], metas[i:i + 1])
            srv.wait(t)
            alone[i] = (ids[0].copy(), d[0].copy())
        st = srv.stats(reset=True)
        assert st["max_batch_seen"] == 1
        # the mix: a client thread submits small bursts while batches run
        outs = []

        def client():
            rng = np.random.default_rng(3)
            i = 0
            while i < q.shape[0]:
                n = int(rng.integers(1, 64))
                outs.append((i, srv.submit(q[i:i + n], metas[i:i + n])))
                i += n
                time.sleep(float(rng.uniform(0, 2e-4)))

        th = threading.Thread(target=client)
        th.start()
        th.join()
        srv.drain(timeout_ms=120_000)
        st = srv.stats()
    mix_ids = np.concatenate([o[1][1] for o in outs])
    mix_d = np.concatenate([o[1][2] for o in outs])
    assert st["completed"] == q.shape[0] and st["failed"] == 0
    assert st["batches"] < q.shape[0] and st["mean_batch"] > 1.0  # requests were batched
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    np.testing.assert_array_equal(mix_ids, direct_ids)
    np.testing.assert_array_equal(mix_d, direct_d)
    for i in probe:
        np.testing.assert_array_equal(alone[i][0], mix_ids[i])
        np.testing.assert_array_equal(alone[i][1], mix_d[i])


def test_budget_limits_batches_and_everything_completes(data):
    idx, q, metas = data
    direct_ids, _ = idx.search(q[:1500], metas[:1500], k=100)
    with fknn.Server(idx, max_batch=1024, slots=2, hbm_budget=24 << 20) as srv:
        t, ids, _ = srv.submit(q[:1500], metas[:1500], with_dists=False)
        srv.drain(timeout_ms=120_000)
        st = srv.stats()
    np.testing.assert_array_equal(ids, direct_ids)
    assert st["completed"] == 1500 and st["failed"] == 0
    assert st["budget_trims"] >= 1  # a 1024-query batch needs more than 24 MB of scratch
    assert st["scratch_bytes"] <= st["budget_bytes"]


def test_invalid_request_is_rejected_at_submit(data):
    idx, q, metas = data
    bad = metas[:4].copy()
    bad[2, 0] = 7.0
    with fknn.Server(idx) as srv:
        with pytest.raises(fknn.FknnError) as e:
            srv.submit(q[:4], bad)
        assert e.value.code == fknn.FKNN_EINVAL
        assert srv.stats()["submitted"] == 0
        t, ids, _ = srv.submit(q[:4], metas[:4])
        srv.drain(timeout_ms=60_000)
