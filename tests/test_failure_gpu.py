"""Failure paths, made to happen without faulting, trapping or hanging the
GPU.

* A bounded device wait runs out: fknn_index_test_withhold_copy makes the
  next BF16 search issue no row-block copy for its first work item, so that
  item's MMA issuer and epilogue wait on barriers nothing completes.  Each
  wait gives up after about a second of the global timer, the kernel
  returns through its error flag, the call reports FKNN_ETIMEOUT with
  complete results (the affected queries re-answered by the exact scan),
  and the next call succeeds.
* The request loop's host waits: fknn_server_wait / fknn_server_drain with
  a short timeout while a batch is still on the device report FKNN_ETIMEOUT
  and leave the server usable.
"""
import time

import numpy as np
import pytest

import fknn
from fknn import datagen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def data():
    vecs, labels, ts, q, metas = datagen.make_workload(2, n=300_000, nq=3000)
    idx = fknn.Index(vecs, labels, ts, build_bf16=True)
    yield idx, q, metas
    idx.close()


def test_device_wait_runs_out_then_next_call_succeeds(data):
    idx, q, metas = data
    lib = fknn.load()
    want, wd = idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=200)
    exact, ed = idx.search(q, metas, mode=fknn.MODE_EXACT_FP32)
    assert lib.fknn_index_test_withhold_copy(idx._h) == fknn.FKNN_OK
    ids = np.full_like(want, 0xFFFFFFFE)  # neither a row id nor the padding value
    dd = np.zeros_like(wd)
    t0 = time.perf_counter()
    with pytest.raises(fknn.FknnError) as e:
        idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=200, ids=ids, dists=dd)
    took = time.perf_counter() - t0
    assert e.value.code == fknn.FKNN_ETIMEOUT
    assert b"bounded device wait" in lib.fknn_last_error()
    assert 0.5 < took < 60.0, took  # the waits give up after about a second
    # complete results: every query is the normal answer or, for the queries
    # of the starved work item, the exact one
    # (the BF16 form keeps equal-screening-distance candidates in arrival
    # order, so a rare row may differ between runs: allow 1 %)
    same = np.all(ids == want, axis=1)
    exact_rows = np.all(ids == exact, axis=1)
    assert (~(same | exact_rows)).sum() <= q.shape[0] // 100
    assert (ids != 0xFFFFFFFE).all() and np.isfinite(dd[ids != 0xFFFFFFFF]).all()
    # the hook is off again and the context is healthy
    again, ad = idx.search(q, metas, mode=fknn.MODE_BF16_RERANK, kprime=200)
    assert (~np.all(again == want, axis=1)).sum() <= q.shape[0] // 100


def test_server_wait_and_drain_time_out_on_the_host(data):
    idx, q, metas = data
    big_q = np.ascontiguousarray(np.repeat(q, 4, axis=0))
    big_m = np.ascontiguousarray(np.repeat(metas, 4, axis=0))
    with fknn.Server(idx, mode=fknn.MODE_EXACT_FP32, max_batch=4096, slots=1) as srv:
        t, ids, d = srv.submit(big_q, big_m)
        last = t + big_q.shape[0] - 1
        with pytest.raises(fknn.FknnError) as e:
            srv.wait(last, timeout_ms=0)
        assert e.value.code == fknn.FKNN_ETIMEOUT
        with pytest.raises(fknn.FknnError) as e:
            srv.drain(timeout_ms=0)
        assert e.value.code == fknn.FKNN_ETIMEOUT
        srv.drain()  # no limit: everything completes
        srv.wait(last)
        direct, _ = idx.search(q[:50], metas[:50])
        np.testing.assert_array_equal(ids[:200:4], direct)
