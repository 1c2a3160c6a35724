"""SQ8 symmetric quantizer and the SQ8 slab brute force on the GPU against
the reference's outputs (golden fixture, heap-array order included) and the
oracle restatement."""
import os

import numpy as np
import pytest

import fknn
import oracle
from fknn import datagen

pytestmark = pytest.mark.gpu


def test_train_encode_match_reference_fixture(golden_dir):
    f = np.load(os.path.join(golden_dir, "sq8.npz"))
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=6000, nq=12)
    quant = fknn.SQ8SymmetricQuantizer(100)
    quant.train(vecs)
    assert np.float32(quant.alpha) == f["alpha"]
    _, ocodes = oracle.sq8_sym_train(vecs)
    np.testing.assert_array_equal(quant.codes, ocodes)
    np.testing.assert_array_equal(quant.encode(q), f["qcodes"])


def test_bruteforce_heap_order_matches_reference_fixture(golden_dir):
    f = np.load(os.path.join(golden_dir, "sq8.npz"))
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=6000, nq=12)
    alpha, codes = oracle.sq8_sym_train(vecs)
    qcodes = f["qcodes"]
    tie_codes = np.repeat(codes[:700], 4, axis=0)
    for j, (k, s, npnt, src) in enumerate(f["cases"]):
        slab = np.ascontiguousarray((codes if src == 0 else tie_codes)[s:s + npnt])
        k = int(k)
        # one query per call, exactly as hybrid_graph.cpp:211 calls it
        for i in range(qcodes.shape[0]):
            out = np.empty(k, dtype=np.int32)
            fknn.bruteforce(100, k, out, int(npnt), slab, alpha, 1, np.ascontiguousarray(qcodes[i]))
            np.testing.assert_array_equal(out, f[f"ids{j}"][i])
        # batched: all queries against the slab in one call, with distances
        outb = np.empty((qcodes.shape[0], k), dtype=np.int32)
        dist = np.empty((qcodes.shape[0], k), dtype=np.float32)
        fknn.bruteforce_subgraph(100, k, outb, dist, int(npnt), slab, alpha, qcodes.shape[0], qcodes)
        np.testing.assert_array_equal(outb, f[f"ids{j}"])
        np.testing.assert_array_equal(dist, f[f"dists{j}"])


@pytest.mark.parametrize("npoints,k", [(140, 140), (5000, 140), (200000, 140), (70000, 1), (30000, 1000)])
def test_bruteforce_matches_oracle(npoints, k):
    rng = np.random.default_rng(npoints + k)
    base = rng.standard_normal((npoints // 3 + 1, 100), dtype=np.float32)
    vecs = np.repeat(base, 3, axis=0)[:npoints]  # many equal distances
    alpha, codes = oracle.sq8_sym_train(vecs)
    qv = oracle.sq8_sym_encode(rng.standard_normal((5, 100), dtype=np.float32), alpha)
    out = np.empty((5, k), dtype=np.int32)
    d = np.empty((5, k), dtype=np.float32)
    fknn.bruteforce_subgraph(100, k, out, d, npoints, codes, alpha, 5, qv)
    for i in range(5):
        oi, od = oracle.sq8_bruteforce(k, codes, alpha, qv[i], with_dists=True)
        np.testing.assert_array_equal(out[i], oi)
        np.testing.assert_array_equal(d[i], od)


@pytest.mark.parametrize("nq,k", [(9, 2048), (17, 140), (2, 7)])
def test_bruteforce_batched_matches_single(nq, k):
    """The batched kernel (eight queries per block, short last block) returns
    what one-query calls return, at the largest k too."""
    rng = np.random.default_rng(nq * 1000 + k)
    base = rng.standard_normal((4000, 100), dtype=np.float32)
    vecs = np.repeat(base, 2, axis=0)
    alpha, codes = oracle.sq8_sym_train(vecs)
    qv = oracle.sq8_sym_encode(rng.standard_normal((nq, 100), dtype=np.float32), alpha)
    out = np.empty((nq, k), dtype=np.int32)
    fknn.bruteforce(100, k, out, codes.shape[0], codes, alpha, nq, qv)
    for i in range(nq):
        one = np.empty(k, dtype=np.int32)
        fknn.bruteforce(100, k, one, codes.shape[0], codes, alpha, 1, np.ascontiguousarray(qv[i]))
        np.testing.assert_array_equal(out[i], one)
        if i % 4 == 0:
            np.testing.assert_array_equal(out[i], oracle.sq8_bruteforce(k, codes, alpha, qv[i]))


@pytest.mark.parametrize("npoints,nq,k", [(20000, 9, 2048), (40000, 130, 140)])
def test_bruteforce_screened_batch(npoints, nq, k):
    """Slabs past the exactly replayed prefix go through the int8 tensor-core
    screen; the batch (a short last query tile included) must give the
    oracle's heap arrays at the largest k and at the reference's K'."""
    rng = np.random.default_rng(npoints + nq)
    base = rng.standard_normal((npoints // 2, 100), dtype=np.float32)
    vecs = np.repeat(base, 2, axis=0)  # many equal distances
    alpha, codes = oracle.sq8_sym_train(vecs)
    qv = oracle.sq8_sym_encode(rng.standard_normal((nq, 100), dtype=np.float32), alpha)
    out = np.empty((nq, k), dtype=np.int32)
    d = np.empty((nq, k), dtype=np.float32)
    fknn.bruteforce_subgraph(100, k, out, d, npoints, codes, alpha, nq, qv)
    for i in list(range(0, nq, max(1, nq // 6))) + [nq - 1]:
        oi, od = oracle.sq8_bruteforce(k, codes, alpha, qv[i], with_dists=True)
        np.testing.assert_array_equal(out[i], oi)
        np.testing.assert_array_equal(d[i], od)


def test_bruteforce_full_width_codes():
    """The distance runs over all 112 code bytes (L2SqrSQ8_sym with d = 112),
    padding bytes included, on the prefix and the screened part alike."""
    rng = np.random.default_rng(7)
    npoints, nq, k = 30000, 5, 140
    codes = rng.integers(-127, 128, size=(npoints, 112), dtype=np.int8)
    qv = rng.integers(-127, 128, size=(nq, 112), dtype=np.int8)
    out = np.empty((nq, k), dtype=np.int32)
    fknn.bruteforce(100, k, out, npoints, codes, 1.0, nq, qv)
    for i in range(nq):
        np.testing.assert_array_equal(out[i], oracle.sq8_bruteforce(k, codes, 1.0, qv[i]))


def test_bruteforce_concurrent_callers():
    """The reference calls bruteforce() one query at a time from concurrent
    OpenMP workers (hybrid_graph.cpp:168,380).  Host threads calling at once,
    each on its own slab (prefix-only and screened sizes), get what the same
    calls return one after another."""
    import concurrent.futures as cf
    rng = np.random.default_rng(11)
    sizes = [3000, 9000, 12000, 20000, 5000, 16000]
    jobs = []
    for n in sizes:
        vecs = np.repeat(rng.standard_normal((n // 2, 100), dtype=np.float32), 2, axis=0)
        alpha, codes = oracle.sq8_sym_train(vecs)
        qv = oracle.sq8_sym_encode(rng.standard_normal((6, 100), dtype=np.float32), alpha)
        jobs.append((n, codes, alpha, qv))
    k = 140

    def run(job):
        n, codes, alpha, qv = job
        out = np.empty((qv.shape[0], k), dtype=np.int32)
        for i in range(qv.shape[0]):
            fknn.bruteforce(100, k, out[i], n, codes, alpha, 1, np.ascontiguousarray(qv[i]))
        return out

    serial = [run(j) for j in jobs]
    for _ in range(2):
        with cf.ThreadPoolExecutor(len(jobs)) as ex:
            par = list(ex.map(run, jobs))
        for a, b in zip(serial, par):
            np.testing.assert_array_equal(a, b)
    n, codes, alpha, qv = jobs[3]
    np.testing.assert_array_equal(serial[3][0], oracle.sq8_bruteforce(k, codes, alpha, qv[0]))


def test_bruteforce_rejects_bad_k():
    codes = np.zeros((10, 112), np.int8)
    out = np.empty(11, np.int32)
    with pytest.raises(fknn.FknnError):
        fknn.bruteforce(100, 11, out, 10, codes, 1.0, 1, np.zeros(112, np.int8))


def test_release_thread_scratch_then_call_again():
    """fknn_sq8_release_thread_scratch frees the calling thread's scratch;
    the next call sets it up again and returns the same heap arrays."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(21)
    vecs = rng.standard_normal((40000, 100), dtype=np.float32)
    alpha, codes = oracle.sq8_sym_train(vecs)
    qv = oracle.sq8_sym_encode(rng.standard_normal((3, 100), dtype=np.float32), alpha)
    k = 140
    a = np.empty((3, k), dtype=np.int32)
    b = np.empty((3, k), dtype=np.int32)
    fknn.bruteforce(100, k, a, codes.shape[0], codes, alpha, 3, qv)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert fknn.load().fknn_sq8_release_thread_scratch() == fknn.FKNN_OK
    free1, _ = torch.cuda.mem_get_info()
    assert free1 > free0  # the scratch went back to the device
    fknn.bruteforce(100, k, b, codes.shape[0], codes, alpha, 3, qv)
    np.testing.assert_array_equal(a, b)
    assert fknn.load().fknn_sq8_release_thread_scratch() == fknn.FKNN_OK
    assert fknn.load().fknn_sq8_release_thread_scratch() == fknn.FKNN_OK  # twice is harmless
