"""The allocation-free predicate compaction (fknn_filter_rows_noalloc).

It serves callers that may not allocate device memory at all -- engines that
run inside a fixed, pre-reserved HBM budget or another allocator's pool, and
latency-critical paths that cannot afford cudaMalloc's implicit device
synchronisation.  Its scratch is a fixed device array shared by every call.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.  It must pass alone in a
fresh process (the first call on the device does the one-time address
set-up) and after the other tests.
"""
import ctypes
from ctypes import byref, c_uint64

import numpy as np
import pytest

import fknn
from fknn import _lib, datagen

pytestmark = pytest.mark.gpu
MAX_ROWS = 65536 * 4096


def call_noalloc(labels_d, ts_d, n, meta4, out_d, stream=None):
    m = np.ascontiguousarray(meta4, dtype=np.float32).reshape(4)
    cnt = c_uint64()
    rc = fknn.load().fknn_filter_rows_noalloc(labels_d.data_ptr(), ts_d.data_ptr(), n, m.ctypes.data,
                                               out_d.data_ptr(), byref(cnt), stream)
    _lib.check(rc)
    return cnt.value


def test_noalloc_matches_filter_rows_on_two_calls_in_a_row():
    torch = pytest.importorskip("torch")
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=300_007, nq=8)
    labels_d = torch.from_numpy(labels).cuda()
    ts_d = torch.from_numpy(ts).cuda()
    out_d = torch.full((labels.shape[0],), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    with fknn.Index(vecs, labels, ts) as idx:
        # two different predicates back to back, then the first one again:
        # the second call must not see the first call's counters
        preds = [metas[0], metas[1], metas[0]]
        for t in range(4):  # make sure every predicate kind is covered
            sel = np.nonzero(metas[:, 0] == t)[0]
            if len(sel):
                preds.append(metas[sel[0]])
        for m in preds:
            want = idx.filter_rows(m)
            c = call_noalloc(labels_d, ts_d, labels.shape[0], m, out_d, stream)
            got = out_d[:c].cpu().numpy().view(np.uint32)
            assert c == len(want)
            np.testing.assert_array_equal(got, want)


def test_noalloc_calls_allocate_no_device_memory():
    """After the first call on the device (its one-time address look-up and
    the kernels' module loading), further calls leave the device's free
    memory exactly where it was."""
    torch = pytest.importorskip("torch")
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=200_003, nq=8)
    labels_d = torch.from_numpy(labels).cuda()
    ts_d = torch.from_numpy(ts).cuda()
    out_d = torch.empty(labels.shape[0], dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    call_noalloc(labels_d, ts_d, labels.shape[0], metas[0], out_d, stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for i in range(6):
        call_noalloc(labels_d, ts_d, labels.shape[0], metas[i % 8], out_d, stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory moved by {free0 - free1} bytes"


def test_noalloc_rejects_sizes_beyond_its_limit_and_host_pointers():
    torch = pytest.importorskip("torch")
    lib = fknn.load()
    small = torch.zeros(16, dtype=torch.float32, device="cuda")
    out = torch.zeros(16, dtype=torch.int32, device="cuda")
    m = np.array([0, -1, -1, -1], dtype=np.float32)
    cnt = c_uint64()
    rc = lib.fknn_filter_rows_noalloc(small.data_ptr(), small.data_ptr(), MAX_ROWS + 1, m.ctypes.data,
                                      out.data_ptr(), byref(cnt), None)
    assert rc == fknn.FKNN_EINVAL
    assert b"limit" in lib.fknn_last_error()
    host = np.zeros(16, dtype=np.float32)
    rc = lib.fknn_filter_rows_noalloc(host.ctypes.data, host.ctypes.data, 16, m.ctypes.data, out.data_ptr(),
                                      byref(cnt), None)
    assert rc == fknn.FKNN_EINVAL
    # still usable afterwards
    assert call_noalloc(small, small, 16, m, out) == 16
