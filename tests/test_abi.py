"""C ABI checks that need no GPU: the library loads, exports every entry
point include/fknn.h declares, and rejects bad arguments before touching a
device."""
import ctypes
import os
import re
from ctypes import byref, c_void_p

import numpy as np
import pytest

import fknn
from fknn import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            names |= set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(fknn_\w+)\s*\(", src, flags=re.M))
    return names


def test_library_loads_and_exports_every_declared_symbol():
    lib = fknn.load()
    decl = declared_symbols()
    assert {"fknn_index_create", "fknn_search", "fknn_sq8_bruteforce"} <= decl
    for name in decl:
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
    # the Python binding covers every declared entry point
    assert decl <= set(_lib.SIGNATURES)


def test_version_and_error_text():
    lib = fknn.load()
    assert lib.fknn_version() >= 100
    assert isinstance(lib.fknn_last_error(), bytes)


def test_bad_arguments_are_rejected_without_a_device():
    lib = fknn.load()
    v = np.zeros((4, 99), dtype=np.float32)
    l = np.zeros(4, dtype=np.float32)
    h = c_void_p()
    opts = _lib.IndexOpts(0, 0, 0, 0)
    assert lib.fknn_index_create(v.ctypes.data, l.ctypes.data, l.ctypes.data, 4, 99, byref(opts), byref(h)) == \
        fknn.FKNN_EINVAL
    assert b"dim" in lib.fknn_last_error()
    assert lib.fknn_index_create(v.ctypes.data, l.ctypes.data, l.ctypes.data, 0, 100, byref(opts), byref(h)) == \
        fknn.FKNN_EINVAL
    assert lib.fknn_search(None, None, None, 1, 100, 0, None, None, None) == fknn.FKNN_EINVAL
    assert lib.fknn_index_destroy(None) == fknn.FKNN_OK


def test_no_cpu_fallback_without_a_device():
    """On a machine without a GPU the library reports ENODEV; it never answers
    from the host."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    v = np.zeros((8, 100), dtype=np.float32)
    l = np.zeros(8, dtype=np.float32)
    with pytest.raises(fknn.FknnError) as e:
        fknn.Index(v, l, l)
    assert e.value.code == _lib.FKNN_ENODEV
    with pytest.raises(fknn.FknnError):
        fknn.Bruteforce(np.zeros((8, 102), np.float32), np.zeros((1, 104), np.float32))


def test_graph_and_server_arguments_are_checked_without_a_device():
    """Malformed Graph::save bytes are rejected while parsing (before any
    device work); the request loop and the re-rank reject NULL arguments."""
    lib = fknn.load()
    vec = np.zeros((4, 100), dtype=np.float32)
    h = c_void_p()
    bad = np.array([0, 4, 2, 1, 2, -1, -1, 0, 0, 0, 0, 0, 0], dtype=np.int32)  # no eps, no initializer
    assert lib.fknn_graph_create(bad.ctypes.data, bad.nbytes, vec.ctypes.data, 0, byref(h)) == fknn.FKNN_EINVAL
    assert b"Graph::save" in lib.fknn_last_error()
    trunc = np.array([1, 0, 4, 2], dtype=np.int32)  # adjacency missing
    assert lib.fknn_graph_create(trunc.ctypes.data, trunc.nbytes, vec.ctypes.data, 0, byref(h)) == fknn.FKNN_EINVAL
    oob = np.concatenate([np.array([1, 0, 2, 1], np.int32), np.array([5, 0], np.int32),
                          np.zeros(2, np.float32).view(np.int32)])  # neighbour id 5 of a 2-point graph
    assert lib.fknn_graph_create(oob.ctypes.data, oob.nbytes, vec.ctypes.data, 0, byref(h)) == fknn.FKNN_EINVAL
    assert lib.fknn_graph_search(None, None, 1, 0, 10, 0, 10, None, None, None, None, None) == fknn.FKNN_EINVAL
    assert lib.fknn_server_create(None, None, byref(h)) == fknn.FKNN_EINVAL
    assert lib.fknn_server_submit(None, None, None, 1, None, None, None, None) == fknn.FKNN_EINVAL
    assert lib.fknn_rerank(None, None, 1, None, 10, 5, None, None, None) == fknn.FKNN_EINVAL
    t = _lib.Tuning(100, 0, 0, 0, 0)  # list_slack below 256
    assert lib.fknn_index_set_tuning(None, 1, byref(t)) == fknn.FKNN_EINVAL
