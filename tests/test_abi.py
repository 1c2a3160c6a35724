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
