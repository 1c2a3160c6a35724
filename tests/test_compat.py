"""include/fknn_compat.hpp: the reference's C++ entry points (Bruteforce,
bruteforce, HybridGraph::BatchSearch) over the C ABI.  The header compiles
here; tests/compat_main.cpp runs it on the GPU against a CPU restatement."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "sigmod-2024-contest_b200", "fknn")


def _build(tmp_path):
    exe = str(tmp_path / "compat_main")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "compat_main.cpp"), "-L", LIBDIR, "-lfknn",
                    f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True, capture_output=True, text=True)
    return exe


def test_compat_header_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_compat_shims_match_reference_semantics(tmp_path):
    r = subprocess.run([_build(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("OK"), r.stdout + r.stderr
