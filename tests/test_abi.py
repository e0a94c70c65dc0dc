"""The C ABI on a CPU-only machine: every declared entry point is exported,
the library loads, and the reference-compatible shim header compiles."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

from simd2_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in ("simd2.h",)]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^(?:const\s+char\s*\*|int|long long|void)\s+(simd2_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


@pytest.fixture(scope="module")
def lib():
    path = build.build()
    return ctypes.CDLL(path)


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 25, names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_version(lib):
    lib.simd2_status_string.restype = ctypes.c_char_p
    lib.simd2_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.simd2_version()
    for code in range(9):
        assert lib.simd2_status_string(code) != b"unknown status"


def test_argument_checks_need_no_gpu(lib):
    # invalid arguments are rejected before any CUDA call
    assert lib.simd2_srgemm(99, 1, 1, 1, None, 1, None, 1, None, 1, None, 1, 0, None) == 1
    assert lib.simd2_srgemm(0, -1, 1, 1, None, 1, None, 1, None, 1, None, 1, 0, None) == 1
    assert lib.simd2_srgemm(0, 0, 5, 5, None, 5, None, 5, None, 5, None, 5, 0, None) == 0  # empty problem
    assert lib.simd2_knn(None, 4, 4, None, 4, 4, 4, 0, None, None, 4, None) == 1  # k = 0


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not available")
def test_shim_header_compiles(tmp_path):
    out = tmp_path / "app.o"
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-I", os.path.join(ROOT, "include"),
           "-c", os.path.join(ROOT, "tests", "compat", "cuasr_app.cu"), "-o", str(out)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr


def test_dense_configs_table_arguments(lib):
    """simd2_set_dense_configs validates its table (ascending sizes, configs
    0..3 without block skipping) without touching the GPU; an empty table
    restores the rule."""
    L = lib
    L.simd2_set_dense_configs.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    L.simd2_set_dense_configs.restype = ctypes.c_int
    arr = lambda *v: (ctypes.c_int * len(v))(*v)
    assert L.simd2_set_dense_configs(arr(2048, 4096), arr(0, 1), 2) == 0
    assert L.simd2_set_dense_configs(arr(4096, 2048), arr(0, 1), 2) == 1   # not ascending
    assert L.simd2_set_dense_configs(arr(2048), arr(4), 1) == 1             # a skip config
    assert L.simd2_set_dense_configs(arr(0), arr(1), 1) == 1                # size below 1
    assert L.simd2_set_dense_configs(None, None, -1) == 1
    assert L.simd2_set_dense_configs(None, None, 0) == 0
