"""Build libsimd2.so in-tree with nvcc for sm_100a.

    python -m simd2_b200.build        (or simd2_b200.build.build())

The library is a plain C-ABI shared object (include/simd2.h); Python loads it
with ctypes.  Nothing here is compiled at import time on a GPU box: the built
.so travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsimd2.so")
SOURCES = ["capi.cu"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "-Xptxas", "-v",
]


def _newest_source_mtime() -> float:
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    paths.append(os.path.join(ROOT, "include", "simd2_cuasr.h"))
    paths.append(os.path.join(ROOT, "include", "simd2.h"))
    return max(os.path.getmtime(p) for p in paths if os.path.isfile(p))


def needs_build() -> bool:
    return not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest_source_mtime()


APP_SRC = os.path.join(HERE, "apps", "closure_app.cu")
APP = os.path.join(HERE, "apps", "simd2_closure_app")


def build_app(force: bool = False) -> str:
    """The drop-in closure app driver, linked against libsimd2.so."""
    build()
    if not force and os.path.exists(APP) and os.path.getmtime(APP) >= max(os.path.getmtime(APP_SRC),
                                                                              os.path.getmtime(LIB)):
        return APP
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), APP_SRC, "-o", APP + ".tmp",
           "-L", HERE, "-lsimd2", f"-Xlinker=-rpath,{HERE}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("building simd2_closure_app failed")
    os.replace(APP + ".tmp", APP)
    return APP


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-o", LIB + ".tmp",
           *[os.path.join(CSRC, s) for s in SOURCES]]
    res = subprocess.run(cmd, capture_output=True, text=True)
    log = os.path.join(HERE, "build.log")
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"nvcc failed (see {log})")
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
    print(build_app(force="--force" in sys.argv))
