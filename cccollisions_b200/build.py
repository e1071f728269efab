"""Build step for the native library (nvcc, sm_100a), in-tree.

    python -m cccollisions_b200.build

Produces ``cccollisions_b200/libccc_b200.so`` from ``csrc/ccc_capi.cu`` (the reference-format
operations) and ``csrc/ccc_engine.cu`` (the resident multi-mesh engine), which share the
kernel headers.  Flags:

* ``-gencode arch=compute_100a,code=sm_100a`` — B200 only;
* ``-fmad=false`` — no multiply-add contraction, so every floating-point expression rounds
  exactly as written (the CPU oracle is built with ``-ffp-contract=off`` to match);
* ``-lineinfo`` for profiler source correlation.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libccc_b200.so")
SOURCES = ["ccc_capi.cu", "ccc_engine.cu"]
HEADERS = ["ccc_kernels.cuh", "ccc_engine.cuh", "ccc_runtime.cuh", "ccc_geom.cuh", "ccc_libm.h", "ccc_ddmul.h"]
ROOT = os.path.dirname(HERE)

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-fmad=false", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", h)
                                                                  for h in ("ccc_b200.h", "ccc_engine.h")]
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", tmp] + [os.path.join(CSRC, f) for f in SOURCES]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
