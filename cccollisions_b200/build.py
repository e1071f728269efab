"""Build step for the native library (nvcc, sm_100a), in-tree.

    python -m cccollisions_b200.build

Produces ``cccollisions_b200/libccc_b200.so`` from ``csrc/ccc_capi.cu`` (the reference-format
operations), ``csrc/ccc_engine.cu`` (the resident multi-mesh engine) and
``csrc/ccc_narrow.cu`` (the continuous narrow phase), which share the kernel headers.  Flags:

* ``-gencode arch=compute_100a,code=sm_100a`` — B200 only;
* ``-fmad=false`` — no multiply-add contraction, so every floating-point expression rounds
  exactly as written (the CPU oracle is built with ``-ffp-contract=off`` to match), except
  in ``ccc_narrow.cu``, built with nvcc's default ``-fmad=true`` as the reference is, so that
  CUDA's pow computes what it computes in the reference's kernels (the library's own
  arithmetic there is written contraction-proof);
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
NARROW_SOURCE = "ccc_narrow.cu"
HEADERS = ["ccc_kernels.cuh", "ccc_engine.cuh", "ccc_runtime.cuh", "ccc_geom.cuh", "ccc_libm.h", "ccc_ddmul.h"]
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC"]
NVCC_FLAGS = COMMON + ["-fmad=false"]
NARROW_FLAGS = COMMON + ["-fmad=true"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + [NARROW_SOURCE] + HEADERS] + [os.path.join(ROOT, "include", h)
                                                                  for h in ("ccc_b200.h", "ccc_engine.h")]
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    tmp = LIB + ".tmp"
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    compiles, objs = [], []
    for f, flags in [(f, NVCC_FLAGS) for f in SOURCES] + [(NARROW_SOURCE, NARROW_FLAGS)]:
        o = os.path.join(objdir, f.replace(".cu", ".o"))
        compiles.append([nvcc()] + flags + ["-c", os.path.join(CSRC, f), "-o", o])
        objs.append(o)
    # the translation units compile in parallel, then link into the shared library
    procs = []
    for cmd in compiles:
        if verbose:
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd)))
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    link = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", tmp] + objs
    if verbose:
        print(" ".join(link))
    subprocess.check_call(link)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
