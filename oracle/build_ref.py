"""Recipe that compiles the reference extension (Dolorousrtur/CCCollisions) from its own
sources, where they lie, into ``oracle/_ref/cccollisions.so``.

TEST INFRASTRUCTURE ONLY: the reference build is the second checker (it generates the
golden fixtures under tests/golden/ on a GPU).  Nothing in the product imports it.

    python oracle/build_ref.py [--src /path/to/reference]

The source checkout comes from ``--src``, else from the ``CCC_REFERENCE_SRC`` environment
variable, else from the checkout location of the machine this recipe was written on.

The reference's own build (setup.py + cuda-samples' helper_math.h) is not run.  Instead:
* ``oracle/ref_shim/helper_math.h`` (project-written) supplies the component-wise float
  vector operators the sources use;
* ``oracle/ref_shim/torch_compat.h`` (project-written, force-included) lets the sources'
  ``AT_DISPATCH_FLOATING_TYPES(t.type(), ...)`` compile against the current torch;
* ``-DAT_CHECK=TORCH_CHECK`` maps the removed AT_CHECK macro;
* nvcc flags are torch's CUDAExtension defaults (``--expt-relaxed-constexpr``, the
  ``__CUDA_NO_HALF*`` defines, default ``-fmad=true``) for sm_100.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SHIM = os.path.join(HERE, "ref_shim")
DEFAULT_SRC = os.environ.get("CCC_REFERENCE_SRC", "/root/reference")


def reference_src(src=None):
    """The reference checkout: the argument, else CCC_REFERENCE_SRC, else DEFAULT_SRC; None when
    that directory holds no ``src/`` (the product build then skips the checker)."""
    src = src or DEFAULT_SRC
    return src if os.path.isdir(os.path.join(src, "src")) else None


def build(src=DEFAULT_SRC, force=False) -> str:
    so = os.path.join(OUT, "cccollisions.so")
    if os.path.exists(so) and not force:
        return so
    if not os.path.isdir(os.path.join(src, "src")):
        raise FileNotFoundError(f"reference sources not found under {src}")
    import torch.utils.cpp_extension as ce
    os.makedirs(OUT, exist_ok=True)
    inc = ce.include_paths()
    py = sysconfig.get_paths()["include"]
    libdir = ce.library_paths()[0]
    common = ["-include", os.path.join(SHIM, "torch_compat.h"), f"-I{os.path.join(src, 'include')}", f"-I{SHIM}"]
    common += [f"-I{p}" for p in inc] + [f"-I{py}"]
    defs = ["-DTORCH_EXTENSION_NAME=cccollisions", "-DTORCH_API_INCLUDE_EXTENSION_H", "-D_GLIBCXX_USE_CXX11_ABI=1",
            "-DAT_CHECK=TORCH_CHECK"]
    nvcc = ["/usr/local/cuda/bin/nvcc", "-c", os.path.join(src, "src", "out.cu"), "-o", os.path.join(OUT, "out.o"),
            "-gencode", "arch=compute_100,code=sm_100", "-Xcompiler", "-fPIC", "-std=c++17",
            "-D__CUDA_NO_HALF_OPERATORS__", "-D__CUDA_NO_HALF_CONVERSIONS__", "-D__CUDA_NO_BFLOAT16_CONVERSIONS__",
            "-D__CUDA_NO_HALF2_OPERATORS__", "--expt-relaxed-constexpr", "-w"] + common + defs
    subprocess.check_call(nvcc)
    gxx = ["g++", "-c", os.path.join(src, "src", "cccollisions.cpp"), "-o", os.path.join(OUT, "cccollisions.o"),
           "-fPIC", "-std=c++17", "-O2", "-w", "-I/usr/local/cuda/include"] + common + defs
    subprocess.check_call(gxx)
    link = ["g++", "-shared", "-o", so, os.path.join(OUT, "out.o"), os.path.join(OUT, "cccollisions.o"),
            f"-L{libdir}", "-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu", "-ltorch_cuda", "-ltorch_python",
            "-L/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{libdir}"]
    subprocess.check_call(link)
    return so


def build_probe(src=DEFAULT_SRC, force=False) -> str:
    """oracle/_ref/libref_probe.so: oracle/ref_probe.cu + the reference sources (stage probe)."""
    so = os.path.join(OUT, "libref_probe.so")
    if os.path.exists(so) and not force:
        return so
    import torch.utils.cpp_extension as ce
    os.makedirs(OUT, exist_ok=True)
    inc = ce.include_paths()
    py = sysconfig.get_paths()["include"]
    libdir = ce.library_paths()[0]
    cmd = ["/usr/local/cuda/bin/nvcc", "-shared", "-Xcompiler", "-fPIC", "-o", so, os.path.join(HERE, "ref_probe.cu"),
           "-gencode", "arch=compute_100,code=sm_100", "-std=c++17", "-D__CUDA_NO_HALF_OPERATORS__",
           "-D__CUDA_NO_HALF_CONVERSIONS__", "-D__CUDA_NO_BFLOAT16_CONVERSIONS__", "-D__CUDA_NO_HALF2_OPERATORS__",
           "--expt-relaxed-constexpr", "-w", "-include", os.path.join(SHIM, "torch_compat.h"),
           f"-I{os.path.join(src, 'src')}", f"-I{os.path.join(src, 'include')}", f"-I{SHIM}", f"-I{py}",
           "-DTORCH_EXTENSION_NAME=ref_probe", "-D_GLIBCXX_USE_CXX11_ABI=1", "-DAT_CHECK=TORCH_CHECK"]
    cmd += [f"-I{p}" for p in inc]
    cmd += [f"-L{libdir}", "-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu", "-ltorch_cuda", f"-Xlinker",
            f"-rpath,{libdir}"]
    subprocess.check_call(cmd)
    return so


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=DEFAULT_SRC)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.src, a.force))
    print(build_probe(a.src, a.force))
