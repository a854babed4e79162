"""Build the sm_100a library in-tree: fasttransforms_b200/_lib/libft_b200.so.

    python fasttransforms_b200/build.py      (by path: the package import loads the library)

nvcc compiles the CUDA kernels and the host plan code for sm_100a only and
links a shared library with a static CUDA runtime that exports only the C ABI
declared in include/ft_b200.h.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libft_b200.so")
BUILD_DIR = os.path.join(HERE, "_build")

SOURCES = ["rotations.cu", "trmm.cu", "blocked.cu", "trmm_mixed.cu", "grid.cu", "spin.cu", "rectdisk.cu", "tet.cu", "ann.cu", "column.cu", "api.cu", "noalloc.cu", "plan.cpp"]
CUDA_LIB = "/usr/local/cuda/lib64"   # cuFFT (grid synthesis / analysis), same path on every box of this image
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-ccbin", "/usr/bin/g++"]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(BUILD_DIR, exist_ok=True)
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD_DIR, src + ".o")
        deps = [path, os.path.join(CSRC, "ft_internal.h"), os.path.join(CSRC, "tc05.h"),
                os.path.join(HERE, os.pardir, "include", "ft_b200.h")]
        if not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(d) for d in deps):
            cmd = [NVCC, *ARCH, *COMMON, "-c", path, "-o", obj]
            if verbose and src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            if src.endswith(".cpp"):
                cmd = [NVCC, *ARCH, *COMMON, "-x", "c++", "-c", path, "-o", obj]
            _run(cmd)
        objs.append(obj)
    link = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static",
            "-Xlinker", "--version-script=" + os.path.join(CSRC, "exports.map"), "-Xlinker", "-Bsymbolic",
            "-L" + CUDA_LIB, "-lcufft", "-Xlinker", "-rpath=" + CUDA_LIB, "-lpthread"]
    _run(link)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
