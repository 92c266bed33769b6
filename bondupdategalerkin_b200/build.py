"""In-tree build of ``libbug_b200.so`` for sm_100a (nvcc cross-compiles without a GPU).

Each translation unit compiles to its own object in ``_build/`` (in parallel), and one link step
makes the shared library next to this file, where the loader and the GPU box find it.
"""

from __future__ import annotations

import os
import subprocess
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
UNITS = ("engine.cu", "kernels.cu", "step.cu", "noalloc.cu", "server.cu", "tcgemm.cu")
SOURCES = [os.path.join(HERE, "csrc", f) for f in UNITS]
HEADERS = ("kernels.cuh", "engine.h", "smallla.h", "tcgemm.cuh")
OUTPUT = os.path.join(HERE, "libbug_b200.so")
OBJDIR = os.path.join(os.path.dirname(HERE), "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Host code: hardware FMA for the explicit std::fma of the Krylov-weight and small dense kernels
# (without it each is a libm call), and no contraction of other a*b+c, so every other host result
# keeps the rounding of plain multiplies and adds.
NVCC_FLAGS = ["-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-mfma,-ffp-contract=off"]


def _deps():
    return [os.path.join(HERE, "csrc", f) for f in HEADERS] + [
        os.path.join(os.path.dirname(HERE), "include", "bug_b200.h")]


def needs_build() -> bool:
    if not os.path.exists(OUTPUT):
        return True
    t = os.path.getmtime(OUTPUT)
    return any(os.path.getmtime(p) > t for p in SOURCES + _deps() if os.path.exists(p))


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OBJDIR, os.path.basename(src).replace(".cu", ".o"))
    cmd = ["nvcc", *NVCC_FLAGS, "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    if force or needs_build():
        os.makedirs(OBJDIR, exist_ok=True)
        srcs = [s for s in SOURCES if os.path.exists(s)]
        with ThreadPoolExecutor(max_workers=len(srcs)) as ex:
            objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
        cmd = ["nvcc", *ARCH, "-shared", *objs, "-o", OUTPUT]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUTPUT


if __name__ == "__main__":
    build(force=True, verbose=True)
