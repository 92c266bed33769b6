"""In-tree build of ``libbug_b200.so`` for sm_100a (nvcc cross-compiles without a GPU)."""

from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("engine.cu", "kernels.cu", "step.cu", "noalloc.cu", "server.cu")]
OUTPUT = os.path.join(HERE, "libbug_b200.so")
NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fcx-limited-range",
              "-Xcompiler", "-fPIC", "-shared"]


def needs_build() -> bool:
    if not os.path.exists(OUTPUT):
        return True
    t = os.path.getmtime(OUTPUT)
    deps = SOURCES + [os.path.join(HERE, "csrc", f) for f in ("kernels.cuh", "engine.h", "smallla.h")] + [
                      os.path.join(os.path.dirname(HERE), "include", "bug_b200.h")]
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force: bool = False, verbose: bool = False) -> str:
    if force or needs_build():
        cmd = ["nvcc", *NVCC_FLAGS, *SOURCES, "-o", OUTPUT]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return OUTPUT


if __name__ == "__main__":
    build(force=True, verbose=True)
