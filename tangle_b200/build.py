"""Builds libtangle_cuda.so, the sm_100a relaxation library, in-tree.

`-fmad=false` keeps nvcc from contracting a*b+c into FMA, and the default
IEEE division and square root stay on, so every kernel expression rounds as
written (the parity contract with the reference's f32 arithmetic).
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libtangle_cuda.so")
SOURCES = [os.path.join(HERE, "csrc", name) for name in ("kernels.cu", "world.cu", "noalloc.cu", "warmstart.cu", "capture.cu", "formation.cu")]
HEADERS = [os.path.join(HERE, "csrc", name) for name in ("common.cuh", "kernels.cuh", "contact.cuh", "umma_gemm.cuh", "umma_gemm_tma.cuh", "warmstart.cuh", "formation.cuh")] + [
    os.path.join(ROOT, "include", "tangle_cuda.h")
]


def nvcc() -> str:
    for candidate in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if candidate and os.path.exists(candidate):
            return candidate
    raise RuntimeError("nvcc not found")


def flags():
    return [
        "-gencode", "arch=compute_100a,code=sm_100a",
        "-O3", "-lineinfo", "-std=c++17",
        "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
        "--expt-relaxed-constexpr",
        "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
        "-Xptxas", "-v",
        "-shared",
    ]


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    built = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > built for p in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> str:
    if force or stale():
        cmd = [nvcc()] + flags() + ["-cudart", "static", "-o", LIB] + SOURCES
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + proc.stdout + proc.stderr)
        if verbose:
            sys.stderr.write(proc.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
