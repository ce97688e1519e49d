"""Build recipe of the CUDA library (sm_100a) and of the CPU oracle.

``python -m mfix_b200.build`` compiles every ``csrc/*.cu`` with nvcc for
``sm_100a`` into ``mfix_b200/libmfixgpu.so`` (in-tree, so the built library
travels with the source tree) and runs ``make -C oracle`` for the oracle's
shared library, which only the tests and the benchmark's CPU leg load.
Objects are rebuilt when a source or header is newer than the library.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmfixgpu.so")
BUILD_DIR = os.path.join(ROOT, "_build")

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-diag-suppress", "177"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(verbose: bool = False) -> str:
    nvcc = _nvcc()
    os.makedirs(BUILD_DIR, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) +
                     glob.glob(os.path.join(ROOT, "include", "*.h")))
    objects = []
    for src in sources:
        obj = os.path.join(BUILD_DIR, os.path.basename(src) + ".o")
        objects.append(obj)
        if _stale(obj, [src] + headers):
            cmd = [nvcc, *ARCH_FLAGS, *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if _stale(LIB, objects):
        cmd = [nvcc, *ARCH_FLAGS, "-shared", "-Xcompiler", "-fPIC", "-o", LIB, *objects, "-lpthread"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


def build_oracle(verbose: bool = False) -> str:
    out = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True,
                         capture_output=not verbose, text=True)
    del out
    return os.path.join(ROOT, "oracle", "liboracle_leq.so")


def main() -> None:
    verbose = "-v" in sys.argv
    print(build_library(verbose))
    print(build_oracle(verbose))


if __name__ == "__main__":
    main()
