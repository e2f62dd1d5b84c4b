"""Build recipe for the in-tree CUDA library (sm_100a only).

    python -m eu3d_b200.build

produces eu3d_b200/libeu3d_gpu.so from eu3d_b200/csrc/eu3d_gpu.cu with
nvcc -gencode arch=compute_100a,code=sm_100a.  The library is loaded from the
package directory by eu3d_b200.gpu; there is no CPU fallback.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libeu3d_gpu.so")
SRC_DIR = os.path.join(HERE, "csrc")
MAIN_SRC = os.path.join(SRC_DIR, "eu3d_gpu.cu")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-shared", "--expt-relaxed-constexpr",
]


def sources():
    out = []
    for d in (SRC_DIR, INCLUDE):
        for f in sorted(os.listdir(d)):
            if f.endswith((".cu", ".cuh", ".h", ".hpp")):
                out.append(os.path.join(d, f))
    return out


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(s) > t for s in sources())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + [MAIN_SRC, "-o", LIB + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
