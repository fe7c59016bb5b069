"""Build the in-tree CUDA library ``gegs_b200/libgegs_b200.so`` for sm_100a.

The library is compiled with ``-fmad=false`` (no FMA contraction) and IEEE
division / square root, which together with the library's own transcendental
functions makes every particle history reproducible bit for bit.
"""
from __future__ import annotations

import os
import pathlib
import subprocess

PKG = pathlib.Path(__file__).resolve().parent
SRC = PKG / "csrc"
INC = PKG.parent / "include"
LIB = PKG / "libgegs_b200.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC", "-shared",
]


def sources():
    return sorted(list(SRC.glob("*.cu")) + list(SRC.glob("*.cuh")) + list(SRC.glob("*.cpp")) + list(SRC.glob("*.h"))
                  + list(INC.glob("*.h")))


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources())


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    if not force and not needs_build():
        return LIB
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    cmd = [nvcc, *NVCC_FLAGS, "-Xcompiler", "-ffp-contract=off", "-o", str(LIB), str(SRC / "engine.cu"),
           str(SRC / "postproc.cu"), str(SRC / "plan_host.cpp")]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    tmp = LIB.with_suffix(".so.tmp")
    cmd[cmd.index(str(LIB))] = str(tmp)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    import sys
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
