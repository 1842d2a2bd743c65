"""In-tree build of libefl_b200.so (nvcc, sm_100a) and of the oracle.

The CUDA library is compiled with -fmad=false and IEEE division/square
root: the parity contract with the CPU oracle is bit-exactness wherever the
reference's arithmetic is not implementation-defined.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG_DIR)
CSRC = os.path.join(PKG_DIR, "csrc")
LIB_NAME = "libefl_b200.so"
LIB_PATH = os.path.join(PKG_DIR, LIB_NAME)

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden,-O2",
    "-shared",
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libefl_b200.so")


def sources() -> list[str]:
    return [os.path.join(CSRC, "efl_sim.cu")]


def deps() -> list[str]:
    out = []
    for d in (CSRC, os.path.join(REPO, "include")):
        for f in sorted(os.listdir(d)):
            if f.endswith((".cu", ".cuh", ".h", ".hpp")):
                out.append(os.path.join(d, f))
    return out


def needs_build(target: str, inputs: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in inputs)


def build_lib(force: bool = False, verbose: bool = True, extra: list[str] | None = None) -> str:
    if not force and not needs_build(LIB_PATH, deps() + [__file__]):
        return LIB_PATH
    cmd = [_nvcc(), *NVCC_FLAGS, *(extra or []), "-o", LIB_PATH, *sources()]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=PKG_DIR)
    return LIB_PATH


def build_oracle(force: bool = False, verbose: bool = True) -> str:
    """Builds oracle/liboracle_efl.so (test infrastructure) with make."""
    odir = os.path.join(REPO, "oracle")
    cmd = ["make", "-C", odir] + (["-B"] if force else [])
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return os.path.join(odir, "liboracle_efl.so")


if __name__ == "__main__":
    force = "--force" in sys.argv
    build_lib(force=force)
    build_oracle(force=force)
