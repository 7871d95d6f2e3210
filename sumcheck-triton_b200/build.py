"""Builds libsumcheck_b200.so (sm_100a) in-tree, next to the Python package.

    python sumcheck-triton_b200/build.py [--verbose]

nvcc cross-compiles for sm_100a without a GPU. The library has no torch dependency: the
Python package loads it with ctypes. The field arithmetic header is regenerated first when
its generator is newer.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "zkduel_b200" / "libsumcheck_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared"]


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> Path:
    gen = CSRC / "gen_field_ptx.py"
    hdr = CSRC / "field_ptx.cuh"
    if _stale(hdr, [gen]):
        subprocess.check_call([sys.executable, str(gen)])
    sources = [CSRC / "capi.cu", CSRC / "batch.cu", CSRC / "noalloc.cu"]
    deps = sources + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [PKG.parent / "include" / "sumcheck_b200.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *ARCH, *FLAGS, *(["-Xptxas", "-v"] if verbose else []), *map(str, sources), "-o", str(LIB)]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force="--force" in sys.argv))
