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
DEFAULT_LIB = PKG / "zkduel_b200" / "libsumcheck_b200.so"
LIB = Path(os.environ.get("SC_LIB_OUT", DEFAULT_LIB))
OBJ = Path(os.environ.get("SC_BUILD_DIR", PKG / "_build"))
CLI = PKG / "bin" / "field_sumcheck_b200"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC"]
SOURCES = ["capi.cu", "batch.cu", "noalloc.cu", "serve.cu", "split.cu"]


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
    gen_w = CSRC / "gen_workload_table.py"
    hdr_w = CSRC / "workload_table.h"
    if _stale(hdr_w, [gen_w, PKG / "zkduel_b200" / "workloads.py", PKG / "zkduel_b200" / "fields.py"]):
        subprocess.check_call([sys.executable, str(gen_w)])
    sources = [CSRC / s for s in SOURCES]
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [PKG.parent / "include" / "sumcheck_b200.h"]
    if not force and not _stale(LIB, sources + headers):
        if LIB == DEFAULT_LIB:
            build_cli(os.environ.get("NVCC", "nvcc"))
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    OBJ.mkdir(exist_ok=True)
    # one nvcc per translation unit, in parallel; then one link
    procs = []
    for src in sources:
        obj = OBJ / (src.stem + ".o")
        if not force and not _stale(obj, [src] + headers):
            continue
        extra = os.environ.get("SC_NVCC_FLAGS", "").split()
        cmd = [nvcc, *ARCH, *FLAGS, *extra, *(["-Xptxas", "-v"] if verbose else []), "-c", str(src), "-o", str(obj)]
        procs.append((src, subprocess.Popen(cmd)))
    failed = [str(src) for src, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, f"nvcc {' '.join(failed)}")
    objs = [str(OBJ / (src.stem + ".o")) for src in sources]
    subprocess.check_call([nvcc, *ARCH, "-shared", *objs, "-o", str(LIB)])
    if LIB == DEFAULT_LIB:  # the command-line tool links the package's own library only
        build_cli(nvcc)
    return LIB


def build_cli(nvcc: str = "nvcc") -> Path:
    """The reference executable's command line over this library (cli/field_sumcheck_b200.cpp)."""
    src = PKG / "cli" / "field_sumcheck_b200.cpp"
    if not CLI.parent.exists():
        CLI.parent.mkdir(parents=True)
    if _stale(CLI, [src, LIB, CSRC / "workload_table.h", PKG.parent / "include" / "sumcheck_b200.h"]):
        rpath = "$ORIGIN/" + os.path.relpath(LIB.parent, CLI.parent)
        subprocess.check_call([nvcc, *ARCH, "-O2", "-std=c++17", str(src), "-o", str(CLI), "-L", str(LIB.parent),
                               "-l" + LIB.stem[3:], "-Xlinker", "-rpath", "-Xlinker", rpath])
    return CLI


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force="--force" in sys.argv))
