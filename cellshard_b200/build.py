"""Builds libcellshard_b200.so in-tree from cellshard_b200/csrc/*.cu.

nvcc cross-compiles for sm_100a only (B200); the CUDA runtime is linked
statically so the library does not depend on which libcudart a host process
(for example torch) has already loaded.  Objects go to cellshard_b200/_build/
and are rebuilt when their source or any shared header is newer.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libcellshard_b200.so"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC,-O3,-fvisibility=hidden",
    "-Xptxas",
    "-O3",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libcellshard_b200")


def _headers() -> list[Path]:
    return list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    header_mtime = max((h.stat().st_mtime for h in _headers()), default=0.0)
    objects = []
    for src in sources:
        obj = BUILD / (src.stem + ".o")
        objects.append(obj)
        if obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, header_mtime) and not ptxas_info:
            continue
        cmd = [nvcc(), *ARCH_FLAGS, *NVCC_FLAGS, "-I", str(ROOT / "include"), "-c", str(src), "-o", str(obj)]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    newest = max(o.stat().st_mtime for o in objects)
    if not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [nvcc(), *ARCH_FLAGS, "-shared", "--cudart", "static", "-o", str(LIB), *map(str, objects),
               "-lpthread", "-ldl", "-lrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas-info" in sys.argv)
    print(LIB)
