"""Build libspgemm_b200.so in-tree with nvcc for sm_100a.

Every translation unit is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked into one
shared library next to this file. The CUDA runtime is linked statically, so the
library carries its own runtime and shares device memory with any other
runtime in the process through the driver's primary context.

Usage: ``python -m spgemm_b200.build`` (or ``build()`` from Python).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "libspgemm_b200.so"

SOURCES = [
    "engine.cu",
    "batch.cu",
    "coo_sort.cu",
    "api.cu",
    "legacy_mm.cu",
    "host_coo.cpp",
    "host_mtx.cpp",
    "host_cm.cpp",
    "host_legacy.cpp",
    "legacy_spgemm.cu",
    "noalloc.cu",
]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-Wall", f"-I{INCLUDE}"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _deps(src: Path) -> list[Path]:
    return [src] + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compile stale objects and relink the library; returns its path."""
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    objs = []
    for name in SOURCES:
        src = CSRC / name
        if not src.exists():
            continue
        obj = BUILD / (name + ".o")
        objs.append(obj)
        if force or _stale(obj, _deps(src)):
            cmd = [nvcc, *ARCH, *COMMON, "-c", str(src), "-o", str(obj)]
            if src.suffix == ".cpp":
                cmd = [nvcc, *ARCH, *COMMON, "-x", "c++", "-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB),
               *map(str, objs), "-lpthread", "-ldl", "-lrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    print(LIB)
