"""Builds libcontinuum_cuda.so in-tree (continuum_b200/lib/) with nvcc for sm_100a.

Usage: python -m continuum_b200.build [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "libcontinuum_cuda.so"
INCLUDE = PKG.parent / "include"

SOURCES = ["visibility.cu", "visibility_splat.cu", "visibility_split.cu", "order.cu", "capi.cu", "batch.cu", "server.cu", "movers.cu", "cache.cu", "static_scratch.cu", "bvh.cpp",
           "raycast.cpp", "cache_plan.cpp"]
# The cone geometry is evaluated without fused multiply-adds: the reference's
# clip and cull decisions are ill-conditioned in f32 for receivers lifted
# 1e-4 off curved surfaces (the plane through the apex and a near edge),
# and contracting a*b+c there changes which side a vertex falls on. Plain
# IEEE multiplies and adds (with IEEE division and square root, nvcc's
# defaults) reproduce the reference arithmetic's rounding.
PER_SOURCE = {"visibility.cu": ["-fmad=false"], "visibility_splat.cu": ["-fmad=false"], "visibility_split.cu": ["-fmad=false"]}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "-Xcompiler", "-fvisibility=hidden",
              "--cudart", "static", "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or Path(cand).exists()):
            return cand
    return "nvcc"


def _inputs() -> list[Path]:
    files = [CSRC / s for s in SOURCES]
    files += sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [INCLUDE / "continuum_cuda.h"]
    return files


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(f.stat().st_mtime <= t for f in _inputs())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    LIB_DIR.mkdir(exist_ok=True)
    objs = []
    obj_dir = PKG / "_build"
    obj_dir.mkdir(exist_ok=True)
    for src in SOURCES:
        obj = obj_dir / (src + ".o")
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *PER_SOURCE.get(src, []), "-I", str(INCLUDE), "-c", str(CSRC / src),
               "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "--cudart", "static", "-o", str(tmp), *objs, "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
