"""Builds the oracle (test infrastructure) into oracle/_build/libcone_oracle.so.

The oracle is the checker: only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline arm load it. It is compiled without floating-point contraction so
FP32 results are plain IEEE single-precision operations.

The reference (Rust + WGSL) cannot be compiled here: there is no Rust
toolchain and no graphics stack, so there is no oracle/_ref build.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "cone_oracle.cpp"
OUT = HERE / "_build" / "libcone_oracle.so"


def build(force: bool = False) -> Path:
    if not force and OUT.exists() and OUT.stat().st_mtime >= SRC.stat().st_mtime:
        return OUT
    OUT.parent.mkdir(exist_ok=True)
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-pthread",
           "-o", str(tmp), str(SRC)]
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
