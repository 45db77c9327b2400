"""Build recipe for the CPU oracle (test infrastructure): oracle/liboracle.so.

    python -m oracle.build [--force]
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
SRCS = [HERE / "gv_oracle.cpp"]
DEPS = SRCS + [HERE / "gv_oracle.h", HERE.parent / "gv_b200" / "csrc" / "rmat.h"]


def build(force: bool = False) -> Path:
    if not force and LIB.exists() and all(p.stat().st_mtime <= LIB.stat().st_mtime for p in DEPS):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = ["g++", "-O3", "-march=x86-64-v3", "-std=c++17", "-fopenmp", "-fPIC", "-shared",
           *map(str, SRCS), "-o", str(tmp)]
    subprocess.run(cmd, check=True)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
