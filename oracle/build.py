"""Builds the CPU oracle (test infrastructure) into oracle/liboracle.so.

The reference itself (Embree, TBB, Eigen, glog) cannot be compiled in this
image, so oracle/_ref is not produced; the oracle is a restatement."""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "shb_oracle.cpp"
LIB = HERE / "liboracle.so"


def build(verbose: bool = False, force: bool = False) -> Path:
    deps = [SRC, HERE / "shb_oracle.h", HERE.parent / "include" / "shb.h", Path(__file__)]
    if force or not LIB.exists() or any(d.stat().st_mtime > LIB.stat().st_mtime for d in deps):
        cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-pthread",
               str(SRC), "-o", str(LIB)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
