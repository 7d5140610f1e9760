"""Builds the CPU oracle (test infrastructure) into oracle/liboracle.so.

The reference's bake path (Embree, TBB, Eigen, glog) cannot be compiled in
this image; the oracle is a restatement.  The reference's vendored EXR
library (src/tinyexr_impl.cpp + src/miniz.c) does compile: build_ref()
compiles it where it lies in the reference tree, together with
oracle/exr_ref_harness.cpp, into oracle/_ref/libexr_ref.so (only when the
reference tree is present).  The reference's `src` folder is
$SHB_REFERENCE_SRC, else `reference/src` beside this repository's folder."""
from __future__ import annotations

import os
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


REF_SRC = Path(os.environ.get("SHB_REFERENCE_SRC", str(HERE.parent.parent / "reference" / "src")))
REF_DIR = HERE / "_ref"
REF_LIB = REF_DIR / "libexr_ref.so"


def build_ref(verbose: bool = False, force: bool = False):
    """oracle/_ref/libexr_ref.so from the reference's tinyexr + miniz and the
    harness; returns its path, or None when the reference tree is absent."""
    if not (REF_SRC / "tinyexr.h").exists():
        return REF_LIB if REF_LIB.exists() else None
    harness = HERE / "exr_ref_harness.cpp"
    deps = [harness, REF_SRC / "tinyexr.h", REF_SRC / "miniz.c", Path(__file__)]
    if force or not REF_LIB.exists() or any(d.stat().st_mtime > REF_LIB.stat().st_mtime for d in deps):
        REF_DIR.mkdir(exist_ok=True)
        mz = REF_DIR / "miniz.o"
        cmds = [["gcc", "-O2", "-fPIC", "-w", "-c", str(REF_SRC / "miniz.c"), "-o", str(mz)],
                ["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-w", "-shared", "-I", str(REF_SRC),
                 str(harness), str(REF_SRC / "tinyexr_impl.cpp"), str(mz), "-o", str(REF_LIB)]]
        for cmd in cmds:
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    return REF_LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    build_ref(verbose=True, force="--force" in sys.argv)
