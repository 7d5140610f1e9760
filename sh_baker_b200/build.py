"""Builds libshb.so (the CUDA bake library) in-tree with nvcc for sm_100a.

Files whose arithmetic must round exactly like the CPU restatement of the
reference are compiled with -fmad=false; the traversal and BVH builder keep
FMA contraction (their exact steps use explicit rounding intrinsics).
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libshb.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
SOURCES = {
    "shb_capi.cu": ["-fmad=false"],
    "raster.cu": ["-fmad=false"],
    "shade.cu": ["-fmad=false"],
    "traverse.cu": ["-fmad=true"],
    "bvh_build.cu": ["-fmad=true"],
    "batch.cu": ["-fmad=false"],
    "exr.cu": ["-fmad=false"],
    "gltf.cpp": [],
    "tspace.cpp": [],
    "jpeg.cpp": [],
    "atlas.cpp": [],
    "preview.cu": ["-fmad=false"],
}
HEADERS = ["shb_internal.h", "shb_math.cuh", "wavefront.h", "tspace.h"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _newer(out: Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False, variant: str | None = None, defines=(),
          file_flags=None) -> Path:
    """Builds libshb.so.  A `variant` builds the same sources with extra
    preprocessor `defines` (tuning options such as SHB_NEE_BLOCKS_PER_SM=2)
    and per-file nvcc flags (`file_flags`, e.g. {"shade.cu": ["-fmad=true"]},
    appended after the file's own) into _build_<variant>/libshb.so, loaded
    through $SHB_LIBRARY."""
    file_flags = file_flags or {}
    build_dir = BUILD if variant is None else PKG / f"_build_{variant}"
    lib = LIB if variant is None else build_dir / "libshb.so"
    build_dir.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [PKG.parent / "include" / "shb.h"]
    objs, cmds = [], []
    dflags = [f"-D{d}" for d in defines]
    for src, flags in SOURCES.items():
        s = CSRC / src
        o = build_dir / (src + ".o")
        objs.append(o)
        if force or _newer(o, [s, *headers, Path(__file__)]):
            cmds.append([nvcc(), *ARCH, *COMMON, *flags, *file_flags.get(src, []), *dflags, "-c", str(s), "-o", str(o)])
    if cmds:
        from concurrent.futures import ThreadPoolExecutor

        def run(cmd):
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)

        with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as pool:
            for f in [pool.submit(run, c) for c in cmds]:
                f.result()
    if force or _newer(lib, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(lib), *map(str, objs), "-lz", "-Xlinker", "--no-undefined"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if variant is None:
        build_cli(verbose, force)
    return lib


CLI = PKG / "bin" / "sh_baker"
CVT = PKG / "bin" / "sh_cvt"


def build_cli(verbose: bool = False, force: bool = False) -> Path:
    """The command lines (the reference's sh_baker and sh_cvt, same flags)
    linked to libshb.so."""
    CLI.parent.mkdir(exist_ok=True)
    for exe in (CLI, CVT):
        src = PKG / "cli" / (exe.name + ".cpp")
        if force or _newer(exe, [src, LIB, PKG.parent / "include" / "shb.h", Path(__file__)]):
            cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", str(PKG.parent / "include"), str(src), "-L", str(PKG),
                   "-lshb", "-Wl,-rpath,$ORIGIN/..", "-o", str(exe)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    return CLI


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
