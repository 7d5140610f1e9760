"""Generates tests/golden/exr_reference.npz: a crafted SH lightmap and what
the reference's own EXR writer path (src/saver.cpp:108-401 restated over the
reference's vendored tinyexr, oracle/_ref/libexr_ref.so) stores for it in
each SaveMode, as read back by the reference's own reader (tinyexr).

The texture is 37 x 21 texels (two ZIP chunks, the second partial) with
seeded random coefficients plus the values where float -> half rounding
differs between rules: exact half-way mantissas, the half overflow edge
(65504 / 65519.99 / 65520), half denormals and their rounding, float
denormals, +-0, +-inf and NaN.

Run from the repository root: python tests/golden/make_exr_golden.py
"""
import ctypes as C
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import build as ob  # noqa: E402
from oracle import exr_read  # noqa: E402

W, H = 37, 21
FILES = {0: ["lightmap.exr"],
         1: [f"lightmap_{n}.exr" for n in ("L0", "L1m1", "L10", "L11", "L2m2", "L2m1", "L20", "L21", "L22")],
         2: [f"lightmap_packed_{k}.exr" for k in range(3)]}


def crafted_texture():
    rng = np.random.default_rng(20241203)
    sh = (rng.standard_normal((H * W, 27)) * rng.choice([1e-4, 1e-2, 1.0, 30.0, 3e3], (H * W, 27))).astype(np.float32)
    env = rng.uniform(0, 1, H * W).astype(np.float32)
    f32 = np.float32
    special = np.array([0.0, -0.0, 1.0 + 2.0 ** -11, 1.0 + 3 * 2.0 ** -11, -(1.0 + 2.0 ** -11), 65504.0, 65519.99,
                        65520.0, -65520.0, 1e5, 2.0 ** -24, 2.0 ** -25, 3 * 2.0 ** -26, 2.0 ** -14, 2.0 ** -15 * 1.5,
                        1e-40, -1e-40, np.inf, -np.inf, np.nan, 0.5 + 2.0 ** -12, 1024.5, 2049.0, 6.1e-5],
                       dtype=f32)
    flat = sh.reshape(-1)
    flat[:special.size] = special
    flat[27 * 5:27 * 5 + special.size] = -special
    env[:4] = [0.0, 1.0, 0.5 + 2.0 ** -12, np.nan]
    return sh, env


def load_ref():
    lib = C.CDLL(str(ob.build_ref()))
    lib.ref_exr_save.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_char_p, C.c_int]
    lib.ref_exr_load.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.c_void_p, C.c_void_p]
    return lib


def tinyexr_read(lib, path, max_ch=32):
    w, h = C.c_int(), C.c_int()
    names = C.create_string_buffer(256 * max_ch)
    halves = np.zeros((max_ch, H, W), np.uint16)
    n = lib.ref_exr_load(str(path).encode(), C.byref(w), C.byref(h), max_ch, names, halves.ctypes.data)
    assert n > 0 and (w.value, h.value) == (W, H)
    nm = [names.raw[256 * c:256 * (c + 1)].split(b"\0")[0].decode() for c in range(n)]
    return nm, halves[:n]


def reference_files(lib, sh, env, mode, out_dir):
    path = Path(out_dir) / "lightmap.exr"
    assert lib.ref_exr_save(sh.ctypes.data, env.ctypes.data, W, H, str(path).encode(), mode) == 0
    return [Path(out_dir) / f for f in FILES[mode]]


def main():
    lib = load_ref()
    sh, env = crafted_texture()
    out = {"sh": sh, "env": env}
    with tempfile.TemporaryDirectory() as d:
        for mode in (0, 1, 2):
            md = Path(d) / str(mode)
            md.mkdir()
            for f in reference_files(lib, sh, env, mode, md):
                names, halves = tinyexr_read(lib, f)
                ex = exr_read.read(f)
                key = f"m{mode}_{f.stem}"
                out[key + "_names"] = np.array(names)
                out[key + "_halves"] = halves
                out[key + "_attr_names"] = np.array([n for n, _, _ in ex.attributes])
                out[key + "_attr_types"] = np.array([t for _, t, _ in ex.attributes])
                out[key + "_attr_values"] = np.array([v.hex() for _, _, v in ex.attributes])
    np.savez_compressed(Path(__file__).with_name("exr_reference.npz"), **out)


if __name__ == "__main__":
    main()
