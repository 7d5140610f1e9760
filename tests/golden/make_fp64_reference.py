"""Generates the FP64 oracle references used by the accuracy tests.

For each workload a crop of the output lightmap (supersample 3) is baked by
the CPU oracle in double precision at 4096 samples per supersampled texel
(Philox stream, seed 987654, independent of every GPU seed), then
box-downsampled like the pipeline.  The crops are lit regions, chosen by a
quick low-spp bake of candidate crops: the lightmaps' corners are dim
enough that 4096 samples still leave much of the signal as noise there.
Written as float32 to tests/golden/fp64_<workload>.npz with the crop
position and per-texel standard errors.

The atrium crop is the 256 x 256 output texels the atrium workload names.
It contains the 128 x 128 crop of an earlier fixture: with --grow, output
texels that an existing fixture of the same scene, seed, spp and bounces
already holds are taken from it (the counter-based stream is keyed by the
global texel index, so they are the values a full run computes) and only
the rest are baked.

    python tests/golden/make_fp64_reference.py [--grow] [--threads N] [room|atrium ...]
"""
from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import pyoracle as O  # noqa: E402
from sh_baker_b200 import scenes  # noqa: E402

CROPS = {
    # workload: (scene factory, width, height, ss, bounces, crop x0, crop y0, crop size)
    "room": (lambda: scenes.procedural_room(seed=2, res=1024), 1024, 1024, 3, 3, 384, 128, 64),
    "atrium": (lambda: scenes.atrium(seed=3, res=2048), 2048, 2048, 3, 4, 448, 192, 256),
}
SPP = 4096
SEED = 987654


def crop_indices(W, ss, x0, y0, size):
    ys, xs = np.meshgrid(np.arange(y0 * ss, (y0 + size) * ss), np.arange(x0 * ss, (x0 + size) * ss), indexing="ij")
    return (ys * (W * ss) + xs).reshape(-1)


def reusable(path, w, h, ss, bounces, x0, y0, size):
    """Output texels of an existing fixture at `path` that lie in the new
    crop, as (sh, se, valid, known-mask) in the new crop's frame; None when
    the fixture is absent or was made with other settings."""
    if not path.exists():
        return None
    d = np.load(path)
    same = (int(d["width"]), int(d["height"]), int(d["ss"]), int(d["bounces"]), int(d["spp"]), int(d["seed"])) == \
        (w, h, ss, bounces, SPP, SEED)
    if not same:
        return None
    ox, oy, os_ = int(d["x0"]) - x0, int(d["y0"]) - y0, int(d["size"])
    if ox < 0 or oy < 0 or ox + os_ > size or oy + os_ > size:
        return None
    sh = np.zeros((size, size, 27), np.float32)
    se = np.zeros((size, size, 27), np.float32)
    valid = np.zeros((size, size), bool)
    known = np.zeros((size, size), bool)
    sh[oy:oy + os_, ox:ox + os_] = d["sh"]
    se[oy:oy + os_, ox:ox + os_] = d["se"]
    valid[oy:oy + os_, ox:ox + os_] = d["valid"]
    known[oy:oy + os_, ox:ox + os_] = True
    return sh, se, valid, known, float(d["seconds"]), int(d["rays"])


def make(name, grow=False, threads=0):
    make_scene, w, h, ss, bounces, x0, y0, size = CROPS[name]
    out = Path(__file__).parent / f"fp64_{name}.npz"
    prev = reusable(out, w, h, ss, bounces, x0, y0, size) if grow else None
    sc = make_scene()
    osc = O.OracleScene(sc)
    pts = osc.rasterize(w, h, ss)
    known = prev[3] if prev else np.zeros((size, size), bool)
    # supersampled texels of the output texels still to bake
    oy, ox = np.nonzero(~known)
    sub_y = (y0 + oy)[:, None, None] * ss + np.arange(ss)[None, :, None]
    sub_x = (x0 + ox)[:, None, None] * ss + np.arange(ss)[None, None, :]
    idx = (sub_y * (w * ss) + sub_x).reshape(-1)
    t0 = time.time()
    r = osc.bake(pts, w, h, ss, samples=SPP, bounces=bounces, seed=SEED, rng=O.RNG_PHILOX, fp64=True, subset=idx,
                 stats=True, threads=threads)
    dt = time.time() - t0
    m64 = r["mean64"].reshape(-1, 27)[idx].reshape(-1, ss * ss, 27)
    var = r["var"].reshape(-1, 27)[idx].reshape(-1, ss * ss, 27)
    valid_sub = (pts["material_id"][idx] >= 0).reshape(-1, ss * ss)
    sh = prev[0] if prev else np.zeros((size, size, 27), np.float32)
    se = prev[1] if prev else np.zeros((size, size, 27), np.float32)
    vmask = prev[2] if prev else np.zeros((size, size), bool)
    # box downsample including invalid (zero) sub-texels, like DownsampleTexture
    sh[oy, ox] = m64.mean(axis=1).astype(np.float32)
    se[oy, ox] = (np.sqrt(var.sum(axis=1) / SPP) / (ss * ss)).astype(np.float32)
    vmask[oy, ox] = valid_sub.any(axis=1)
    rays = int(r["rays"]) + (prev[5] if prev else 0)
    seconds = dt + (prev[4] if prev else 0.0)
    np.savez_compressed(out, sh=sh, se=se, valid=vmask, x0=x0, y0=y0, size=size, ss=ss, spp=SPP, seed=SEED, width=w,
                        height=h, bounces=bounces, rays=rays, seconds=seconds)
    print(f"{name}: {int(vmask.sum())} valid texels ({int(known.sum())} reused), {rays} rays, {seconds:.0f} s -> {out}")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("names", nargs="*")
    ap.add_argument("--grow", action="store_true")
    ap.add_argument("--threads", type=int, default=0)
    args = ap.parse_args()
    for n in (args.names or list(CROPS)):
        make(n, grow=args.grow, threads=args.threads)
