"""Generates the FP64 oracle references used by the accuracy tests.

For each workload a crop of the output lightmap (64 x 64 texels,
supersample 3) is baked by the CPU oracle in double precision at 4096
samples per supersampled texel (Philox stream, seed 987654, independent of
every GPU seed), then box-downsampled like the pipeline.  The crops are lit
regions, chosen by a quick low-spp bake of candidate crops: the lightmaps'
corners are dim enough that 4096 samples still leave much of the signal
as noise there.  Written as float32 to
tests/golden/fp64_<workload>.npz with the crop position and per-texel
standard errors.

    python tests/golden/make_fp64_reference.py [room|atrium ...]
"""
from __future__ import annotations

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
    "atrium": (lambda: scenes.atrium(seed=3, res=2048), 2048, 2048, 3, 4, 512, 256, 128),
}
SPP = 4096
SEED = 987654


def crop_indices(W, ss, x0, y0, size):
    ys, xs = np.meshgrid(np.arange(y0 * ss, (y0 + size) * ss), np.arange(x0 * ss, (x0 + size) * ss), indexing="ij")
    return (ys * (W * ss) + xs).reshape(-1)


def make(name):
    make_scene, w, h, ss, bounces, x0, y0, size = CROPS[name]
    sc = make_scene()
    osc = O.OracleScene(sc)
    pts = osc.rasterize(w, h, ss)
    idx = crop_indices(w, ss, x0, y0, size)
    t0 = time.time()
    r = osc.bake(pts, w, h, ss, samples=SPP, bounces=bounces, seed=SEED, rng=O.RNG_PHILOX, fp64=True, subset=idx,
                 stats=True)
    dt = time.time() - t0
    W = w * ss
    sub = (r["mean64"].reshape(-1, 27)[idx]).reshape(size * ss, size * ss, 27)
    var = (r["var"].reshape(-1, 27)[idx]).reshape(size * ss, size * ss, 27)
    valid = (pts["material_id"][idx] >= 0).reshape(size * ss, size * ss)
    # box downsample including invalid (zero) sub-texels, like DownsampleTexture
    sh = sub.reshape(size, ss, size, ss, 27).mean(axis=(1, 3))
    se = np.sqrt(var.reshape(size, ss, size, ss, 27).sum(axis=(1, 3)) / SPP) / (ss * ss)
    vmask = valid.reshape(size, ss, size, ss).any(axis=(1, 3))
    out = Path(__file__).parent / f"fp64_{name}.npz"
    np.savez_compressed(out, sh=sh.astype(np.float32), se=se.astype(np.float32), valid=vmask, x0=x0, y0=y0,
                        size=size, ss=ss, spp=SPP, seed=SEED, width=w, height=h, bounces=bounces,
                        rays=r["rays"], seconds=dt)
    print(f"{name}: {int(vmask.sum())} valid texels, {r['rays']} rays, {dt:.0f} s -> {out}")


if __name__ == "__main__":
    for n in (sys.argv[1:] or list(CROPS)):
        make(n)
