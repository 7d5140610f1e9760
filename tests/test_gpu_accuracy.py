"""Global relative RMSE of the GPU bake against the 4096-spp FP64 CPU oracle
(tests/golden/fp64_<workload>.npz, made by tests/golden/make_fp64_reference.py)
on a crop of the output lightmap (room 64x64, atrium 256x256), at the
workload's own spp.

The reference estimator samples primary directions uniformly over the
hemisphere (src/baker.cpp:38-46), so at matched spp its Monte-Carlo noise
alone exceeds 1 %.  The yardstick is therefore the error an unbiased
estimator of the same variance has at that spp, which the fixture's
per-texel standard errors predict: ||se|| sqrt(4096 / spp + 1) / ||ref||
(the bake's noise plus the fixture's own).  The GPU must reach 1 % or stay
within 25 % of that prediction.  The reference algorithm itself (the oracle
on the reference's mt19937 stream) is held to the same gate, which checks
the prediction; both errors are printed.  To keep the CPU run to about a
minute, the reference algorithm bakes the central 128x128 of a larger crop
and is held to that region's own prediction.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import pyoracle as O
from sh_baker_b200 import api, scenes

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).parent / "golden"
FACTORY = {"room": lambda: scenes.procedural_room(seed=2, res=1024), "atrium": lambda: scenes.atrium(seed=3, res=2048)}


def rel_rmse(x, ref, valid):
    d = (x - ref)[valid]
    return float(np.linalg.norm(d) / np.linalg.norm(ref[valid]))


@pytest.mark.parametrize("name,spp", [("room", 128), ("atrium", 256)])
def test_relative_rmse_vs_fp64_oracle(gpu_ctx, name, spp):
    ref = np.load(GOLDEN / f"fp64_{name}.npz")
    w, h, ss, size, x0, y0 = (int(ref[k]) for k in ("width", "height", "ss", "size", "x0", "y0"))
    bounces = int(ref["bounces"])
    sc = FACTORY[name]()
    pts = api.RasterizeScene(sc, api.RasterConfig(w, h, ss), ctx=gpu_ctx).reshape(h * ss, w * ss)
    crop = np.ascontiguousarray(pts[y0 * ss:(y0 + size) * ss, x0 * ss:(x0 + size) * ss]).reshape(-1)
    rc = api.RasterConfig(size, size, ss)
    got = api.BakeSHLightMap(sc, crop, rc, api.BakeConfig(samples=spp, bounces=bounces, seed=2024), ctx=gpu_ctx)
    g = api.DownsampleSHTexture(got.sh_texture, ss, ctx=gpu_ctx).reshape(size, size, 27)
    valid = ref["valid"]
    r = ref["sh"]

    def predicted(v):
        floor = float(np.linalg.norm(ref["se"][v]) / np.linalg.norm(r[v]))
        return floor, floor * float(np.sqrt(int(ref["spp"]) / spp + 1.0))

    e_gpu = rel_rmse(g, r, valid)
    floor, expected = predicted(valid)
    # the reference algorithm on the central (at most) 128x128 of the crop
    sub = min(size, 128)
    o = (size - sub) // 2
    cpts = np.ascontiguousarray(crop.reshape(size * ss, size * ss)[o * ss:(o + sub) * ss, o * ss:(o + sub) * ss])
    osc = O.OracleScene(sc)
    cpu = osc.bake(cpts.reshape(-1), sub, sub, ss, samples=spp, bounces=bounces, rng=O.RNG_MT19937)
    c = O.downsample(cpu["sh"], sub * ss, sub * ss, 27, ss).reshape(sub, sub, 27)
    vsub = np.zeros_like(valid)
    vsub[o:o + sub, o:o + sub] = valid[o:o + sub, o:o + sub]
    cfull = np.zeros_like(r)
    cfull[o:o + sub, o:o + sub] = c
    e_cpu = rel_rmse(cfull, r, vsub)
    _, expected_cpu = predicted(vsub)
    print(f"{name}: rel. RMSE vs FP64@{int(ref['spp'])}: GPU {e_gpu:.4f} (predicted {expected:.4f}, "
          f"{size}x{size}), reference algorithm {e_cpu:.4f} (predicted {expected_cpu:.4f}, {sub}x{sub}); "
          f"FP64 reference's own error {floor:.4f}; {spp} spp")
    assert e_cpu <= max(0.01, 1.25 * expected_cpu), (e_cpu, expected_cpu)
    assert e_gpu <= max(0.01, 1.25 * expected), (e_gpu, expected)


def channel_bias(x, o, se, valid):
    """Per SH coefficient channel c: the relative bias sum(x_c - o_c) /
    sum |o_c| over the valid texels, and its standard error when x and o
    are independent estimates with the fixture's per-texel standard errors."""
    d = (x - o)[valid].astype(np.float64)
    a = np.abs(o[valid].astype(np.float64)).sum(axis=0)
    se_sum = np.sqrt(2.0 * (se[valid].astype(np.float64) ** 2).sum(axis=0))
    return d.sum(axis=0) / a, se_sum / a


@pytest.mark.parametrize("name", ["room", "atrium"])
def test_systematic_error_below_one_percent(gpu_ctx, name):
    """The GPU bake at the fixture's own 4096 spp against the FP64 fixture.
    Two independent 4096-spp estimates differ by their noise, which the
    fixture's per-texel standard errors give.  (1) The relative RMSE stays
    within 25 % of that noise floor (sqrt 2 times the fixture's own error).
    (2) The 1 % gate on what is systematic: in every one of the 27 SH
    channels the summed difference over the crop, relative to the summed
    magnitude, is at most 1 % plus 3 of its standard errors.  Summing over
    the crop's texels averages the noise down, so the bias is resolved far
    below 1 %, where the RMSE itself is dominated by noise."""
    ref = np.load(GOLDEN / f"fp64_{name}.npz")
    w, h, ss, size, x0, y0 = (int(ref[k]) for k in ("width", "height", "ss", "size", "x0", "y0"))
    sc = FACTORY[name]()
    pts = api.RasterizeScene(sc, api.RasterConfig(w, h, ss), ctx=gpu_ctx).reshape(h * ss, w * ss)
    crop = np.ascontiguousarray(pts[y0 * ss:(y0 + size) * ss, x0 * ss:(x0 + size) * ss]).reshape(-1)
    rc = api.RasterConfig(size, size, ss)
    got = api.BakeSHLightMap(sc, crop, rc, api.BakeConfig(samples=int(ref["spp"]), bounces=int(ref["bounces"]),
                                                          seed=777), ctx=gpu_ctx)
    g = api.DownsampleSHTexture(got.sh_texture, ss, ctx=gpu_ctx).reshape(size, size, 27).astype(np.float64)
    valid = ref["valid"]
    r = ref["sh"].astype(np.float64)
    total = rel_rmse(g, r, valid)
    noise = float(np.sqrt(2.0) * np.linalg.norm(ref["se"][valid]) / np.linalg.norm(r[valid]))
    bias, bias_se = channel_bias(g, r, ref["se"], valid)
    worst = int(np.argmax(np.abs(bias) - 3 * bias_se))
    print(f"{name}: at {int(ref['spp'])} spp rel. RMSE {total:.4f} (noise floor {noise:.4f}); channel bias "
          f"|b| max {np.abs(bias).max():.4f}, L0 {bias[0]:+.4f} {bias[1]:+.4f} {bias[2]:+.4f}, "
          f"worst channel {worst}: {bias[worst]:+.4f} +- {bias_se[worst]:.4f}")
    assert total <= 1.25 * noise, (total, noise)
    assert (np.abs(bias) <= 0.01 + 3 * bias_se).all(), (bias, bias_se)
