"""Path-replay adjoint (shb_backward) of the bake.

1. Parity: on a 64x64 crop of a 256x256 room lightmap the GPU gradient equals
   the oracle's FP64 forward-mode gradient of the same Philox paths
   (light-selection pdfs held constant on both sides).
2. Finite differences: for Loss = sum (SH - SH_target)^2 with the target baked
   at albedos x U[0.8, 1.2] and intensities x U[0.5, 2], the adjoint agrees
   with central differences (h = 1e-3, common random numbers) of the GPU
   forward bake within 1e-2 (relative L2 over all 8x3 + 5 parameters).
3. The torch.autograd wrapper returns the same gradients; argument errors.
"""
import numpy as np
import pytest

from oracle.pyoracle import OracleScene, srgb_to_linear
from sh_baker_b200 import api, scenes

pytestmark = pytest.mark.gpu


def room(res, seed=11, n_boxes=40):
    return scenes.procedural_room(seed=seed, n_boxes=n_boxes, res=res, n_point_lights=4)


def linear_albedo(sc):
    """The materials' own 1x1 sRGB albedos as linear floats."""
    lut = np.array([srgb_to_linear(i) for i in range(256)], np.float32)
    return np.stack([lut[m.albedo.pixel_data[:3]] for m in sc.materials]).astype(np.float32)


def make_bake(ctx, sc, res, spp, bounces, seed=5, ss=1):
    ds = api.DeviceScene(ctx, sc)
    rc = api.RasterConfig(res, res, ss)
    g = api.rasterize_to_device(ds, rc)
    return api.BatchBake(ds, g, rc, api.BakeConfig(samples=spp, bounces=bounces, seed=seed))


def test_adjoint_matches_fp64_forward_mode_on_crop(gpu_ctx):
    res, spp, bounces = 256, 8, 3
    sc = room(res)
    b = make_bake(gpu_ctx, sc, res, spp, bounces)
    rng = np.random.default_rng(3)
    albedo = linear_albedo(sc) * rng.uniform(0.8, 1.2, (len(sc.materials), 3)).astype(np.float32)
    inten = np.array([l.intensity for l in sc.lights], np.float32)
    b.scene.set_params(albedo, inten)
    # dLoss/dSH nonzero on a 64x64 crop only
    dsh = np.zeros((res, res, 27), np.float32)
    y0, x0 = 96, 80
    dsh[y0:y0 + 64, x0:x0 + 64] = rng.normal(size=(64, 64, 27))
    d_alb, d_li = api.Backward(b, dsh.reshape(-1))
    o = OracleScene(sc)
    o.set_params(albedo, inten)
    pts = b.gbuffer.download()
    crop = (np.arange(y0, y0 + 64)[:, None] * res + np.arange(x0, x0 + 64)[None, :]).reshape(-1)
    r_alb, r_li = o.bake_grad(pts, res, res, 1, spp, bounces, dsh.reshape(-1), seed=5, subset=crop)
    got = np.concatenate([d_alb.reshape(-1), d_li])
    ref = np.concatenate([r_alb.reshape(-1), r_li])
    assert np.abs(ref).max() > 0
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err < 2e-3, (err, got, ref)
    assert np.all(np.abs(got - ref) <= 5e-3 * np.abs(ref).max())


def test_adjoint_matches_central_differences(gpu_ctx):
    """Config of the adjoint workload: room at 512x512, supersample 3, 64 spp,
    3 bounces.  Central differences also see light-selection switches (the
    adjoint holds the selection pdfs constant); that noise falls as
    1/sqrt(samples), and at 88 M texel-samples it is well inside 1e-2."""
    import torch
    res, spp, bounces = 512, 64, 3
    sc = room(res, seed=2, n_boxes=200)
    b = make_bake(gpu_ctx, sc, res, spp, bounces, seed=9, ss=3)
    rng = np.random.default_rng(4)
    albedo = linear_albedo(sc)
    inten = np.array([l.intensity for l in sc.lights], np.float32)
    n = b.gbuffer.width * b.gbuffer.height
    sh = torch.empty(n * 27, dtype=torch.float32, device="cuda")
    env = torch.empty(n, dtype=torch.float32, device="cuda")
    target = torch.empty_like(sh)
    b.scene.set_params(albedo * rng.uniform(0.8, 1.2, albedo.shape).astype(np.float32),
                       inten * rng.uniform(0.5, 2.0, inten.shape).astype(np.float32))
    api.bake_plain_device(b, target, env)

    def loss(a, i):
        b.scene.set_params(a, i)
        api.bake_plain_device(b, sh, env)
        return float(((sh.double() - target.double()) ** 2).sum())

    loss(albedo, inten)
    d_alb, d_li = api.Backward(b, (2.0 * (sh - target)).contiguous())
    fd_alb = np.zeros_like(d_alb)
    fd_li = np.zeros_like(d_li)
    h = 1e-3
    for m in range(len(sc.materials)):
        for c in range(3):
            ap, am = albedo.copy(), albedo.copy()
            ap[m, c] += h
            am[m, c] -= h
            fd_alb[m, c] = (loss(ap, inten) - loss(am, inten)) / (float(ap[m, c]) - float(am[m, c]))
    for l in range(len(sc.lights)):
        ip, im = inten.copy(), inten.copy()
        ip[l] *= 1 + h
        im[l] *= 1 - h
        fd_li[l] = (loss(albedo, ip) - loss(albedo, im)) / (float(ip[l]) - float(im[l]))
    got = np.concatenate([d_alb.reshape(-1), d_li * inten])  # intensities: relative sensitivity
    fd = np.concatenate([fd_alb.reshape(-1), fd_li * inten])
    err = np.linalg.norm(got - fd) / np.linalg.norm(fd)
    assert err < 1e-2, (err, got, fd)


def test_autograd_wrapper_matches_backward(gpu_ctx):
    import torch

    from sh_baker_b200.autograd import bake_sh
    res = 64
    sc = room(res, seed=13, n_boxes=15)
    b = make_bake(gpu_ctx, sc, res, 8, 2)
    albedo = torch.tensor(linear_albedo(sc), requires_grad=True)
    inten = torch.tensor([l.intensity for l in sc.lights], dtype=torch.float32, requires_grad=True)
    sh = bake_sh(albedo, inten, b)
    w = torch.linspace(-1, 1, sh.numel(), device="cuda").view_as(sh)
    (sh * w).sum().backward()
    d_alb, d_li = api.Backward(b, w.contiguous().view(-1).cpu().numpy())
    np.testing.assert_allclose(albedo.grad.numpy(), d_alb, rtol=1e-4, atol=1e-6 * np.abs(d_alb).max())
    np.testing.assert_allclose(inten.grad.numpy(), d_li, rtol=1e-4, atol=1e-6 * np.abs(d_li).max())


def test_backward_rejects_bad_arguments(gpu_ctx):
    sc = room(32, seed=14, n_boxes=4)
    b = make_bake(gpu_ctx, sc, 32, 4, 17)
    with pytest.raises(api.A.ShbError):
        api.Backward(b, np.zeros(32 * 32 * 27, np.float32))  # more than 16 bounces
    with pytest.raises(ValueError):
        api.Backward(make_bake(gpu_ctx, sc, 32, 4, 2), np.zeros(5, np.float32))
    with pytest.raises(api.A.ShbError):
        b.scene.set_params(np.full((len(sc.materials), 3), np.nan, np.float32))
