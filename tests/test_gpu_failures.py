"""Failure paths, made without faulting, trapping or hanging the GPU.

Every device loop and queue of the bake is bounded.  These tests lower the
bounds until they run out, or refuse an allocation on the host, and check
that the entry point reports it with its status code and error flags, that
the kernels still end, and that the same context then bakes the same bits
as an undisturbed bake.  The reference has no counterpart (it logs and
returns nullopt, src/occlusion.cpp:10-13).
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from sh_baker_b200 import _capi as A
from sh_baker_b200 import api, scenes

pytestmark = pytest.mark.gpu

TIMEOUT, INTERNAL, OOM = 4, 5, 2
ERR_STACK, ERR_QUEUE, ERR_ITER = 1, 2, 4


@pytest.fixture(scope="module")
def room(gpu_ctx):
    import torch
    sc = scenes.procedural_room(seed=8, n_boxes=20, res=64)
    ds = api.DeviceScene(gpu_ctx, sc)
    rc = api.RasterConfig(64, 64, 2)
    g = api.rasterize_to_device(ds, rc)
    bake = api.BatchBake(ds, g, rc, api.BakeConfig(samples=16, bounces=3, seed=31))
    n = g.width * g.height
    clean = (torch.empty(n * 27, dtype=torch.float32, device="cuda"), torch.empty(n, dtype=torch.float32, device="cuda"))
    api.bake_plain_device(bake, *clean)
    torch.cuda.synchronize()
    yield sc, ds, g, bake, clean
    g.close()
    ds.close()


def same(a, b):
    return a[0].cpu().numpy().tobytes() == b[0].cpu().numpy().tobytes() and \
        a[1].cpu().numpy().tobytes() == b[1].cpu().numpy().tobytes()


def test_traversal_step_limit_returns_timeout_and_context_recovers(gpu_ctx, room):
    sc, ds, g, bake, clean = room
    outs, st, status = api.bake_batch(gpu_ctx, [bake], use_graph=False, max_traversal_steps=2, check=False)
    assert status == TIMEOUT, A.STATUS_NAMES.get(status)
    assert st.error_flags & ERR_ITER
    assert b"step limit" in gpu_ctx.lib.shb_last_error()
    outs, st = api.bake_batch(gpu_ctx, [bake], use_graph=False)
    assert st.error_flags == 0
    assert same(outs[0], clean)


def test_queue_capacity_overflow_returns_internal_and_context_recovers(gpu_ctx, room):
    sc, ds, g, bake, clean = room
    outs, st, status = api.bake_batch(gpu_ctx, [bake], use_graph=True, queue_capacity=1000, check=False)
    assert status == INTERNAL, A.STATUS_NAMES.get(status)
    assert st.error_flags & ERR_QUEUE
    assert b"queue overflow" in gpu_ctx.lib.shb_last_error()
    outs, st = api.bake_batch(gpu_ctx, [bake], use_graph=True)
    assert st.error_flags == 0
    assert same(outs[0], clean)


def test_negative_bounds_are_invalid_arguments(gpu_ctx, room):
    sc, ds, g, bake, clean = room
    _, _, status = api.bake_batch(gpu_ctx, [bake], max_traversal_steps=-1, check=False)
    assert status == 1
    _, _, status = api.bake_batch(gpu_ctx, [bake], queue_capacity=-5, check=False)
    assert status == 1


def test_refused_allocation_returns_oom_and_context_recovers(room):
    """A fresh context has no scratch yet, so its first bake allocates; the
    hook refuses that allocation before cudaMalloc is called."""
    sc = room[0]
    ctx = api.Context(device=0)
    try:
        pts = O.OracleScene(sc).rasterize(32, 32, 1)
        rc = api.RasterConfig(32, 32, 1)
        cfg = api.BakeConfig(samples=8, bounces=2, seed=3)
        ds = api.DeviceScene(ctx, sc)
        g = api.GBuffer.from_points(ctx, pts, 32, 32)
        ctx.lib.shb_test_fail_allocation_after(0)
        try:
            with pytest.raises(A.ShbError) as e:
                api.BakeSHLightMap(sc, g, rc, cfg, ctx=ctx)
            assert e.value.status == OOM
            assert b"refused" in ctx.lib.shb_last_error()
        finally:
            ctx.lib.shb_test_fail_allocation_after(-1)
        a = api.BakeSHLightMap(sc, g, rc, cfg, ctx=ctx)
        b = api.BakeSHLightMap(sc, pts, rc, cfg, ctx=ctx)
        assert a.sh_texture.tobytes() == b.sh_texture.tobytes()
        g.close()
        ds.close()
    finally:
        ctx.close()


def test_refused_allocation_in_scene_upload(room):
    sc = room[0]
    ctx = api.Context(device=0)
    try:
        ctx.lib.shb_test_fail_allocation_after(3)
        try:
            with pytest.raises(A.ShbError) as e:
                api.DeviceScene(ctx, sc)
            assert e.value.status == OOM
        finally:
            ctx.lib.shb_test_fail_allocation_after(-1)
        ds = api.DeviceScene(ctx, sc)  # the same context uploads once the hook is off
        assert ds.bvh_info()["triangles"] == sc.triangle_count
        ds.close()
    finally:
        ctx.close()


def test_find_occlusion_ends_without_flags(gpu_ctx, room):
    """FindOcclusion keeps the default bound: a query of ordinary rays ends
    with no error and the oracle's hits."""
    sc = room[0]
    rng = np.random.default_rng(3)
    n = 4096
    rays = np.hstack([rng.uniform(-4.5, 4.5, (n, 3)) * [1, 0.3, 1] + [0, 1.5, 0], rng.normal(size=(n, 3)),
                      np.full((n, 1), 0.001), np.full((n, 1), np.inf)]).astype(np.float32)
    h = api.FindOcclusion(sc, rays, ctx=gpu_ctx)
    r = O.OracleScene(sc).find_occlusion(rays)
    assert (h["hit"] == r["hit"]).mean() >= 0.999
