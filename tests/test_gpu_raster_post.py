"""Bit-exact parity of the CUDA raster, mask, downsample and dilation
kernels against the CPU oracle (src/rasterizer.cpp, src/baker.cpp:151-182,
src/dilation.cpp), called through the C ABI."""
import numpy as np
import pytest

from oracle import pyoracle as O
from sh_baker_b200 import api, scenes
from sh_baker_b200.scene import Geometry, Material, Scene

pytestmark = pytest.mark.gpu


def ref_quad(material_id=0):
    return Geometry(
        vertices=np.array([[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]], np.float32),
        normals=np.array([[0, 0, 1]] * 4, np.float32),
        texture_uvs=np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32),
        lightmap_uvs=np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32),
        tangents=np.array([[1, 0, 0, 1]] * 4, np.float32),
        indices=np.array([0, 1, 2, 0, 2, 3], np.uint32), material_id=material_id)


def soup(seed, n_geoms=6, tris=400, tiny=True, with_negative_material=True, uv_spread=1.0):
    rng = np.random.default_rng(seed)
    geoms = []
    for g in range(n_geoms):
        n = tris
        centers = rng.uniform(-0.1 * uv_spread, 1.0 + 0.1 * uv_spread, (n, 2))
        scale = rng.uniform(0.0005, 0.004, (n, 1)) if tiny else rng.uniform(0.01, 0.3, (n, 1))
        uv = (centers[:, None, :] + scale[:, None, :] * rng.normal(size=(n, 3, 2))).reshape(-1, 2)
        v = rng.normal(size=(3 * n, 3)).astype(np.float32)
        nrm = rng.normal(size=(3 * n, 3))
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        t = rng.normal(size=(3 * n, 3))
        tan = np.hstack([t, np.where(rng.uniform(size=(3 * n, 1)) < 0.5, -1.0, 1.0)])
        mid = -1 if (with_negative_material and g % 3 == 2) else int(rng.integers(0, 3))
        geoms.append(Geometry(vertices=v, normals=nrm.astype(np.float32), tangents=tan.astype(np.float32),
                              lightmap_uvs=uv.astype(np.float32), texture_uvs=uv.astype(np.float32),
                              indices=np.arange(3 * n, dtype=np.uint32), material_id=mid))
    return Scene(geoms, [Material(), Material(), Material()], [])


def rotated_room():
    sc = scenes.procedural_room(seed=5, n_boxes=20, res=128)
    a = 0.7
    R = np.array([[np.cos(a), 0, np.sin(a)], [0, 1, 0], [-np.sin(a), 0, np.cos(a)]], np.float32)
    for i, g in enumerate(sc.geometries):
        if i % 2 == 1:
            g.transform = np.hstack([R, np.array([[0.5], [0.1], [-0.25]], np.float32)])
    return sc


CASES = {
    "ref_quad_4": (lambda: Scene([ref_quad()], [Material()], []), 4, 4, 1),
    "ref_quad_4_ss2": (lambda: Scene([ref_quad()], [Material()], []), 4, 4, 2),
    "unit_quad_256": (scenes.unit_quad, 256, 256, 1),
    "room_128_ss3": (lambda: scenes.procedural_room(seed=2, res=128), 128, 128, 3),
    "room_rotated": (rotated_room, 128, 128, 2),
    "soup_tiny": (lambda: soup(1), 97, 61, 1),
    "soup_large_overlap": (lambda: soup(2, tiny=False, tris=60), 64, 48, 2),
    "soup_uv_outside": (lambda: soup(3, tiny=False, tris=50, uv_spread=4.0), 33, 40, 1),
    "soup_degenerate": (lambda: soup(4, tris=300, tiny=True), 512, 512, 1),
    "empty": (lambda: Scene([], [], []), 8, 8, 1),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_rasterize_bit_exact(gpu_ctx, name):
    make, w, h, s = CASES[name]
    sc = make()
    ref = O.OracleScene(sc).rasterize(w, h, s)
    got = api.RasterizeScene(sc, api.RasterConfig(w, h, s), ctx=gpu_ctx)
    assert got.tobytes() == ref.tobytes(), np.flatnonzero(got.view(np.uint8).reshape(-1, 64).tobytes() !=
                                                          ref.view(np.uint8).reshape(-1, 64).tobytes())[:10]


def test_rasterize_reference_known_answer(gpu_ctx):
    # src/rasterizer_test.cpp:7-43 on the GPU
    got = api.RasterizeScene(Scene([ref_quad()], [Material()], []), api.RasterConfig(4, 4, 1), ctx=gpu_ctx)
    assert (got["material_id"] >= 0).all()
    assert abs(got[5]["position"][0] + 0.25) < 1e-3 and abs(got[5]["position"][1] + 0.25) < 1e-3
    assert abs(got[5]["normal"][2] - 1.0) < 1e-3


def test_rasterize_rejects_missing_tangents(gpu_ctx):
    g = ref_quad()
    g.tangents = None
    with pytest.raises(Exception, match="INVALID_ARG"):
        api.RasterizeScene(Scene([g], [Material()], []), api.RasterConfig(4, 4, 1), ctx=gpu_ctx)


def test_validity_mask_and_downsample(gpu_ctx):
    sc = scenes.procedural_room(seed=2, n_boxes=40, res=64)
    pts = O.OracleScene(sc).rasterize(64, 64, 3)
    m = api.CreateValidityMask(pts, ctx=gpu_ctx)
    np.testing.assert_array_equal(m, O.validity_mask(pts))
    d = api.DownsampleValidityMask(m, 64, 64, 3, ctx=gpu_ctx)
    np.testing.assert_array_equal(d, O.downsample_validity_mask(m, 64, 64, 3))


@pytest.mark.parametrize("w,h,s", [(1, 1, 1), (3, 5, 2), (17, 9, 3), (64, 64, 4)])
def test_downsample_validity_mask_random(gpu_ctx, w, h, s):
    rng = np.random.default_rng(w * 100 + h)
    m = (rng.uniform(size=w * s * h * s) < 0.1).astype(np.uint8)
    np.testing.assert_array_equal(api.DownsampleValidityMask(m, w, h, s, ctx=gpu_ctx),
                                  O.downsample_validity_mask(m, w, h, s))


@pytest.mark.parametrize("w,h,ch,s", [(6, 6, 27, 3), (10, 7, 27, 3), (64, 32, 1, 2), (5, 5, 1, 1), (96, 96, 27, 4),
                                      (3, 3, 1, 3)])
def test_downsample_bit_exact(gpu_ctx, w, h, ch, s):
    rng = np.random.default_rng(w * 7 + ch)
    x = rng.normal(size=(h, w, ch)).astype(np.float32)
    x[rng.uniform(size=(h, w)) < 0.3] = 0.0
    ref = O.downsample(x, w, h, ch, s)
    if ch == 27:
        got = api.DownsampleSHTexture(x.reshape(h, w, 9, 3), s, ctx=gpu_ctx).reshape(-1)
    else:
        got = api.DownsampleEnvironmentVisibilityTexture(x.reshape(h, w), s, ctx=gpu_ctx).reshape(-1)
    assert got.tobytes() == ref.tobytes()


@pytest.mark.parametrize("kind", [0, 1, 2])
@pytest.mark.parametrize("w,h,passes,density", [(1, 1, 1, 0.0), (3, 3, 1, 0.2), (37, 19, 2, 0.1), (256, 256, 5, 0.02),
                                                (64, 64, 16, 0.3), (40, 40, 0, 0.3), (50, 30, 40, 0.001)])
def test_dilate_bit_exact(gpu_ctx, kind, w, h, passes, density):
    rng = np.random.default_rng(w + 1000 * passes + kind)
    n = w * h
    ch = 27 if kind == 0 else 1
    mask = (rng.uniform(size=n) < density).astype(np.uint8)
    if kind == 2:
        px = rng.integers(0, 256, size=n).astype(np.uint8)
    else:
        px = rng.normal(size=n * ch).astype(np.float32)
    px_ref, m_ref = px.copy(), mask.copy()
    O.dilate(kind, w, h, px_ref, m_ref, passes)
    px_gpu, m_gpu = px.copy(), mask.copy()
    api.Dilate(w, h, px_gpu, m_gpu, passes, ctx=gpu_ctx)
    assert m_gpu.tobytes() == m_ref.tobytes()
    assert px_gpu.tobytes() == px_ref.tobytes()


def test_dilate_reference_known_answers(gpu_ctx):
    # src/dilation_test.cpp:11-58
    px = np.zeros(9 * 27, np.float32)
    m = np.zeros(9, np.uint8)
    m[4] = 1
    px[4 * 27] = 1.0
    api.Dilate(3, 3, px, m, 1, ctx=gpu_ctx)
    assert m[1] == 1 and abs(px[27] - 1.0) < 1e-3 and m[0] == 1 and abs(px[0] - 1.0) < 1e-3
    px = np.zeros(9 * 27, np.float32)
    m = np.zeros(9, np.uint8)
    m[3] = m[5] = 1
    px[3 * 27] = 1.0
    px[5 * 27 + 2] = 1.0
    api.Dilate(3, 3, px, m, 1, ctx=gpu_ctx)
    assert m[4] == 1 and abs(px[4 * 27] - 0.5) < 1e-3 and abs(px[4 * 27 + 2] - 0.5) < 1e-3
