"""GPU BVH queries and Monte-Carlo bakes against the CPU oracle, through the
C ABI.

Hits: the GPU and the oracle use the same watertight triangle test, so hit
flags, triangle ids and t agree except for exact ties between triangles.
Bakes: with the counter-based Philox stream both consume the same random
numbers, so texels agree to float rounding except where a 1-ulp
transcendental difference changes a path.  Agreement with the reference's
own mt19937 stream is statistical; tests/test_gpu_parity_full.py checks it
per texel at 3 standard errors.
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from sh_baker_b200 import api, scenes
from sh_baker_b200.scene import AREA, Geometry, Light, Material, Scene, Texture

pytestmark = pytest.mark.gpu


def tri_scene():
    g = Geometry(vertices=np.array([[-1, -1, 0], [1, -1, 0], [0, 1, 0]], np.float32),
                 indices=np.array([0, 1, 2], np.uint32))
    return Scene([g], [], [])


def ray(o, d, tnear=0.0, tfar=np.inf):
    return np.array([*o, *d, tnear, tfar], np.float32)


# ------------------------------------------------------------------ BVH ---

def test_occlusion_reference_cases(gpu_ctx):
    # src/occlusion_test.cpp:18-115
    rays = np.stack([ray((0, 0, 1), (0, 0, -1)), ray((2, 0, 1), (0, 0, -1)), ray((0, 0, 1), (0, 0, 1)),
                     ray((0, 0, 1), (0, 0, -1), 0.0, 0.5), ray((0, 0, 1), (0, 0, -1), 1.2),
                     ray((0, 0, 1), (0, 0, -1), 0.1, 10.0)])
    h = api.FindOcclusion(tri_scene(), rays, ctx=gpu_ctx)
    assert list(h["hit"]) == [1, 0, 0, 0, 0, 1]
    assert abs(h["position"][0][2]) < 1e-4 and abs(h["normal"][0][2] - 1.0) < 1e-4


def test_occlusion_multi_geometry(gpu_ctx):
    # src/occlusion_test.cpp:117-184
    quads = []
    for x0, mid in ((-3.0, 10), (1.0, 20)):
        quads.append(Geometry(vertices=np.array([[x0, -1, 0], [x0 + 2, -1, 0], [x0, 1, 0], [x0 + 2, 1, 0]], np.float32),
                              indices=np.array([0, 1, 2, 1, 3, 2], np.uint32), material_id=mid))
    h = api.FindOcclusion(Scene(quads, [Material() for _ in range(21)], []), ray((2.8, 0.8, 5.0), (0, 0, -1))[None],
                          ctx=gpu_ctx)
    assert h["hit"][0] == 1 and h["material_id"][0] == 20
    np.testing.assert_allclose(h["position"][0], [2.8, 0.8, 0.0], atol=1e-4)


def random_rays(rng, n, lo, hi):
    o = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    d[rng.uniform(size=n) < 0.02, rng.integers(0, 3)] = 0.0  # axis-parallel rays
    scale = rng.uniform(0.3, 3.0, (n, 1))  # unnormalised directions (t in units of |d|)
    tn = np.full((n, 1), 0.001)
    tf = np.where(rng.uniform(size=(n, 1)) < 0.3, rng.uniform(0.5, 4.0, (n, 1)), np.inf)
    return np.hstack([o, d * scale, tn, tf]).astype(np.float32)


def degenerate_scene(name, rng):
    """Inputs that stress the builder's splits and the collapse: identical
    triangles stacked on one another (no SAH split exists), a flat grid
    (zero extent on one axis) and long needles across the scene."""
    if name == "stack":
        v = np.tile(np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]]], np.float32), (300, 1, 1))
    elif name == "grid":
        k = 60
        x, y = np.meshgrid(np.linspace(-2, 2, k + 1), np.linspace(-2, 2, k + 1), indexing="ij")
        pts = np.stack([x, y, np.zeros_like(x)], -1).astype(np.float32)
        a, b, c, d = pts[:-1, :-1], pts[1:, :-1], pts[1:, 1:], pts[:-1, 1:]
        v = np.concatenate([np.stack([a, b, c], -2), np.stack([a, c, d], -2)]).reshape(-1, 3, 3)
    else:  # needles
        n = 2000
        p0 = rng.uniform(-2, 2, (n, 3))
        p1 = -p0 + rng.normal(scale=0.05, size=(n, 3))
        v = np.stack([p0, p1, p1 + rng.normal(scale=0.01, size=(n, 3))], 1)
    return Scene([Geometry(vertices=v.reshape(-1, 3).astype(np.float32), indices=np.arange(v.shape[0] * 3,
                                                                                            dtype=np.uint32),
                           material_id=0)], [Material()], [])


@pytest.mark.parametrize("name", ["room", "soup1", "soup3", "soup100", "soup5000", "stack", "grid", "needles"])
def test_closest_hit_matches_oracle(gpu_ctx, name):
    rng = np.random.default_rng(len(name))
    if name == "room":
        sc = scenes.procedural_room(seed=2, res=256)
        lo, hi = [-5, 0, -5], [5, 3, 5]
    elif name in ("stack", "grid", "needles"):
        sc = degenerate_scene(name, rng)
        lo, hi = [-3, -3, -3], [3, 3, 3]
    else:
        n = int(name[4:])
        v = rng.uniform(-1, 1, (n, 3, 3)) * 0.3 + rng.uniform(-2, 2, (n, 1, 3))
        sc = Scene([Geometry(vertices=v.reshape(-1, 3).astype(np.float32), indices=np.arange(3 * n, dtype=np.uint32),
                             material_id=0)], [Material()], [])
        lo, hi = [-3, -3, -3], [3, 3, 3]
    rays = random_rays(rng, 20000, lo, hi)
    g = api.FindOcclusion(sc, rays, ctx=gpu_ctx)
    r = O.OracleScene(sc).find_occlusion(rays)
    assert (g["hit"] == r["hit"]).mean() >= 0.9995
    both = (g["hit"] == 1) & (r["hit"] == 1)
    if name == "stack":  # every hit is an exact tie of identical triangles: any of them is right
        same = np.ones(both.sum(), bool)
    else:
        same = g["prim_id"][both] == r["prim_id"][both]
    assert same.mean() >= 0.999
    np.testing.assert_allclose(g["t"][both], r["t"][both], rtol=1e-5, atol=1e-6)
    np.testing.assert_array_equal(g["position"][both][same], r["position"][both][same])
    np.testing.assert_array_equal(g["normal"][both][same], r["normal"][both][same])


def test_bvh_info(gpu_ctx):
    sc = scenes.procedural_room(seed=2, res=256)
    ds = api.DeviceScene(gpu_ctx, sc)
    info = ds.bvh_info()
    assert info["triangles"] == 2412 and info["wide_nodes"] >= 1 and info["depth"] <= 64
    ds.rebuild_bvh()
    assert ds.bvh_info() == info


# ----------------------------------------------------------------- bakes ---

def bake_pair(gpu_ctx, sc, w, h, s, spp, bounces, seed=7, rng=O.RNG_PHILOX, stats=False, nls=1):
    osc = O.OracleScene(sc)
    pts = osc.rasterize(w, h, s)
    ref = osc.bake(pts, w, h, s, samples=spp, bounces=bounces, seed=seed, rng=rng, stats=stats,
                   num_light_samples=nls)
    got = api.BakeSHLightMap(sc, pts, api.RasterConfig(w, h, s),
                             api.BakeConfig(samples=spp, bounces=bounces, seed=seed, num_light_samples=nls),
                             ctx=gpu_ctx, with_stats=True)
    return pts, ref, got


def test_unit_quad_closed_form_gpu(gpu_ctx):
    from test_oracle_known_answers import unit_quad_expectation
    sc = scenes.unit_quad()
    pts, ref, got = bake_pair(gpu_ctx, sc, 32, 32, 1, 512, 3, seed=1, stats=True)
    assert (got.environment_visibility_texture == 1.0).all()
    exp = unit_quad_expectation(sc, pts)
    mean = got.sh_texture.reshape(-1, 27).astype(np.float64)
    tol = 4.5 * np.sqrt(ref["var"].reshape(-1, 27) / 512) + 3e-5 * np.abs(exp) + 1e-6
    assert (np.abs(mean - exp) <= tol).mean() > 0.999


def test_unit_quad_gpu_equals_oracle_philox(gpu_ctx):
    pts, ref, got = bake_pair(gpu_ctx, scenes.unit_quad(), 64, 64, 1, 64, 3, seed=1)
    np.testing.assert_allclose(got.sh_texture, ref["sh"], rtol=2e-5, atol=2e-6)
    np.testing.assert_array_equal(got.environment_visibility_texture, ref["env"])


def small_room(res=32, seed=2):
    # few boxes so that one chart per face fits a small atlas
    return scenes.procedural_room(seed=seed, n_boxes=max(2, res // 5), res=res)


def test_room_gpu_matches_oracle_philox(gpu_ctx):
    pts, ref, got = bake_pair(gpu_ctx, small_room(32), 32, 32, 1, 32, 3, seed=11)
    valid = (pts["material_id"] >= 0).reshape(32, 32)
    g = got.sh_texture[valid].reshape(-1, 27)
    r = ref["sh"][valid].reshape(-1, 27)
    close = np.isclose(g, r, rtol=1e-3, atol=1e-5).all(axis=1)
    assert close.mean() >= 0.98, close.mean()
    np.testing.assert_allclose(got.environment_visibility_texture, ref["env"], atol=1.0 / 32 + 1e-6)
    rel = np.linalg.norm(g - r) / max(np.linalg.norm(r), 1e-12)
    assert rel < 1e-2, rel
    st = got.stats
    assert st.error_flags == 0 and st.texel_samples == valid.sum() * 32 and st.extend_rays > 0


def test_bake_deterministic_and_split(gpu_ctx):
    sc = small_room(32, seed=4)
    pts = O.OracleScene(sc).rasterize(32, 32, 1)
    rc = api.RasterConfig(32, 32, 1)
    a = api.BakeSHLightMap(sc, pts, rc, api.BakeConfig(samples=16, bounces=2, seed=9), ctx=gpu_ctx)
    b = api.BakeSHLightMap(sc, pts, rc, api.BakeConfig(samples=16, bounces=2, seed=9), ctx=gpu_ctx)
    assert a.sh_texture.tobytes() == b.sh_texture.tobytes()
    h1 = api.BakeSHLightMap(sc, pts, rc, api.BakeConfig(samples=8, bounces=2, seed=9), ctx=gpu_ctx)
    h2 = api.BakeSHLightMap(sc, pts, rc, api.BakeConfig(samples=8, bounces=2, seed=9, sample_offset=8), ctx=gpu_ctx)
    np.testing.assert_allclose(0.5 * (h1.sh_texture + h2.sh_texture), a.sh_texture, rtol=1e-4, atol=1e-5)


def area_alpha_scene():
    """Emissive patches (area lights), a spot light and an RGBA (alpha)
    material exercise every light type and transmission."""
    sc = scenes.procedural_room(seed=6, n_boxes=12, res=48)
    sc.materials.append(Material(name="glow", albedo=Texture(1, 1, 3, np.array([250, 200, 120], np.uint8)),
                                 emission_intensity=3.0))
    sc.materials.append(Material(name="screen", albedo=Texture(2, 1, 4, np.array([200, 200, 200, 100,
                                                                                  90, 200, 90, 255], np.uint8))))
    sc.geometries[3].material_id = len(sc.materials) - 2
    sc.geometries[5].material_id = len(sc.materials) - 1
    scenes.mark_area_lights(sc)
    sc.lights.append(Light(type=2, position=(0.0, 2.9, 0.0), direction=(0.0, -1.0, 0.0), intensity=30.0,
                           cos_inner_cone=0.9, cos_outer_cone=0.6))
    return sc


def test_all_light_types_and_alpha_match_oracle(gpu_ctx):
    sc = area_alpha_scene()
    assert any(L.type == AREA for L in sc.lights)
    pts, ref, got = bake_pair(gpu_ctx, sc, 48, 48, 1, 32, 3, seed=21, nls=2)
    valid = (pts["material_id"] >= 0).reshape(48, 48)
    g = got.sh_texture[valid].reshape(-1, 27)
    r = ref["sh"][valid].reshape(-1, 27)
    close = np.isclose(g, r, rtol=1e-3, atol=1e-5).all(axis=1)
    assert close.mean() >= 0.97, close.mean()
    assert np.linalg.norm(g - r) / max(np.linalg.norm(r), 1e-12) < 2e-2


def test_bake_rejects_bad_arguments(gpu_ctx):
    sc = small_room(32)
    pts = O.OracleScene(sc).rasterize(16, 16, 1)
    with pytest.raises(Exception, match="INVALID_ARG"):
        api.BakeSHLightMap(sc, pts, api.RasterConfig(16, 16, 1), api.BakeConfig(samples=0), ctx=gpu_ctx)
    # a 16x16 G-buffer baked with a raster config of 32x16 texels
    g = api.GBuffer.from_points(gpu_ctx, pts, 16, 16)
    with pytest.raises(Exception, match="INVALID_ARG"):
        api.BakeSHLightMap(sc, g, api.RasterConfig(16, 8, 2), api.BakeConfig(samples=4), ctx=gpu_ctx)


def test_bake_all_invalid_texels(gpu_ctx):
    sc = small_room(32)
    from sh_baker_b200.scene import surface_points_empty
    pts = surface_points_empty(16 * 16)
    out = api.BakeSHLightMap(sc, pts, api.RasterConfig(16, 16, 1), api.BakeConfig(samples=4), ctx=gpu_ctx)
    assert not out.sh_texture.any() and not out.environment_visibility_texture.any()
