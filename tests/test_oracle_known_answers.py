"""Pins the CPU oracle to the reference's own known-answer tests.

Each test restates one GoogleTest case of the reference (cited file:line)
against oracle/shb_oracle.cpp.  The values are the reference's; the
machine-readable copy with citations is tests/golden/reference_known_answers.json.
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from oracle import pyoracle as O
from sh_baker_b200 import scenes
from sh_baker_b200.scene import AREA, DIRECTIONAL, POINT, SPOT, Geometry, Light, Material, Scene, Texture

GOLDEN = json.loads((Path(__file__).parent / "golden" / "reference_known_answers.json").read_text())


def K(name):
    return GOLDEN[name]["value"]


def quad_geometry(with_tangents=True, material_id=0):
    # src/rasterizer_test.cpp:9-17
    g = Geometry(
        vertices=np.array([[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]], np.float32),
        normals=np.array([[0, 0, 1]] * 4, np.float32),
        texture_uvs=np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32),
        lightmap_uvs=np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32),
        tangents=np.array([[1, 0, 0, 1]] * 4, np.float32) if with_tangents else None,
        indices=np.array([0, 1, 2, 0, 2, 3], np.uint32),
        material_id=material_id,
    )
    return g


# ------------------------------------------------------------------ SH ----

def test_sh_basis_plus_z():
    # src/sh_coeffs_test.cpp:7-38
    acc = O.accumulate_radiance([1, 1, 1], [0, 0, 1]).reshape(9, 3)
    expect = K("sh_basis_plus_z")
    for i in range(9):
        assert abs(acc[i, 0] - expect[i]) <= 1e-5


def test_sh_accumulate_adds():
    # src/sh_coeffs_test.cpp:40-50: accumulation adds component-wise
    a = O.accumulate_radiance([1, 2, 3], [0, 0, 1])
    b = O.accumulate_radiance([1, 2, 3], [0, 0, 1], a)
    np.testing.assert_allclose(b, 2 * a, rtol=0, atol=1e-7)


# ------------------------------------------------------------- materials --

def mat_scene(mats):
    return O.OracleScene(Scene([], mats, []))


def test_get_albedo_srgb():
    # src/material_test.cpp:43-54
    s = mat_scene([Material(albedo=Texture(1, 1, 3, np.array([255, 128, 0], np.uint8)))])
    a = s.albedo(0, [0.5, 0.5])
    exp = K("get_albedo_255_128_0")
    assert abs(a[0] - exp[0]) < 1e-5 and abs(a[1] - exp[1]) < 1e-3 and abs(a[2] - exp[2]) < 1e-5


def test_get_albedo_default_grey():
    # src/material.cpp:70: Vector3f(0.8f, 0.8f, 0.8f) without texture
    s = mat_scene([Material()])
    np.testing.assert_array_equal(s.albedo(0, [0.3, 0.3]), np.float32([0.8, 0.8, 0.8]))


def test_get_emission():
    # src/material_test.cpp:87-99
    s = mat_scene([Material(albedo=Texture(1, 1, 3, np.array([255, 255, 255], np.uint8)), emission_intensity=5.0)])
    np.testing.assert_allclose(s.emission(0, [0.5, 0.5]), K("get_emission_white_5"), atol=1e-5)


def test_get_alpha():
    # src/material_test.cpp:101-121
    s = mat_scene([Material(albedo=Texture(1, 1, 4, np.array([255, 255, 255, 128], np.uint8))),
                   Material(albedo=Texture(1, 1, 3, np.array([255, 255, 255], np.uint8)))])
    assert abs(s.alpha(0, [0.5, 0.5]) - K("get_alpha_128")) < 1e-5
    assert abs(s.alpha(1, [0.5, 0.5]) - 1.0) < 1e-5


def test_srgb_to_linear_endpoints():
    # src/colorspace.h:10-14
    assert O.srgb_to_linear(0) == 0.0
    assert O.srgb_to_linear(255) == 1.0
    assert abs(O.srgb_to_linear(10) - (10 / 255.0) / 12.92) < 1e-9


# ---------------------------------------------------------------- lights --

def light_test_scene(area_emission=0.0):
    # src/light_test.cpp:13-67: point light (0,10,0) I=100 and an area light
    area_geo = Geometry(vertices=np.array([[10, -1, 1], [10, 1, 0], [10, -1, -1]], np.float32),
                        normals=np.array([[-1, 0, 0]] * 3, np.float32), indices=np.array([0, 1, 2], np.uint32),
                        material_id=0)
    return Scene([area_geo], [Material(name="default", emission_intensity=area_emission)],
                 [Light(type=POINT, position=(0, 10, 0), intensity=100.0),
                  Light(type=AREA, geometry_index=0, material_index=0, intensity=10.0, area=2.0)])


def test_evaluate_point_light():
    # src/light_test.cpp:74-109
    s = O.OracleScene(light_test_scene())
    r = s.evaluate_light_samples([0, 0, 0], [0, 1, 0], [0, 1, 0], 0, [0, 0], 1, seed=12345)
    exp, tol = K("evaluate_point_light")
    assert abs(r[0] - exp) <= tol


def test_evaluate_area_light():
    # src/light_test.cpp:111-169 (100 samples, result within (0.01, 10))
    geo = Geometry(vertices=np.array([[-1, 10, 1], [1, 10, 1], [0, 10, -1]], np.float32),
                   normals=np.array([[0, -1, 0]] * 3, np.float32), indices=np.array([0, 2, 1], np.uint32),
                   material_id=0)
    sc = Scene([geo], [Material(name="emit", emission_intensity=10.0)],
               [Light(type=AREA, geometry_index=0, material_index=0, intensity=10.0, area=2.0)])
    s = O.OracleScene(sc)
    r = s.evaluate_light_samples([0, 0, 0], [0, 1, 0], [0, 1, 0], 0, [0, 0], 100, seed=12345)
    lo, hi = K("evaluate_area_light_bounds")
    assert lo < r[0] < hi


def test_directional_light_radiance():
    # src/light_test.cpp:171-201
    sc = Scene([], [Material()], [Light(type=DIRECTIONAL, direction=(0, -1, 0), intensity=2.0)])
    s = O.OracleScene(sc)
    rad, ray = s.light_radiance_unit_brdf(0, [0, 0, 0], [0, 1, 0])
    assert abs(rad[0] - K("directional_radiance")) < 1e-5
    assert list(ray.direction) == [0.0, 1.0, 0.0]
    assert ray.tfar == np.float32(1.0e10)


@pytest.mark.parametrize("angle,expect_kind", [(0.0, "inside"), (50.0, "between"), (70.0, "outside")])
def test_spot_light_falloff(angle, expect_kind):
    # src/light_test.cpp:203-276
    spot = Light(type=SPOT, position=(0, 10, 0), direction=(0, -1, 0), intensity=100.0, cos_inner_cone=0.70710678,
                 cos_outer_cone=0.5)
    s = O.OracleScene(Scene([], [Material()], [spot]))
    if angle == 0.0:
        rad, _ = s.light_radiance_unit_brdf(0, [0, 0, 0], [0, 1, 0])
        assert abs(rad[0] - K("spot_inside")) < 1e-5
        return
    a = np.float32(angle * math.pi / 180.0)
    ld = np.array([np.sin(a), -np.cos(a), 0], np.float32)
    p = np.array([0, 10, 0], np.float32) + ld * np.float32(10.0)
    rad, _ = s.light_radiance_unit_brdf(0, p, -ld)
    if expect_kind == "between":
        cos_l = math.cos(angle * math.pi / 180.0)
        expected = 100.0 * ((cos_l - 0.5) / (0.70710678 - 0.5)) / 100.0
        assert abs(rad[0] - expected) < 1e-4 and 0 < rad[0] < 1
    else:
        assert abs(rad[0]) < 1e-5


def test_sample_area_light():
    # src/light_test.cpp:278-306
    s = O.OracleScene(light_test_scene(area_emission=10.0))
    smp = s.sample_area_light(1, seed=12345)
    exp = K("sample_area_light")
    assert abs(smp["point"][0] - exp["point_x"]) < 1e-4
    assert abs(smp["normal"][0] - exp["normal_x"]) < 1e-4
    assert abs(smp["pdf"] - exp["pdf"]) < 1e-4
    assert abs(smp["radiance"][0] - exp["radiance_x"]) < 1e-4


# ------------------------------------------------------------ rasterizer --

def test_rasterize_quad():
    # src/rasterizer_test.cpp:7-43
    s = O.OracleScene(Scene([quad_geometry()], [Material()], []))
    r = s.rasterize(4, 4, 1)
    assert r.size == 16
    assert (r["material_id"] >= 0).all()
    exp = K("rasterize_quad_texel5")
    assert abs(r[5]["position"][0] - exp["position"][0]) < 1e-3
    assert abs(r[5]["position"][1] - exp["position"][1]) < 1e-3
    assert abs(r[5]["normal"][2] - exp["normal_z"]) < 1e-3


def test_rasterize_quad_supersampled():
    # src/rasterizer_test.cpp:45-72
    s = O.OracleScene(Scene([quad_geometry()], [Material()], []))
    r = s.rasterize(4, 4, 2)
    assert r.size == 64 and (r["material_id"] >= 0).all()


def test_validity_mask():
    # src/rasterizer_test.cpp:74-87
    from sh_baker_b200.scene import surface_points_empty
    p = surface_points_empty(3)
    p["material_id"] = [0, -1, 0]
    np.testing.assert_array_equal(O.validity_mask(p), K("validity_mask"))


def test_downsample_validity_mask():
    # src/rasterizer_test.cpp:89-126
    hi = np.zeros(16, np.uint8)
    hi[[2, 8, 9, 12, 13, 15]] = 1
    np.testing.assert_array_equal(O.downsample_validity_mask(hi, 2, 2, 2), K("downsample_validity_mask"))


# -------------------------------------------------------------- dilation --

def test_dilation_simple_fill():
    # src/dilation_test.cpp:11-34
    px = np.zeros((9, 27), np.float32)
    m = np.zeros(9, np.uint8)
    m[4] = 1
    px[4, 0] = 1.0
    O.dilate(0, 3, 3, px, m, 1)
    assert m[1] == 1 and abs(px[1, 0] - 1.0) < 1e-3
    assert m[0] == 1 and abs(px[0, 0] - 1.0) < 1e-3


def test_dilation_average_neighbors():
    # src/dilation_test.cpp:36-58
    px = np.zeros((9, 27), np.float32)
    m = np.zeros(9, np.uint8)
    m[3] = 1
    px[3, 0] = 1.0
    m[5] = 1
    px[5, 2] = 1.0
    O.dilate(0, 3, 3, px, m, 1)
    assert m[4] == 1
    assert abs(px[4, 0] - 0.5) < 1e-3 and abs(px[4, 2] - 0.5) < 1e-3


# ----------------------------------------------------------------- baker --

def test_bake_simple_quad_mt19937():
    # src/baker_test.cpp:10-65: 64 samples, 0 bounces, lit quad texel 5
    g = quad_geometry(with_tangents=False)
    mat = Material(name="white", albedo=Texture(1, 1, 4, np.array([255, 255, 255, 255], np.uint8)))
    sc = Scene([g], [mat], [Light(type=DIRECTIONAL, direction=(0, 0, -1), intensity=1.0)])
    from sh_baker_b200.scene import surface_points_empty
    pts = surface_points_empty(16)
    pts[5]["material_id"] = 0
    pts[5]["position"] = (-0.25, -0.25, 0)
    pts[5]["normal"] = (0, 0, 1)
    pts[5]["tangent"] = (1, 0, 0, 1)
    out = O.OracleScene(sc).bake(pts, 4, 4, 1, samples=64, bounces=0, rng=O.RNG_MT19937)
    assert out["sh"][1, 1, 0, 0] > K("bake_simple_quad_min_l0")


def test_downsample_sh_texture_ones():
    # src/baker_test.cpp:67-88
    x = np.ones((2, 2, 27), np.float32)
    y = O.downsample(x, 2, 2, 27, 2)
    assert y.shape == (27,)
    np.testing.assert_array_equal(y, np.ones(27, np.float32))


# ------------------------------------------------------------- occlusion --

def tri_scene(material_id=-1):
    g = Geometry(vertices=np.array([[-1, -1, 0], [1, -1, 0], [0, 1, 0]], np.float32),
                 indices=np.array([0, 1, 2], np.uint32), material_id=material_id)
    return Scene([g], [], [])


def ray(o, d, tnear=0.0, tfar=np.inf):
    return np.array([*o, *d, tnear, tfar], np.float32)


def test_occlusion_triangle_intersection():
    # src/occlusion_test.cpp:18-62
    s = O.OracleScene(tri_scene())
    h = s.find_occlusion(np.stack([ray((0, 0, 1), (0, 0, -1)), ray((2, 0, 1), (0, 0, -1)),
                                   ray((0, 0, 1), (0, 0, 1))]))
    assert h["hit"][0] == 1 and abs(h["position"][0][2]) < 1e-4 and abs(h["normal"][0][2] - 1.0) < 1e-4
    assert h["hit"][1] == 0 and h["hit"][2] == 0


def test_occlusion_ray_clipping():
    # src/occlusion_test.cpp:64-115
    s = O.OracleScene(tri_scene())
    h = s.find_occlusion(np.stack([ray((0, 0, 1), (0, 0, -1), 0.0, 0.5), ray((0, 0, 1), (0, 0, -1), 1.2),
                                   ray((0, 0, 1), (0, 0, -1), 0.1, 10.0)]))
    assert list(h["hit"]) == [0, 0, 1]
    assert abs(h["position"][2][2]) < 1e-4


def test_occlusion_multi_geometry_material():
    # src/occlusion_test.cpp:117-184
    quads = []
    for x0, mid in ((-3.0, 10), (1.0, 20)):
        quads.append(Geometry(vertices=np.array([[x0, -1, 0], [x0 + 2, -1, 0], [x0, 1, 0], [x0 + 2, 1, 0]], np.float32),
                              indices=np.array([0, 1, 2, 1, 3, 2], np.uint32), material_id=mid))
    mats = [Material() for _ in range(21)]
    s = O.OracleScene(Scene(quads, mats, []))
    h = s.find_occlusion(ray((2.8, 0.8, 5.0), (0, 0, -1))[None])
    exp = K("occlusion_multi_geometry")
    assert h["hit"][0] == 1 and h["material_id"][0] == exp["material_id"]
    np.testing.assert_allclose(h["position"][0], exp["position"], atol=1e-4)


# ---------------------------------------------------------------- philox --

def test_philox_known_answers():
    # Philox4x32-10 known-answer vectors (Salmon et al., SC'11, Random123 KAT)
    for case in GOLDEN["philox4x32_10_kat"]["value"]:
        out = O.philox([int(x, 16) for x in case["ctr"]], [int(x, 16) for x in case["key"]])
        assert [f"{int(v):08x}" for v in out] == case["out"]


# --------------------------------------------------- unit-quad closed form --

def unit_quad_expectation(scene_obj, points):
    """Config-1 closed form: no occluders, so E[SH] = sum_i w_i Y(d_i) over
    front-facing lights (d_i unnormalised for the point light, src/light.cpp:291)
    and every primary ray misses (env visibility exactly 1)."""
    exp = np.zeros((len(points), 27))
    for k, p in enumerate(points):
        if p["material_id"] < 0:
            continue
        P = p["position"].astype(np.float64)
        N = p["normal"].astype(np.float64)
        for L in scene_obj.lights:
            if L.type == DIRECTIONAL:
                d = -np.asarray(L.direction, np.float64)
                if N @ d < 0:
                    continue
                rad = L.intensity
            else:
                d = np.asarray(L.position, np.float64) - P
                dist = np.linalg.norm(d)
                if N @ (d / dist) < 0:
                    continue
                rad = L.intensity / dist ** 2
            exp[k] += np.asarray(O.accumulate_radiance([rad] * 3, d), np.float64)
    return exp


def test_unit_quad_closed_form_oracle():
    sc = scenes.unit_quad()
    s = O.OracleScene(sc)
    pts = s.rasterize(16, 16, 1)
    out = s.bake(pts, 16, 16, 1, samples=256, bounces=3, seed=1, stats=True)
    valid = pts["material_id"] >= 0
    assert valid.all()
    np.testing.assert_array_equal(out["env"].reshape(-1), np.ones(256, np.float32))
    exp = unit_quad_expectation(sc, pts)
    mean = out["sh"].reshape(-1, 27).astype(np.float64)
    # 4.5 standard errors, floored at float32 rounding of the accumulation
    tol = 4.5 * np.sqrt(out["var"].reshape(-1, 27) / 256) + 3e-5 * np.abs(exp) + 1e-6
    ok = np.abs(mean - exp) <= tol
    assert ok.mean() > 0.999, np.abs(mean - exp)[~ok][:5]
    assert abs(mean[:, 0].mean() - exp[:, 0].mean()) / exp[:, 0].mean() < 0.01
