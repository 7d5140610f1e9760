"""Lightmap atlas (src/atlas.h, src/atlas.cpp): CalculateGeometryScales
against the reference's known answers (src/atlas_test.cpp:67-170), the
SimpleQuad case (src/atlas_test.cpp:9-65), and the contract of
CreateAtlasGeometries on meshes that need seams, folds cut apart and
degenerate faces: no texel shared by two charts, `padding` free texels
between charts, source attributes kept, one density per chart, one page.
Host code only (no GPU)."""
import numpy as np
import pytest

from atlas_check import charts_of, check_atlas
from sh_baker_b200 import _capi as A
from sh_baker_b200 import api, scenes
from sh_baker_b200.scene import Geometry, Material, Scene, Texture


def uv_geo(uvs, mid):
    return Geometry(vertices=None, indices=np.zeros(0, np.uint32), texture_uvs=np.array(uvs, np.float32),
                    material_id=mid)


def mat(w, h=None):
    return Material(albedo=Texture(w, w if h is None else h, 4, np.zeros(0, np.uint8)))


def test_geometry_scales_basic():
    s = api.CalculateGeometryScales([uv_geo([[0, 0], [1, 0], [0, 1]], 0)], [mat(100)], 1.0)
    assert s.shape == (1,) and abs(s[0] - 100.0) <= 1e-4


def test_geometry_scales_tiling():
    s = api.CalculateGeometryScales([uv_geo([[0, 0], [2, 0], [0, 2]], 0)], [mat(10)], 1.0)
    assert abs(s[0] - 20.0) <= 1e-4


def test_geometry_scales_clamping():
    g = [uv_geo([[0, 0], [1, 1]], k) for k in range(3)]
    s = api.CalculateGeometryScales(g, [mat(10), mat(10), mat(1000)], 1.0)
    np.testing.assert_allclose(s, [10.0, 10.0, 50.0], atol=1e-4)


def test_geometry_scales_density_multiplier():
    s = api.CalculateGeometryScales([uv_geo([[0, 0], [1, 1]], 0)], [mat(100)], 2.0)
    assert abs(s[0] - 200.0) <= 1e-4


def test_geometry_scales_errors_and_floors():
    """Zero UV range counts as 0.001 (src/atlas.cpp:60-62); a degenerate
    median is floored at 0.001 (:77-78); no texture UVs or a material out
    of range is an error (the reference CHECKs / indexes out of bounds)."""
    s = api.CalculateGeometryScales([uv_geo([[0.5, 0.5], [0.5, 0.5]], 0)], [mat(100)], 1.0)
    assert s[0] == np.float32(100.0) * np.sqrt(np.float32(0.001) * np.float32(0.001), dtype=np.float32)
    s = api.CalculateGeometryScales([uv_geo([[0, 0], [1, 1]], 0)] * 3, [mat(0)], 1.0)
    np.testing.assert_array_equal(s, [0, 0, 0])
    with pytest.raises(A.ShbError):
        api.CalculateGeometryScales([uv_geo(np.zeros((0, 2)), 0)], [mat(4)], 1.0)
    with pytest.raises(A.ShbError):
        api.CalculateGeometryScales([uv_geo([[0, 0]], 1)], [mat(4)], 1.0)


def mesh(v, idx, mid=0, transform=None):
    v = np.asarray(v, np.float32)
    n = len(v)
    g = Geometry(vertices=v, indices=np.asarray(idx, np.uint32).reshape(-1),
                 normals=np.tile(np.float32([0, 0, 1]), (n, 1)), tangents=np.tile(np.float32([1, 0, 0, 1]), (n, 1)),
                 texture_uvs=np.random.default_rng(n).uniform(0, 1, (n, 2)).astype(np.float32), material_id=mid)
    if transform is not None:
        g.transform = np.asarray(transform, np.float32)
    return g


def quad_scene():
    g = mesh([[-1, -1, 0], [1, -1, 0], [-1, 1, 0], [1, 1, 0]], [0, 1, 2, 2, 1, 3])
    g.texture_uvs = np.float32([[0, 0], [1, 0], [0, 1], [1, 1]])
    return Scene(geometries=[g], materials=[mat(256)])


def test_simple_quad():
    sc = quad_scene()
    r = api.CreateAtlasGeometries(sc, 256, 2)
    assert r is not None and r.width >= 0 and r.height >= 0
    assert len(r.geometries) == 1
    g = r.geometries[0]
    assert len(g.lightmap_uvs) == len(g.vertices)
    assert g.lightmap_uvs.min() >= 0.0 and g.lightmap_uvs.max() <= 1.0
    assert len(g.indices) == 6 and len(g.vertices) >= 4
    assert check_atlas(sc, r, 256, 2)[0] == 1  # a planar quad is one chart


def uv_sphere(nu=24, nv=12, r=1.0):
    v = [[0, 0, r]]
    for i in range(1, nv):
        th = np.pi * i / nv
        for j in range(nu):
            ph = 2 * np.pi * j / nu
            v.append([r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th)])
    v.append([0, 0, -r])
    idx = []
    ring = lambda i, j: 1 + (i - 1) * nu + (j % nu)  # noqa: E731
    for j in range(nu):
        idx += [0, ring(1, j), ring(1, j + 1)]
    for i in range(1, nv - 1):
        for j in range(nu):
            a, b, c, d = ring(i, j), ring(i, j + 1), ring(i + 1, j), ring(i + 1, j + 1)
            idx += [a, c, b, b, c, d]
    s = len(v) - 1
    for j in range(nu):
        idx += [s, ring(nv - 1, j + 1), ring(nv - 1, j)]
    return np.array(v, np.float32), np.array(idx, np.uint32)


def helicoid(turns=2.5, nu=80, nv=3):
    """A ramp winding round an axis, almost flat: every face is within a few
    degrees of +Z, so only the overlap test can split it."""
    v, idx = [], []
    n = int(turns * nu)
    for i in range(n + 1):
        a = 2 * np.pi * i / nu
        for k in range(nv + 1):
            r = 0.5 + 0.5 * k / nv
            v.append([r * np.cos(a), r * np.sin(a), 0.02 * a])
    for i in range(n):
        for k in range(nv):
            p, q = i * (nv + 1) + k, (i + 1) * (nv + 1) + k
            idx += [p, p + 1, q, q, p + 1, q + 1]
    return np.array(v, np.float32), np.array(idx, np.uint32)


def cylinder(n=32, h=2.0):
    v, idx = [], []
    for i in range(n):
        a = 2 * np.pi * i / n
        v += [[np.cos(a), np.sin(a), 0], [np.cos(a), np.sin(a), h]]
    for i in range(n):
        p, q = 2 * i, 2 * ((i + 1) % n)
        idx += [p, q, p + 1, p + 1, q, q + 1]
    return np.array(v, np.float32), np.array(idx, np.uint32)


def test_sphere_cylinder_and_helicoid():
    geos = [mesh(*uv_sphere()), mesh(*cylinder()), mesh(*helicoid())]
    sc = Scene(geometries=geos, materials=[mat(64)])
    r = api.CreateAtlasGeometries(sc, 512, 2)
    assert r is not None
    charts, covered = check_atlas(sc, r, 512, 2)
    assert covered > 0.3 * 512 * 512
    # a closed cylinder cannot be one planar chart; the helicoid (2.5 turns)
    # overlaps itself when flattened whole
    assert charts_of(r.geometries[1]).max() >= 2 and charts_of(r.geometries[2]).max() >= 2
    # seams split vertices
    assert len(r.geometries[1].vertices) > len(geos[1].vertices)


def test_degenerate_faces_duplicates_and_transform():
    """Repeated indices, zero-area faces, vertices duplicated at one position
    (split normals) and a non-uniform transform."""
    v = np.float32([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0], [1, 0, 0], [2, 2, 0], [3, 3, 0]])
    idx = [0, 1, 2, 2, 4, 3, 1, 1, 2, 0, 5, 6]  # face 2 repeats an index, face 3 is collinear
    tr = np.float32([[3, 0, 0, 5], [0, 0.5, 0, -1], [0, 0, 1, 2]])
    g = mesh(v, idx, transform=tr)
    g.normals[4] = [0, 0.6, 0.8]
    unused = mesh(np.vstack([v, [[9, 9, 9]]]), idx)  # vertex 7 is used by no face
    sc = Scene(geometries=[g, unused], materials=[mat(16)])
    r = api.CreateAtlasGeometries(sc, 64, 1)
    assert r is not None
    check_atlas(sc, r, 64, 1)
    assert len(r.geometries[1].vertices) <= 7 + 2 * 4


def test_density_follows_geometry_scale():
    """Two equal quads whose materials give scales 10 and 40: the second
    gets 4x the texels per unit (16x the area)."""
    q = quad_scene().geometries[0]
    a, b = mesh(q.vertices, q.indices, 0), mesh(q.vertices, q.indices, 1)
    a.texture_uvs = b.texture_uvs = q.texture_uvs
    b.transform = np.float32([[1, 0, 0, 10], [0, 1, 0, 0], [0, 0, 1, 0]])
    sc = Scene(geometries=[a, b], materials=[mat(10), mat(40)])
    r = api.CreateAtlasGeometries(sc, 256, 2)

    def uv_area(g):
        u = g.lightmap_uvs[np.asarray(g.indices).reshape(-1, 3)]
        e1, e2 = u[:, 1] - u[:, 0], u[:, 2] - u[:, 0]
        return 0.5 * np.abs(e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]).sum()

    ratio = uv_area(r.geometries[1]) / uv_area(r.geometries[0])
    assert 16 * 0.8 < ratio < 16 * 1.25
    check_atlas(sc, r, 256, 2)


def test_procedural_room():
    sc = scenes.procedural_room(seed=2, res=256)
    r = api.CreateAtlasGeometries(sc, 1024, 2)
    charts, covered = check_atlas(sc, r, 1024, 2)
    assert charts >= 200 * 5 and covered > 0.6 * 1024 * 1024


def test_deterministic_and_failures():
    sc = scenes.procedural_room(seed=5, n_boxes=20, res=64)
    a = api.CreateAtlasGeometries(sc, 256, 3)
    b = api.CreateAtlasGeometries(sc, 256, 3)
    for x, y in zip(a.geometries, b.geometries):
        np.testing.assert_array_equal(x.lightmap_uvs, y.lightmap_uvs)
        np.testing.assert_array_equal(x.indices, y.indices)
    err = []
    assert api.CreateAtlasGeometries(Scene(materials=[mat(4)]), 64, 2, error=err) is None and "no geometries" in err[0]
    err = []
    assert api.CreateAtlasGeometries(sc, 8, 4, error=err) is None and "could not fit" in err[0]
    g = quad_scene()
    g.geometries[0].tangents = None
    err = []
    assert api.CreateAtlasGeometries(g, 64, 2, error=err) is None and "tangents" in err[0]
    g = quad_scene()
    g.geometries[0].texture_uvs = None
    err = []
    assert api.CreateAtlasGeometries(g, 64, 2, error=err) is None and "texture_uvs" in err[0]


@pytest.mark.gpu
def test_atlas_rasterizes_without_overlaps(gpu_ctx):
    """The atlas of the procedural room through RasterizeScene on the GPU.
    The valid texels are at most the texel centres the charts cover plus one
    centroid texel per face.  They are at least 95 % of the covered ones:
    the rasterizer, like the reference's Barycentric (src/rasterizer.cpp:28),
    drops UV triangles whose |d00*d11 - d01^2| < 1e-8 in UV units (UV area
    under ~5e-5 of the page), keeping only their centroid texel."""
    sc = scenes.procedural_room(seed=2, res=256)
    W = 512
    r = api.CreateAtlasGeometries(sc, W, 2)
    charts, covered = check_atlas(sc, r, W, 2)
    sc.geometries = r.geometries
    pts = api.RasterizeScene(sc, api.RasterConfig(W, W, 1), ctx=gpu_ctx)
    valid = int((pts["material_id"] >= 0).sum())
    assert 0.95 * covered <= valid <= covered + sc.triangle_count
