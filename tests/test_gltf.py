"""LoadScene (shb_load_gltf, src/loader.cpp:144-844) on glTF files written
by tests/gltf_fixture.py; host code only, no GPU."""
import math
from pathlib import Path

import numpy as np
import pytest

from sh_baker_b200 import api
from sh_baker_b200.scene import AREA, DIRECTIONAL, POINT, SPOT
from tests.gltf_fixture import GltfBuilder, png_bytes, quad


def quat_matrix(q):
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def affine(R, t):
    m = np.eye(4)
    m[:3, :3] = R
    m[:3, 3] = t
    return m


def linear_to_srgb(x):
    x = np.float32(x)
    if x <= np.float32(0.0031308):
        return int(np.rint(x * np.float32(12.92) * np.float32(255.0)))
    return int(np.rint((np.float32(1.055) * np.float32(x) ** np.float32(1 / 2.4) - np.float32(0.055)) *
                       np.float32(255.0)))


def build_scene():
    b = GltfBuilder()
    pos, nrm, uv, idx = quad(2.0)
    m_factor = b.material(factor=[0.5, 0.2, 0.3, 0.7], name="factor")
    tex = np.array([[[255, 0, 0, 255], [0, 255, 0, 128], [0, 0, 255, 0]],
                    [[10, 20, 30, 40], [50, 60, 70, 80], [90, 100, 110, 120]]], np.uint8)
    m_tex = b.material(texture_png=png_bytes(tex), name="tex")
    m_emit = b.material(factor=[1, 1, 1, 1], emissive_strength=3.0, name="emit")
    # a degenerate triangle (repeated index) that the loader drops
    idx_d = np.concatenate([idx, [1, 1, 2]]).astype(np.uint32)
    p0 = b.primitive(pos, nrm, uv, uv * 0.5, idx=idx_d, material=m_factor, pad=4)
    p1 = b.primitive(pos, nrm, uv, idx=idx.astype(np.uint16), material=m_tex, idx_type=5123)
    p2 = b.primitive(pos * 0.5, nrm, uv, uv, idx=idx.astype(np.uint8), material=m_emit, idx_type=5121)
    mesh0 = b.mesh([p0, p1])
    mesh1 = b.mesh([p2])
    q = [0.0, math.sin(math.pi / 8), 0.0, math.cos(math.pi / 8)]  # 45 deg about Y
    child_m = affine(quat_matrix([math.sin(math.pi / 4), 0, 0, math.cos(math.pi / 4)]), [0, 0, 5])
    child = b.node(root=False, mesh=mesh1, matrix=list(child_m.T.reshape(-1)))
    parent = b.node(mesh=mesh0, translation=[1, 2, 3], rotation=q, scale=[2, 2, 2], children=[child])
    lp = b.light(type="point", color=[1, 0.5, 0.25], intensity=20.0)
    ls = b.light(type="spot", intensity=7.0, spot={"innerConeAngle": 0.3, "outerConeAngle": 0.6})
    ld = b.light(type="directional", intensity=2.5)
    b.node(translation=[0, 4, 0], extensions={"KHR_lights_punctual": {"light": lp}})
    b.node(translation=[1, 1, 1], rotation=q, extensions={"KHR_lights_punctual": {"light": ls}})
    b.node(rotation=[math.sin(math.pi / 4), 0, 0, math.cos(math.pi / 4)],
           extensions={"KHR_lights_punctual": {"light": ld}})
    expect = {"parent": affine(quat_matrix(q) * 2.0, [1, 2, 3]), "child_local": child_m, "q": q, "tex": tex,
              "pos": pos, "nrm": nrm, "uv": uv, "idx": idx}
    return b, expect


@pytest.mark.parametrize("container", ["data", "bin", "glb"])
def test_load_scene(tmp_path, container):
    b, ex = build_scene()
    path = b.write(tmp_path / ("scene.glb" if container == "glb" else "scene.gltf"), container)
    sc = api.LoadScene(path)
    assert sc is not None
    assert len(sc.geometries) == 3 and len(sc.materials) == 3
    g0, g1, g2 = sc.geometries
    # transforms: parent TRS, child = parent * child matrix
    np.testing.assert_allclose(g0.transform, ex["parent"][:3], atol=1e-6)
    np.testing.assert_allclose(g2.transform, (ex["parent"] @ ex["child_local"])[:3], atol=1e-5)
    # attributes, strided accessors, u8/u16/u32 indices, degenerate triangle dropped
    np.testing.assert_array_equal(g0.vertices, ex["pos"])
    np.testing.assert_array_equal(g0.normals, ex["nrm"])
    np.testing.assert_array_equal(g0.lightmap_uvs, ex["uv"] * 0.5)
    np.testing.assert_array_equal(g0.indices, ex["idx"])
    np.testing.assert_array_equal(g1.indices, ex["idx"])
    assert g1.lightmap_uvs is None
    np.testing.assert_array_equal(g2.indices, ex["idx"])
    # materials: baseColorFactor through LinearToSRGB, PNG texture, emission
    m0, m1, m2 = sc.materials
    assert (m0.albedo.width, m0.albedo.height, m0.albedo.channels) == (1, 1, 4)
    assert list(m0.albedo.pixel_data) == [linear_to_srgb(0.5), linear_to_srgb(0.2), linear_to_srgb(0.3),
                                          int(np.rint(0.7 * 255))]
    assert (m1.albedo.width, m1.albedo.height, m1.albedo.channels) == (3, 2, 4)
    np.testing.assert_array_equal(m1.albedo.pixel_data, ex["tex"].reshape(-1))
    assert m2.emission_intensity == 3.0 and m0.emission_intensity == 0.0
    # lights: area light for the emissive primitive (added while traversing),
    # then point, spot, directional in node order
    kinds = [L.type for L in sc.lights]
    assert kinds == [AREA, POINT, SPOT, DIRECTIONAL]
    area, point, spot, sun = sc.lights
    assert area.material_index == 2 and area.geometry_index == 2 and area.intensity == 3.0
    assert area.area == pytest.approx(1.0)  # object-space area of the 1x1 quad
    np.testing.assert_allclose(point.position, [0, 4, 0])
    np.testing.assert_allclose(point.color, [1, 0.5, 0.25])
    assert point.intensity == 20.0
    np.testing.assert_allclose(spot.position, [1, 1, 1])
    d = quat_matrix(ex["q"]) @ np.array([0, 0, -1.0])
    np.testing.assert_allclose(spot.direction, d / np.linalg.norm(d), atol=1e-6)
    assert spot.cos_inner_cone == pytest.approx(math.cos(0.3)) and spot.cos_outer_cone == pytest.approx(math.cos(0.6))
    np.testing.assert_allclose(sun.direction, [0, 1, 0], atol=1e-6)


def test_generated_tangents(tmp_path):
    b = GltfBuilder()
    pos, nrm, uv, idx = quad()
    b.node(mesh=b.mesh([b.primitive(pos, nrm, uv, idx=idx, material=b.material(factor=[1, 1, 1, 1]))]))
    # second primitive: v flipped -> left-handed frame
    g = api.LoadScene(b.write(tmp_path / "t.gltf")).geometries[0]
    np.testing.assert_allclose(g.tangents, np.tile([[1, 0, 0, 1]], (4, 1)), atol=1e-6)
    b2 = GltfBuilder()
    b2.node(mesh=b2.mesh([b2.primitive(pos, nrm, uv * [1, -1], idx=idx, material=b2.material(factor=[1, 1, 1, 1]))]))
    g2 = api.LoadScene(b2.write(tmp_path / "t2.gltf")).geometries[0]
    np.testing.assert_allclose(g2.tangents, np.tile([[1, 0, 0, -1]], (4, 1)), atol=1e-6)
    # a TANGENT attribute is kept as given
    t = np.tile(np.array([[0, 1, 0, -1]], np.float32), (4, 1))
    b3 = GltfBuilder()
    b3.node(mesh=b3.mesh([b3.primitive(pos, nrm, uv, tan=t, idx=idx, material=b3.material(factor=[1, 1, 1, 1]))]))
    np.testing.assert_array_equal(api.LoadScene(b3.write(tmp_path / "t3.gltf")).geometries[0].tangents, t)


def test_png_colour_types(tmp_path):
    gray = np.array([[[0], [128]], [[255], [7]]], np.uint8)
    pal = np.array([[0, 1], [2, 1]], np.uint8)
    palette = np.array([[10, 20, 30], [40, 50, 60], [70, 80, 90]], np.uint8)
    b = GltfBuilder()
    pos, nrm, uv, idx = quad()
    m_g = b.material(texture_png=png_bytes(gray))
    m_p = b.material(texture_png=png_bytes(pal, palette=palette, trns=[255, 128]))
    b.node(mesh=b.mesh([b.primitive(pos, nrm, uv, idx=idx, material=m_g),
                        b.primitive(pos, nrm, uv, idx=idx, material=m_p)]))
    sc = api.LoadScene(b.write(tmp_path / "p.gltf"))
    mg, mp = sc.materials
    assert mg.albedo.channels == 3
    np.testing.assert_array_equal(mg.albedo.pixel_data.reshape(2, 2, 3), np.repeat(gray, 3, axis=2))
    assert mp.albedo.channels == 4
    exp = np.concatenate([palette[pal], np.array([255, 128, 255])[pal][..., None]], axis=2)
    np.testing.assert_array_equal(mp.albedo.pixel_data.reshape(2, 2, 4), exp)


def test_jpeg_textures_match_libjpeg(tmp_path):
    """JPEG base-colour textures (the reference decodes them with stb_image)
    against Pillow's libjpeg decode of the same files
    (tests/golden/make_jpeg_golden.py): 4:4:4 / 4:2:2 / 4:2:0 sampling,
    restart markers, greyscale, partial MCUs, sequential and progressive
    files.  Both use exact-enough inverse DCTs and the same chroma filter, so
    pixels differ by at most 2 levels."""
    ref = np.load(Path(__file__).parent / "golden" / "jpeg_reference.npz")
    names = sorted({k[:-5] for k in ref.files if k.endswith("_jpeg")})
    assert len(names) == 14
    pos, nrm, uv, idx = quad()
    for n in names:
        b = GltfBuilder()
        m = b.material(texture_png=ref[n + "_jpeg"].tobytes())
        b.node(mesh=b.mesh([b.primitive(pos, nrm, uv, idx=idx, material=m)]))
        err = []
        sc = api.LoadScene(b.write(tmp_path / f"{n}.gltf"), err)
        assert sc is not None, (n, err)
        a = sc.materials[0].albedo
        want = ref[n + "_rgb"]
        assert (a.height, a.width, a.channels) == (*want.shape[:2], 3), n
        diff = np.abs(a.pixel_data.reshape(want.shape).astype(int) - want.astype(int))
        assert diff.max() <= 2 and diff.mean() <= 0.5, (n, diff.max(), diff.mean())


def load_texture(tmp_path, data, name):
    pos, nrm, uv, idx = quad()
    b = GltfBuilder()
    b.material(texture_png=data)
    b.node(mesh=b.mesh([b.primitive(pos, nrm, uv, idx=idx, material=0)]))
    err = []
    sc = api.LoadScene(b.write(tmp_path / f"{name}.gltf"), err)
    return (sc.materials[0].albedo if sc is not None else None), err


def test_progressive_jpeg_equals_its_sequential_twin(tmp_path):
    """A progressive file (T.81 annex G: DC and AC first and refinement
    scans, end-of-band runs) holds the same quantised coefficients as the
    sequential file of the same image and settings, so the two decode to
    the same bytes."""
    ref = np.load(Path(__file__).parent / "golden" / "jpeg_reference.npz")
    twins = sorted(k[5:-5] for k in ref.files if k.startswith("prog_") and k.endswith("_jpeg"))
    assert len(twins) == 6
    for n in twins:
        seq, err = load_texture(tmp_path, ref[n + "_jpeg"].tobytes(), n)
        assert seq is not None, (n, err)
        prog, err = load_texture(tmp_path, ref["prog_" + n + "_jpeg"].tobytes(), "prog_" + n)
        assert prog is not None, (n, err)
        assert (prog.width, prog.height) == (seq.width, seq.height)
        np.testing.assert_array_equal(prog.pixel_data, seq.pixel_data, err_msg=n)


def test_bad_progressive_scans_are_rejected(tmp_path):
    # SOF2 with no scan before EOI
    data = bytes([0xFF, 0xD8, 0xFF, 0xC2, 0x00, 0x0B, 8, 0, 1, 0, 1, 1, 1, 0x11, 0, 0xFF, 0xD9])
    tex, err = load_texture(tmp_path, data, "p")
    assert tex is None and "no image data" in err[0], err
    # an AC scan with its Ss set to 0: a DC scan (Ss = 0) must have Se = 0
    good = np.load(Path(__file__).parent / "golden" / "jpeg_reference.npz")["prog_s420_q90_jpeg"].tobytes()
    k = 2
    while True:
        k = good.index(b"\xff\xda", k)
        ns = good[k + 4]
        ss = good[k + 5 + 2 * ns]
        if ss > 0:
            break
        k += 2
    bad = bytearray(good)
    bad[k + 5 + 2 * ns] = 0  # Ss = 0 with Se > 0
    tex, err = load_texture(tmp_path, bytes(bad), "q")
    assert tex is None and "progressive scan parameters" in err[0], err


def test_defaults_and_errors(tmp_path):
    pos, nrm, uv, idx = quad()
    # no materials: a white default (a primitive must still name material 0)
    b = GltfBuilder()
    b.node(mesh=b.mesh([b.primitive(pos, nrm, uv, idx=idx, material=0)]))
    sc = api.LoadScene(b.write(tmp_path / "d.gltf"))
    assert len(sc.materials) == 1 and list(sc.materials[0].albedo.pixel_data) == [255, 255, 255, 255]
    # no indices: no triangles
    b = GltfBuilder()
    b.node(mesh=b.mesh([b.primitive(pos, nrm, uv, material=b.material(factor=[1, 1, 1, 1]))]))
    assert len(api.LoadScene(b.write(tmp_path / "n.gltf")).geometries[0].indices) == 0
    # missing NORMAL / material / TEXCOORD_0, unreadable file, JPEG texture
    for kw, what in [({"nrm": None}, "NORMAL"), ({"material": None}, "material"), ({"uv0": None}, "TEXCOORD_0")]:
        b = GltfBuilder()
        args = dict(pos=pos, nrm=nrm, uv0=uv, idx=idx, material=0)
        args.update(kw)
        if args["material"] is not None:
            b.material(factor=[1, 1, 1, 1])
        b.node(mesh=b.mesh([b.primitive(**args)]))
        err = []
        assert api.LoadScene(b.write(tmp_path / "e.gltf"), err) is None
        assert what in err[0]
    err = []
    assert api.LoadScene(tmp_path / "missing.gltf", err) is None and "cannot read" in err[0]
    b = GltfBuilder()
    b.material(texture_png=b"\xff\xd8\xff\xe0 a damaged jpeg")
    b.node(mesh=b.mesh([b.primitive(pos, nrm, uv, idx=idx, material=0)]))
    err = []
    assert api.LoadScene(b.write(tmp_path / "j.gltf"), err) is None and "JPEG" in err[0]
    b = GltfBuilder()
    b.material(texture_png=b"GIF89a neither")
    b.node(mesh=b.mesh([b.primitive(pos, nrm, uv, idx=idx, material=0)]))
    err = []
    assert api.LoadScene(b.write(tmp_path / "g.gltf"), err) is None and "PNG or JPEG" in err[0]


def test_save_scene_round_trip(tmp_path):
    """SaveScene then LoadScene gives back geometry, transforms, lightmap
    UVs, 1x1 albedos (through SRGBToLinear / LinearToSRGB) and the punctual
    lights; like the reference, emission strength is not written, so area
    lights do not come back."""
    b, ex = build_scene()
    sc = api.LoadScene(b.write(tmp_path / "in.gltf"))
    out = tmp_path / "out" / "scene.gltf"
    out.parent.mkdir()
    assert api.SaveScene(sc, out)
    assert (out.parent / "scene.bin").exists()
    back = api.LoadScene(out)
    assert back is not None and len(back.geometries) == 3
    for a, c in zip(sc.geometries, back.geometries):
        np.testing.assert_array_equal(a.vertices, c.vertices)
        np.testing.assert_array_equal(a.indices, c.indices)
        np.testing.assert_array_equal(a.tangents, c.tangents)
        np.testing.assert_allclose(a.transform, c.transform, rtol=0, atol=1e-6)
        if a.lightmap_uvs is None:
            assert c.lightmap_uvs is None
        else:
            np.testing.assert_array_equal(a.lightmap_uvs, c.lightmap_uvs)
    np.testing.assert_array_equal(sc.materials[0].albedo.pixel_data, back.materials[0].albedo.pixel_data)
    punctual = [L for L in sc.lights if L.type != AREA]
    assert [L.type for L in back.lights] == [L.type for L in punctual]
    for a, c in zip(punctual, back.lights):
        np.testing.assert_allclose(a.position, c.position, atol=1e-6)
        np.testing.assert_allclose(a.color, c.color, atol=1e-7)
        assert a.intensity == c.intensity
        if a.type != POINT:
            np.testing.assert_allclose(a.direction, c.direction, atol=1e-5)
        if a.type == SPOT:
            assert c.cos_outer_cone == pytest.approx(a.cos_outer_cone, abs=1e-6)


def test_srgb_bytes_round_trip_through_factor(tmp_path):
    """A 1x1 albedo byte survives SaveScene's SRGBToLinear and the loader's
    LinearToSRGB for all 256 values."""
    from sh_baker_b200.scene import Geometry, Material, Scene, Texture
    pos, nrm, uv, idx = quad()
    mats = [Material(albedo=Texture(1, 1, 4, np.array([v, 255 - v, (v * 7) % 256, v], np.uint8)))
            for v in range(256)]
    sc = Scene([Geometry(pos, idx, nrm, uv, uv, None, 0)], mats, [])
    assert api.SaveScene(sc, tmp_path / "s.gltf")
    back = api.LoadScene(tmp_path / "s.gltf")
    for a, c in zip(mats, back.materials):
        np.testing.assert_array_equal(a.albedo.pixel_data, c.albedo.pixel_data)


def test_damaged_jpeg_files_fail_cleanly(tmp_path):
    """Truncated and bit-flipped copies of the JPEG fixtures: the loader
    either decodes them or reports an error, without crashing."""
    ref = np.load(Path(__file__).parent / "golden" / "jpeg_reference.npz")
    rng = np.random.default_rng(0)
    pos, nrm, uv, idx = quad()
    for n in ("s420_restart", "s444_q90", "grey"):
        good = ref[n + "_jpeg"].tobytes()
        for t in range(40):
            data = bytearray(good)
            if t % 2:
                data = data[: int(rng.integers(2, len(data)))]
            else:
                for _ in range(int(rng.integers(1, 6))):
                    data[int(rng.integers(2, len(data)))] = int(rng.integers(0, 256))
            b = GltfBuilder()
            b.material(texture_png=bytes(data))
            b.node(mesh=b.mesh([b.primitive(pos, nrm, uv, idx=idx, material=0)]))
            err = []
            sc = api.LoadScene(b.write(tmp_path / f"{n}_{t}.gltf"), err)
            assert sc is not None or "JPEG" in err[0], err


@pytest.mark.parametrize("field,value,what", [
    ("count", 2 ** 53, "exceeds its buffer"),         # (count - 1) * stride would wrap 64 bits at 2^62
    ("count", 2 ** 62, "non-negative integers"),
    ("count", 1e300, "non-negative integers"),
    ("count", -1, "non-negative integers"),
    ("count", 2.5, "non-negative integers"),
    ("byteOffset", 2 ** 62, "non-negative integers"),
    ("bufferView", 1e300, "bufferView"),
])
def test_malformed_accessor_numbers_are_errors(tmp_path, field, value, what):
    """Accessor sizes and indices that are not integers in range are load
    errors, checked before any arithmetic on them (a count near 2^62 used to
    wrap the bounds check of (count - 1) * stride)."""
    pos, nrm, uv, idx = quad()
    b = GltfBuilder()
    b.node(mesh=b.mesh([b.primitive(pos, nrm, uv, idx=idx, material=b.material(factor=[1, 1, 1, 1]))]))
    acc = b.j["meshes"][0]["primitives"][0]["attributes"]["POSITION"]
    b.j["accessors"][acc][field] = value
    err = []
    assert api.LoadScene(b.write(tmp_path / "m.gltf"), err) is None
    assert what in err[0], err


def test_out_of_range_indices_are_not_cast(tmp_path):
    pos, nrm, uv, idx = quad()

    def build():
        b = GltfBuilder()
        b.node(mesh=b.mesh([b.primitive(pos, nrm, uv, idx=idx, material=b.material(factor=[1, 1, 1, 1]))]))
        return b

    b = build()
    b.j["nodes"][0]["children"] = [1e300]
    err = []
    assert api.LoadScene(b.write(tmp_path / "c.gltf"), err) is None and "node" in err[0]
    b = build()
    b.j["meshes"][0]["primitives"][0]["material"] = 1e20
    err = []
    assert api.LoadScene(b.write(tmp_path / "m.gltf"), err) is None and "material" in err[0]
    b = build()
    b.j["meshes"][0]["primitives"][0]["indices"] = -1e300  # not an index: the primitive has no triangles
    assert len(api.LoadScene(b.write(tmp_path / "i.gltf")).geometries[0].indices) == 0


def test_base_colour_factor_outside_unit_range_keeps_the_low_byte(tmp_path):
    """LinearToSRGB (src/colorspace.h:17-21) casts the rounded value to
    uint8_t.  For factors outside [0, 1] that cast is undefined in C++; the
    reference compiled for x86-64 converts to a 32-bit integer and keeps its
    low byte, and the loader writes out those steps: 1.5 rounds to 305 (byte
    49), -0.5 to -1647 (byte 145)."""
    pos, nrm, uv, idx = quad()
    b = GltfBuilder()
    b.node(mesh=b.mesh([b.primitive(pos, nrm, uv, idx=idx, material=b.material(factor=[1.5, -0.5, 0.25, 1]))]))
    px = list(api.LoadScene(b.write(tmp_path / "f.gltf")).materials[0].albedo.pixel_data)
    assert linear_to_srgb(1.5) == 305 and linear_to_srgb(-0.5) == -1647
    assert px == [305 & 0xFF, -1647 & 0xFF, linear_to_srgb(0.25), 255]
