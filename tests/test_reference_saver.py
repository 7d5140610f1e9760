"""The reference's SaveScene tests (src/saver_test.cpp:105-350) through
api.SaveScene (shb_save_gltf).  Where the reference reloads the file with
tinygltf, these read its JSON directly.  Host code only, no GPU."""
import json
import math

import numpy as np

from sh_baker_b200 import api
from sh_baker_b200.scene import DIRECTIONAL, POINT, SPOT, Geometry, Light, Material, Scene, Texture
from tests.gltf_fixture import png_bytes


def test_save_scene_with_texture(tmp_path):
    """src/saver_test.cpp:105-181 (SaveSceneWithTexture): a material whose
    albedo comes from an image file gets the file copied beside the output
    and referenced by name; buffers go to <stem>.bin."""
    src = tmp_path / "source" / "test_albedo.png"
    src.parent.mkdir()
    src.write_bytes(png_bytes(np.array([[[255, 0, 0]]], np.uint8)))
    mat = Material(name="TestMat", albedo=Texture(width=1, height=1, file_path=str(src)))
    geo = Geometry(vertices=np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32),
                   indices=np.array([0, 1, 2], np.uint32), material_id=0)
    out = tmp_path / "output" / "scene.gltf"
    out.parent.mkdir()
    assert api.SaveScene(Scene(geometries=[geo], materials=[mat]), out)
    assert out.exists()
    assert (out.parent / "test_albedo.png").exists()
    assert (out.parent / "scene.bin").exists()
    j = json.loads(out.read_text())
    assert len(j["materials"]) == 1 and j["materials"][0]["name"] == "TestMat"
    t = j["materials"][0]["pbrMetallicRoughness"]["baseColorTexture"]["index"]
    assert 0 <= t < len(j["textures"])
    s = j["textures"][t]["source"]
    assert 0 <= s < len(j["images"])
    assert j["images"][s]["uri"] == "test_albedo.png"


def test_save_scene_fallback_1x1(tmp_path):
    """src/saver_test.cpp:183-215 (SaveSceneFallback1x1): a 1x1 albedo is
    written as a linear baseColorFactor."""
    mat = Material(name="FallbackMat", albedo=Texture(width=1, height=1, channels=4,
                                                      pixel_data=np.array([255, 0, 0, 255], np.uint8)))
    out = tmp_path / "fallback.gltf"
    api.SaveScene(Scene(materials=[mat]), out)
    j = json.loads(out.read_text())
    assert len(j["materials"]) == 1
    base = j["materials"][0]["pbrMetallicRoughness"]["baseColorFactor"]
    assert len(base) == 4
    np.testing.assert_allclose(base, [1.0, 0.0, 0.0, 1.0], atol=1e-4)


def test_save_complex_scene(tmp_path):
    """src/saver_test.cpp:261-350 (SaveComplexScene): five materials, three
    geometries and a point, a spot and a directional light survive a save
    and a LoadScene."""
    white = dict(width=1, height=1, channels=4, pixel_data=np.array([255, 255, 255, 255], np.uint8))
    mats = [Material(name=f"Mat_{i}", albedo=Texture(**white)) for i in range(5)]
    geos = [Geometry(vertices=np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32),
                     normals=np.array([[0, 0, 1]] * 3, np.float32),
                     texture_uvs=np.array([[0, 0], [1, 0], [0, 1]], np.float32),
                     indices=np.array([0, 1, 2], np.uint32), material_id=i) for i in range(3)]
    lights = [Light(type=POINT, position=(10.0, 10.0, 10.0), intensity=5.0),
              Light(type=SPOT, position=(0.0, 5.0, 0.0), direction=(0.0, -1.0, 0.0),
                    cos_inner_cone=math.cos(0.5), cos_outer_cone=math.cos(0.8)),
              Light(type=DIRECTIONAL, direction=(1.0, 0.0, 0.0))]
    out = tmp_path / "complex.gltf"
    assert api.SaveScene(Scene(geometries=geos, materials=mats, lights=lights), out)
    err = []
    sc = api.LoadScene(out, err)
    assert sc is not None, err
    assert len(sc.materials) == 5 and len(sc.geometries) == 3 and len(sc.lights) == 3
    types = [l.type for l in sc.lights]
    assert types.count(POINT) == 1 and types.count(SPOT) == 1 and types.count(DIRECTIONAL) == 1
    assert [m.name for m in sc.materials] == [f"Mat_{i}" for i in range(5)]
