"""The reference's own loader tests (src/loader_test.cpp) on the glTF scenes
of its data folder, through LoadScene (shb_load_gltf).  Host code only, no
GPU.  The scenes are read where they lie in the reference tree (the folder
beside $SHB_REFERENCE_SRC, else reference/data beside this repository's
folder); the tests skip where the tree is absent."""
import os
from pathlib import Path

import pytest

from oracle import build as OB
from sh_baker_b200 import api

DATA = Path(os.environ.get("SHB_REFERENCE_SRC", str(OB.REF_SRC))).parent / "data"


def scene_path(*parts):
    p = DATA.joinpath(*parts)
    if not p.exists():
        pytest.skip(f"reference data not present ({p.name})")
    return p


def test_load_cube():
    """src/loader_test.cpp:9-50 (LoadCube)."""
    sc = api.LoadScene(scene_path("cube", "Cube.gltf"))
    assert sc is not None
    assert len(sc.geometries) == 1
    g = sc.geometries[0]
    assert len(g.indices) == 36
    assert len(g.vertices) > 0
    assert len(g.vertices) == len(g.normals) == len(g.texture_uvs)
    assert len(sc.materials) == 1
    m = sc.materials[0]
    assert m.name == "Cube"
    assert m.albedo.width > 0 and m.albedo.height > 0  # Cube_BaseColor.png
    assert m.albedo.file_path is not None and Path(m.albedo.file_path).is_absolute()
    assert Path(m.albedo.file_path).exists()


def test_missing_file():
    """src/loader_test.cpp:52-55 (MissingFile)."""
    err = []
    assert api.LoadScene(DATA / "no_such_scene.gltf", err) is None and err


def test_load_box_fallback_color():
    """src/loader_test.cpp:57-81 (LoadBoxFallbackColor): an untextured
    material becomes a 1x1 RGBA texture of its baseColorFactor in sRGB."""
    sc = api.LoadScene(scene_path("box", "scene.gltf"))
    assert sc is not None
    assert len(sc.materials) == 1
    m = sc.materials[0]
    assert m.name == "Red"
    assert (m.albedo.width, m.albedo.height, m.albedo.channels) == (1, 1, 4)
    px = [int(v) for v in m.albedo.pixel_data]
    assert abs(px[0] - 231) <= 1 and px[1:] == [0, 0, 255]


@pytest.mark.parametrize("name,expect", [
    (("plane", "scene.gltf"), dict(geometries=1, triangles=2, lights=1)),
    (("DirectionalLight", "scene.gltf"), dict(geometries=3, triangles=3174, lights=1)),
    (("LightsPunctualLamp", "LightsPunctualLamp.gltf"), dict(geometries=3, triangles=6000, lights=5)),
])
def test_other_reference_scenes_load(name, expect):
    """The data folder's other complete scenes load, with their punctual
    lights and a tangent per vertex.  ABeautifulGame and Sponza lack their
    .bin buffers in the reference tree: the last test only checks that they
    fail cleanly."""
    sc = api.LoadScene(scene_path(*name))
    assert sc is not None
    assert len(sc.geometries) == expect["geometries"]
    assert sum(len(g.indices) // 3 for g in sc.geometries) == expect["triangles"]
    assert len(sc.lights) == expect["lights"]
    for g in sc.geometries:
        assert g.tangents is not None and len(g.tangents) == len(g.vertices)


@pytest.mark.parametrize("name", [("ABeautifulGame", "ABeautifulGame.gltf"), ("Sponza", "scene.gltf")])
def test_scenes_without_their_buffers_fail_cleanly(name):
    p = scene_path(*name)
    err = []
    sc = api.LoadScene(p, err)
    if sc is None:
        assert "cannot read" in err[0], err
