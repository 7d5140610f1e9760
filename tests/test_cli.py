"""The sh_baker command line (sh_baker_b200/cli/sh_baker.cpp): the reference's
flags (src/main.cpp:14-35) and output files (lightmap.exr in the three save
modes, scene.gltf, material_map.png)."""
import subprocess

import numpy as np
import pytest

from oracle import exr_read
from sh_baker_b200 import api, scenes
from sh_baker_b200 import build as B


def cli():
    B.build()
    return str(B.CLI)


def run(*args, timeout=600):
    return subprocess.run([cli(), *map(str, args)], capture_output=True, text=True, timeout=timeout)


def room_gltf(path, res=64):
    sc = scenes.procedural_room(seed=3, n_boxes=10, res=res)
    assert api.SaveScene(sc, path)
    return path


def test_usage_and_flag_errors(tmp_path):
    r = run()
    assert r.returncode == 1 and "Usage" in r.stderr
    assert run("--no_such_flag=1").returncode == 1
    assert run("--width", "abc", "--input", "x").returncode == 1
    # int32 flags, as gflags parses them: values beyond int32 are errors, not wrapped
    for v in ("4294967297", "-2147483649", "99999999999999999999"):
        r = run(f"--width={v}", "--input", "x")
        assert r.returncode == 1 and "bad value for --width" in r.stderr, v
    r = run("--input", tmp_path / "missing.gltf")
    assert r.returncode == 1 and "does not exist" in r.stderr


def no_lightmap_uvs_gltf(path):
    sc = scenes.procedural_room(seed=3, n_boxes=4, res=32)
    for g in sc.geometries:
        g.lightmap_uvs = None
    assert api.SaveScene(sc, path)
    return path


def test_keep_lightmap_uvs_needs_them(tmp_path):
    src = no_lightmap_uvs_gltf(tmp_path / "s.gltf")
    r = run("--input", src, "--output", tmp_path / "out", "--keep_lightmap_uvs")
    assert r.returncode == 1 and "TEXCOORD_1" in r.stderr


def test_atlas_that_cannot_fit_fails(tmp_path):
    """The atlas runs before any GPU work; 200+ charts cannot fit a 16x16
    page with 8 texels of padding (src/main.cpp:76-83)."""
    src = room_gltf(tmp_path / "in.gltf")
    r = run("--input", src, "--output", tmp_path / "out", "--width", 16, "--height", 16, "--dilation", 8)
    assert r.returncode == 1 and "Atlas generation failed" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("flags,files", [([], ["lightmap.exr"]),
                                         (["--luminance_only"], [f"lightmap_packed_{k}.exr" for k in range(3)]),
                                         (["--split_channels=true"], ["lightmap_L0.exr", "lightmap_L22.exr"]),
                                         (["--keep_lightmap_uvs", "--density_multiplier=2"], ["lightmap.exr"])])
def test_bake_matches_library_pipeline(tmp_path, flags, files):
    """The CLI's files decode to what LoadScene + CreateAtlasGeometries +
    the bake pipeline + SaveSHLightMap give for the same scene, config and
    seed; scene.gltf carries the atlas UVs as TEXCOORD_1."""
    src = room_gltf(tmp_path / "in.gltf")
    out = tmp_path / "out"
    r = run("--input", src, "--output", out, "--width", 64, "--height", 64, "--samples", 8, "--bounces", 2,
            "--dilation", 2, "--supersample_scale", 2, "--seed", 7, "--debug_output", *flags)
    assert r.returncode == 0, r.stderr
    assert (out / "scene.gltf").exists() and (out / "scene.bin").exists() and (out / "material_map.png").exists()
    sc = api.LoadScene(src)
    if "--keep_lightmap_uvs" not in flags:
        atlas = api.CreateAtlasGeometries(sc, 64, 2, 1.0)
        sc.geometries = atlas.geometries
    saved = api.LoadScene(out / "scene.gltf")
    assert saved is not None
    for a, b in zip(saved.geometries, sc.geometries):
        np.testing.assert_array_equal(a.lightmap_uvs, b.lightmap_uvs)
    res = api.bake_lightmap(sc, 64, 64, samples=8, bounces=2, supersample_scale=2, dilation=2, seed=7)
    ref = tmp_path / "ref"
    ref.mkdir()
    mode = (api.SaveMode.kLuminancePacked if "--luminance_only" in flags else
            api.SaveMode.kSplitChannels if "--split_channels=true" in flags else api.SaveMode.kCombined)
    assert api.SaveSHLightMap(res.sh, res.env, ref / "lightmap.exr", mode)
    for f in files:
        a, b = exr_read.read(out / f), exr_read.read(ref / f)
        assert a.channels == b.channels
        for name, _ in a.channels:
            np.testing.assert_array_equal(a.raw[name], b.raw[name])


@pytest.mark.gpu
def test_scene_without_lightmap_uvs_bakes(tmp_path):
    """Like the reference, the CLI makes its own lightmap UVs: a scene with
    no TEXCOORD_1 bakes and gets them in scene.gltf."""
    src = no_lightmap_uvs_gltf(tmp_path / "s.gltf")
    out = tmp_path / "out"
    r = run("--input", src, "--output", out, "--width", 64, "--height", 64, "--samples", 4, "--bounces", 1,
            "--dilation", 2)
    assert r.returncode == 0, r.stderr
    ex = exr_read.read(out / "lightmap.exr")
    assert ex.half("L0.R").max() > 0
    saved = api.LoadScene(out / "scene.gltf")
    assert all(g.lightmap_uvs is not None for g in saved.geometries)
