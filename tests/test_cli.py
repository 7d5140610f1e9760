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
    r = run("--input", tmp_path / "missing.gltf")
    assert r.returncode == 1 and "does not exist" in r.stderr


def test_scene_without_lightmap_uvs_is_an_error(tmp_path):
    sc = scenes.procedural_room(seed=3, n_boxes=4, res=32)
    for g in sc.geometries:
        g.lightmap_uvs = None
    assert api.SaveScene(sc, tmp_path / "s.gltf")
    r = run("--input", tmp_path / "s.gltf", "--output", tmp_path / "out")
    assert r.returncode == 1 and "TEXCOORD_1" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("flags,files", [([], ["lightmap.exr"]),
                                         (["--luminance_only"], [f"lightmap_packed_{k}.exr" for k in range(3)]),
                                         (["--split_channels=true"], ["lightmap_L0.exr", "lightmap_L22.exr"])])
def test_bake_matches_library_pipeline(tmp_path, flags, files):
    """The CLI's files decode to what LoadScene + the bake pipeline +
    SaveSHLightMap give for the same scene, config and seed."""
    src = room_gltf(tmp_path / "in.gltf")
    out = tmp_path / "out"
    r = run("--input", src, "--output", out, "--width", 64, "--height", 64, "--samples", 8, "--bounces", 2,
            "--dilation", 2, "--supersample_scale", 2, "--seed", 7, "--debug_output", *flags)
    assert r.returncode == 0, r.stderr
    assert (out / "scene.gltf").exists() and (out / "scene.bin").exists() and (out / "material_map.png").exists()
    assert api.LoadScene(out / "scene.gltf") is not None
    sc = api.LoadScene(src)
    res = api.bake_lightmap(sc, 64, 64, samples=8, bounces=2, supersample_scale=2, dilation=2, seed=7)
    ref = tmp_path / "ref"
    ref.mkdir()
    mode = (api.SaveMode.kLuminancePacked if "--luminance_only" in flags else
            api.SaveMode.kSplitChannels if flags else api.SaveMode.kCombined)
    assert api.SaveSHLightMap(res.sh, res.env, ref / "lightmap.exr", mode)
    for f in files:
        a, b = exr_read.read(out / f), exr_read.read(ref / f)
        assert a.channels == b.channels
        for name, _ in a.channels:
            np.testing.assert_array_equal(a.raw[name], b.raw[name])
