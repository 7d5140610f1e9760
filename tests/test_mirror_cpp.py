"""The C++ mirror (include/sh_baker/sh_baker.h): the reference's own unit
tests restated in C++ against it.  Compiling is checked on the CPU; the run
needs the GPU."""
import subprocess
from pathlib import Path

import pytest

from sh_baker_b200 import build as B

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "mirror_test.cpp"


def compile_mirror(out: Path) -> Path:
    lib = B.build()
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(SRC), "-L",
           str(lib.parent), "-lshb", f"-Wl,-rpath,{lib.parent}", "-o", str(out)]
    subprocess.run(cmd, check=True)
    return out


def test_mirror_compiles_and_runs_host_tests(tmp_path):
    """Compiles; the host-side tests (atlas) run without a GPU."""
    exe = compile_mirror(tmp_path / "mirror_test")
    r = subprocess.run([str(exe), "--host"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "OK (0 failures)" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_mirror_runs_reference_unit_tests(tmp_path):
    exe = compile_mirror(tmp_path / "mirror_test")
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK (0 failures)" in r.stdout


def test_mirror_load_and_save_scene(tmp_path):
    """sh_baker::LoadScene / SaveScene and the scene.h helpers
    (tests/cpp/scene_io_test.cpp, host code): a save and load round trip
    keeps names, lightmap UVs, tangents and lights; an emissive primitive's
    area light points at its material and geometry in the returned scene; a
    missing file is nullopt; the reference's TransformedVertices / Normals /
    Tangents tests hold, the rotation part strips a non-uniform scale, and
    SurfaceArea sums object-space triangle areas."""
    import numpy as np

    from tests.gltf_fixture import GltfBuilder, quad
    lib = B.build()
    exe = tmp_path / "scene_io_test"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "cpp" / "scene_io_test.cpp"), "-L", str(lib.parent), "-lshb",
                    f"-Wl,-rpath,{lib.parent}", "-o", str(exe)], check=True)

    def run(*args):
        r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stdout + r.stderr

    run("roundtrip", tmp_path)
    pos, nrm, uv, idx = quad()
    b = GltfBuilder()
    plain = b.material(factor=[1, 1, 1, 1], name="Plain")
    glow = b.material(factor=[1, 0.5, 0.2, 1], emissive_strength=4.0, name="Glow")
    b.node(mesh=b.mesh([b.primitive(pos, nrm, uv, idx=idx, material=plain)]))
    b.node(mesh=b.mesh([b.primitive(pos + np.float32(1), nrm, uv, idx=idx, material=glow)]))
    run("emissive", b.write(tmp_path / "glow.gltf"))
    run("missing", tmp_path / "no_such.gltf")
    run("transforms", "-")
