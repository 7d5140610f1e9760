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
