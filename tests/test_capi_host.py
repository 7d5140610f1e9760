"""CPU-only checks of the C ABI boundary and the host-side logic (no GPU
compute is called here)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from sh_baker_b200 import _capi as A
from sh_baker_b200 import build as B
from sh_baker_b200 import scenes
from sh_baker_b200.scene import SURFACE_POINT_DTYPE, pack_scene

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "shb.h"


@pytest.fixture(scope="module")
def lib():
    B.build()
    return A.load()


def declared_symbols():
    text = HEADER.read_text()
    return re.findall(r"SHB_API\s+[\w\s\*]+?\b(shb_\w+)\s*\(", text)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert len(names) >= 20
    assert set(names) == set(A.SIGNATURES), set(names) ^ set(A.SIGNATURES)


def test_library_exports_every_declared_symbol(lib):
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert lib.shb_abi_version() == 1


def test_library_exports_nothing_else():
    out = subprocess.run(["nm", "-D", "--defined-only", str(A.LIB_PATH)], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if " T " in line}
    ours = {s for s in exported if s.startswith("shb_")}
    assert ours == set(declared_symbols())


def test_context_without_gpu_fails_cleanly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    st = lib.shb_context_create(None, C.byref(h))
    assert st == 6  # SHB_ERR_NO_DEVICE
    assert h.value is None
    assert b"CUDA" in lib.shb_last_error() or b"device" in lib.shb_last_error()


def test_oversized_arguments_are_rejected_before_any_device_work(lib):
    """Sizes whose byte counts could wrap are refused by the C ABI itself:
    image arguments above 2^31 - 1 texels (the limit shb_rasterize applies to
    its G-buffer) and more than 2^31 - 1 rays per shb_find_occlusion call.
    The size checks come before the handle checks, so NULL handles show which
    check answered."""
    big = (65536, 32768)  # 2^31 texels
    out = C.c_void_p()

    def err(st):
        assert st == 1, st  # SHB_ERR_INVALID_ARG
        return lib.shb_last_error().decode()

    assert "2^31 - 1 texels" in err(lib.shb_gbuffer_upload(None, None, *big, C.byref(out)))
    assert "NULL" in err(lib.shb_gbuffer_upload(None, None, 4, 4, C.byref(out)))
    assert "2^31 - 1 texels" in err(lib.shb_downsample_validity_mask(None, None, 30000, 30000, 3, None, 0))
    assert "NULL" in err(lib.shb_downsample_validity_mask(None, None, 100, 100, 3, None, 0))
    assert "2^31 - 1 texels" in err(lib.shb_downsample(None, None, 46341, 46341, 1, 1, None, 0))
    assert "floats" in err(lib.shb_downsample(None, None, 2**31 - 1, 1, 28, 1, None, 0))
    assert "NULL" in err(lib.shb_downsample(None, None, 2**31 - 1, 1, 27, 1, None, 0))
    assert "2^31 - 1 texels" in err(lib.shb_dilate(None, A.DILATE_SH9, *big, None, None, 1, 0))
    assert "NULL" in err(lib.shb_dilate(None, A.DILATE_SH9, 0, 5, None, None, 1, 0))
    assert "2^31 - 1 texels" in err(lib.shb_save_sh_lightmap(None, None, None, *big, 0, b"x.exr", 0))
    assert "2^31 - 1 texels" in err(lib.shb_sh_preview(None, None, *big, None, None, 0, 0, 0, None))
    assert "rays" in err(lib.shb_find_occlusion(None, None, 2**31, None, 0))
    assert "NULL" in err(lib.shb_find_occlusion(None, None, 2**31 - 1, None, 0))


def test_scene_limits_are_checked_from_the_counts(lib):
    """Scenes whose 32-bit device indices could wrap (4 * vertex id,
    3 * triangle id) are refused from the descriptor's counts alone, before
    any data is read or the context is used: at most 2^30 - 1 vertices and
    2^30 - 1 triangles."""
    out = C.c_void_p()

    def upload(geoms):
        arr = (A.GeometryDesc * len(geoms))(*geoms)
        d = A.SceneDesc()
        d.geometries = C.cast(arr, C.POINTER(A.GeometryDesc))
        d.geometry_count = len(geoms)
        st = lib.shb_scene_upload(None, C.byref(d), C.byref(out))
        return st, lib.shb_last_error().decode()

    def geo(nv, ni):
        g = A.GeometryDesc()
        g.vertex_count, g.index_count = nv, ni
        return g

    st, msg = upload([geo(2 ** 29, 0), geo(2 ** 29, 0)])  # 2^30 vertices in total
    assert st == 1 and "scene too large" in msg, msg
    st, msg = upload([geo(3, 3 * 2 ** 29), geo(3, 3 * 2 ** 29)])  # 2^30 triangles
    assert st == 1 and "scene too large" in msg, msg
    st, msg = upload([geo(2 ** 30 - 1, 0)])  # at the limit: only the missing context is refused
    assert st == 1 and msg == "NULL argument", msg


def test_struct_layouts_match_header(tmp_path):
    """Compiles a probe against include/shb.h and compares sizes/offsets
    with the ctypes mirror."""
    src = tmp_path / "probe.c"
    fields = {
        "shb_surface_point": ["position", "normal", "tangent", "material_id"],
        "shb_geometry_desc": ["vertices", "vertex_count", "indices", "index_count", "material_id", "transform"],
        "shb_material_desc": ["albedo_pixels", "albedo_channels", "emission_intensity"],
        "shb_light_desc": ["type", "position", "intensity", "area", "material_index", "geometry_index"],
        "shb_bake_config": ["samples", "seed", "rng_mode"],
        "shb_bake_stats": ["texel_samples", "error_flags", "bvh_build_ms", "shadow_launches"],
        "shb_hit": ["position", "uv", "normal", "material_id", "hit", "t", "prim_id"],
        "shb_ray": ["origin", "direction", "tnear", "tfar"],
        "shb_scene_desc": ["geometries", "lights", "light_count"],
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for s, fs in fields.items():
        lines.append(f'printf("{s} %zu\\n", sizeof({s}));')
        for f in fs:
            lines.append(f'printf("{s}.{f} %zu\\n", offsetof({s}, {f}));')
    lines.append("return 0;}")
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    mirror = {"shb_surface_point": A.SurfacePoint, "shb_geometry_desc": A.GeometryDesc,
              "shb_material_desc": A.MaterialDesc, "shb_light_desc": A.LightDesc, "shb_bake_config": A.BakeConfig,
              "shb_bake_stats": A.BakeStats, "shb_hit": A.Hit, "shb_ray": A.Ray, "shb_scene_desc": A.SceneDesc}
    for s, fs in fields.items():
        assert int(got[s]) == C.sizeof(mirror[s]), s
        for f in fs:
            assert int(got[f"{s}.{f}"]) == getattr(mirror[s], f).offset, (s, f)
    # numpy view of SurfacePoint matches too
    assert SURFACE_POINT_DTYPE.itemsize == 64
    assert SURFACE_POINT_DTYPE.fields["tangent"][1] == int(got["shb_surface_point.tangent"])


def test_shelf_pack_no_overlap():
    rng = np.random.default_rng(0)
    sizes = [tuple(rng.uniform(0.1, 3.0, 2)) for _ in range(300)]
    res, pad = 512, 2
    _, rects = scenes.shelf_pack(sizes, res, pad)
    occ = np.zeros((res, res), np.int32)
    for x0, y0, cw, ch in rects:
        assert x0 >= 0 and y0 >= 0 and x0 + cw <= res and y0 + ch <= res
        occ[y0:y0 + ch, x0:x0 + cw] += 1
    assert occ.max() == 1


def test_room_scene_counts():
    sc = scenes.procedural_room(seed=2)
    assert sc.triangle_count == 2412
    assert len(sc.geometries) == 201 and len(sc.materials) == 8 and len(sc.lights) == 5
    desc, keep = pack_scene(sc)
    assert desc.geometry_count == 201 and desc.light_count == 5
    for g in sc.geometries:
        uv = g.lightmap_uvs
        assert (uv >= 0).all() and (uv <= 1).all()


def test_unit_quad_scene():
    sc = scenes.unit_quad()
    assert sc.triangle_count == 2 and len(sc.lights) == 2


def test_srgb_table_matches_oracle():
    """shb_srgb_to_linear_table (GetAlbedo's SRGBToLinear, src/colorspace.h:10-14)
    against the oracle's restatement, all 256 values bit for bit; host only."""
    import numpy as np

    from oracle import pyoracle as O
    from sh_baker_b200 import api
    got = api.srgb_to_linear_table()
    want = np.array([O.srgb_to_linear(i) for i in range(256)], np.float32)
    assert got.tobytes() == want.tobytes()


def test_entry_point_guard_maps_exceptions(tmp_path):
    """Every status-returning C ABI entry point runs its body in
    shb::guarded: no C++ exception reaches a C, ctypes or cgo caller.
    tests/cpp/guard_test.cpp checks the mapping (host compiler only)."""
    cuda_inc = Path("/usr/local/cuda/include")
    if not (cuda_inc / "cuda_runtime.h").exists():
        pytest.skip("CUDA headers not found")
    exe = tmp_path / "guard_test"
    subprocess.run(["g++", "-std=c++17", "-O1", "-pthread", "-I", str(cuda_inc), "-I", str(ROOT / "sh_baker_b200" / "csrc"),
                    str(ROOT / "tests" / "cpp" / "guard_test.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    # and every definition of a status-returning entry point goes through it
    csrc = ROOT / "sh_baker_b200" / "csrc"
    defs = 0
    for f in list(csrc.glob("*.cu")) + list(csrc.glob("*.cpp")):
        lines = f.read_text().split("\n")
        for i, line in enumerate(lines):
            m = re.match(r'^(extern "C" )?(SHB_API )?shb_status (shb_\w+)\(', line)
            if m:
                j = i
                while not lines[j].rstrip().endswith("{"):
                    j += 1
                assert f'guarded("{m.group(3)}"' in lines[j + 1], (f.name, m.group(3))
                defs += 1
    assert defs == 35, defs
