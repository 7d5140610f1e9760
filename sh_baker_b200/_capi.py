"""ctypes mirror of include/shb.h and the loader of libshb.so.

The library is the CUDA implementation of the bake; there is no CPU
fallback.  load() raises if libshb.so is missing or cannot be loaded.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libshb.so"

SHB_OK = 0
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "CUDA", 4: "TIMEOUT", 5: "INTERNAL", 6: "NO_DEVICE"}

LIGHT_POINT, LIGHT_DIRECTIONAL, LIGHT_SPOT, LIGHT_AREA = 0, 1, 2, 3
DILATE_SH9, DILATE_F32, DILATE_U8 = 0, 1, 2
RNG_PHILOX = 0

f32p = C.POINTER(C.c_float)
u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)


class GeometryDesc(C.Structure):
    _fields_ = [
        ("vertices", f32p), ("normals", f32p), ("texture_uvs", f32p), ("lightmap_uvs", f32p),
        ("tangents", f32p), ("vertex_count", C.c_uint32), ("indices", u32p), ("index_count", C.c_uint32),
        ("material_id", C.c_int32), ("transform", C.c_float * 12),
    ]


class MaterialDesc(C.Structure):
    _fields_ = [
        ("albedo_pixels", u8p), ("albedo_width", C.c_uint32), ("albedo_height", C.c_uint32),
        ("albedo_channels", C.c_uint32), ("emission_intensity", C.c_float),
    ]


class LightDesc(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("position", C.c_float * 3), ("direction", C.c_float * 3), ("color", C.c_float * 3),
        ("intensity", C.c_float), ("cos_inner_cone", C.c_float), ("cos_outer_cone", C.c_float),
        ("area", C.c_float), ("material_index", C.c_int32), ("geometry_index", C.c_int32),
    ]


class SceneDesc(C.Structure):
    _fields_ = [
        ("geometries", C.POINTER(GeometryDesc)), ("geometry_count", C.c_uint32),
        ("materials", C.POINTER(MaterialDesc)), ("material_count", C.c_uint32),
        ("lights", C.POINTER(LightDesc)), ("light_count", C.c_uint32),
    ]


class RasterConfig(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("supersample_scale", C.c_int32)]


class SurfacePoint(C.Structure):
    _fields_ = [
        ("position", C.c_float * 3), ("normal", C.c_float * 3), ("_pad0", C.c_float * 2),
        ("tangent", C.c_float * 4), ("material_id", C.c_int32), ("_pad1", C.c_int32 * 3),
    ]


class BakeConfig(C.Structure):
    _fields_ = [
        ("samples", C.c_int32), ("bounces", C.c_int32), ("num_light_samples", C.c_int32), ("seed", C.c_uint32),
        ("sample_offset", C.c_int32), ("rng_mode", C.c_int32), ("reserved", C.c_int32 * 2),
    ]


class BakeOutput(C.Structure):
    _fields_ = [("sh", C.c_void_p), ("env_visibility", C.c_void_p), ("device_ptrs", C.c_int32),
                ("reserved", C.c_int32)]


class Ray(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("direction", C.c_float * 3), ("tnear", C.c_float), ("tfar", C.c_float)]


class Hit(C.Structure):
    _fields_ = [
        ("position", C.c_float * 3), ("uv", C.c_float * 2), ("normal", C.c_float * 3), ("material_id", C.c_int32),
        ("hit", C.c_int32), ("t", C.c_float), ("prim_id", C.c_uint32),
    ]


class BakeStats(C.Structure):
    _fields_ = [
        ("texel_samples", C.c_uint64), ("valid_texels", C.c_uint64), ("extend_rays", C.c_uint64),
        ("shadow_rays", C.c_uint64), ("kernel_launches", C.c_uint64), ("error_flags", C.c_uint32),
        ("waves", C.c_uint32), ("bvh_build_ms", C.c_double), ("trace_ms", C.c_double),
        ("extend_kernel_ms", C.c_double), ("shadow_kernel_ms", C.c_double), ("shade_kernel_ms", C.c_double),
        ("extend_launches", C.c_uint64), ("shadow_launches", C.c_uint64),
    ]


class PipelineConfig(C.Structure):
    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32), ("supersample_scale", C.c_int32), ("samples", C.c_int32),
        ("bounces", C.c_int32), ("dilation", C.c_int32), ("num_light_samples", C.c_int32), ("seed", C.c_uint32),
    ]


class BatchItem(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("gbuffer", C.c_void_p), ("raster", RasterConfig), ("config", BakeConfig),
                ("sh", C.c_void_p), ("env_visibility", C.c_void_p)]


class BatchOptions(C.Structure):
    _fields_ = [("use_graph", C.c_int32), ("autotune", C.c_int32), ("wave_paths", C.c_int32),
                ("tile_texels", C.c_int32), ("grid_scale", C.c_int32), ("share_paths", C.c_int32),
                ("nee_split", C.c_int32), ("max_traversal_steps", C.c_int32),
                ("tune_cache", C.c_char_p), ("queue_capacity", C.c_int32), ("reserved", C.c_int32 * 3)]


class Options(C.Structure):
    _fields_ = [("device", C.c_int32), ("profiling", C.c_int32), ("reserved", C.c_int32 * 6)]


assert C.sizeof(SurfacePoint) == 64
assert C.sizeof(Hit) == 48

SAVE_COMBINED, SAVE_SPLIT_CHANNELS, SAVE_LUMINANCE_PACKED = 0, 1, 2
PREVIEW_L0, PREVIEW_SH, PREVIEW_SH_PACKED = 0, 1, 2

vp = C.c_void_p
# name -> (restype, argtypes); every symbol declared in include/shb.h
SIGNATURES = {
    "shb_abi_version": (C.c_int32, []),
    "shb_last_error": (C.c_char_p, []),
    "shb_srgb_to_linear_table": (None, [vp]),
    "shb_test_fail_allocation_after": (None, [C.c_int32]),
    "shb_context_create": (C.c_int, [C.POINTER(Options), C.POINTER(vp)]),
    "shb_context_destroy": (C.c_int, [vp]),
    "shb_context_set_stream": (C.c_int, [vp, vp]),
    "shb_context_synchronize": (C.c_int, [vp]),
    "shb_context_kernel_launches": (C.c_uint64, [vp]),
    "shb_scene_upload": (C.c_int, [vp, C.POINTER(SceneDesc), C.POINTER(vp)]),
    "shb_scene_destroy": (C.c_int, [vp]),
    "shb_scene_rebuild_bvh": (C.c_int, [vp]),
    "shb_scene_bvh_info": (C.c_int, [vp, u32p, u32p, u32p]),
    "shb_rasterize": (C.c_int, [vp, C.POINTER(RasterConfig), vp, C.POINTER(vp)]),
    "shb_gbuffer_upload": (C.c_int, [vp, vp, C.c_int32, C.c_int32, C.POINTER(vp)]),
    "shb_gbuffer_download": (C.c_int, [vp, vp]),
    "shb_gbuffer_dims": (C.c_int, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "shb_gbuffer_destroy": (C.c_int, [vp]),
    "shb_validity_mask": (C.c_int, [vp, vp, vp, C.c_int32]),
    "shb_downsample_validity_mask": (C.c_int, [vp, vp, C.c_int32, C.c_int32, C.c_int32, vp, C.c_int32]),
    "shb_bake": (C.c_int, [vp, vp, C.POINTER(RasterConfig), C.POINTER(BakeConfig), C.POINTER(BakeOutput),
                           C.POINTER(BakeStats)]),
    "shb_downsample": (C.c_int, [vp, vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, vp, C.c_int32]),
    "shb_dilate": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32, vp, vp, C.c_int32, C.c_int32]),
    "shb_find_occlusion": (C.c_int, [vp, vp, C.c_int64, vp, C.c_int32]),
    "shb_bake_pipeline": (C.c_int, [vp, C.POINTER(PipelineConfig), vp, vp, vp, C.POINTER(BakeStats)]),
    "shb_dilate_noalloc": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32, vp, vp, C.c_int32]),
    "shb_bake_batch": (C.c_int, [vp, vp, C.c_int32, C.POINTER(BatchOptions), C.POINTER(BakeStats)]),
    "shb_scene_set_params": (C.c_int, [vp, vp, vp, vp]),
    "shb_load_gltf": (C.c_int, [C.c_char_p, C.POINTER(vp)]),
    "shb_host_scene_desc": (C.POINTER(SceneDesc), [vp]),
    "shb_host_scene_destroy": (C.c_int, [vp]),
    "shb_rotation_part": (C.c_int, [vp, vp]),
    "shb_host_scene_material_info": (C.c_int, [vp, C.c_int32, C.POINTER(C.c_char_p), C.POINTER(C.c_char_p)]),
    "shb_save_gltf": (C.c_int, [C.POINTER(SceneDesc), vp, vp, C.c_char_p]),
    "shb_atlas_geometry_scales": (C.c_int, [C.POINTER(SceneDesc), C.c_float, vp]),
    "shb_create_atlas": (C.c_int, [C.POINTER(SceneDesc), C.c_uint32, C.c_uint32, C.c_float, C.POINTER(vp),
                                   C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "shb_sh_preview": (C.c_int, [vp, vp, C.c_int32, C.c_int32, vp, vp, C.c_int32, C.c_int32, C.c_int32, vp]),
    "shb_exr_load_channels": (C.c_int, [C.c_char_p, vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                        vp]),
    "shb_write_png": (C.c_int, [C.c_char_p, C.c_int32, C.c_int32, C.c_int32, vp]),
    "shb_save_sh_lightmap": (C.c_int, [vp, vp, vp, C.c_int32, C.c_int32, C.c_int32, C.c_char_p, C.c_int32]),
    "shb_backward": (C.c_int, [vp, vp, C.POINTER(RasterConfig), C.POINTER(BakeConfig), vp, C.c_int32, vp, vp,
                               C.POINTER(BakeStats)]),
}

_lib = None


class ShbError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"shb status {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def load(path: Path | str | None = None):
    """Loads libshb.so (building is a separate step: sh_baker_b200.build).
    $SHB_LIBRARY names another build of the same sources (a tuning variant
    from sh_baker_b200.build.build(variant=...))."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    env = os.environ.get("SHB_LIBRARY")
    p = Path(path) if path else (Path(env) if env else LIB_PATH)
    if not p.exists():
        raise RuntimeError(f"libshb.so not found at {p}; run `python -m sh_baker_b200.build` (no CPU fallback exists)")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(status: int):
    if status != SHB_OK:
        msg = load().shb_last_error()
        raise ShbError(status, msg.decode() if msg else "")
