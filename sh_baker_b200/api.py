"""Host-side mirror of sh_baker's bake API over the C ABI.

Names, argument meaning and return values follow the reference:
RasterizeScene (src/rasterizer.h:27-28), CreateValidityMask /
DownsampleValidityMask (src/rasterizer.h:31-39), BakeSHLightMap
(src/baker.h:25-28), DownsampleSHTexture /
DownsampleEnvironmentVisibilityTexture (src/baker.h:31-36), Dilate
(src/dilation.h:14-16), FindOcclusion (src/occlusion.h:27) and
CreateAtlasGeometries / CalculateGeometryScales (src/atlas.h).  Where the
reference aborts (CHECK) these raise ShbError.  All compute runs in
libshb.so on the GPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _capi as A
from .scene import SURFACE_POINT_DTYPE, Scene, pack_scene


@dataclass
class RasterConfig:
    width: int = 1024
    height: int = 1024
    supersample_scale: int = 1

    def c(self) -> A.RasterConfig:
        return A.RasterConfig(self.width, self.height, self.supersample_scale)


@dataclass
class BakeConfig:
    samples: int = 128
    bounces: int = 3
    num_light_samples: int = 1
    seed: int = 12345
    sample_offset: int = 0

    def c(self) -> A.BakeConfig:
        cfg = A.BakeConfig()
        cfg.samples = self.samples
        cfg.bounces = self.bounces
        cfg.num_light_samples = self.num_light_samples
        cfg.seed = self.seed & 0xFFFFFFFF
        cfg.sample_offset = self.sample_offset
        cfg.rng_mode = A.RNG_PHILOX
        return cfg


@dataclass
class BakeResult:
    """sh_texture: (H*s, W*s, 9, 3) float32; environment_visibility_texture:
    (H*s, W*s) float32 (src/baker.h:16-19)."""
    sh_texture: np.ndarray
    environment_visibility_texture: np.ndarray
    stats: Optional[A.BakeStats] = None


class Context:
    """One CUDA stream on one device (shb_context)."""

    def __init__(self, device: int = 0, profiling: bool = False):
        self.lib = A.load()
        opts = A.Options()
        opts.device = device
        opts.profiling = int(profiling)
        h = C.c_void_p()
        A.check(self.lib.shb_context_create(C.byref(opts), C.byref(h)))
        self.h = h

    def kernel_launches(self) -> int:
        return int(self.lib.shb_context_kernel_launches(self.h))

    def set_stream(self, stream_ptr: int) -> None:
        A.check(self.lib.shb_context_set_stream(self.h, C.c_void_p(stream_ptr)))

    def synchronize(self) -> None:
        A.check(self.lib.shb_context_synchronize(self.h))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.shb_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceScene:
    """An uploaded scene with its GPU BVH (shb_scene)."""

    def __init__(self, ctx: Context, scene: Scene):
        self.ctx = ctx
        self.lib = ctx.lib
        desc, keep = pack_scene(scene)
        h = C.c_void_p()
        A.check(self.lib.shb_scene_upload(ctx.h, C.byref(desc), C.byref(h)))
        self.h = h
        self.n_materials = len(scene.materials)
        self.n_lights = len(scene.lights)

    def set_params(self, albedo=None, light_intensity=None, use_override=None) -> None:
        """Adjoint parameters (shb_scene_set_params): albedo (materials, 3)
        linear base colours replacing the albedo textures (of the materials
        where use_override is true; None: all), light_intensity (lights,)."""
        alb = None if albedo is None else np.ascontiguousarray(albedo, np.float32).reshape(self.n_materials, 3)
        use = None if use_override is None else np.ascontiguousarray(use_override, np.uint8).reshape(self.n_materials)
        li = None if light_intensity is None else np.ascontiguousarray(light_intensity, np.float32).reshape(
            self.n_lights)
        A.check(self.lib.shb_scene_set_params(self.h, None if alb is None else alb.ctypes.data,
                                              None if use is None else use.ctypes.data,
                                              None if li is None else li.ctypes.data))

    def bvh_info(self):
        n, t, d = C.c_uint32(), C.c_uint32(), C.c_uint32()
        A.check(self.lib.shb_scene_bvh_info(self.h, C.byref(n), C.byref(t), C.byref(d)))
        return {"wide_nodes": n.value, "triangles": t.value, "depth": d.value}

    def rebuild_bvh(self) -> None:
        A.check(self.lib.shb_scene_rebuild_bvh(self.h))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.shb_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GBuffer:
    """Device-resident texel G-buffer (shb_gbuffer)."""

    def __init__(self, ctx: Context, handle: C.c_void_p):
        self.ctx = ctx
        self.lib = ctx.lib
        self.h = handle
        w, hh = C.c_int32(), C.c_int32()
        A.check(self.lib.shb_gbuffer_dims(handle, C.byref(w), C.byref(hh)))
        self.width, self.height = w.value, hh.value

    @staticmethod
    def from_points(ctx: Context, points: np.ndarray, width: int, height: int) -> "GBuffer":
        pts = np.ascontiguousarray(points, dtype=SURFACE_POINT_DTYPE)
        if pts.size != width * height:
            raise ValueError("points size must be width*height")
        h = C.c_void_p()
        A.check(ctx.lib.shb_gbuffer_upload(ctx.h, pts.ctypes.data, width, height, C.byref(h)))
        return GBuffer(ctx, h)

    def download(self) -> np.ndarray:
        out = np.empty(self.width * self.height, dtype=SURFACE_POINT_DTYPE)
        A.check(self.lib.shb_gbuffer_download(self.h, out.ctypes.data))
        return out

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.shb_gbuffer_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default: Optional[Context] = None


def default_context() -> Context:
    global _default
    if _default is None:
        _default = Context()
    return _default


def _scene_handle(scene, ctx: Context) -> DeviceScene:
    return scene if isinstance(scene, DeviceScene) else DeviceScene(ctx, scene)


# ------------------------------------------------------ reference-named API --

def RasterizeScene(scene, config: RasterConfig, ctx: Optional[Context] = None) -> np.ndarray:
    """src/rasterizer.cpp:68-211.  Returns (W*s)*(H*s) surface points."""
    ctx = ctx or default_context()
    ds = _scene_handle(scene, ctx)
    n = config.width * config.supersample_scale * config.height * config.supersample_scale
    out = np.empty(n, dtype=SURFACE_POINT_DTYPE)
    A.check(ctx.lib.shb_rasterize(ds.h, C.byref(config.c()), out.ctypes.data, None))
    return out


def rasterize_to_device(ds: DeviceScene, config: RasterConfig) -> GBuffer:
    h = C.c_void_p()
    A.check(ds.lib.shb_rasterize(ds.h, C.byref(config.c()), None, C.byref(h)))
    return GBuffer(ds.ctx, h)


def CreateValidityMask(points: np.ndarray, ctx: Optional[Context] = None) -> np.ndarray:
    """src/rasterizer.cpp:213-220."""
    ctx = ctx or default_context()
    g = GBuffer.from_points(ctx, points, len(points), 1)
    out = np.empty(len(points), np.uint8)
    A.check(ctx.lib.shb_validity_mask(ctx.h, g.h, out.ctypes.data, 0))
    return out


def DownsampleValidityMask(high_res_mask: np.ndarray, width: int, height: int, scale: int,
                           ctx: Optional[Context] = None) -> np.ndarray:
    """src/rasterizer.cpp:222-241."""
    ctx = ctx or default_context()
    m = np.ascontiguousarray(high_res_mask, dtype=np.uint8).reshape(-1)
    if m.size != width * height * scale * scale:
        raise A.ShbError(1, "high_res_mask size != width*height*scale*scale")
    out = np.empty(width * height, np.uint8)
    A.check(ctx.lib.shb_downsample_validity_mask(ctx.h, m.ctypes.data, width, height, scale, out.ctypes.data, 0))
    return out


def BakeSHLightMap(scene, surface_points, raster_config: RasterConfig, config: BakeConfig,
                   ctx: Optional[Context] = None, with_stats: bool = False) -> BakeResult:
    """src/baker.cpp:186-304 on the GPU.  surface_points: numpy array of
    SURFACE_POINT_DTYPE or a GBuffer."""
    ctx = ctx or default_context()
    ds = _scene_handle(scene, ctx)
    W = raster_config.width * raster_config.supersample_scale
    H = raster_config.height * raster_config.supersample_scale
    g = surface_points if isinstance(surface_points, GBuffer) else GBuffer.from_points(ctx, surface_points, W, H)
    sh = np.empty((H, W, 9, 3), np.float32)
    env = np.empty((H, W), np.float32)
    out = A.BakeOutput(sh.ctypes.data, env.ctypes.data, 0, 0)
    st = A.BakeStats()
    A.check(ctx.lib.shb_bake(ds.h, g.h, C.byref(raster_config.c()), C.byref(config.c()), C.byref(out), C.byref(st)))
    return BakeResult(sh, env, st if with_stats else None)


def _downsample(x: np.ndarray, w: int, h: int, ch: int, scale: int, ctx: Context) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float32)
    ow, oh = (w, h) if scale <= 1 else (w // scale, h // scale)
    out = np.empty(ow * oh * ch, np.float32)
    A.check(ctx.lib.shb_downsample(ctx.h, x.ctypes.data, w, h, ch, scale, out.ctypes.data, 0))
    return out


def DownsampleSHTexture(sh_texture: np.ndarray, scale: int, ctx: Optional[Context] = None) -> np.ndarray:
    """src/baker.cpp:306-313: (H, W, 9, 3) -> (H/s, W/s, 9, 3)."""
    ctx = ctx or default_context()
    h, w = sh_texture.shape[:2]
    out = _downsample(sh_texture, w, h, 27, scale, ctx)
    return out.reshape((h if scale <= 1 else h // scale), (w if scale <= 1 else w // scale), 9, 3)


def DownsampleEnvironmentVisibilityTexture(env: np.ndarray, scale: int, ctx: Optional[Context] = None) -> np.ndarray:
    """src/baker.cpp:315-323."""
    ctx = ctx or default_context()
    h, w = env.shape[:2]
    out = _downsample(env, w, h, 1, scale, ctx)
    return out.reshape((h if scale <= 1 else h // scale), (w if scale <= 1 else w // scale))


def Dilate(width: int, height: int, pixels: np.ndarray, mask: np.ndarray, passes: int = 1,
           ctx: Optional[Context] = None) -> None:
    """src/dilation.cpp:7-73; pixels and mask are updated in place.  The
    element type follows the reference's instantiations: 27 floats per texel
    (SHCoeffs), float32, or uint8."""
    ctx = ctx or default_context()
    if pixels.size == 0 or mask.size == 0:
        return
    n = width * height
    if mask.dtype != np.uint8 or not mask.flags.c_contiguous or not pixels.flags.c_contiguous:
        raise TypeError("pixels and mask must be C-contiguous; mask uint8")
    if pixels.dtype == np.uint8:
        kind = A.DILATE_U8
    elif pixels.dtype == np.float32 and pixels.size == 27 * n:
        kind = A.DILATE_SH9
    elif pixels.dtype == np.float32 and pixels.size == n:
        kind = A.DILATE_F32
    else:
        raise TypeError("unsupported pixel layout")
    if mask.size != n or (kind == A.DILATE_U8 and pixels.size != n):
        return  # the reference returns when sizes disagree
    A.check(ctx.lib.shb_dilate(ctx.h, kind, width, height, pixels.ctypes.data, mask.ctypes.data, passes, 0))


def srgb_to_linear_table() -> np.ndarray:
    """SRGBToLinear (src/colorspace.h:10-14) of every 8-bit value, as the
    library computes it for GetAlbedo."""
    out = np.empty(256, np.float32)
    A.load().shb_srgb_to_linear_table(out.ctypes.data)
    return out


def material_linear_albedo(scene) -> np.ndarray:
    """Linear RGB albedo of each material's first albedo texel (the 1x1
    textures of the procedural scenes): the starting values of the adjoint's
    base-colour parameters (shb_scene_set_params)."""
    lut = srgb_to_linear_table()
    out = np.full((len(scene.materials), 3), 0.8, np.float32)
    for m, mat in enumerate(scene.materials):
        px = mat.albedo.pixel_data
        if px is not None and np.size(px) >= 3:
            out[m] = lut[np.asarray(px).reshape(-1)[:3]]
    return out


@dataclass
class BatchBake:
    """One bake of a batch: an uploaded scene, its device G-buffer and the
    BakeSHLightMap arguments."""
    scene: DeviceScene
    gbuffer: GBuffer
    raster: RasterConfig
    config: BakeConfig


def bake_batch(ctx: Context, bakes, use_graph: bool = True, autotune: bool = False, tune_cache: Optional[str] = None,
               wave_paths: int = 0, tile_texels: int = 0, grid_scale: int = 0, share_paths: int = 0,
               nee_split: int = 0, outputs=None, max_traversal_steps: int = 0, queue_capacity: int = 0,
               check: bool = True):
    """Runs many bakes through one shared sequence of wavefront launches
    (shb_bake_batch; small bakes share waves).  Returns
    ([(sh, env)] device tensors of W*s*H*s*27 and W*s*H*s floats, stats).
    `outputs` may supply those tensors (reused across calls).  Bakes of fewer
    than `share_paths` paths share waves, larger ones get their own (0: half
    a wave or the tuned value; -1: no sharing).  `nee_split`: next-event
    estimation as its own kernel by light-loop cost (0), never (1) or
    always (2); the results do not change.  `max_traversal_steps` and
    `queue_capacity` lower the device bounds (0: defaults).  With
    check=False a failing status is returned as a third value instead of
    raised, with the stats of the failed call."""
    import torch
    n = len(bakes)
    items = (A.BatchItem * max(1, n))()
    outs = []
    for i, b in enumerate(bakes):
        texels = b.gbuffer.width * b.gbuffer.height
        if outputs is not None:
            sh, env = outputs[i]
        else:
            sh = torch.empty(texels * 27, dtype=torch.float32, device="cuda")
            env = torch.empty(texels, dtype=torch.float32, device="cuda")
        outs.append((sh, env))
        items[i] = A.BatchItem(b.scene.h, b.gbuffer.h, b.raster.c(), b.config.c(), sh.data_ptr(), env.data_ptr())
    opts = A.BatchOptions()
    opts.use_graph = int(use_graph)
    opts.autotune = int(autotune)
    opts.wave_paths = wave_paths
    opts.tile_texels = tile_texels
    opts.grid_scale = grid_scale
    opts.share_paths = share_paths
    opts.nee_split = nee_split
    opts.tune_cache = tune_cache.encode() if tune_cache else None
    opts.max_traversal_steps = max_traversal_steps
    opts.queue_capacity = queue_capacity
    st = A.BakeStats()
    status = ctx.lib.shb_bake_batch(ctx.h, C.addressof(items), n, C.byref(opts), C.byref(st))
    if not check:
        return outs, st, status
    A.check(status)
    return outs, st


def bake_plain_device(b: BatchBake, sh, env) -> A.BakeStats:
    """One plain BakeSHLightMap (shb_bake) into device tensors."""
    out = A.BakeOutput(sh.data_ptr(), env.data_ptr(), 1, 0)
    st = A.BakeStats()
    A.check(b.scene.lib.shb_bake(b.scene.h, b.gbuffer.h, C.byref(b.raster.c()), C.byref(b.config.c()), C.byref(out),
                                 C.byref(st)))
    return st


def Backward(b: BatchBake, d_sh, stats: bool = False):
    """Path-replay adjoint of BakeSHLightMap (shb_backward) for the bake
    `b` (same scene parameters, G-buffer and config as its forward bake).
    d_sh: dLoss/dSH, W*s*H*s*27 floats, a CUDA tensor or a host array.
    Returns (d_albedo (materials, 3), d_light_intensity (lights,)) as
    float64 arrays, and the stats when asked."""
    ds = b.scene
    n = b.gbuffer.width * b.gbuffer.height * 27
    on_device = hasattr(d_sh, "is_cuda") and d_sh.is_cuda
    if on_device:
        import torch
        if d_sh.numel() != n or not d_sh.is_contiguous() or d_sh.dtype != torch.float32:
            raise ValueError("d_sh must be a contiguous float32 tensor of W*s*H*s*27 values")
        torch.cuda.current_stream(d_sh.device).synchronize()  # d_sh may come from torch's stream
        ptr = d_sh.data_ptr()
    else:
        host = np.ascontiguousarray(d_sh, np.float32).reshape(-1)
        if host.size != n:
            raise ValueError("d_sh must hold W*s*H*s*27 floats")
        ptr = host.ctypes.data
    d_alb = np.zeros((ds.n_materials, 3), np.float64)
    d_li = np.zeros(ds.n_lights, np.float64)
    st = A.BakeStats()
    A.check(ds.lib.shb_backward(ds.h, b.gbuffer.h, C.byref(b.raster.c()), C.byref(b.config.c()), ptr,
                                int(on_device), d_alb.ctypes.data, d_li.ctypes.data, C.byref(st)))
    return (d_alb, d_li, st) if stats else (d_alb, d_li)


@dataclass
class LightmapResult:
    """Final lightmap at width x height: sh (H, W, 9, 3), env (H, W), mask."""
    sh: np.ndarray
    env: np.ndarray
    mask: np.ndarray
    stats: A.BakeStats


def bake_lightmap(scene, width: int, height: int, samples: int = 128, bounces: int = 3, supersample_scale: int = 1,
                  dilation: int = 16, seed: int = 12345, num_light_samples: int = 1,
                  ctx: Optional[Context] = None, out: Optional[tuple] = None) -> LightmapResult:
    """The sh_baker CLI's sequence (src/main.cpp:91-163) in one device
    pipeline: raster, bake, validity mask, downsample, dilation.  `out` may
    supply (sh, env, mask) host arrays (for example pinned memory)."""
    ctx = ctx or default_context()
    ds = _scene_handle(scene, ctx)
    cfg = A.PipelineConfig(width, height, supersample_scale, samples, bounces, dilation, num_light_samples,
                           seed & 0xFFFFFFFF)
    if out is None:
        out = (np.empty((height, width, 9, 3), np.float32), np.empty((height, width), np.float32),
               np.empty((height, width), np.uint8))
    sh, env, mask = out
    st = A.BakeStats()
    A.check(ctx.lib.shb_bake_pipeline(ds.h, C.byref(cfg), sh.ctypes.data, env.ctypes.data, mask.ctypes.data,
                                      C.byref(st)))
    return LightmapResult(sh, env, mask, st)


def LoadScene(path, error: Optional[list] = None) -> Optional[Scene]:
    """src/loader.h LoadScene: a .gltf / .glb file read by shb_load_gltf
    (host only, no GPU).  None on failure, like the reference's nullopt; the
    reason is appended to `error` when given."""
    from .scene import unpack_scene
    lib = A.load()
    h = C.c_void_p()
    st = lib.shb_load_gltf(str(path).encode(), C.byref(h))
    if st != 0:
        if error is not None:
            error.append(lib.shb_last_error().decode())
        return None
    try:
        scene = unpack_scene(lib.shb_host_scene_desc(h).contents)
        # names and albedo image paths (src/loader.cpp:428-432,470)
        for i, m in enumerate(scene.materials):
            name, path = C.c_char_p(), C.c_char_p()
            A.check(lib.shb_host_scene_material_info(h, i, C.byref(name), C.byref(path)))
            m.name = (name.value or b"").decode()
            m.albedo.file_path = path.value.decode() if path.value else None
        return scene
    finally:
        lib.shb_host_scene_destroy(h)


@dataclass
class AtlasResult:
    """src/atlas.h:26-35: atlas geometries and the page size."""
    geometries: list
    width: int
    height: int


def CalculateGeometryScales(geometries, materials, density_multiplier: float) -> np.ndarray:
    """atlas_internal::CalculateGeometryScales (src/atlas.cpp:21-93) through
    shb_atlas_geometry_scales.  Only texture_uvs, material_id and the
    materials' albedo sizes are read, so geometries may carry nothing else
    (as in the reference's tests).  Raises ShbError where the reference
    CHECKs (no texture UVs, material out of range)."""
    from .scene import _f32, _ptr
    lib = A.load()
    keep = []
    geos = (A.GeometryDesc * max(1, len(geometries)))()
    for i, g in enumerate(geometries):
        uv = _f32(g.texture_uvs, 2)
        keep.append(uv)
        geos[i].texture_uvs = _ptr(uv, C.c_float)
        geos[i].vertex_count = 0 if uv is None else len(uv)
        geos[i].material_id = int(g.material_id)
    mats = (A.MaterialDesc * max(1, len(materials)))()
    for i, m in enumerate(materials):
        mats[i].albedo_width = m.albedo.width
        mats[i].albedo_height = m.albedo.height
    desc = A.SceneDesc(geos, len(geometries), mats, len(materials), None, 0)
    out = np.zeros(max(1, len(geometries)), np.float32)
    A.check(lib.shb_atlas_geometry_scales(C.byref(desc), float(density_multiplier), out.ctypes.data))
    return out[:len(geometries)]


def CreateAtlasGeometries(scene: Scene, target_resolution: int, padding: int, density_multiplier: float = 1.0,
                          error: Optional[list] = None) -> Optional[AtlasResult]:
    """src/atlas.h:49-51 CreateAtlasGeometries through shb_create_atlas (host
    only): new geometries with non-overlapping lightmap UVs in one page of
    target_resolution^2 texels, `padding` texels apart.  None when it fails
    (no geometries, charts that do not fit), like the reference's nullopt;
    the reason is appended to `error` when given."""
    from .scene import unpack_scene
    lib = A.load()
    desc, keep = pack_scene(scene)
    h = C.c_void_p()
    w, hh = C.c_int32(), C.c_int32()
    st = lib.shb_create_atlas(C.byref(desc), int(target_resolution), int(padding), float(density_multiplier),
                              C.byref(h), C.byref(w), C.byref(hh))
    if st != 0:
        if error is not None:
            error.append(lib.shb_last_error().decode())
        return None
    try:
        geos = unpack_scene(lib.shb_host_scene_desc(h).contents).geometries
    finally:
        lib.shb_host_scene_destroy(h)
    return AtlasResult(geos, w.value, hh.value)


def SaveScene(scene: Scene, path, material_names=None, albedo_files=None) -> bool:
    """src/saver.h:50-53 SaveScene: glTF + <stem>.bin (host only).  False
    on failure, like the reference.  Material names and albedo image files
    default to the materials' own (Material.name, albedo.file_path), as the
    reference reads them."""
    lib = A.load()
    desc, keep = pack_scene(scene)
    n = len(scene.materials)
    if material_names is None:
        material_names = [m.name for m in scene.materials]
    if albedo_files is None:
        albedo_files = [getattr(m.albedo, "file_path", None) for m in scene.materials]

    def strs(v):
        if v is None:
            return None
        arr = (C.c_char_p * max(1, n))()
        for i in range(n):
            arr[i] = v[i].encode() if v[i] else None
        keep.append(arr)
        return C.cast(arr, C.c_void_p)

    return lib.shb_save_gltf(C.byref(desc), strs(material_names), strs(albedo_files), str(path).encode()) == 0


class SaveMode:
    """src/saver.h:21-25."""
    kCombined = A.SAVE_COMBINED
    kSplitChannels = A.SAVE_SPLIT_CHANNELS
    kLuminancePacked = A.SAVE_LUMINANCE_PACKED


def SaveSHLightMap(sh_texture: np.ndarray, environment_visibility_texture: Optional[np.ndarray], path,
                   mode: int = SaveMode.kCombined, ctx: Optional[Context] = None) -> bool:
    """src/saver.h:45-48: sh_texture (H, W, 9, 3) float32, env (H, W) or
    None.  Returns False where the reference does (empty texture, write
    failure), with the reason in shb_last_error."""
    ctx = ctx or default_context()
    sh = np.ascontiguousarray(sh_texture, np.float32)
    if sh.ndim != 4 or sh.shape[2:] != (9, 3):
        raise ValueError("sh_texture must be (H, W, 9, 3)")
    H, W = sh.shape[:2]
    env = None
    if environment_visibility_texture is not None:
        env = np.zeros((H, W), np.float32)
        e = np.ascontiguousarray(environment_visibility_texture, np.float32).reshape(-1)[:H * W]
        env.reshape(-1)[:e.size] = e  # missing texels are 0, as in the reference
    st = ctx.lib.shb_save_sh_lightmap(ctx.h, sh.ctypes.data, None if env is None else env.ctypes.data, W, H, 0,
                                      str(path).encode(), int(mode))
    return st == 0


def FindOcclusion(scene, rays: np.ndarray, ctx: Optional[Context] = None):
    """Batched src/occlusion.cpp:9-107.  rays: (N, 8) float32 rows of
    origin(3), direction(3), tnear, tfar.  Returns a structured hit array."""
    ctx = ctx or default_context()
    ds = _scene_handle(scene, ctx)
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    hits = (A.Hit * max(1, len(r)))()
    A.check(ctx.lib.shb_find_occlusion(ds.h, r.ctypes.data, len(r), C.addressof(hits), 0))
    return hits_to_numpy(hits, len(r))


HIT_DTYPE = np.dtype([("position", "<f4", 3), ("uv", "<f4", 2), ("normal", "<f4", 3), ("material_id", "<i4"),
                      ("hit", "<i4"), ("t", "<f4"), ("prim_id", "<u4")])


def hits_to_numpy(hits, n: int) -> np.ndarray:
    buf = (C.c_char * (C.sizeof(A.Hit) * n)).from_address(C.addressof(hits))
    return np.frombuffer(bytes(buf), dtype=HIT_DTYPE, count=n).copy()
