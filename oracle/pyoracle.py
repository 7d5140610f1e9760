"""ctypes bindings of the CPU oracle (oracle/shb_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as
the checker and by bench.py's CPU-baseline leg; never by the product.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from sh_baker_b200 import _capi as A
from sh_baker_b200.scene import SURFACE_POINT_DTYPE, Scene, pack_scene

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

RNG_MT19937 = 0
RNG_PHILOX = 1


class BakeArgs(C.Structure):
    _fields_ = [
        ("samples", C.c_int32), ("bounces", C.c_int32), ("num_light_samples", C.c_int32), ("seed", C.c_uint32),
        ("sample_offset", C.c_int32), ("rng_mode", C.c_int32), ("fp64", C.c_int32), ("threads", C.c_int32),
        ("texel_subset", C.POINTER(C.c_int64)), ("subset_count", C.c_int64),
        ("sh_out", C.POINTER(C.c_float)), ("env_out", C.POINTER(C.c_float)),
        ("sh_var_out", C.POINTER(C.c_double)), ("sh_mean64_out", C.POINTER(C.c_double)),
        ("rays_traced", C.c_uint64), ("texel_samples", C.c_uint64),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        from . import build as _build
        _build.build()
        _lib = C.CDLL(str(LIB))
        vp = C.c_void_p
        f = _lib
        f.oracle_scene_create.restype = vp
        f.oracle_scene_create.argtypes = [C.POINTER(A.SceneDesc)]
        f.oracle_scene_destroy.argtypes = [vp]
        f.oracle_rasterize.restype = C.c_int
        f.oracle_rasterize.argtypes = [vp, C.POINTER(A.RasterConfig), vp]
        f.oracle_validity_mask.argtypes = [vp, C.c_int64, vp]
        f.oracle_downsample_validity_mask.restype = C.c_int
        f.oracle_downsample_validity_mask.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp]
        f.oracle_downsample.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp]
        f.oracle_dilate.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp, C.c_int]
        f.oracle_bake.restype = C.c_int
        f.oracle_bake.argtypes = [vp, vp, C.POINTER(A.RasterConfig), C.POINTER(BakeArgs)]
        f.oracle_find_occlusion.argtypes = [vp, vp, C.c_int64, vp]
        f.oracle_accumulate_radiance.argtypes = [vp, vp, vp]
        f.oracle_srgb_to_linear.restype = C.c_float
        f.oracle_srgb_to_linear.argtypes = [C.c_uint8]
        f.oracle_get_albedo.argtypes = [vp, C.c_int, vp, vp]
        f.oracle_get_alpha.restype = C.c_float
        f.oracle_get_alpha.argtypes = [vp, C.c_int, vp]
        f.oracle_get_emission.argtypes = [vp, C.c_int, vp, vp]
        f.oracle_evaluate_light_samples.argtypes = [vp, vp, vp, vp, C.c_int, vp, C.c_uint, C.c_uint32, C.c_int, vp]
        f.oracle_sample_area_light.argtypes = [vp, C.c_int, C.c_uint32, vp]
        f.oracle_light_radiance_unit_brdf.argtypes = [vp, C.c_int, vp, vp, vp, vp]
        f.oracle_philox4x32_10.argtypes = [vp, vp, vp]
        f.oracle_scene_set_params.argtypes = [vp, vp, vp, vp]
        f.oracle_bake_grad.restype = C.c_int
        f.oracle_bake_grad.argtypes = [vp, vp, C.POINTER(A.RasterConfig), C.POINTER(BakeArgs), vp, vp, vp]
    return _lib


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class OracleScene:
    def __init__(self, scene: Scene):
        desc, keep = pack_scene(scene)
        self.h = lib().oracle_scene_create(C.byref(desc))
        self.scene = scene

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_scene_destroy(self.h)
            self.h = None

    def rasterize(self, width: int, height: int, scale: int = 1) -> np.ndarray:
        n = width * scale * height * scale
        out = np.empty(n, dtype=SURFACE_POINT_DTYPE)
        rc = lib().oracle_rasterize(self.h, C.byref(A.RasterConfig(width, height, scale)), out.ctypes.data)
        if rc != 0:
            raise ValueError(f"oracle_rasterize failed ({rc})")
        return out

    def bake(self, points: np.ndarray, width: int, height: int, scale: int, samples: int, bounces: int,
             seed: int = 12345, rng: int = RNG_PHILOX, fp64: bool = False, num_light_samples: int = 1,
             subset=None, threads: int = 0, stats: bool = False, sample_offset: int = 0):
        W, H = width * scale, height * scale
        pts = np.ascontiguousarray(points, dtype=SURFACE_POINT_DTYPE)
        sh = np.zeros((H * W, 27), np.float32)
        env = np.zeros(H * W, np.float32)
        var = np.zeros((H * W, 27), np.float64) if stats else None
        m64 = np.zeros((H * W, 27), np.float64) if stats else None
        a = BakeArgs()
        a.samples, a.bounces, a.num_light_samples = samples, bounces, num_light_samples
        a.seed, a.sample_offset, a.rng_mode, a.fp64, a.threads = seed & 0xFFFFFFFF, sample_offset, rng, int(fp64), threads
        sub = None
        if subset is not None:
            sub = np.ascontiguousarray(subset, dtype=np.int64)
            a.texel_subset = sub.ctypes.data_as(C.POINTER(C.c_int64))
            a.subset_count = sub.size
        a.sh_out = sh.ctypes.data_as(C.POINTER(C.c_float))
        a.env_out = env.ctypes.data_as(C.POINTER(C.c_float))
        if stats:
            a.sh_var_out = var.ctypes.data_as(C.POINTER(C.c_double))
            a.sh_mean64_out = m64.ctypes.data_as(C.POINTER(C.c_double))
        rc = lib().oracle_bake(self.h, pts.ctypes.data, C.byref(A.RasterConfig(width, height, scale)), C.byref(a))
        if rc != 0:
            raise ValueError(f"oracle_bake failed ({rc})")
        out = {"sh": sh.reshape(H, W, 9, 3), "env": env.reshape(H, W), "rays": a.rays_traced,
               "texel_samples": a.texel_samples}
        if stats:
            out["var"] = var.reshape(H, W, 9, 3)
            out["mean64"] = m64.reshape(H, W, 9, 3)
        return out

    def set_params(self, albedo=None, light_intensity=None, use_override=None) -> None:
        nm, nl = len(self.scene.materials), len(self.scene.lights)
        alb = None if albedo is None else _f(albedo).reshape(nm, 3)
        use = None if use_override is None else np.ascontiguousarray(use_override, np.uint8).reshape(nm)
        li = None if light_intensity is None else _f(light_intensity).reshape(nl)
        lib().oracle_scene_set_params(self.h, None if alb is None else alb.ctypes.data,
                                      None if use is None else use.ctypes.data, None if li is None else li.ctypes.data)

    def bake_grad(self, points: np.ndarray, width: int, height: int, scale: int, samples: int, bounces: int,
                  dsh: np.ndarray, seed: int = 12345, num_light_samples: int = 1, subset=None, threads: int = 0,
                  sample_offset: int = 0):
        """FP64 forward-mode gradient of sum(dsh * SH): (d_albedo (M, 3), d_light (L,))."""
        pts = np.ascontiguousarray(points, dtype=SURFACE_POINT_DTYPE)
        g = np.ascontiguousarray(dsh, np.float32).reshape(-1)
        if g.size != pts.size * 27:
            raise ValueError("dsh must hold 27 floats per texel")
        a = BakeArgs()
        a.samples, a.bounces, a.num_light_samples = samples, bounces, num_light_samples
        a.seed, a.sample_offset, a.rng_mode, a.fp64, a.threads = seed & 0xFFFFFFFF, sample_offset, RNG_PHILOX, 1, threads
        sub = None
        if subset is not None:
            sub = np.ascontiguousarray(subset, dtype=np.int64)
            a.texel_subset = sub.ctypes.data_as(C.POINTER(C.c_int64))
            a.subset_count = sub.size
        d_alb = np.zeros((len(self.scene.materials), 3), np.float64)
        d_li = np.zeros(max(1, len(self.scene.lights)), np.float64)
        rc = lib().oracle_bake_grad(self.h, pts.ctypes.data, C.byref(A.RasterConfig(width, height, scale)),
                                    C.byref(a), g.ctypes.data, d_alb.ctypes.data, d_li.ctypes.data)
        if rc != 0:
            raise ValueError(f"oracle_bake_grad failed ({rc})")
        return d_alb, d_li[:len(self.scene.lights)]

    def find_occlusion(self, rays: np.ndarray) -> np.ndarray:
        from sh_baker_b200.api import HIT_DTYPE
        r = _f(rays).reshape(-1, 8)
        out = np.zeros(len(r), dtype=HIT_DTYPE)
        lib().oracle_find_occlusion(self.h, r.ctypes.data, len(r), out.ctypes.data)
        return out

    def albedo(self, m: int, uv) -> np.ndarray:
        o = np.zeros(3, np.float32)
        lib().oracle_get_albedo(self.h, m, _f(uv).ctypes.data, o.ctypes.data)
        return o

    def alpha(self, m: int, uv) -> float:
        return float(lib().oracle_get_alpha(self.h, m, _f(uv).ctypes.data))

    def emission(self, m: int, uv) -> np.ndarray:
        o = np.zeros(3, np.float32)
        lib().oracle_get_emission(self.h, m, _f(uv).ctypes.data, o.ctypes.data)
        return o

    def evaluate_light_samples(self, p, n, wo, mat: int, uv, num_samples: int, seed: int = 12345,
                               empty_bvh: bool = True) -> np.ndarray:
        o = np.zeros(3, np.float32)
        pp, nn, ww, uu = _f(p), _f(n), _f(wo), _f(uv)
        lib().oracle_evaluate_light_samples(self.h, pp.ctypes.data, nn.ctypes.data, ww.ctypes.data, mat,
                                            uu.ctypes.data, num_samples, seed, int(empty_bvh), o.ctypes.data)
        return o

    def sample_area_light(self, light: int, seed: int = 12345) -> dict:
        o = np.zeros(10, np.float32)
        lib().oracle_sample_area_light(self.h, light, seed, o.ctypes.data)
        return {"point": o[0:3], "normal": o[3:6], "radiance": o[6:9], "pdf": float(o[9])}

    def light_radiance_unit_brdf(self, light: int, p, n):
        rad = np.zeros(3, np.float32)
        ray = A.Ray()
        pp, nn = _f(p), _f(n)
        lib().oracle_light_radiance_unit_brdf(self.h, light, pp.ctypes.data, nn.ctypes.data, rad.ctypes.data,
                                              C.addressof(ray))
        return rad, ray


def accumulate_radiance(radiance, direction, acc=None) -> np.ndarray:
    out = np.zeros(27, np.float32) if acc is None else np.ascontiguousarray(acc, np.float32).copy()
    r, d = _f(radiance), _f(direction)
    lib().oracle_accumulate_radiance(r.ctypes.data, d.ctypes.data, out.ctypes.data)
    return out


def srgb_to_linear(x: int) -> float:
    return float(lib().oracle_srgb_to_linear(x))


def philox(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    o = np.zeros(4, np.uint32)
    lib().oracle_philox4x32_10(c.ctypes.data, k.ctypes.data, o.ctypes.data)
    return o


def validity_mask(points: np.ndarray) -> np.ndarray:
    pts = np.ascontiguousarray(points, dtype=SURFACE_POINT_DTYPE)
    out = np.empty(len(pts), np.uint8)
    lib().oracle_validity_mask(pts.ctypes.data, len(pts), out.ctypes.data)
    return out


def downsample_validity_mask(mask, w: int, h: int, scale: int) -> np.ndarray:
    m = np.ascontiguousarray(mask, np.uint8)
    out = np.empty(w * h, np.uint8)
    lib().oracle_downsample_validity_mask(m.ctypes.data, w, h, scale, out.ctypes.data)
    return out


def downsample(x: np.ndarray, w: int, h: int, ch: int, scale: int) -> np.ndarray:
    x = _f(x)
    ow, oh = (w, h) if scale <= 1 else (w // scale, h // scale)
    out = np.empty(ow * oh * ch, np.float32)
    lib().oracle_downsample(x.ctypes.data, w, h, ch, scale, out.ctypes.data)
    return out


def dilate(kind: int, w: int, h: int, pixels: np.ndarray, mask: np.ndarray, passes: int) -> None:
    """In place, like the reference."""
    lib().oracle_dilate(kind, w, h, pixels.ctypes.data, mask.ctypes.data, passes)
