"""Scene data model mirroring sh_baker's structs (src/scene.h:18-115,
src/rasterizer.h:12-23, src/baker.h:10-19) and its packing into the C ABI's
shb_scene_desc."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _capi as A

POINT, DIRECTIONAL, SPOT, AREA = A.LIGHT_POINT, A.LIGHT_DIRECTIONAL, A.LIGHT_SPOT, A.LIGHT_AREA

# sh_baker::SurfacePoint with Eigen alignment (64 bytes).
SURFACE_POINT_DTYPE = np.dtype({
    "names": ["position", "normal", "tangent", "material_id"],
    "formats": [("<f4", 3), ("<f4", 3), ("<f4", 4), "<i4"],
    "offsets": [0, 12, 32, 48],
    "itemsize": 64,
})


@dataclass
class Texture:
    width: int = 0
    height: int = 0
    channels: int = 0
    pixel_data: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint8))
    file_path: Optional[str] = None  # the image file it was read from, absolute (src/scene.h:19-22)


@dataclass
class Material:
    name: str = ""
    albedo: Texture = field(default_factory=Texture)
    emission_intensity: float = 0.0


@dataclass
class Geometry:
    vertices: np.ndarray
    indices: np.ndarray
    normals: Optional[np.ndarray] = None
    texture_uvs: Optional[np.ndarray] = None
    lightmap_uvs: Optional[np.ndarray] = None
    tangents: Optional[np.ndarray] = None
    material_id: int = -1
    transform: np.ndarray = field(default_factory=lambda: np.hstack([np.eye(3), np.zeros((3, 1))]).astype(np.float32))


@dataclass
class Light:
    type: int = POINT
    position: tuple = (0.0, 0.0, 0.0)
    direction: tuple = (0.0, 0.0, -1.0)
    color: tuple = (1.0, 1.0, 1.0)
    intensity: float = 1.0
    cos_inner_cone: float = 1.0
    cos_outer_cone: float = 0.70710678118654752440
    area: float = 0.0
    material_index: int = -1
    geometry_index: int = -1


@dataclass
class Scene:
    geometries: List[Geometry] = field(default_factory=list)
    materials: List[Material] = field(default_factory=list)
    lights: List[Light] = field(default_factory=list)

    @property
    def triangle_count(self) -> int:
        return int(sum(len(g.indices) // 3 for g in self.geometries))


def _f32(a, cols):
    if a is None:
        return None
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32).reshape(-1, cols))
    return a


def _ptr(a, ctype):
    return None if a is None else a.ctypes.data_as(C.POINTER(ctype))


def pack_scene(scene: Scene):
    """Returns (SceneDesc, keepalive).  keepalive holds every buffer the
    descriptor points at; keep it alive while the descriptor is used."""
    keep = []
    geos = (A.GeometryDesc * max(1, len(scene.geometries)))()
    for i, g in enumerate(scene.geometries):
        v = _f32(g.vertices, 3)
        n = _f32(g.normals, 3)
        tuv = _f32(g.texture_uvs, 2)
        luv = _f32(g.lightmap_uvs, 2)
        t = _f32(g.tangents, 4)
        idx = np.ascontiguousarray(np.asarray(g.indices, dtype=np.uint32).reshape(-1))
        keep += [v, n, tuv, luv, t, idx]
        d = geos[i]
        d.vertices = _ptr(v, C.c_float)
        d.normals = _ptr(n, C.c_float)
        d.texture_uvs = _ptr(tuv, C.c_float)
        d.lightmap_uvs = _ptr(luv, C.c_float)
        d.tangents = _ptr(t, C.c_float)
        d.vertex_count = len(v)
        d.indices = _ptr(idx, C.c_uint32) if idx.size else None
        d.index_count = idx.size
        d.material_id = int(g.material_id)
        tr = np.asarray(g.transform, dtype=np.float32).reshape(3, 4)
        for k in range(12):
            d.transform[k] = float(tr.reshape(-1)[k])
    mats = (A.MaterialDesc * max(1, len(scene.materials)))()
    for i, m in enumerate(scene.materials):
        px = np.ascontiguousarray(np.asarray(m.albedo.pixel_data, dtype=np.uint8).reshape(-1))
        keep.append(px)
        d = mats[i]
        d.albedo_pixels = _ptr(px, C.c_uint8) if px.size else None
        d.albedo_width = m.albedo.width
        d.albedo_height = m.albedo.height
        d.albedo_channels = m.albedo.channels
        d.emission_intensity = float(m.emission_intensity)
    lights = (A.LightDesc * max(1, len(scene.lights)))()
    for i, L in enumerate(scene.lights):
        d = lights[i]
        d.type = int(L.type)
        for k in range(3):
            d.position[k] = float(L.position[k])
            d.direction[k] = float(L.direction[k])
            d.color[k] = float(L.color[k])
        d.intensity = float(L.intensity)
        d.cos_inner_cone = float(L.cos_inner_cone)
        d.cos_outer_cone = float(L.cos_outer_cone)
        d.area = float(L.area)
        d.material_index = int(L.material_index)
        d.geometry_index = int(L.geometry_index)
    keep += [geos, mats, lights]
    desc = A.SceneDesc(geos, len(scene.geometries), mats, len(scene.materials), lights, len(scene.lights))
    return desc, keep


def surface_points_empty(n: int) -> np.ndarray:
    sp = np.zeros(n, dtype=SURFACE_POINT_DTYPE)
    sp["material_id"] = -1
    return sp


def unpack_scene(desc: A.SceneDesc) -> Scene:
    """Copies a shb_scene_desc (for example one returned by shb_load_gltf)
    into a Scene."""
    def arr(ptr, n, cols, dt=np.float32):
        if not ptr or n == 0:
            return None
        return np.ctypeslib.as_array(ptr, shape=(n * cols,)).astype(dt).reshape(n, cols)

    sc = Scene()
    for i in range(desc.geometry_count):
        d = desc.geometries[i]
        nv = d.vertex_count
        idx = (np.ctypeslib.as_array(d.indices, shape=(d.index_count,)).astype(np.uint32)
               if d.indices and d.index_count else np.zeros(0, np.uint32))
        sc.geometries.append(Geometry(vertices=arr(d.vertices, nv, 3), indices=idx, normals=arr(d.normals, nv, 3),
                                      texture_uvs=arr(d.texture_uvs, nv, 2), lightmap_uvs=arr(d.lightmap_uvs, nv, 2),
                                      tangents=arr(d.tangents, nv, 4), material_id=int(d.material_id),
                                      transform=np.array(list(d.transform), np.float32).reshape(3, 4)))
    for i in range(desc.material_count):
        d = desc.materials[i]
        n = d.albedo_width * d.albedo_height * d.albedo_channels
        px = (np.ctypeslib.as_array(d.albedo_pixels, shape=(n,)).astype(np.uint8)
              if d.albedo_pixels and n else np.zeros(0, np.uint8))
        sc.materials.append(Material(albedo=Texture(d.albedo_width, d.albedo_height, d.albedo_channels, px),
                                     emission_intensity=float(d.emission_intensity)))
    for i in range(desc.light_count):
        d = desc.lights[i]
        sc.lights.append(Light(type=int(d.type), position=tuple(d.position), direction=tuple(d.direction),
                               color=tuple(d.color), intensity=float(d.intensity),
                               cos_inner_cone=float(d.cos_inner_cone), cos_outer_cone=float(d.cos_outer_cone),
                               area=float(d.area), material_index=int(d.material_index),
                               geometry_index=int(d.geometry_index)))
    return sc
