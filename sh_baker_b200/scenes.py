"""Seeded synthetic scenes with the shapes and sizes of the bake workloads.

Every generator is deterministic in its seed.  Lightmap UVs come from this
module's own chart packer (one chart per planar patch or unwrapped
cylinder, shelf-packed with a texel padding); the reference's xatlas
unwrapper (src/atlas.cpp) is not used.  Emissive geometries become area
lights the way the reference's loader does it (src/loader.cpp:391-411).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Tuple

import numpy as np

from .scene import AREA, DIRECTIONAL, POINT, Geometry, Light, Material, Scene, Texture


def linear_to_srgb_byte(x: float) -> int:
    """src/colorspace.h:16-21."""
    if x <= 0.0031308:
        return int(np.rint(x * 12.92 * 255.0))
    return int(np.rint((1.055 * math.pow(x, 1.0 / 2.4) - 0.055) * 255.0))


def solid_material(rgb, emission: float = 0.0, name: str = "") -> Material:
    px = np.array([linear_to_srgb_byte(float(c)) for c in rgb], dtype=np.uint8)
    return Material(name=name, albedo=Texture(1, 1, 3, px), emission_intensity=float(emission))


def _normalize(v):
    v = np.asarray(v, dtype=np.float64)
    return v / np.linalg.norm(v)


# ------------------------------------------------------------------ patches --

@dataclass
class Patch:
    """A chart: a planar grid (corner, eu, ev) or a cylinder side."""
    geom: int
    kind: str  # "quad" | "cyl"
    corner: np.ndarray
    eu: np.ndarray
    ev: np.ndarray
    nu: int = 1
    nv: int = 1
    radius: float = 0.0
    height: float = 0.0
    inward: bool = False

    # "arch": half barrel vault; corner = centre of the springing line,
    # eu = half-span vector (radius), ev = depth vector; "cloth": quad with a
    # sinusoidal sag of amplitude `radius` along its normal.
    def world_size(self) -> Tuple[float, float]:
        if self.kind in ("quad", "cloth"):
            return float(np.linalg.norm(self.eu)), float(np.linalg.norm(self.ev))
        if self.kind == "arch":
            return math.pi * float(np.linalg.norm(self.eu)), float(np.linalg.norm(self.ev))
        return 2.0 * math.pi * self.radius, self.height


def _shelf_try(order, cws, chs, res: int, padding: int):
    rects = [None] * len(cws)
    x = y = shelf_h = 0
    for i in order:
        cw, ch = cws[i], chs[i]
        ow, oh = cw + padding, ch + padding
        if ow > res:
            return None
        if x + ow > res:
            x = 0
            y += shelf_h
            shelf_h = 0
        if y + oh > res:
            return None
        rects[i] = (x + padding // 2, y + padding // 2, cw, ch)
        x += ow
        if oh > shelf_h:
            shelf_h = oh
    return rects


def shelf_pack(sizes: List[Tuple[float, float]], res: int, padding: int):
    """Packs world-size charts into a res x res atlas at one texel density.
    The density starts at 55 % fill and coarsens by 4 % steps until the
    shelves fit.  Returns (texel_size, [(x0, y0, cw, ch)]) in texels."""
    if len(sizes) * (1 + padding) ** 2 > res * res:
        raise RuntimeError("chart packing failed")
    total = sum(w * h for w, h in sizes)
    s0 = math.sqrt(total / (res * res * 0.55)) if total > 0 else 1.0
    order = sorted(range(len(sizes)), key=lambda i: -sizes[i][1])
    W = np.array([w for w, _ in sizes], np.float64)
    H = np.array([h for _, h in sizes], np.float64)

    def attempt(k):
        s = s0 * (1.04 ** k) if k else s0
        # the same arithmetic as a scalar loop: ceil(size / s), at least 1
        cws = [max(1, int(math.ceil(w / s))) for w in W.tolist()]
        chs = [max(1, int(math.ceil(h / s))) for h in H.tolist()]
        return s, _shelf_try(order, cws, chs, res, padding)

    for k in range(12):  # most atlases fit within a few steps
        s, rects = attempt(k)
        if rects is not None:
            return s, rects
    lo, hi, step, k = 11, None, 1, 12
    while k < 200:  # grow the step exponentially, then bisect
        if attempt(k)[1] is not None:
            hi = k
            break
        lo = k
        step *= 2
        k = lo + step if lo < 199 else 200
        k = min(k, 199) if lo < 199 else k
    if hi is None:
        raise RuntimeError("chart packing failed")
    while hi - lo > 1:
        mid = (lo + hi) // 2
        if attempt(mid)[1] is not None:
            hi = mid
        else:
            lo = mid
    return attempt(hi)


class MeshBuilder:
    def __init__(self, n_geoms: int):
        self.v = [[] for _ in range(n_geoms)]
        self.n = [[] for _ in range(n_geoms)]
        self.t = [[] for _ in range(n_geoms)]
        self.tuv = [[] for _ in range(n_geoms)]
        self.luv = [[] for _ in range(n_geoms)]
        self.idx = [[] for _ in range(n_geoms)]

    def add_patch(self, p: Patch, rect, res: int):
        g = p.geom
        x0, y0, cw, ch = rect
        base = sum(len(a) for a in self.v[g])
        nu, nv = p.nu, p.nv
        a = np.linspace(0.0, 1.0, nu + 1)
        b = np.linspace(0.0, 1.0, nv + 1)
        A, B = np.meshgrid(a, b)  # (nv+1, nu+1)
        A = A.reshape(-1)
        B = B.reshape(-1)
        if p.kind == "quad":
            pos = p.corner[None, :] + A[:, None] * p.eu[None, :] + B[:, None] * p.ev[None, :]
            nrm = np.repeat(_normalize(np.cross(p.eu, p.ev))[None, :], len(A), 0)
            tan = np.repeat(_normalize(p.eu)[None, :], len(A), 0)
        elif p.kind == "cloth":
            n0 = _normalize(np.cross(p.eu, p.ev))
            sag = p.radius * np.sin(math.pi * A) * np.sin(math.pi * B)
            pos = (p.corner[None, :] + A[:, None] * p.eu[None, :] + B[:, None] * p.ev[None, :]
                   + sag[:, None] * n0[None, :])
            # analytic normal of the sagging sheet
            du = p.eu[None, :] + (p.radius * math.pi * np.cos(math.pi * A) * np.sin(math.pi * B))[:, None] * n0[None, :]
            dv = p.ev[None, :] + (p.radius * math.pi * np.sin(math.pi * A) * np.cos(math.pi * B))[:, None] * n0[None, :]
            nrm = np.cross(du, dv)
            nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
            tan = du / np.linalg.norm(du, axis=1, keepdims=True)
        elif p.kind == "arch":
            r = float(np.linalg.norm(p.eu))
            span = p.eu / r
            up = np.array([0.0, 1.0, 0.0])
            ang = A * math.pi
            radial = np.cos(ang)[:, None] * span[None, :] + np.sin(ang)[:, None] * up[None, :]
            pos = p.corner[None, :] + r * radial + B[:, None] * p.ev[None, :]
            nrm = -radial  # the intrados faces the axis
            tan = -np.sin(ang)[:, None] * span[None, :] + np.cos(ang)[:, None] * up[None, :]
        else:
            ang = A * 2.0 * math.pi
            radial = np.stack([np.cos(ang), np.zeros_like(ang), np.sin(ang)], 1)
            pos = p.corner[None, :] + p.radius * radial + (B * p.height)[:, None] * np.array([0.0, 1.0, 0.0])[None, :]
            nrm = -radial if p.inward else radial
            tan = np.stack([-np.sin(ang), np.zeros_like(ang), np.cos(ang)], 1)
        luv = np.stack([(x0 + A * cw) / res, (y0 + B * ch) / res], 1)
        self.v[g].append(pos.astype(np.float32))
        self.n[g].append(nrm.astype(np.float32))
        self.t[g].append(np.hstack([tan, np.ones((len(A), 1))]).astype(np.float32))
        self.tuv[g].append(np.stack([A, B], 1).astype(np.float32))
        self.luv[g].append(luv.astype(np.float32))
        ii = []
        for j in range(nv):
            for i in range(nu):
                q0 = j * (nu + 1) + i
                q1, q2, q3 = q0 + 1, q0 + nu + 2, q0 + nu + 1
                if (p.kind == "cyl" and not p.inward) or (p.kind == "arch" and not p.inward):
                    ii += [q0, q2, q1, q0, q3, q2]
                else:
                    ii += [q0, q1, q2, q0, q2, q3]
        self.idx[g].append(np.asarray(ii, dtype=np.uint32) + base)

    def geometries(self, material_ids: List[int]) -> List[Geometry]:
        out = []
        for g in range(len(self.v)):
            if not self.v[g]:
                continue
            out.append(Geometry(
                vertices=np.vstack(self.v[g]), indices=np.concatenate(self.idx[g]), normals=np.vstack(self.n[g]),
                texture_uvs=np.vstack(self.tuv[g]), lightmap_uvs=np.vstack(self.luv[g]),
                tangents=np.vstack(self.t[g]), material_id=material_ids[g]))
        return out


def grid_pack(sizes: List[Tuple[float, float]], res: int):
    """Fallback for atlases too small for one texel-aligned chart per patch:
    a uniform grid of cells, each patch scaled into its cell (charts may be
    smaller than a texel; the rasteriser's centroid rule then covers them)."""
    n = len(sizes)
    cols = max(1, int(math.ceil(math.sqrt(n))))
    cell = res / cols
    rects = []
    for i, (w, h) in enumerate(sizes):
        s = 0.8 * cell / max(w, h, 1e-9)
        cx, cy = (i % cols) * cell, (i // cols) * cell
        rects.append((cx + 0.1 * cell, cy + 0.1 * cell, w * s, h * s))
    return rects


def build_from_patches(patches: List[Patch], material_ids: List[int], res: int, padding: int) -> List[Geometry]:
    sizes = [p.world_size() for p in patches]
    try:
        _, rects = shelf_pack(sizes, res, padding)
    except RuntimeError:
        rects = grid_pack(sizes, res)
    mb = MeshBuilder(len(material_ids))
    for p, r in zip(patches, rects):
        mb.add_patch(p, r, res)
    return mb.geometries(material_ids)


def box_patches(geom: int, lo, hi, inward: bool, subdiv: int = 1) -> List[Patch]:
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    d = hi - lo
    X, Y, Z = np.array([d[0], 0, 0]), np.array([0, d[1], 0]), np.array([0, 0, d[2]])
    # (corner, eu, ev) with eu x ev pointing outward
    faces = [
        (lo, Z, Y),                # -x
        (lo + X, Y, Z),            # +x
        (lo, X, Z),                # -y
        (lo + Y, Z, X),            # +y
        (lo, Y, X),                # -z
        (lo + Z, X, Y),            # +z
    ]
    out = []
    for c, eu, ev in faces:
        if inward:
            eu, ev = ev, eu
        out.append(Patch(geom, "quad", np.asarray(c, np.float64), np.asarray(eu, np.float64),
                         np.asarray(ev, np.float64), subdiv, subdiv))
    return out


def mark_area_lights(scene: Scene) -> None:
    """Every geometry with an emissive material becomes an area light
    (src/loader.cpp:391-411)."""
    for gi, g in enumerate(scene.geometries):
        m = scene.materials[g.material_id]
        if m.emission_intensity > 0.0:
            v = np.asarray(g.vertices, np.float64)
            i = np.asarray(g.indices).reshape(-1, 3)
            area = 0.5 * np.linalg.norm(np.cross(v[i[:, 1]] - v[i[:, 0]], v[i[:, 2]] - v[i[:, 0]]), axis=1).sum()
            scene.lights.append(Light(type=AREA, material_index=g.material_id, geometry_index=gi,
                                      area=float(area), intensity=m.emission_intensity))


# ---------------------------------------------------------------- configs --

def unit_quad() -> Scene:
    """Unit quad [-0.5,0.5]^2 in the XZ plane at y=0, normal +Y, tangent +X,
    UV = lightmap UV = [0,1]^2, default albedo 0.8; directional light
    (0.3,-1,0.2)/|.| radiance 3 and a point light at (0,1,0) intensity 10."""
    v = np.array([[-0.5, 0, -0.5], [0.5, 0, -0.5], [0.5, 0, 0.5], [-0.5, 0, 0.5]], np.float32)
    uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    g = Geometry(vertices=v, indices=np.array([0, 2, 1, 0, 3, 2], np.uint32),
                 normals=np.tile([0, 1, 0], (4, 1)).astype(np.float32), texture_uvs=uv, lightmap_uvs=uv,
                 tangents=np.tile([1, 0, 0, 1], (4, 1)).astype(np.float32), material_id=0)
    d = np.array([0.3, -1.0, 0.2], np.float32)
    d = d / np.linalg.norm(d)
    lights = [Light(type=DIRECTIONAL, direction=tuple(float(x) for x in d), intensity=3.0),
              Light(type=POINT, position=(0.0, 1.0, 0.0), intensity=10.0)]
    return Scene([g], [Material(name="grey")], lights)


def _box_faces(lo: np.ndarray, hi: np.ndarray, inward: bool):
    """The six (corner, eu, ev) faces of each box, in box_patches' order,
    eu x ev pointing out of the box (or into it when inward)."""
    d = hi - lo
    n = len(lo)
    X = np.zeros((n, 3)); X[:, 0] = d[:, 0]
    Y = np.zeros((n, 3)); Y[:, 1] = d[:, 1]
    Z = np.zeros((n, 3)); Z[:, 2] = d[:, 2]
    corners = np.stack([lo, lo + X, lo, lo + Y, lo, lo + Z], 1)
    eu = np.stack([Z, Y, X, Z, Y, X], 1)
    ev = np.stack([Y, Z, Z, X, X, Y], 1)
    if inward:
        eu, ev = ev, eu
    return corners.reshape(-1, 3), eu.reshape(-1, 3), ev.reshape(-1, 3)


def _box_geometries(corners, eu, ev, n_geoms: int, material_ids: List[int], res: int, padding: int):
    """Axis-aligned single-quad charts (6 per geometry), packed and turned
    into geometries with the same arithmetic as MeshBuilder.add_patch."""
    wu = np.abs(eu).max(1)  # |eu| of an axis-aligned vector, exact
    wv = np.abs(ev).max(1)
    sizes = list(zip(wu.tolist(), wv.tolist()))
    try:
        _, rects = shelf_pack(sizes, res, padding)
    except RuntimeError:
        rects = grid_pack(sizes, res)
    R = np.asarray(rects, np.float64)
    x0, y0, cw, ch = R[:, 0:1], R[:, 1:2], R[:, 2:3], R[:, 3:4]
    A = np.array([0.0, 1.0, 0.0, 1.0])
    B = np.array([0.0, 0.0, 1.0, 1.0])
    pos = corners[:, None, :] + A[None, :, None] * eu[:, None, :] + B[None, :, None] * ev[:, None, :]
    cr = np.cross(eu, ev)
    nrm = cr / np.sqrt((cr * cr).sum(1))[:, None]
    tan = eu / np.sqrt((eu * eu).sum(1))[:, None]
    luv = np.stack([(x0 + A[None, :] * cw) / res, (y0 + B[None, :] * ch) / res], 2)
    nf = len(corners)
    V = pos.astype(np.float32)
    N = np.repeat(nrm[:, None, :], 4, 1).astype(np.float32)
    T = np.concatenate([np.repeat(tan[:, None, :], 4, 1), np.ones((nf, 4, 1))], 2).astype(np.float32)
    TUV = np.repeat(np.stack([A, B], 1)[None], nf, 0).astype(np.float32)
    LUV = luv.astype(np.float32)
    quad = np.array([0, 1, 3, 0, 3, 2], np.uint32)
    out = []
    per = nf // n_geoms
    for g in range(n_geoms):
        f = slice(g * per, (g + 1) * per)
        idx = (quad[None, :] + 4 * np.arange(per, dtype=np.uint32)[:, None]).reshape(-1)
        out.append(Geometry(vertices=V[f].reshape(-1, 3), indices=idx, normals=N[f].reshape(-1, 3),
                            texture_uvs=TUV[f].reshape(-1, 2), lightmap_uvs=LUV[f].reshape(-1, 2),
                            tangents=T[f].reshape(-1, 4), material_id=material_ids[g]))
    return out


def procedural_room(seed: int = 2, n_boxes: int = 200, res: int = 1024, padding: int = 2,
                    n_materials: int = 8, n_point_lights: int = 4, box_subdiv: int = 1) -> Scene:
    """Closed 10x3x10 room (12 inward triangles) plus `n_boxes` axis-aligned
    boxes with uniform positions inside and edges U[0.1, 1.0]; one chart per
    face; 8 Lambertian materials with albedo U[0.1, 0.9]; one directional and
    `n_point_lights` point lights with intensity U[5, 50]."""
    rng = np.random.default_rng(seed)
    mats = [solid_material(rng.uniform(0.1, 0.9, 3), name=f"m{i}") for i in range(n_materials)]
    room_lo, room_hi = np.array([-5.0, 0.0, -5.0]), np.array([5.0, 3.0, 5.0])
    mat_ids = [0]
    los, his = [], []
    for b in range(n_boxes):
        size = rng.uniform(0.1, 1.0, 3)
        lo = rng.uniform(room_lo, room_hi - size)
        los.append(lo)
        his.append(lo + size)
        mat_ids.append(int(rng.integers(0, n_materials)))
    if box_subdiv == 1:
        rc, ru, rv = _box_faces(room_lo[None], room_hi[None], inward=True)
        if n_boxes:
            bc, bu, bv = _box_faces(np.array(los), np.array(his), inward=False)
            rc, ru, rv = np.vstack([rc, bc]), np.vstack([ru, bu]), np.vstack([rv, bv])
        geoms = _box_geometries(rc, ru, rv, n_boxes + 1, mat_ids, res, padding)
    else:
        patches = box_patches(0, room_lo, room_hi, inward=True)
        for b in range(n_boxes):
            patches += box_patches(b + 1, los[b], his[b], inward=False, subdiv=box_subdiv)
        geoms = build_from_patches(patches, mat_ids, res, padding)
    d = _normalize([rng.uniform(-0.5, 0.5), -1.0, rng.uniform(-0.5, 0.5)])
    lights = [Light(type=DIRECTIONAL, direction=tuple(float(x) for x in d), intensity=3.0)]
    for _ in range(n_point_lights):
        pos = (rng.uniform(-4, 4), rng.uniform(1.5, 2.8), rng.uniform(-4, 4))
        lights.append(Light(type=POINT, position=tuple(float(x) for x in pos), intensity=float(rng.uniform(5, 50))))
    return Scene(geoms, mats, lights)


def atrium(seed: int = 3, res: int = 2048, padding: int = 2, column_segments: Tuple[int, int] = (50, 20),
           n_cloth: int = 100, cloth_grid: Tuple[int, int] = (22, 23), wall_grid: int = 22) -> Scene:
    """Two-storey colonnaded courtyard (~262k triangles): 64 columns of
    2,000-triangle cylinders (32 per storey on the courtyard edge), half-barrel
    arches between neighbouring columns, tiled ground floor, gallery slabs and
    roof, subdivided outer and courtyard walls, and 100 hanging cloth quads of
    about 1,000 triangles.  25 materials with albedo U[0.1, 0.9]; 10 % of the
    planar patches are emissive with radiance U[1, 5] (area lights); one sun
    of radiance 20 and 8 point lights in the galleries."""
    rng = np.random.default_rng(seed)
    n_mat = 25
    n_emissive = 3  # materials 22..24 are emissive
    mats = [solid_material(rng.uniform(0.1, 0.9, 3), name=f"m{i}") for i in range(n_mat - n_emissive)]
    mats += [solid_material(rng.uniform(0.6, 1.0, 3), emission=float(rng.uniform(1.0, 5.0)), name=f"e{i}")
             for i in range(n_emissive)]
    X, Z, H, S = 20.0, 15.0, 10.0, 5.0  # outer half-extents, height, storey height
    CX, CZ = 14.0, 9.0                   # courtyard half-extents
    patches: List[Patch] = []
    mat_ids: List[int] = []
    planar: List[int] = []  # geometry ids of planar patches (candidates for emission)

    def add(p_list, mat, is_planar):
        gid = len(mat_ids)
        for p in p_list:
            p.geom = gid
            patches.append(p)
        mat_ids.append(mat)
        if is_planar:
            planar.append(gid)
        return gid

    def quad(corner, eu, ev, nu=1, nv=1):
        return Patch(0, "quad", np.asarray(corner, np.float64), np.asarray(eu, np.float64),
                     np.asarray(ev, np.float64), nu, nv)

    def rmat():
        return int(rng.integers(0, n_mat - n_emissive))

    # ground floor tiles: 5 m x 5 m patches of 1 m tiles, facing up
    for x0 in np.arange(-X, X, 5.0):
        for z0 in np.arange(-Z, Z, 5.0):
            add([quad((x0, 0.0, z0), (0, 0, 5.0), (5.0, 0, 0), 5, 5)], rmat(), True)
    # gallery slab (y = S, both faces) and roof (y = H, underside) over the ring
    ring = [((-X, -Z), (2 * X, Z - CZ)), ((-X, CZ), (2 * X, Z - CZ)), ((-X, -CZ), (X - CX, 2 * CZ)),
            ((CX, -CZ), (X - CX, 2 * CZ))]
    for (x0, z0), (dx, dz) in ring:
        nx, nz = max(1, int(dx / 2.5)), max(1, int(dz / 2.5))
        add([quad((x0, S, z0), (0, 0, dz), (dx, 0, 0), nz, nx)], rmat(), True)           # slab top
        add([quad((x0, S - 0.01, z0), (dx, 0, 0), (0, 0, dz), nx, nz)], rmat(), True)    # ceiling below
        add([quad((x0, H, z0), (dx, 0, 0), (0, 0, dz), nx, nz)], rmat(), True)           # roof underside
    # outer walls (inward) and courtyard-facing upper walls, per storey, as panels
    for s in range(2):
        y0 = s * S
        for (c, eu) in (((-X, y0, -Z), (2 * X, 0, 0)), ((X, y0, Z), (-2 * X, 0, 0)),
                        ((-X, y0, Z), (0, 0, -2 * Z)), ((X, y0, -Z), (0, 0, 2 * Z))):
            L = np.linalg.norm(eu)
            n_pan = int(L // 10)
            step = np.asarray(eu, np.float64) / n_pan
            for k in range(n_pan):
                corner = np.asarray(c, np.float64) + k * step
                add([quad(corner, step, (0, S, 0), wall_grid, wall_grid)], rmat(), True)
    # 64 columns (2 storeys x 32 on the courtyard edge)
    col_xz = []
    for x in np.linspace(-CX, CX, 10):
        col_xz += [(x, -CZ), (x, CZ)]
    for z in np.linspace(-CZ, CZ, 8)[1:-1]:
        col_xz += [(-CX, z), (CX, z)]
    assert len(col_xz) == 32
    nseg, nring = column_segments
    for s in range(2):
        for (x, z) in col_xz:
            add([Patch(0, "cyl", np.array([x, s * S, z]), np.zeros(3), np.zeros(3), nseg, nring, radius=0.35,
                       height=S - 1.0)], rmat(), False)
    # arches between neighbouring columns along each courtyard side, per storey
    for s in range(2):
        ytop = s * S + (S - 1.0)
        sides = [([(x, -CZ) for x in np.linspace(-CX, CX, 10)], (0, 0, 0.8)),
                 ([(x, CZ) for x in np.linspace(-CX, CX, 10)], (0, 0, -0.8)),
                 ([(-CX, z) for z in np.linspace(-CZ, CZ, 8)], (0.8, 0, 0)),
                 ([(CX, z) for z in np.linspace(-CZ, CZ, 8)], (-0.8, 0, 0))]
        for pts, depth in sides:
            for a, b in zip(pts[:-1], pts[1:]):
                mid = np.array([(a[0] + b[0]) / 2, ytop, (a[1] + b[1]) / 2])
                half = np.array([(b[0] - a[0]) / 2, 0.0, (b[1] - a[1]) / 2])
                d = np.asarray(depth, np.float64)
                add([Patch(0, "arch", mid - d / 2, half, d, 16, 2)], rmat(), True)
    # 100 hanging cloth quads in the courtyard and the galleries
    nu, nv = cloth_grid
    for _ in range(n_cloth):
        w, h = rng.uniform(1.0, 3.0), rng.uniform(1.0, 3.0)
        cx, cz = rng.uniform(-X + 2, X - 2), rng.uniform(-Z + 2, Z - 2)
        top = rng.uniform(3.0, 9.5)
        ang = rng.uniform(0, math.pi)
        eu = np.array([math.cos(ang) * w, 0.0, math.sin(ang) * w])
        corner = np.array([cx, top - h, cz]) - eu / 2
        add([Patch(0, "cloth", corner, eu, np.array([0.0, h, 0.0]), nu, nv, radius=0.15 * min(w, h))], rmat(), False)
    # 10 % of the planar patches emissive
    n_em = max(1, len(planar) // 10)
    for gid in rng.choice(planar, size=n_em, replace=False):
        mat_ids[int(gid)] = int(rng.integers(n_mat - n_emissive, n_mat))
    geoms = build_from_patches(patches, mat_ids, res, padding)
    scene = Scene(geoms, mats, [])
    scene.lights.append(Light(type=DIRECTIONAL, direction=tuple(float(x) for x in _normalize([-0.35, -1.0, -0.45])),
                              intensity=20.0))
    for _ in range(8):
        side = rng.integers(0, 4)
        if side < 2:
            pos = (rng.uniform(-X + 1, X - 1), rng.uniform(1.5, 4.5) + S * rng.integers(0, 2),
                   (Z - 3.0) * (1 if side == 0 else -1))
        else:
            pos = ((X - 3.0) * (1 if side == 2 else -1), rng.uniform(1.5, 4.5) + S * rng.integers(0, 2),
                   rng.uniform(-Z + 1, Z - 1))
        scene.lights.append(Light(type=POINT, position=tuple(float(v) for v in pos),
                                  intensity=float(rng.uniform(5.0, 50.0))))
    mark_area_lights(scene)
    return scene


def batched_mix(seed: int = 4, n: int = 64):
    """The batched-bake mix: `n` independent procedural rooms with triangle
    counts log-uniform in [1k, 100k], lightmaps of {128, 256, 512, 1024}^2,
    {32, 64, 128, 256} spp, 2-4 bounces and 1-8 point lights each.  Returns
    a list of dicts (scene, width, height, spp, bounces, seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        tris = math.exp(rng.uniform(math.log(1_000), math.log(100_000)))
        n_boxes = max(1, int(round((tris - 12) / 12)))
        res = int(rng.choice([128, 256, 512, 1024]))
        spp = int(rng.choice([32, 64, 128, 256]))
        bounces = int(rng.integers(2, 5))
        lights = int(rng.integers(1, 9))
        sc = procedural_room(seed=1000 + i, n_boxes=n_boxes, res=res, n_point_lights=lights)
        out.append({"scene": sc, "width": res, "height": res, "spp": spp, "bounces": bounces, "seed": 77 + i})
    return out
