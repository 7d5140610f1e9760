"""Property checks of a lightmap atlas (CreateAtlasGeometries): charts are
the connected components of the output faces in UV space; every output face keeps its source face's vertex attributes; no
texel centre is covered by two charts; texels of different charts are more
than `padding` texels apart; each chart keeps one texels-per-area density."""
import numpy as np


def charts_of(geo):
    """Charts as connected components of faces through shared lightmap UV
    points (vertices are split on chart seams, and two charts never share a
    UV point when they are padded apart)."""
    idx = np.asarray(geo.indices, np.int64).reshape(-1, 3)
    uv = np.ascontiguousarray(geo.lightmap_uvs, np.float32)
    _, key = np.unique(uv.view(np.uint64).reshape(-1), return_inverse=True)
    parent = np.arange(key.max() + 1 if len(key) else 0)

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    k = key[idx] if len(idx) else np.zeros((0, 3), np.int64)
    for f in k:
        r0 = find(f[0])
        for v in f[1:]:
            r = find(v)
            if r != r0:
                parent[r] = r0
    roots = np.array([find(f[0]) for f in k]) if len(k) else np.zeros(0, np.int64)
    _, comp = np.unique(roots, return_inverse=True)
    return comp


def covered_texels(uv, W, H):
    """Texel centres ((x+0.5)/W, (y+0.5)/H) inside a UV triangle (edges
    included), as flat indices."""
    p = uv * np.array([W, H])
    x0, y0 = np.floor(p.min(0) - 0.5).astype(int)
    x1, y1 = np.ceil(p.max(0) - 0.5).astype(int)
    x0, y0 = max(x0, 0), max(y0, 0)
    x1, y1 = min(x1, W - 1), min(y1, H - 1)
    if x1 < x0 or y1 < y0:
        return np.zeros(0, np.int64)
    xs, ys = np.meshgrid(np.arange(x0, x1 + 1) + 0.5, np.arange(y0, y1 + 1) + 0.5)
    a, b, c = p
    d = (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0])
    if d == 0:
        return np.zeros(0, np.int64)
    w1 = ((xs - a[0]) * (c[1] - a[1]) - (ys - a[1]) * (c[0] - a[0])) / d
    w2 = ((b[0] - a[0]) * (ys - a[1]) - (b[1] - a[1]) * (xs - a[0])) / d
    m = (w1 >= -1e-7) & (w2 >= -1e-7) & (w1 + w2 <= 1 + 1e-7)
    return (np.floor(ys[m]).astype(np.int64) * W + np.floor(xs[m]).astype(np.int64))


def check_atlas(scene, res, W, padding):
    """Asserts the atlas properties; returns (charts, covered texels)."""
    assert res is not None and res.width == W and res.height == W
    assert len(res.geometries) == len(scene.geometries)
    owner = np.full(W * W, -1, np.int64)
    base = 0
    for g_in, g in zip(scene.geometries, res.geometries):
        idx_in = np.asarray(g_in.indices, np.int64).reshape(-1, 3)
        idx = np.asarray(g.indices, np.int64).reshape(-1, 3)
        assert idx.shape == idx_in.shape
        if len(idx) == 0:
            continue
        for attr in ("vertices", "normals", "tangents", "texture_uvs"):
            np.testing.assert_array_equal(getattr(g, attr)[idx], getattr(g_in, attr)[idx_in])
        uv = g.lightmap_uvs
        assert uv.min() >= 0.0 and uv.max() <= 1.0
        comp = charts_of(g)
        # one density per chart: uv area / world area within a factor 1/0.7
        # (projection onto the chart plane) for faces of non-zero area
        L = np.asarray(g.transform, np.float64).reshape(3, 4)
        wv = g.vertices.astype(np.float64) @ L[:, :3].T + L[:, 3]
        e1, e2 = wv[idx[:, 1]] - wv[idx[:, 0]], wv[idx[:, 2]] - wv[idx[:, 0]]
        area = 0.5 * np.linalg.norm(np.cross(e1, e2), axis=1)
        u1, u2 = uv[idx[:, 1]] - uv[idx[:, 0]], uv[idx[:, 2]] - uv[idx[:, 0]]
        uva = 0.5 * np.abs(u1[:, 0] * u2[:, 1] - u1[:, 1] * u2[:, 0]).astype(np.float64)
        ok = area > 1e-9 * max(area.max(), 1e-30)
        for c in np.unique(comp[ok]):
            r = uva[ok & (comp == c)] / area[ok & (comp == c)]
            assert r.min() >= 0.69 * r.max() - 1e-12, (c, r.min(), r.max())
        for f in range(len(idx)):
            t = covered_texels(uv[idx[f]].astype(np.float64), W, W)
            cid = base + comp[f]
            prev = owner[t]
            clash = (prev >= 0) & (prev != cid)
            assert not clash.any(), f"texel covered by charts {set(prev[clash])} and {cid}"
            owner[t] = cid
        base += comp.max() + 1
    # padding: no texel of another chart within `padding` texels (Chebyshev)
    grid = owner.reshape(W, W)
    for dy in range(-padding, padding + 1):
        for dx in range(-padding, padding + 1):
            if dx == 0 and dy == 0:
                continue
            a = grid[max(dy, 0):W + min(dy, 0), max(dx, 0):W + min(dx, 0)]
            b = grid[max(-dy, 0):W + min(-dy, 0), max(-dx, 0):W + min(-dx, 0)]
            bad = (a >= 0) & (b >= 0) & (a != b)
            assert not bad.any(), f"charts closer than {padding + 1} texels at offset {(dx, dy)}"
    return base, int((owner >= 0).sum())
