"""Tangent frames built by the loader for primitives without a TANGENT
attribute: the MikkTSpace method the reference applies through that library
(src/loader.cpp:88-109,363-385).  The library itself is not in the
reference tree, so these are property checks of the published method:
the UV-space direction dP/du, orientation from the UV winding, welding of
identical corners, grouping by orientation, angle weighting, the write order
of shared vertex indices, and the reference's geometric fallback.  Host code
only, no GPU."""
import math

import numpy as np
import pytest

from sh_baker_b200 import api
from tests.gltf_fixture import GltfBuilder


def load_tangents(tmp_path, pos, nrm, uv, idx, name="m.gltf"):
    b = GltfBuilder()
    prim = b.primitive(np.asarray(pos, np.float32), np.asarray(nrm, np.float32), np.asarray(uv, np.float32),
                       idx=np.asarray(idx, np.uint32), material=b.material(factor=[1, 1, 1, 1]))
    b.node(mesh=b.mesh([prim]))
    return np.asarray(api.LoadScene(b.write(tmp_path / name)).geometries[0].tangents, np.float64)


def unit(v):
    v = np.asarray(v, np.float64)
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def fallback(n):
    a = np.array([1.0, 0, 0]) if abs(n[0]) < 0.9 else np.array([0, 1.0, 0])
    return unit(a - n * np.dot(n, a))


def cylinder(segs=24, rings=3, radius=1.5, height=2.0):
    """Open cylinder about +Y with a UV seam: u = angle / 2 pi (the seam
    column is duplicated at u = 0 and u = 1), v = y / height."""
    pos, nrm, uv = [], [], []
    for r in range(rings + 1):
        for s in range(segs + 1):
            a = 2 * math.pi * s / segs
            pos.append([radius * math.cos(a), height * r / rings, radius * math.sin(a)])
            nrm.append([math.cos(a), 0, math.sin(a)])
            uv.append([s / segs, r / rings])
    idx = []
    for r in range(rings):
        for s in range(segs):
            i0 = r * (segs + 1) + s
            i1, i2, i3 = i0 + 1, i0 + segs + 2, i0 + segs + 1
            idx += [i0, i2, i1, i0, i3, i2]  # outward-facing winding
    return np.array(pos), np.array(nrm), np.array(uv), np.array(idx)


def test_cylinder_tangents_follow_du(tmp_path):
    pos, nrm, uv, idx = cylinder()
    t = load_tangents(tmp_path, pos, nrm, uv, idx)
    a = 2 * math.pi * uv[:, 0]
    du = np.stack([-np.sin(a), np.zeros_like(a), np.cos(a)], 1)  # dP/du direction
    np.testing.assert_allclose(np.linalg.norm(t[:, :3], axis=1), 1.0, atol=1e-6)
    np.testing.assert_allclose(np.abs((t[:, :3] * nrm).sum(1)), 0.0, atol=1e-6)
    # the two faces beside a column are mirror images about dP/du there
    np.testing.assert_allclose(t[:, :3], du, atol=1e-6)
    # u grows along +angle seen from outside, v along +Y: a left-handed UV
    # frame about the outward normal, sign -1, bitangent (n x t) w along +Y
    bit = np.cross(nrm, t[:, :3]) * t[:, 3:4]
    assert (bit[:, 1] > 0.99).all()
    expect_sign = np.sign(np.einsum("ij,ij->i", np.cross(nrm, du), np.array([[0, 1, 0]] * len(nrm))))
    np.testing.assert_array_equal(t[:, 3], expect_sign)


def strip(mirror_right):
    """Two unit quads side by side in z = 0 facing +Z sharing the column
    x = 1; the right one's u runs back from 1 to 0 when mirrored."""
    pos = np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0], [0, 1, 0], [1, 1, 0], [2, 1, 0]], np.float64)
    u_right = 0.0 if mirror_right else 2.0
    uv = np.array([[0, 0], [1, 0], [u_right, 0], [0, 1], [1, 1], [u_right, 1]], np.float64)
    nrm = np.tile([0, 0, 1.0], (6, 1))
    idx = np.array([0, 1, 4, 0, 4, 3, 1, 2, 5, 1, 5, 4])
    return pos, nrm, uv, idx


def test_mirrored_half_gets_its_own_group_and_the_last_write(tmp_path):
    pos, nrm, uv, idx = strip(mirror_right=True)
    t = load_tangents(tmp_path, pos, nrm, uv, idx)
    np.testing.assert_allclose(t[[0, 3]], [[1, 0, 0, 1]] * 2, atol=1e-6)
    np.testing.assert_allclose(t[[2, 5]], [[-1, 0, 0, -1]] * 2, atol=1e-6)
    # the shared column belongs to both groups; the right quad's corners come
    # later in face order, so its frame is the one kept
    np.testing.assert_allclose(t[[1, 4]], [[-1, 0, 0, -1]] * 2, atol=1e-6)
    # faces reordered: the left quad's frame is kept instead
    t2 = load_tangents(tmp_path, pos, nrm, uv, np.concatenate([idx[6:], idx[:6]]), "m2.gltf")
    np.testing.assert_allclose(t2[[1, 4]], [[1, 0, 0, 1]] * 2, atol=1e-6)
    # unmirrored, one group spans both quads
    p, n, u, i = strip(mirror_right=False)
    np.testing.assert_allclose(load_tangents(tmp_path, p, n, u, i, "m3.gltf"), [[1, 0, 0, 1]] * 6, atol=1e-6)


def fan(center_split):
    """Non-planar fan of four triangles around a raised centre vertex whose
    corner angles differ; the centre is one index, or two indices with equal
    attributes (welded) for alternate triangles."""
    rim = np.array([[1, 0, 0], [0.2, 1.3, 0], [-1, 0.1, 0.1], [0, -1, -0.2], [1, 0, 0]], np.float64)
    c = np.array([0.1, 0.05, 0.6])
    pos = np.vstack([rim[:4], c, c])
    n_rim = unit(np.tile([0, 0, 1.0], (4, 1)) + 0.2 * rim[:4])
    nc = unit([0.05, 0.02, 1.0])
    nrm = np.vstack([n_rim, nc, nc])
    # UV: an affine image of xy with a shear, so dP/du differs per face
    uv = np.column_stack([pos[:, 0] + 0.3 * pos[:, 1], pos[:, 1] - 0.2 * pos[:, 0] + 0.5 * pos[:, 2]])
    idx = []
    for k in range(4):
        centre = 5 if (center_split and k % 2) else 4
        idx += [k, (k + 1) % 4, centre]
    return pos, nrm, uv, np.array(idx)


def expected_centre(pos, nrm, uv, idx, centre_ids):
    """Angle-weighted sum of the faces' in-plane dP/du at the centre."""
    acc = np.zeros(3)
    n = nrm[centre_ids[0]]
    for f in range(len(idx) // 3):
        tri = idx[3 * f:3 * f + 3]
        k = [i for i in range(3) if tri[i] in centre_ids][0]
        i0, i1, i2 = tri[k], tri[(k + 1) % 3], tri[(k + 2) % 3]
        e1, e2 = pos[tri[1]] - pos[tri[0]], pos[tri[2]] - pos[tri[0]]
        d1, d2 = uv[tri[1]] - uv[tri[0]], uv[tri[2]] - uv[tri[0]]
        area2 = d1[0] * d2[1] - d1[1] * d2[0]
        s = (d2[1] * e1 - d1[1] * e2) * np.sign(area2)
        proj = lambda v: unit(v - n * np.dot(n, v))
        ang = math.acos(np.clip(np.dot(proj(pos[i1] - pos[i0]), proj(pos[i2] - pos[i0])), -1, 1))
        acc += ang * proj(unit(s))
    return unit(acc)


@pytest.mark.parametrize("split", [False, True])
def test_angle_weighted_sum_and_welding(tmp_path, split):
    pos, nrm, uv, idx = fan(split)
    t = load_tangents(tmp_path, pos, nrm, uv, idx)
    ids = [4, 5] if split else [4]
    want = expected_centre(pos, nrm, uv, idx, ids)
    for i in ids:
        np.testing.assert_allclose(t[i, :3], want, atol=2e-6)
        assert t[i, 3] == 1.0
    if split:
        np.testing.assert_array_equal(t[4], t[5])
        single = load_tangents(tmp_path, *fan(False), "single.gltf")
        np.testing.assert_allclose(t[4], single[4], atol=1e-7)


def test_zero_uv_area_triangles(tmp_path):
    # one triangle of the quad has collinear UVs: its corners contribute
    # nothing; vertices only it touches get the fallback
    pos = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [2, 0.5, 0]], np.float64)
    nrm = np.tile([0, 0, 1.0], (5, 1))
    uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1], [1, 0.5]], np.float64)
    idx = np.array([0, 1, 2, 0, 2, 3, 1, 4, 2])  # the last one: UV (1,0),(1,.5),(1,1) collinear
    t = load_tangents(tmp_path, pos, nrm, uv, idx)
    np.testing.assert_allclose(t[:4], [[1, 0, 0, 1]] * 4, atol=1e-6)
    np.testing.assert_allclose(t[4, :3], fallback(nrm[4]), atol=1e-6)
    assert t[4, 3] == 1.0
    # no UV frame anywhere: every vertex takes the reference's fallback
    n2 = unit(np.array([[0.95, 0.1, 0.2]] * 4))
    t2 = load_tangents(tmp_path, pos[:4], n2, np.zeros((4, 2)), idx[:6], "z.gltf")
    for i in range(4):
        np.testing.assert_allclose(t2[i, :3], fallback(n2[i]), atol=1e-6)
        assert t2[i, 3] == 1.0


def test_unreferenced_vertex_keeps_the_fallback(tmp_path):
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [5, 5, 5]], np.float64)
    nrm = np.tile([0, 0, 1.0], (4, 1))
    uv = np.array([[0, 0], [1, 0], [0, 1], [0.5, 0.5]], np.float64)
    t = load_tangents(tmp_path, pos, nrm, uv, [0, 1, 2])
    np.testing.assert_allclose(t[:3], [[1, 0, 0, 1]] * 3, atol=1e-6)
    np.testing.assert_allclose(t[3], [1, 0, 0, 1], atol=1e-6)
