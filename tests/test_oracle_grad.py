"""The FP64 forward-mode gradient of the oracle (oracle_bake_grad), pinned
on the CPU against central differences of the oracle's own FP64 bake.  With
a single light the light pick does not depend on the parameters, so for
fixed random numbers the estimator is a polynomial in each parameter and
central differences agree with the forward-mode derivative to O(h^2)."""
import numpy as np
import pytest

from oracle.pyoracle import OracleScene
from sh_baker_b200 import scenes


def one_light_room():
    sc = scenes.procedural_room(seed=5, n_boxes=6, res=16, n_point_lights=1)
    sc.lights = [sc.lights[1]]  # the point light inside the closed room
    return sc


def fd_loss(o, pts, dsh, albedo, intensity, samples, bounces, seed=99):
    o.set_params(albedo, intensity)
    r = o.bake(pts, 16, 16, 1, samples, bounces, seed=seed, fp64=True, stats=True)
    return float(np.sum(r["mean64"].reshape(-1).astype(np.float64) * dsh.reshape(-1)))


@pytest.fixture(scope="module")
def setup():
    sc = one_light_room()
    o = OracleScene(sc)
    pts = o.rasterize(16, 16, 1)
    rng = np.random.default_rng(7)
    albedo = rng.uniform(0.2, 0.8, (len(sc.materials), 3)).astype(np.float32)
    intensity = np.array([sc.lights[0].intensity], np.float32)
    dsh = rng.normal(size=(pts.size, 27)).astype(np.float32)
    return sc, o, pts, albedo, intensity, dsh


def test_forward_mode_matches_central_differences(setup):
    sc, o, pts, albedo, intensity, dsh = setup
    samples, bounces = 4, 2
    o.set_params(albedo, intensity)
    d_alb, d_li = o.bake_grad(pts, 16, 16, 1, samples, bounces, dsh, seed=99)
    assert np.all(np.isfinite(d_alb)) and np.isfinite(d_li).all()
    # the materials the G-buffer sees most
    mats, counts = np.unique(pts["material_id"][pts["material_id"] >= 0], return_counts=True)
    checks = [("light", 0, 0)] + [("albedo", int(m), c) for m in mats[np.argsort(-counts)][:2] for c in range(3)]
    h = 1e-3
    for kind, i, c in checks:
        a_p, a_m = albedo.copy(), albedo.copy()
        l_p, l_m = intensity.copy(), intensity.copy()
        # parameters are float32: difference by the step they really took
        if kind == "light":
            l_p[0] += h * float(intensity[0])
            l_m[0] -= h * float(intensity[0])
            step2 = float(l_p[0]) - float(l_m[0])
            got = d_li[0]
        else:
            a_p[i, c] += h
            a_m[i, c] -= h
            step2 = float(a_p[i, c]) - float(a_m[i, c])
            got = d_alb[i, c]
        fd = (fd_loss(o, pts, dsh, a_p, l_p, samples, bounces) -
              fd_loss(o, pts, dsh, a_m, l_m, samples, bounces)) / step2
        assert got == pytest.approx(fd, rel=2e-5, abs=1e-7 * (1 + abs(fd))), (kind, i, c, got, fd)


def test_materials_without_override_get_no_gradient(setup):
    sc, o, pts, albedo, intensity, dsh = setup
    use = np.zeros(len(sc.materials), np.uint8)
    use[0] = 1
    o.set_params(albedo, intensity, use_override=use)
    d_alb, _ = o.bake_grad(pts, 16, 16, 1, 2, 2, dsh, seed=99)
    assert np.all(d_alb[1:] == 0.0)
    o.set_params(albedo, intensity)


def test_area_light_emission_gradient_matches_central_differences():
    """One emissive box as the only light: the gradient of its material's
    albedo flows through the area-light NEE and the depth-0 emission."""
    from sh_baker_b200.scene import Material, Texture
    sc = scenes.procedural_room(seed=6, n_boxes=6, res=16, n_point_lights=0)
    sc.lights = []
    sc.materials.append(Material(albedo=Texture(1, 1, 3, np.array([220, 200, 180], np.uint8)),
                                 emission_intensity=3.0))
    em = len(sc.materials) - 1
    sc.geometries[3].material_id = em
    scenes.mark_area_lights(sc)
    assert len(sc.lights) == 1
    o = OracleScene(sc)
    pts = o.rasterize(16, 16, 1)
    rng = np.random.default_rng(8)
    albedo = rng.uniform(0.2, 0.8, (len(sc.materials), 3)).astype(np.float32)
    inten = np.array([1.0], np.float32)
    dsh = rng.normal(size=(pts.size, 27)).astype(np.float32)
    o.set_params(albedo, inten)
    d_alb, d_li = o.bake_grad(pts, 16, 16, 1, 4, 2, dsh, seed=99)
    assert d_li[0] == 0.0 and abs(d_alb[em]).sum() > 0
    for c in range(3):
        a_p, a_m = albedo.copy(), albedo.copy()
        a_p[em, c] += 1e-3
        a_m[em, c] -= 1e-3
        fd = (fd_loss(o, pts, dsh, a_p, inten, 4, 2) - fd_loss(o, pts, dsh, a_m, inten, 4, 2)) / (
            float(a_p[em, c]) - float(a_m[em, c]))
        assert d_alb[em, c] == pytest.approx(fd, rel=2e-5, abs=1e-7 * (1 + abs(fd)))
