"""Batched bakes (shb_bake_batch): uneven scenes, sizes, spp and bounces run
through one shared launch sequence give results bit-identical to one plain
bake each, with and without the CUDA graph, and with autotuned launch
parameters."""
import numpy as np
import pytest

from sh_baker_b200 import api, scenes
from sh_baker_b200.scene import Material, Texture

pytestmark = pytest.mark.gpu


def make_batch(ctx):
    specs = []
    for i, (boxes, res, ss, spp, bounces, lights) in enumerate(
            [(10, 32, 1, 16, 2, 1), (30, 64, 2, 8, 3, 4), (4, 24, 1, 32, 4, 8), (60, 48, 1, 5, 2, 2),
             (20, 40, 3, 4, 3, 3)]):
        sc = scenes.procedural_room(seed=100 + i, n_boxes=boxes, res=res, n_point_lights=lights)
        specs.append((sc, res, ss, spp, bounces))
    q = scenes.unit_quad()
    specs.append((q, 16, 1, 24, 3))
    alpha = scenes.procedural_room(seed=7, n_boxes=8, res=32)
    alpha.materials.append(Material(albedo=Texture(1, 1, 4, np.array([200, 180, 160, 120], np.uint8)),
                                    emission_intensity=2.0))
    alpha.geometries[2].material_id = len(alpha.materials) - 1
    scenes.mark_area_lights(alpha)
    specs.append((alpha, 32, 1, 8, 3))
    bakes = []
    for k, (sc, res, ss, spp, bounces) in enumerate(specs):
        ds = api.DeviceScene(ctx, sc)
        rc = api.RasterConfig(res, res, ss)
        g = api.rasterize_to_device(ds, rc)
        bakes.append(api.BatchBake(ds, g, rc, api.BakeConfig(samples=spp, bounces=bounces, seed=31 + k,
                                                             num_light_samples=1 + (k % 2))))
    return bakes


def plain(bakes):
    import torch
    outs = []
    for b in bakes:
        n = b.gbuffer.width * b.gbuffer.height
        sh = torch.empty(n * 27, dtype=torch.float32, device="cuda")
        env = torch.empty(n, dtype=torch.float32, device="cuda")
        api.bake_plain_device(b, sh, env)
        outs.append((sh.cpu().numpy(), env.cpu().numpy()))
    return outs


@pytest.mark.parametrize("use_graph,tile,share", [(False, 0, 0), (True, 0, 0), (True, 7, 0), (False, 100, 0),
                                                  (False, 0, -1), (True, 7, 2**31 - 1), (True, 0, 3000)])
def test_batch_equals_plain(gpu_ctx, use_graph, tile, share):
    """share: 0 = bakes under half a wave share waves; -1 = every bake has
    waves of its own (one-bake traversal); 2^31-1 = all bakes share."""
    bakes = make_batch(gpu_ctx)
    ref = plain(bakes)
    outs, st = api.bake_batch(gpu_ctx, bakes, use_graph=use_graph, tile_texels=tile, wave_paths=1 << 14,
                              share_paths=share)
    assert st.error_flags == 0 and st.waves >= (len(bakes) if share == -1 else 2)
    for (sh, env), (rsh, renv) in zip(outs, ref):
        assert sh.cpu().numpy().tobytes() == rsh.tobytes()
        assert env.cpu().numpy().tobytes() == renv.tobytes()


def test_autotune_persists_per_shape_class(gpu_ctx, tmp_path):
    bakes = make_batch(gpu_ctx)
    ref = plain(bakes)
    cache = tmp_path / "tune.txt"
    outs, _ = api.bake_batch(gpu_ctx, bakes, autotune=True, tune_cache=str(cache))
    lines = cache.read_text().splitlines()
    assert len(lines) == 1
    key, wave, tile, grid, share, cost = lines[0].split()
    assert int(wave) > 0 and int(tile) > 0 and int(grid) >= 1 and int(share) >= 0 and float(cost) > 0
    outs2, _ = api.bake_batch(gpu_ctx, bakes, autotune=True, tune_cache=str(cache))
    assert cache.read_text().splitlines() == lines  # second batch reads the entry
    for (sh, env), (sh2, env2), (rsh, renv) in zip(outs, outs2, ref):
        assert sh.cpu().numpy().tobytes() == rsh.tobytes() == sh2.cpu().numpy().tobytes()


def test_nee_kernel_split_is_bit_identical(gpu_ctx):
    """Next-event estimation inline in the hit kernel (nee_split=1) or as its
    own kernel over per-hit records (nee_split=2) gives the same bits, with
    one and two light samples, alpha branching and area lights."""
    bakes = make_batch(gpu_ctx)
    ref = plain(bakes)
    for split in (1, 2):
        outs, st = api.bake_batch(gpu_ctx, bakes, use_graph=False, wave_paths=1 << 14, nee_split=split)
        assert st.error_flags == 0
        for (sh, env), (rsh, renv) in zip(outs, ref):
            assert sh.cpu().numpy().tobytes() == rsh.tobytes()
            assert env.cpu().numpy().tobytes() == renv.tobytes()
