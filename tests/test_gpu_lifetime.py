"""Object lifetimes through the C ABI: scenes and G-buffers keep their
context alive, so they may be destroyed after it, in any order, and a
process may exit with them still alive.  Each case runs in a child process
so that a crash fails the test instead of the test run."""
import subprocess
import sys
import textwrap
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]

PRELUDE = """
import sys
sys.path.insert(0, {root!r})
from sh_baker_b200 import api, scenes
sc = scenes.procedural_room(seed=2, n_boxes=6, res=32)
rc = api.RasterConfig(32, 32, 1)
cfg = api.BakeConfig(samples=4, bounces=2, seed=1)
"""


def run(body):
    code = PRELUDE.format(root=str(ROOT)) + textwrap.dedent(body)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    assert "done" in r.stdout


def test_destroy_context_before_scene_and_gbuffer():
    run("""
        ctx = api.Context(device=0)
        ds = api.DeviceScene(ctx, sc)
        g = api.rasterize_to_device(ds, rc)
        ctx.close()
        g.close()
        ds.close()
        ctx2 = api.Context(device=0)
        ds2 = api.DeviceScene(ctx2, sc)
        r = api.BakeSHLightMap(ds2, api.RasterizeScene(ds2, rc, ctx=ctx2), rc, cfg, ctx=ctx2)
        assert float(abs(r.sh_texture).sum()) > 0
        ds2.close()
        ctx2.close()
        print("done")
    """)


def test_exit_with_scene_alive_after_context_closed():
    run("""
        ctx = api.Context(device=0)
        ds = api.DeviceScene(ctx, sc)
        pts = api.RasterizeScene(ds, rc, ctx=ctx)
        api.BakeSHLightMap(ds, pts, rc, cfg, ctx=ctx)
        ctx.close()
        print("done")
    """)
