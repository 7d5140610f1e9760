"""The warp-cooperative triangle phase of the traversal kernels (the default
build) against the per-lane triangle loop (the same sources built with
SHB_TRI_COOP=0): whole bakes, whose closest-hit and any-hit queries all go
through the two phases, give the same bits.  The cooperative phase replays
each ray's accepted tests in triangle order against its shrinking tmax, so
its hits are the sequential loop's, ties included.

Each library runs in its own process (one libshb.so per process)."""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

BAKE = r"""
import sys
import numpy as np
from sh_baker_b200 import api, scenes
out = []
for sc, res, ss in ((scenes.atrium(seed=3, res=128), 128, 1), (scenes.procedural_room(seed=4, res=64), 64, 2)):
    r = api.bake_lightmap(sc, res, res, samples=16, bounces=4, supersample_scale=ss, dilation=0, seed=5)
    out += [r.sh.reshape(-1), r.env.reshape(-1)]
    b = api.bake_lightmap(sc, res, res, samples=4, bounces=2, supersample_scale=ss, dilation=0, seed=6,
                          num_light_samples=3)
    out += [b.sh.reshape(-1), b.env.reshape(-1)]
np.save(sys.argv[1], np.concatenate(out))
"""


def run_bake(path: Path, library=None) -> np.ndarray:
    env = dict(os.environ)
    env.pop("SHB_LIBRARY", None)
    if library is not None:
        env["SHB_LIBRARY"] = str(library)
    subprocess.run([sys.executable, "-c", BAKE, str(path)], check=True, env=env, cwd=ROOT, timeout=600)
    return np.load(path)


def test_cooperative_triangle_phase_matches_per_lane_loop(tmp_path):
    from sh_baker_b200 import build as B
    per_lane = B.build(variant="tri_per_lane", defines=["SHB_TRI_COOP=0"])
    coop = run_bake(tmp_path / "coop.npy")
    seq = run_bake(tmp_path / "seq.npy", per_lane)
    assert coop.size > 0 and np.isfinite(coop).all()
    assert coop.tobytes() == seq.tobytes()
