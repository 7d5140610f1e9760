"""bench.py's CPU side: the reference arm (`--impl reference`, the oracle
port on the host cores) prints one JSON line with the contract's keys, and
under several ranks only rank 0 prints.  The GPU arms run in the -m gpu
suite's environment only."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def run_ref(extra_env=None):
    env = dict(os.environ, **(extra_env or {}))
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", "unit_quad",
                        "--steps", "2", "--warmup", "1", "--ref-step-seconds", "0.2"],
                       capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    return [ln for ln in r.stdout.splitlines() if ln.startswith("{")]


def test_reference_arm_line():
    lines = run_ref()
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert "unit_quad" in d["config"]["workload"] and "fit in the 126 MB L2" in d["config"]["l2"]


def test_reference_arm_other_ranks_are_silent():
    assert run_ref({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []


def test_default_workload_is_the_atrium():
    import argparse
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    w = bench.WORKLOADS["atrium"]
    assert (w["width"], w["height"], w["ss"], w["spp"], w["bounces"], w["dilation"]) == (2048, 2048, 3, 256, 4, 4)
    src = (ROOT / "bench.py").read_text()
    assert 'ap.add_argument("--workload", default="atrium"' in src
    del argparse


def test_traversal_profile_rows_parse(tmp_path, monkeypatch):
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod2", ROOT / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    (tmp_path / "profiles").mkdir()
    (tmp_path / "profiles" / "traversal_demo_small.md").write_text(
        "| kernel | rays | DRAM B/ray | L2 B/ray | warp inst/ray | lanes |\n|---|---|---|---|---|---|\n"
        "| closest_hit | 1000 | 49.6 | 812.5 | 210.0 | 13.5 |\n")
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    got = bench.traversal_profile("demo", "closest_hit")
    assert got["warp_inst_per_ray"] == 210.0 and got["l2_bytes_per_ray"] == 812.5 and got["profiled_rays"] == 1000
    assert bench.traversal_profile("demo", "any_hit") is None
