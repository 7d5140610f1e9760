#!/usr/bin/env python
"""Throughput of the SH9 lightmap bake on B200 (texel-samples/s).

One step = one BakeSHLightMap pass (BVH build + path tracing + SH9
projection, the region src/main.cpp:131-136 times) over the whole
supersampled G-buffer of the workload, inputs resident in HBM.  `e2e` is the
same metric through the public C ABI from pinned host buffers: scene upload,
raster, bake, masks, downsample, dilation and the read-back of the final
lightmap.  The CPU baseline is the oracle restatement on the host cores.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "texel-samples/s on 1 B200 at ≤1% rel. RMSE; batched and adjoint vs plain bake"
UNIT = "texel-samples/s"

WORKLOADS = {
    # procedural room: 12-triangle closed room + 200 boxes (2,412 triangles),
    # lightmap 1024^2, supersample 3, 128 spp, 3 bounces, dilation 2
    "room": dict(kind="room", width=1024, height=1024, ss=3, spp=128, bounces=3, dilation=2, seed=2),
    "room_small": dict(kind="room", width=256, height=256, ss=2, spp=32, bounces=3, dilation=2, seed=2),
    "unit_quad": dict(kind="unit_quad", width=256, height=256, ss=1, spp=64, bounces=3, dilation=0, seed=1),
    # two-storey colonnaded courtyard (~262k triangles), lightmap 2048^2,
    # supersample 3, 256 spp, 4 bounces, dilation 4
    "atrium": dict(kind="atrium", width=2048, height=2048, ss=3, spp=256, bounces=4, dilation=4, seed=3),
    "atrium_small": dict(kind="atrium", width=512, height=512, ss=1, spp=32, bounces=4, dilation=4, seed=3),
    # the atrium at a quarter of its supersampled texels: tuning runs of a few seconds per step
    "atrium_mid": dict(kind="atrium", width=1024, height=1024, ss=3, spp=64, bounces=4, dilation=4, seed=3),
}


def make_scene(w):
    from sh_baker_b200 import scenes
    if w["kind"] == "room":
        return scenes.procedural_room(seed=w["seed"], res=w["width"])
    if w["kind"] == "atrium":
        return scenes.atrium(seed=w["seed"], res=w["width"])
    if w["kind"] == "unit_quad":
        return scenes.unit_quad()
    raise ValueError(w["kind"])


def bytes_per_ray(n_tris: int) -> int:
    """Algorithmic bytes of one ray: L node fetches of an 80-byte 8-wide
    node plus one leaf of four 48-byte triangles, L = ceil(log8(ceil(N/4)))."""
    leaves = max(1, math.ceil(n_tris / 4))
    L = max(1, math.ceil(math.log(leaves, 8) - 1e-12))
    return L * 80 + 4 * 48


def traversal_profile(kind: str, kernel: str):
    """Per-ray ncu figures of a traversal kernel from the committed summary
    of the small case of the same scene (profiles/traversal_<kind>_small.md,
    its table row `| closest_hit | ... |`): DRAM bytes, L2 bytes and warp
    instructions per ray and active lanes per warp instruction.  None when
    absent.  The per-ray figures do not depend on the lightmap size, so they
    are scaled by the live ray counts of the full workload."""
    import re
    p = ROOT / "profiles" / f"traversal_{kind}_small.md"
    if not p.exists():
        return None
    m = re.search(rf"^\| {kernel} \| ([0-9.]+) \| ([0-9.]+) \| ([0-9.]+) \| ([0-9.]+) \| ([0-9.]+) \|$",
                  p.read_text(), re.M)
    if not m:
        return None
    rays, dram, l2, inst, lanes = (float(g) for g in m.groups())
    return {"profiled_rays": int(rays), "dram_bytes_per_ray": dram, "l2_bytes_per_ray": l2,
            "warp_inst_per_ray": inst, "active_lanes": lanes, "source": f"profiles/{p.name}"}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback 6650 GB/s, earlier measurement on this pool (MEASURED_PEAKS.json absent)"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "200"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        rows = [r.split(",") for r in Path(self.file.name).read_text().splitlines() if r.count(",") >= 8]
        os.unlink(self.file.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_baseline(scene, pts, w, seconds: float, threads: int, rng_seed: int = 1):
    """The oracle (float, the reference's mt19937 stream) on a seeded random
    subset of valid texels at full spp, sized to about `seconds` of work."""
    import numpy as np

    from oracle import pyoracle as O
    osc = O.OracleScene(scene)
    valid = np.flatnonzero(pts["material_id"] >= 0)
    rng = np.random.default_rng(rng_seed)
    # the probe gives every thread work, so its rate is the loaded rate
    probe = rng.choice(valid, size=min(len(valid), 32 * threads), replace=False)
    t0 = time.perf_counter()
    r = osc.bake(pts, w["width"], w["height"], w["ss"], samples=w["spp"], bounces=w["bounces"], rng=O.RNG_MT19937,
                 subset=probe, threads=threads)
    dt = max(time.perf_counter() - t0, 1e-3)
    rate = r["texel_samples"] / dt
    n = int(min(len(valid), max(64, rate * seconds / w["spp"])))
    for _ in range(2):  # a run far shorter than asked is resized once from its own rate
        sub = rng.choice(valid, size=n, replace=False)
        t0 = time.perf_counter()
        r = osc.bake(pts, w["width"], w["height"], w["ss"], samples=w["spp"], bounces=w["bounces"],
                     rng=O.RNG_MT19937, subset=sub, threads=threads)
        dt = time.perf_counter() - t0
        if dt >= 0.5 * seconds or n >= len(valid):
            break
        n = int(min(len(valid), n * seconds / max(dt, 1e-3)))
    return {"value": r["texel_samples"] / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} random valid texels of the workload at {w['spp']} spp (oracle restatement, "
                      f"std::mt19937 stream, {r['rays']} rays, {dt:.1f} s)"}


def run_reference(args, w):
    """CPU arm: the reference algorithm as restated by the oracle (the
    reference itself cannot be compiled here), all host threads."""
    import numpy as np

    from oracle import pyoracle as O
    from sh_baker_b200 import scenes  # noqa: F401
    scene = make_scene(w)
    osc = O.OracleScene(scene)
    pts = osc.rasterize(w["width"], w["height"], w["ss"])
    threads = os.cpu_count() or 1
    valid = np.flatnonzero(pts["material_id"] >= 0)
    rng = np.random.default_rng(7)
    probe = rng.choice(valid, size=min(len(valid), 32 * threads), replace=False)
    t0 = time.perf_counter()
    r = osc.bake(pts, w["width"], w["height"], w["ss"], samples=w["spp"], bounces=w["bounces"], rng=O.RNG_MT19937,
                 subset=probe, threads=threads)
    rate = r["texel_samples"] / max(time.perf_counter() - t0, 1e-3)
    n = int(min(len(valid), max(64, rate * args.ref_step_seconds / w["spp"])))
    times, ts = [], 0
    for step in range(args.warmup + args.steps):
        sub = rng.choice(valid, size=n, replace=False)
        t0 = time.perf_counter()
        r = osc.bake(pts, w["width"], w["height"], w["ss"], samples=w["spp"], bounces=w["bounces"],
                     rng=O.RNG_MT19937, subset=sub, threads=threads)
        dt = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(dt)
            ts += r["texel_samples"]
    total = sum(times)
    value = ts / total
    sample = f"{n} random valid texels per step at {w['spp']} spp (oracle restatement of the reference, mt19937)"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_of(w, scene),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def pinned_scene(scene, pin):
    """Copy of the scene whose arrays live in pinned (page-locked) memory."""
    import copy

    import numpy as np
    import torch

    def p(a, dt):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=dt)
        out = pin(a.shape, {np.float32: torch.float32, np.uint32: torch.int32, np.uint8: torch.uint8}[dt])
        out = out.view(dt) if dt == np.uint32 else out
        out[...] = a
        return out

    s = copy.deepcopy(scene)
    for g in s.geometries:
        g.vertices, g.normals = p(g.vertices, np.float32), p(g.normals, np.float32)
        g.texture_uvs, g.lightmap_uvs = p(g.texture_uvs, np.float32), p(g.lightmap_uvs, np.float32)
        g.tangents, g.indices = p(g.tangents, np.float32), p(g.indices, np.uint32)
    for m in s.materials:
        m.albedo.pixel_data = p(m.albedo.pixel_data, np.uint8)
    return s


def batched_result(steps: int, warmup: int):
    """64 independent procedural rooms (1k-100k triangles, 128^2-1024^2,
    32-256 spp, 2-4 bounces, 1-8 point lights): one shb_bake_batch (CUDA
    graph, autotuned launch structure) per step versus the same 64 bakes
    through the plain shb_bake path one at a time.  Scenes are uploaded and
    rasterised once, untimed, for both; the first warm-up call tunes."""
    import tempfile

    import torch

    from sh_baker_b200 import api, scenes
    torch.cuda.set_device(0)
    mix = scenes.batched_mix(seed=4, n=64)
    ctx = api.Context(device=0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    bakes, outs = [], []
    for m in mix:
        ds = api.DeviceScene(ctx, m["scene"])
        rc = api.RasterConfig(m["width"], m["height"], 1)
        g = api.rasterize_to_device(ds, rc)
        bakes.append(api.BatchBake(ds, g, rc, api.BakeConfig(samples=m["spp"], bounces=m["bounces"], seed=m["seed"])))
        n = g.width * g.height
        outs.append((torch.empty(n * 27, dtype=torch.float32, device="cuda"),
                     torch.empty(n, dtype=torch.float32, device="cuda")))
    tune = str(Path(tempfile.mkdtemp()) / "autotune.txt")
    for _ in range(max(warmup, 1)):  # the first batched call tunes and caches
        api.bake_batch(ctx, bakes, use_graph=True, autotune=True, tune_cache=tune, outputs=outs)
    for b, (sh, env) in zip(bakes, outs):
        api.bake_plain_device(b, sh, env)
    torch.cuda.synchronize()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), r

    clocks = ClockSampler(0)
    clocks.start()
    l0 = ctx.kernel_launches()
    b_ms, ts = 0.0, 0
    for _ in range(steps):
        ms, (_, st) = timed(lambda: api.bake_batch(ctx, bakes, use_graph=True, autotune=True, tune_cache=tune,
                                                   outputs=outs))
        b_ms += ms
        ts += st.texel_samples
    launches = ctx.kernel_launches() - l0
    s_ms = 0.0
    for _ in range(steps):
        ms, _ = timed(lambda: [api.bake_plain_device(b, sh, env) for b, (sh, env) in zip(bakes, outs)])
        s_ms += ms
    clk = clocks.stop()
    head = batched_headroom(api, bakes, outs, stream, timed)
    tuned = Path(tune).read_text().split()
    tris = [m["scene"].triangle_count for m in mix]
    res = {"value": ts / (b_ms / 1e3), "ms_per_step": b_ms / steps, "steps": steps, "warmup": warmup,
           "sequential": {"value": ts / (s_ms / 1e3), "ms_per_step": s_ms / steps},
           "speedup_vs_sequential": s_ms / b_ms,
           "autotuned": {"wave_paths": int(tuned[1]), "tile_texels": int(tuned[2]), "grid_scale": int(tuned[3]),
                         "share_paths": int(tuned[4])},
           "workload": "64 procedural rooms, 1k-100k triangles, 128^2-1024^2, 32-256 spp, 2-4 bounces, "
                       "1-8 point lights; shb_bake_batch in a CUDA graph vs 64 plain shb_bake calls",
           "bakes": 64, "triangles_total": int(sum(tris)), "texel_samples_per_step": ts // steps,
           "gpu_launches": int(launches), "clocks": clk, "headroom": head}
    ctx.close()
    return res


def batched_headroom(api, bakes, outs, stream, timed, target_paths: int = 1 << 24):
    """How much any batching can gain on this mix.  Each bake is timed alone
    through the plain path, and again with its sample count multiplied
    until it traces at least `target_paths` paths: the same texels, scene,
    bounces and per-path work, enough to fill the GPU, so its rate there is
    the bake's saturated rate.  A bake's idle time is its plain time minus
    its texel-samples at the saturated rate; no launch structure can beat
    the sum of the saturated times, which bounds the batched speed-up."""
    import torch
    plain_ms = sat_ms = 0.0
    per = []
    for b, (sh, env) in zip(bakes, outs):
        ms, st = timed(lambda: api.bake_plain_device(b, sh, env))
        n = st.texel_samples
        m = max(1, -(-target_paths // max(n, 1)))
        cfg = api.BakeConfig(samples=b.config.samples * m, bounces=b.config.bounces, seed=b.config.seed)
        big = api.BatchBake(b.scene, b.gbuffer, b.raster, cfg)
        ms_big, st_big = timed(lambda: api.bake_plain_device(big, sh, env))
        sat = n / (st_big.texel_samples / ms_big)  # ms at the saturated rate
        plain_ms += ms
        sat_ms += sat
        per.append((n, ms, sat))
    torch.cuda.synchronize()
    small = [x for x in per if x[0] < 5_000_000]
    return {"plain_ms": plain_ms, "saturated_ms": sat_ms, "idle_ms": plain_ms - sat_ms,
            "max_speedup": plain_ms / sat_ms,
            "bakes_under_5M_texel_samples": {"count": len(small), "plain_ms": sum(x[1] for x in small),
                                             "saturated_ms": sum(x[2] for x in small)},
            "method": "per bake: plain time vs its texel-samples at the rate of the same bake with samples "
                      f"multiplied to >= {target_paths} paths"}


def run_batched(args):
    from sh_baker_b200 import build as B
    B.build()
    r = batched_result(args.steps, args.warmup)
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": r["workload"], "bakes": r["bakes"], "triangles_total": r["triangles_total"],
                       "texel_samples_per_step": r["texel_samples_per_step"]},
            "sequential": r["sequential"], "speedup_vs_sequential": r["speedup_vs_sequential"],
            "autotuned": r["autotuned"], "headroom": r["headroom"], "gpu_launches": r["gpu_launches"],
            "clocks": r["clocks"]}
    print(json.dumps(line), flush=True)


def adjoint_result(steps: int, warmup: int):
    """Adjoint bake: procedural room (2,412 triangles) at lightmap 512^2,
    supersample 3 (the room workload's), 64 spp, 3 bounces.  Loss = sum
    (SH - SH_target)^2 with the target baked at albedos x U[0.8, 1.2] and
    light intensities x U[0.5, 2].  A step = forward bake + dLoss/dSH +
    path-replay backward; both halves are timed with CUDA events.  The
    gradient of all 8x3 albedos and 5 intensities is compared with central
    differences (h = 1e-3, common random numbers)."""
    import numpy as np
    import torch

    from sh_baker_b200 import api, scenes
    torch.cuda.set_device(0)
    res, spp, bounces = 512, 64, 3
    sc = scenes.procedural_room(seed=2, res=res)
    ctx = api.Context(device=0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ds = api.DeviceScene(ctx, sc)
    rc = api.RasterConfig(res, res, 3)
    g = api.rasterize_to_device(ds, rc)
    bake = api.BatchBake(ds, g, rc, api.BakeConfig(samples=spp, bounces=bounces, seed=2))
    albedo = api.material_linear_albedo(sc)
    inten = np.array([l.intensity for l in sc.lights], np.float32)
    rng = np.random.default_rng(5)
    n = g.width * g.height
    sh = torch.empty(n * 27, dtype=torch.float32, device="cuda")
    env = torch.empty(n, dtype=torch.float32, device="cuda")
    target = torch.empty_like(sh)
    ds.set_params(albedo * rng.uniform(0.8, 1.2, albedo.shape).astype(np.float32),
                  inten * rng.uniform(0.5, 2.0, inten.shape).astype(np.float32))
    api.bake_plain_device(bake, target, env)
    ds.set_params(albedo, inten)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def step():
        e0, e1, e2 = ev(), ev(), ev()
        with torch.cuda.stream(stream):
            e0.record(stream)
            st = api.bake_plain_device(bake, sh, env)
            e1.record(stream)
            dsh = 2.0 * (sh - target)
        d_alb, d_li = api.Backward(bake, dsh)
        e2.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), e1.elapsed_time(e2), st.texel_samples, (d_alb, d_li)

    for _ in range(warmup):
        step()
    clocks = ClockSampler(0)
    clocks.start()
    l0 = ctx.kernel_launches()
    f_ms = b_ms = 0.0
    ts = 0
    for _ in range(steps):
        fm, bm, t, grads = step()
        f_ms += fm
        b_ms += bm
        ts += t
    launches = ctx.kernel_launches() - l0
    clk = clocks.stop()

    def loss(a, i):  # central differences under common random numbers (same seed)
        ds.set_params(a, i)
        with torch.cuda.stream(stream):
            api.bake_plain_device(bake, sh, env)
            v = float(((sh.double() - target.double()) ** 2).sum())
        return v

    h = 1e-3
    fd_alb = np.zeros_like(albedo, dtype=np.float64)
    fd_li = np.zeros_like(inten, dtype=np.float64)
    for m in range(albedo.shape[0]):
        for c in range(3):
            ap, am = albedo.copy(), albedo.copy()
            ap[m, c] += h
            am[m, c] -= h
            fd_alb[m, c] = (loss(ap, inten) - loss(am, inten)) / (float(ap[m, c]) - float(am[m, c]))
    for l in range(len(inten)):
        ip, im = inten.copy(), inten.copy()
        ip[l] *= 1 + h
        im[l] *= 1 - h
        fd_li[l] = (loss(albedo, ip) - loss(albedo, im)) / (float(ip[l]) - float(im[l]))
    ds.set_params(albedo, inten)
    d_alb, d_li = grads
    got = np.concatenate([d_alb.reshape(-1), d_li * inten])
    fd = np.concatenate([fd_alb.reshape(-1), fd_li * inten])
    rel = float(np.linalg.norm(got - fd) / np.linalg.norm(fd))
    worst = float(np.max(np.abs(got - fd)) / np.max(np.abs(fd)))
    out = {"value": ts / (b_ms / 1e3), "ms_per_step": (f_ms + b_ms) / steps, "steps": steps, "warmup": warmup,
           "workload": "adjoint bake: procedural room 2,412 triangles, lightmap 512x512, supersample 3, 64 spp, "
                       "3 bounces; loss sum (SH - SH_target)^2, 8x3 albedos + 5 intensities",
           "texel_samples_per_step": ts // steps, "forward_ms": f_ms / steps, "backward_ms": b_ms / steps,
           "backward_over_forward": b_ms / f_ms, "fd_rel_l2": rel,
           "fd_check": {"h": h, "rel_l2_err": rel, "max_err_over_max": worst},
           "gpu_launches": int(launches), "clocks": clk}
    ctx.close()
    return out


def run_adjoint(args):
    from sh_baker_b200 import build as B
    B.build()
    r = adjoint_result(args.steps, args.warmup)
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": r["workload"], "texel_samples_per_step": r["texel_samples_per_step"]},
            "forward_ms": r["forward_ms"], "backward_ms": r["backward_ms"],
            "backward_over_forward": r["backward_over_forward"], "fd_check": r["fd_check"],
            "gpu_launches": r["gpu_launches"], "clocks": r["clocks"]}
    print(json.dumps(line), flush=True)


def accuracy(w, scene, ctx):
    """Global relative RMSE of a GPU bake, at the workload's spp and bounces,
    against the committed 4096-spp FP64 oracle fixture of the workload
    (tests/golden/fp64_<kind>.npz, a crop of the output lightmap), over all
    valid texels x 27 coefficients.  None when no fixture matches the
    workload's size."""
    import numpy as np

    from sh_baker_b200 import api
    path = ROOT / "tests" / "golden" / f"fp64_{w['kind']}.npz"
    if not path.exists():
        return None
    ref = np.load(path)
    W, H, ss, size, x0, y0 = (int(ref[k]) for k in ("width", "height", "ss", "size", "x0", "y0"))
    if (W, H, ss, int(ref["bounces"])) != (w["width"], w["height"], w["ss"], w["bounces"]):
        return None
    pts = api.RasterizeScene(scene, api.RasterConfig(W, H, ss), ctx=ctx).reshape(H * ss, W * ss)
    crop = np.ascontiguousarray(pts[y0 * ss:(y0 + size) * ss, x0 * ss:(x0 + size) * ss]).reshape(-1)
    rc = api.RasterConfig(size, size, ss)
    got = api.BakeSHLightMap(scene, crop, rc, api.BakeConfig(samples=w["spp"], bounces=w["bounces"], seed=2024),
                             ctx=ctx)
    g = api.DownsampleSHTexture(got.sh_texture, ss, ctx=ctx).reshape(size, size, 27)
    valid, r = ref["valid"], ref["sh"]
    err = float(np.linalg.norm((g - r)[valid]) / np.linalg.norm(r[valid]))
    err_l0 = float(np.linalg.norm((g - r)[valid][:, :3]) / np.linalg.norm(r[valid][:, :3]))
    floor = float(np.linalg.norm(ref["se"][valid]) / np.linalg.norm(r[valid]))
    expected = floor * float(np.sqrt(int(ref["spp"]) / w["spp"] + 1.0))
    return {"rel_rmse_vs_fp64": err, "rel_rmse_l0_vs_fp64": err_l0, "fp64_own_error": floor,
            "unbiased_predicted": expected, "fp64_spp": int(ref["spp"]),
            "crop": f"{size}x{size} output texels at ({x0},{y0}), supersample {ss}", "spp": w["spp"]}


def config_of(w, scene):
    return {"workload": f"procedural {w['kind']}: {scene.triangle_count} triangles, lightmap {w['width']}x{w['height']}"
                        f" supersample {w['ss']}, {w['spp']} spp, {w['bounces']} bounces, dilation {w['dilation']}",
            "triangles": scene.triangle_count, "width": w["width"], "height": w["height"],
            "supersample_scale": w["ss"], "samples": w["spp"], "bounces": w["bounces"], "dilation": w["dilation"],
            "l2": l2_note(w)}


def l2_note(w):
    """Whether one step's G-buffer reads and SH/env writes exceed the 126 MB
    L2, so that steps do not hit each other's data in cache."""
    n = w["width"] * w["ss"] * w["height"] * w["ss"]
    gb, out = n * 64 / 1e6, n * 112 / 1e6
    kind = "inputs larger than L2" if gb + out > 126 else "inputs fit in the 126 MB L2 (a parity case)"
    return "%s: G-buffer %.0f MB + outputs %.0f MB per step" % (kind, gb, out)


def exr_result(steps: int, warmup: int, reference: bool = True, ref_runs: int = 1):
    """SaveSHLightMap of a 2048^2 lightmap (the atrium's output size) in the
    three save modes from host buffers: the library (channel packing,
    float->half and the ZIP pre-pass on the GPU, zlib on all host threads)
    against the reference's own saver code path (tinyexr + miniz compiled
    from the reference tree into oracle/_ref, one host thread; the
    cpu_baseline leg).  The texture is a seeded smooth field with 1 %
    sample noise, like a converged bake.  Wall clock per save, files to a
    temporary directory: `warmup` untimed then `steps` timed saves per mode
    (the median), and `ref_runs` timed reference saves after one untimed."""
    import ctypes as C
    import tempfile

    import numpy as np

    from sh_baker_b200 import _capi as A
    from sh_baker_b200 import api
    W = H = 2048
    rng = np.random.default_rng(11)
    y, x = np.mgrid[0:H, 0:W].astype(np.float32) / np.float32(W)
    sh = np.empty((H, W, 9, 3), np.float32)
    for k in range(9):
        for c in range(3):
            f = rng.uniform(1, 6, 2).astype(np.float32)
            base = np.sin(f[0] * x + k) * np.cos(f[1] * y + c)
            sh[:, :, k, c] = (1.0 + base) if k == 0 else 0.3 * base
    sh *= (1.0 + 0.01 * rng.standard_normal(sh.shape)).astype(np.float32)
    env = np.clip(0.5 + 0.5 * np.sin(3 * x) * np.cos(2 * y), 0, 1).astype(np.float32)
    ctx = api.Context(device=0)
    modes = {"combined": A.SAVE_COMBINED, "split_channels": A.SAVE_SPLIT_CHANNELS,
             "luminance_packed": A.SAVE_LUMINANCE_PACKED}
    tmp = Path(tempfile.mkdtemp())
    ours, ref, files = {}, {}, {}
    ref_lib = None
    if reference:
        try:
            from oracle import build as OB
            path = OB.REF_LIB if OB.REF_LIB.exists() else OB.build_ref()
            if path is not None and Path(path).exists():
                ref_lib = C.CDLL(str(path))
                ref_lib.ref_exr_save.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_char_p, C.c_int]
        except OSError:
            ref_lib = None
    clocks = ClockSampler(0)
    clocks.start()
    for name, m in modes.items():
        out = tmp / f"ours_{name}.exr"
        ts = []
        for i in range(warmup + steps):
            t0 = time.perf_counter()
            A.check(ctx.lib.shb_save_sh_lightmap(ctx.h, sh.ctypes.data, env.ctypes.data, W, H, 0, str(out).encode(), m))
            if i >= warmup:
                ts.append(time.perf_counter() - t0)
        ours[name] = float(np.median(ts))
        files[name] = sum(p.stat().st_size for p in tmp.glob(f"ours_{name}*.exr"))
        if ref_lib is not None:
            rout = tmp / f"ref_{name}.exr"
            rts = []
            for i in range(1 + max(1, ref_runs)):
                t0 = time.perf_counter()
                assert ref_lib.ref_exr_save(sh.ctypes.data, env.ctypes.data, W, H, str(rout).encode(), m) == 0
                if i >= 1:
                    rts.append(time.perf_counter() - t0)
            ref[name] = float(np.median(rts))
    clk = clocks.stop()
    ctx.close()
    texels = W * H
    return {"value": texels / ours["combined"], "unit": "texels/s", "ms_per_save": ours["combined"] * 1e3,
            "steps": steps, "warmup": warmup,
            "workload": "SaveSHLightMap 2048x2048 SH9 + env visibility from host buffers, three save modes",
            "width": W, "height": H, "host_threads": os.cpu_count(),
            "modes": {n: {"ms": ours[n] * 1e3, "bytes": files[n],
                          "reference_ms": ref[n] * 1e3 if n in ref else None,
                          "speedup": ref[n] / ours[n] if n in ref else None} for n in modes},
            "reference_saver": ({"value": texels / ref["combined"], "unit": "texels/s", "cores": 1,
                                 "kind": "reference",
                                 "sample": "the whole 2048x2048 texture, the reference's tinyexr + miniz saver"}
                                if "combined" in ref else None),
            "h2d_bytes_per_save": int(sh.nbytes + env.nbytes), "clocks": clk}


def run_exr(args):
    from sh_baker_b200 import build as B
    B.build()
    r = exr_result(args.steps, args.warmup, reference=not args.no_cpu_baseline, ref_runs=max(1, args.steps // 2))
    line = {"metric": "lightmap texels saved/s (SaveSHLightMap, host buffers, median over saves)",
            "value": r["value"], "unit": "texels/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_save"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32->f16", "data": "synthetic",
            "config": {"workload": r["workload"], "width": r["width"], "height": r["height"],
                       "host_threads": r["host_threads"]},
            "modes": r["modes"], "cpu_baseline": r["reference_saver"],
            "e2e": {"value": r["value"], "unit": "texels/s", "h2d_bytes_per_step": r["h2d_bytes_per_save"],
                    "d2h_bytes_per_step": 0},
            "clocks": r["clocks"]}
    print(json.dumps(line), flush=True)


def roofline_of(stats, steps, scene, w, ms, clk):
    """Roofline of the dominant traversal kernel.  Traversal of incoherent
    rays is bound by instruction issue (dependent node fetches hit L1/L2,
    ncu shows ~80 % issue activity and DRAM traffic < 10 % of the model's
    bytes), so the bound reported is issue: warp instructions per ray (ncu,
    small case of the same scene) x rays traced / kernel time, against the
    SMs' issue slots (SMs x 4 schedulers x median SM clock under load).  The
    model-byte HBM figure (the algorithmic bytes of bytes_per_ray over the
    measured copy bandwidth) is kept beside it as `hbm_model`."""
    import torch
    ext_ms = sum(s.extend_kernel_ms for s in stats)
    sh_ms = sum(s.shadow_kernel_ms for s in stats)
    ext_rays = sum(s.extend_rays for s in stats)
    sh_rays = sum(s.shadow_rays for s in stats)
    bpr = bytes_per_ray(scene.triangle_count)
    dom = "closest_hit" if ext_ms >= sh_ms else "any_hit"
    k_ms, k_rays = (ext_ms, ext_rays) if dom == "closest_hit" else (sh_ms, sh_rays)
    k_launch = sum((s.extend_launches if dom == "closest_hit" else s.shadow_launches) for s in stats)
    rays_per_launch = k_rays / max(k_launch, 1)
    hbm_achieved = k_rays * bpr / (k_ms / 1e3) / 1e9 if k_ms > 0 else 0.0
    peak, peak_kind = measured_peak()
    prof = traversal_profile(w["kind"], dom)
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = (clk or {}).get("sm_mhz") or (clk or {}).get("sm_max_mhz") or 1965.0
    issue_peak = sms * 4 * mhz * 1e6 / 1e9  # G warp instructions / s
    roof = {"kernel": dom, "bound": "issue", "unit": "G warp-inst/s",
            "peak": issue_peak, "peak_source": f"{sms} SMs x 4 schedulers x {mhz:.0f} MHz (median SM clock sampled "
                                              "during the timed region)",
            "achieved": None, "frac": None, "traffic": None,
            "rays_per_launch": rays_per_launch, "launch_ms": k_ms / max(k_launch, 1),
            "kernel_ms": {"closest_hit": ext_ms / steps, "any_hit": sh_ms / steps,
                          "shade": sum(s.shade_kernel_ms for s in stats) / steps},
            "rays_per_s": (ext_rays + sh_rays) / (ms / 1e3),
            "hbm_model": {"bytes_per_ray": bpr, "achieved": hbm_achieved, "peak": peak, "unit": "GB/s",
                          "frac": hbm_achieved / peak, "peak_source": peak_kind}}
    if prof:
        inst = prof["warp_inst_per_ray"] * k_rays / (k_ms / 1e3) / 1e9 if k_ms > 0 else 0.0
        roof.update({"achieved": inst, "frac": inst / issue_peak,
                     "traffic": prof["dram_bytes_per_ray"] * rays_per_launch,
                     "warp_inst_per_ray": prof["warp_inst_per_ray"], "active_lanes": prof["active_lanes"],
                     "l2_bytes_per_ray": prof["l2_bytes_per_ray"], "dram_bytes_per_ray": prof["dram_bytes_per_ray"],
                     "profile": prof["source"]})
    return roof


def accuracy_at_fixture_spp(w, scene, ctx):
    """The bake of the FP64 fixture's crop at the fixture's own spp (4096):
    relative RMSE against the fixture, the noise floor two independent
    4096-spp estimates have (sqrt 2 x the fixture's own error), the
    systematic part as the per-channel relative bias of the summed
    difference (with its standard error), and the rate of that bake."""
    import numpy as np
    import torch

    from sh_baker_b200 import _capi as A
    from sh_baker_b200 import api
    path = ROOT / "tests" / "golden" / f"fp64_{w['kind']}.npz"
    if not path.exists():
        return None
    ref = np.load(path)
    W, H, ss, size, x0, y0 = (int(ref[k]) for k in ("width", "height", "ss", "size", "x0", "y0"))
    if (W, H, ss, int(ref["bounces"])) != (w["width"], w["height"], w["ss"], w["bounces"]):
        return None
    spp = int(ref["spp"])
    pts = api.RasterizeScene(scene, api.RasterConfig(W, H, ss), ctx=ctx).reshape(H * ss, W * ss)
    crop = np.ascontiguousarray(pts[y0 * ss:(y0 + size) * ss, x0 * ss:(x0 + size) * ss]).reshape(-1)
    ds = api.DeviceScene(ctx, scene)
    g = api.GBuffer.from_points(ctx, crop, size * ss, size * ss)
    rc = api.RasterConfig(size, size, ss)
    n = (size * ss) ** 2
    sh = torch.empty(n * 27, dtype=torch.float32, device="cuda")
    env = torch.empty(n, dtype=torch.float32, device="cuda")
    bake = api.BatchBake(ds, g, rc, api.BakeConfig(samples=spp, bounces=w["bounces"], seed=4242))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = api.bake_plain_device(bake, sh, env)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    got = sh.cpu().numpy().reshape(size, ss, size, ss, 27).mean(axis=(1, 3))
    valid, r = ref["valid"], ref["sh"].astype(np.float64)
    d2 = float(np.sum((got - r)[valid] ** 2))
    o2 = float(np.sum(r[valid] ** 2))
    se = ref["se"].astype(np.float64)
    se2 = float(np.sum(se[valid] ** 2))
    # systematic part: per SH channel, the summed difference over the crop
    # relative to the summed magnitude (the noise averages down)
    mag = np.abs(r[valid]).sum(axis=0)
    bias = (got - r)[valid].sum(axis=0) / mag
    bias_se = np.sqrt(2.0 * (se[valid] ** 2).sum(axis=0)) / mag
    g.close()
    ds.close()
    return {"spp": spp, "rel_rmse_vs_fp64": (d2 / o2) ** 0.5, "noise_floor": (2 * se2 / o2) ** 0.5,
            "channel_bias": {"l0_rgb": [float(v) for v in bias[:3]], "max_abs": float(np.abs(bias).max()),
                             "max_abs_over_se": float(np.max(np.abs(bias) / bias_se)),
                             "se_of_max": float(bias_se[int(np.argmax(np.abs(bias)))])},
            "texel_samples_per_s": st.texel_samples / dt, "seconds": dt}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="atrium", choices=sorted(WORKLOADS) + ["batched", "adjoint", "exr"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-step-seconds", type=float, default=5.0)
    ap.add_argument("--e2e-steps", type=int, default=3, help="timed end-to-end steps (after one warm-up)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-sub", action="store_true", help="skip the batched, adjoint and EXR sub-results")
    args = ap.parse_args()
    if args.workload in ("batched", "adjoint", "exr"):
        if args.impl == "ours" and int(os.environ.get("RANK", "0")) == 0:
            {"batched": run_batched, "adjoint": run_adjoint, "exr": run_exr}[args.workload](args)
        return
    w = WORKLOADS[args.workload]

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args, w)
        return

    import numpy as np
    import torch

    from sh_baker_b200 import _capi as A
    from sh_baker_b200 import api
    from sh_baker_b200 import build as B
    from sh_baker_b200.replicas import job_rate

    B.build()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    scene = make_scene(w)
    ctx = api.Context(device=local, profiling=True)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ds = api.DeviceScene(ctx, scene)
    rc = api.RasterConfig(w["width"], w["height"], w["ss"])
    g = api.rasterize_to_device(ds, rc)
    n = g.width * g.height
    sh = torch.empty(n * 27, dtype=torch.float32, device="cuda")
    env = torch.empty(n, dtype=torch.float32, device="cuda")
    out = A.BakeOutput(sh.data_ptr(), env.data_ptr(), 1, 0)
    lib = ctx.lib
    import ctypes as C

    def step(i):
        A.check(lib.shb_scene_rebuild_bvh(ds.h))
        cfg = api.BakeConfig(samples=w["spp"], bounces=w["bounces"], seed=1000 + 7919 * rank + i).c()
        st = A.BakeStats()
        A.check(lib.shb_bake(ds.h, g.h, C.byref(rc.c()), C.byref(cfg), C.byref(out), C.byref(st)))
        return st

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = ctx.kernel_launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    stats = [step(args.warmup + i) for i in range(args.steps)]
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = ctx.kernel_launches() - launches0
    clk = clocks.stop()
    ts = sum(s.texel_samples for s in stats)
    ms, ts, value = job_rate(ms, ts, dist)
    roof = roofline_of(stats, args.steps, scene, w, ms, clk)
    ext_rays = sum(s.extend_rays for s in stats)
    sh_rays = sum(s.shadow_rays for s in stats)

    # end to end through the public API from pinned host memory
    e2e = None
    if not args.no_e2e:
        from sh_baker_b200.scene import pack_scene
        H, W = w["height"], w["width"]
        pin = lambda shape, dt: torch.empty(shape, dtype=dt, pin_memory=True).numpy()  # noqa: E731
        o_sh, o_env, o_mask = pin((H, W, 9, 3), torch.float32), pin((H, W), torch.float32), pin((H, W), torch.uint8)
        pscene = pinned_scene(scene, pin)
        desc, keep = pack_scene(pscene)
        h2d = sum(a.nbytes for a in keep if isinstance(a, np.ndarray))
        e_times, e_ts = [], 0
        e_steps = max(1, min(args.steps, args.e2e_steps))
        for i in range(1 + e_steps):
            ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            ea.record(stream)
            h = C.c_void_p()
            A.check(lib.shb_scene_upload(ctx.h, C.byref(desc), C.byref(h)))
            cfg = A.PipelineConfig(W, H, w["ss"], w["spp"], w["bounces"], w["dilation"], 1, 5000 + i)
            st = A.BakeStats()
            A.check(lib.shb_bake_pipeline(h, C.byref(cfg), o_sh.ctypes.data, o_env.ctypes.data, o_mask.ctypes.data,
                                          C.byref(st)))
            lib.shb_scene_destroy(h)
            eb.record(stream)
            torch.cuda.synchronize()
            if i >= 1:
                e_times.append(ea.elapsed_time(eb))
                e_ts += st.texel_samples
        e_ms, e_ts, e_val = job_rate(sum(e_times), e_ts, dist)
        e2e = {"value": e_val, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(o_sh.nbytes + o_env.nbytes + o_mask.nbytes),
               "ms_per_step": e_ms / e_steps, "steps": e_steps, "warmup": 1,
               "region": "scene upload from pinned host memory, raster, BVH build, bake, masks, downsample, "
                         "dilation, read-back of SH, env visibility and mask (shb_bake_pipeline)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        pts = g.download()
        cpu = cpu_baseline(scene, pts, w, args.cpu_seconds, os.cpu_count() or 1)
        del pts

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config_of(w, scene),
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches), "clocks": clk,
                "bvh": ds.bvh_info(), "valid_texels": int(stats[0].valid_texels),
                "traversal_per_step": {
                    "closest_hit": {"rays": ext_rays // args.steps,
                                    "launches": sum(s.extend_launches for s in stats) // args.steps},
                    "any_hit": {"rays": sh_rays // args.steps,
                                "launches": sum(s.shadow_launches for s in stats) // args.steps}},
                "rays_per_texel_sample": (ext_rays + sh_rays) / max(ts, 1)}
    del sh, env
    g.close()
    ds.close()
    if rank == 0 and world == 1:
        acc = accuracy(w, scene, ctx)
        if acc is not None:
            acc["at_fixture_spp"] = accuracy_at_fixture_spp(w, scene, ctx)
        line["accuracy"] = acc
        if not args.no_sub:
            # the metric's other two parts, shortened: batched vs sequential and adjoint vs forward
            line["batched"] = batched_result(steps=2, warmup=1)
            line["adjoint"] = adjoint_result(steps=2, warmup=1)
            line["exr"] = exr_result(steps=3, warmup=1, reference=not args.no_cpu_baseline, ref_runs=1)
    elif rank == 0:
        line["accuracy"] = None
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
