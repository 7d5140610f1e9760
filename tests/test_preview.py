"""SH previews and the EXR -> PNG tool (src/sh_cvt_main.cpp, the viewer's
EvalSHBasis in glsl/viz.frag:42-99 as arithmetic): shb_sh_preview,
shb_exr_load_channels, shb_write_png and the sh_cvt command line."""
import ctypes as C
import subprocess
import zlib
from pathlib import Path

import numpy as np
import pytest

from oracle import exr_read
from sh_baker_b200 import _capi as A

f32 = np.float32


def read_png(path):
    """Decoder for the filter-0 PNGs shb_write_png writes."""
    b = Path(path).read_bytes()
    assert b[:8] == b"\x89PNG\r\n\x1a\n"
    i, idat, hdr = 8, b"", None
    while i < len(b):
        n = int.from_bytes(b[i:i + 4], "big")
        t, d = b[i + 4:i + 8], b[i + 8:i + 8 + n]
        assert zlib.crc32(t + d) == int.from_bytes(b[i + 8 + n:i + 12 + n], "big")
        if t == b"IHDR":
            hdr = d
        elif t == b"IDAT":
            idat += d
        i += 12 + n
    w, h = int.from_bytes(hdr[:4], "big"), int.from_bytes(hdr[4:8], "big")
    ch = {0: 1, 4: 2, 2: 3, 6: 4}[hdr[9]]
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, w * ch + 1)
    assert np.all(raw[:, 0] == 0)
    return raw[:, 1:].reshape(h, w, ch)


def test_write_png_round_trip(tmp_path):
    lib = A.load()
    rng = np.random.default_rng(1)
    for ch in (1, 2, 3, 4):
        px = rng.integers(0, 256, (7, 5, ch), dtype=np.uint8)
        p = tmp_path / f"t{ch}.png"
        A.check(lib.shb_write_png(str(p).encode(), 5, 7, ch, px.ctypes.data))
        np.testing.assert_array_equal(read_png(p), px)
        # and an independent decoder (Pillow's) reads the same pixels
        from PIL import Image
        im = Image.open(p)
        assert im.mode == {1: "L", 2: "LA", 3: "RGB", 4: "RGBA"}[ch]
        np.testing.assert_array_equal(np.asarray(im).reshape(7, 5, ch), px)
    assert lib.shb_write_png(str(tmp_path / "bad.png").encode(), 0, 7, 3, px.ctypes.data) == 1


def load_channels(path, names):
    lib = A.load()
    arr = (C.c_char_p * len(names))(*[n.encode() for n in names])
    w, h = C.c_int32(), C.c_int32()
    st = lib.shb_exr_load_channels(str(path).encode(), C.cast(arr, C.c_void_p), len(names), C.byref(w), C.byref(h),
                                   None)
    if st != 0:
        return None
    out = np.zeros((len(names), h.value, w.value), np.float32)
    A.check(lib.shb_exr_load_channels(str(path).encode(), C.cast(arr, C.c_void_p), len(names), C.byref(w),
                                      C.byref(h), out.ctypes.data))
    return out


def test_exr_reader_every_half_against_reference_library(tmp_path):
    """Every half pattern written by the reference's tinyexr decodes to the
    same float bits (NaN payloads too) through shb_exr_load_channels."""
    try:
        from oracle import build as ob
        if ob.build_ref() is None:
            raise RuntimeError
        import sys
        sys.path.insert(0, str(Path(__file__).parent / "golden"))
        import make_exr_golden as mk
        lib = mk.load_ref()
    except Exception:
        pytest.skip("reference EXR library not available (needs the reference tree)")
    W, H = 256, 256
    halves = np.arange(65536, dtype=np.uint32).astype(np.uint16)
    vals = halves.view(np.float16).astype(np.float32)
    sh = np.zeros((W * H, 27), np.float32)
    sh[:, 0] = vals
    sh[:, 4] = -vals[::-1]
    env = np.linspace(0, 1, W * H, dtype=np.float32)
    p = tmp_path / "all.exr"
    assert lib.ref_exr_save(sh.ctypes.data, env.ctypes.data, W, H, str(p).encode(), 0) == 0
    ex = exr_read.read(p)
    got = load_channels(p, ["L0.R", "L1m1.G", "EnvVisibility"])
    for k, name in enumerate(["L0.R", "L1m1.G", "EnvVisibility"]):
        want = ex.raw[name].view(np.float16).astype(np.float32)
        np.testing.assert_array_equal(got[k].view(np.uint32), want.view(np.uint32))
    assert load_channels(p, ["L0.R", "nope"]) is None
    assert "nope" in A.load().shb_last_error().decode()


def preview_ref(sh, normals, d, mode, reinhard):
    """numpy float32 restatement of k_sh_preview (same operation order)."""
    sh = sh.reshape(-1, 27).astype(f32)
    n = len(sh)
    if mode == A.PREVIEW_L0:
        rgb = sh[:, :3].copy()
    else:
        x, y, z = ((normals[:, 0], normals[:, 1], normals[:, 2]) if normals is not None else
                   (np.full(n, d[0], f32), np.full(n, d[1], f32), np.full(n, d[2], f32)))
        b = [np.full(n, f32(0.282095)), f32(0.488603) * y, f32(0.488603) * z, f32(0.488603) * x,
             f32(1.092548) * x * y, f32(1.092548) * y * z, f32(0.315392) * (f32(3.0) * z * z - f32(1.0)),
             f32(1.092548) * x * z, f32(0.546274) * (x * x - y * y)]
        coef = sh.copy()
        if mode == A.PREVIEW_SH_PACKED:
            l0 = coef[:, 0] * f32(0.2126) + coef[:, 1] * f32(0.7152) + coef[:, 2] * f32(0.0722)
            chroma = np.ones((n, 3), f32)
            big = l0 > f32(1e-6)
            chroma[big] = coef[big, :3] / l0[big, None]
            for k in range(1, 9):
                q = sh[:, 3 * k:3 * k + 3]
                lum = q[:, 0] * f32(0.2126) + (q[:, 1] * f32(0.7152) + q[:, 2] * f32(0.0722))
                coef[:, 3 * k:3 * k + 3] = lum[:, None] * chroma
        rgb = np.zeros((n, 3), f32)
        for c in range(3):
            s = coef[:, c] * b[0]
            for k in range(1, 9):
                s = s + coef[:, 3 * k + c] * b[k]
            rgb[:, c] = np.maximum(s, f32(0))
    if reinhard:
        rgb = rgb / (f32(1.0) + rgb)
    rgb = np.clip(rgb, f32(0), f32(1))
    return (rgb * f32(255.0) + f32(0.5)).astype(np.uint8)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("reinhard", [0, 1])
@pytest.mark.parametrize("device", [False, True])
def test_preview_matches_restatement(gpu_ctx, mode, reinhard, device):
    import torch
    W, H = 19, 11
    rng = np.random.default_rng(mode * 4 + reinhard)
    sh = (rng.standard_normal((W * H, 27)) * 0.7).astype(np.float32)
    sh[:, :3] = np.abs(sh[:, :3]) * 2
    sh[:5, :3] = 0  # luminance below 1e-6: chroma 1
    nrm = rng.standard_normal((W * H, 3)).astype(np.float32)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    d = np.array([0.0, 0.6, 0.8], np.float32)
    for normals in (None, nrm):
        out = np.zeros((W * H, 3), np.uint8)
        if device:
            tsh = torch.from_numpy(sh).cuda()
            tn = torch.from_numpy(nrm).cuda() if normals is not None else None
            torch.cuda.synchronize()
            A.check(gpu_ctx.lib.shb_sh_preview(gpu_ctx.h, tsh.data_ptr(), W, H, tn.data_ptr() if tn is not None else
                                               None, d.ctypes.data, mode, reinhard, 1, out.ctypes.data))
        else:
            A.check(gpu_ctx.lib.shb_sh_preview(gpu_ctx.h, sh.ctypes.data, W, H,
                                               normals.ctypes.data if normals is not None else None, d.ctypes.data,
                                               mode, reinhard, 0, out.ctypes.data))
        np.testing.assert_array_equal(out, preview_ref(sh, normals, d, mode, reinhard))


@pytest.mark.gpu
def test_sh_cvt_tool(gpu_ctx, tmp_path):
    """sh_cvt turns every .exr with L0.R/G/B (else R/G/B) channels of the
    folder into <stem>_L0.png: combined, split and packed files alike."""
    from sh_baker_b200 import build as B
    B.build()
    W, H = 23, 17
    rng = np.random.default_rng(5)
    sh = (np.abs(rng.standard_normal((H, W, 9, 3))) * 1.5).astype(np.float32)
    env = rng.uniform(0, 1, (H, W)).astype(np.float32)
    for mode in (A.SAVE_COMBINED, A.SAVE_SPLIT_CHANNELS, A.SAVE_LUMINANCE_PACKED):
        A.check(gpu_ctx.lib.shb_save_sh_lightmap(gpu_ctx.h, sh.ctypes.data, env.ctypes.data, W, H, 0,
                                                 str(tmp_path / "lightmap.exr").encode(), mode))
    (tmp_path / "notes.txt").write_text("not an image")
    r = subprocess.run([str(B.CVT), "--input", str(tmp_path), "--reinhard"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    exrs = sorted(p for p in tmp_path.iterdir() if p.suffix == ".exr")
    assert len(exrs) == 1 + 9 + 3
    for p in exrs:
        ex = exr_read.read(p)
        names = [n for n, _ in ex.channels]
        use = ["L0.R", "L0.G", "L0.B"] if "L0.R" in names else ["R", "G", "B"]
        rgb = np.stack([ex.half(n) for n in use], axis=-1).reshape(-1, 3)
        v = rgb / (f32(1.0) + rgb)
        want = (np.clip(v, f32(0), f32(1)) * f32(255.0) + f32(0.5)).astype(np.uint8).reshape(H, W, 3)
        np.testing.assert_array_equal(read_png(tmp_path / (p.stem + "_L0.png")), want)
    assert run_fails([str(B.CVT)]) and run_fails([str(B.CVT), "--input", str(tmp_path / "missing")])


def run_fails(cmd):
    return subprocess.run(cmd, capture_output=True, text=True, timeout=60).returncode != 0
