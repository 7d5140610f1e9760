"""SaveSHLightMap (shb_save_sh_lightmap): OpenEXR output in the reference's
three layouts.

CPU: the checker (oracle/exr_read.py) is pinned against the reference's own
EXR library (tinyexr, built from the reference tree into oracle/_ref) on
files the reference's writer path produces; the committed fixture
(tests/golden/exr_reference.npz, made by tests/golden/make_exr_golden.py)
is what that path stores.
GPU: the CUDA writer's files carry the same attributes, channel names and
order, and bit-identical half samples as the fixture.
"""
import ctypes as C
import tempfile
from pathlib import Path

import numpy as np
import pytest

from oracle import exr_read

ROOT = Path(__file__).resolve().parents[1]
GOLD = ROOT / "tests" / "golden" / "exr_reference.npz"
FILES = {0: ["lightmap"],
         1: [f"lightmap_{n}" for n in ("L0", "L1m1", "L10", "L11", "L2m2", "L2m1", "L20", "L21", "L22")],
         2: [f"lightmap_packed_{k}" for k in range(3)]}


def gold():
    return np.load(GOLD)


def check_file(path, g, key):
    ex = exr_read.read(path)
    assert [n for n, _ in ex.channels] == list(g[key + "_names"])
    assert all(t == 1 for _, t in ex.channels)  # HALF
    assert [n for n, _, _ in ex.attributes] == list(g[key + "_attr_names"])
    assert [t for _, t, _ in ex.attributes] == list(g[key + "_attr_types"])
    assert [v.hex() for _, _, v in ex.attributes] == list(g[key + "_attr_values"])
    halves = np.stack([ex.raw[n] for n, _ in ex.channels])
    np.testing.assert_array_equal(halves, g[key + "_halves"])


def ref_lib():
    try:
        from oracle import build as ob
        p = ob.build_ref()
    except Exception:
        p = None
    if p is None or not Path(p).exists():
        pytest.skip("reference EXR library not available (needs the reference tree)")
    import sys
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    import make_exr_golden as mk
    return mk, mk.load_ref()


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_reader_matches_reference_library(mode):
    """Files written by the reference's writer path decode identically in
    the checker and in tinyexr, and equal the committed fixture."""
    mk, lib = ref_lib()
    sh, env = mk.crafted_texture()
    g = gold()
    np.testing.assert_array_equal(g["sh"].view(np.uint32), sh.view(np.uint32))
    with tempfile.TemporaryDirectory() as d:
        for f in mk.reference_files(lib, sh, env, mode, d):
            names, halves = mk.tinyexr_read(lib, f)
            ex = exr_read.read(f)
            assert [n for n, _ in ex.channels] == names
            np.testing.assert_array_equal(np.stack([ex.raw[n] for n in names]), halves)
            check_file(f, g, f"m{mode}_{f.stem}")


def test_fixture_half_rule():
    """The stored halves follow round-half-up in magnitude on the mantissa
    (1 + 2^-11 -> 1 + 2^-10, where round-to-nearest-even gives 1.0), flush
    float denormals, saturate to inf from 65520 and keep NaN a NaN."""
    g = gold()
    h = g["m0_lightmap_halves"]  # (28, H, W), channel 0 = L0.R = sh[:, 0]
    flat = h.transpose(1, 2, 0).reshape(-1, 28)[:, :27].reshape(-1)
    # positions of the crafted values (tests/golden/make_exr_golden.py)
    expect = {0: 0x0000, 1: 0x8000, 2: 0x3C01, 3: 0x3C02, 4: 0xBC01, 5: 0x7BFF, 6: 0x7BFF, 7: 0x7C00, 8: 0xFC00,
              9: 0x7C00, 10: 0x0001, 11: 0x0001, 15: 0x0000, 16: 0x8000, 17: 0x7C00, 18: 0xFC00}
    for i, hv in expect.items():
        assert flat[i] == hv, (i, hex(flat[i]), hex(hv))
    assert flat[19] & 0x7C00 == 0x7C00 and flat[19] & 0x3FF  # NaN stays NaN


def save(gpu_ctx, sh, env, path, mode, device=False):
    from sh_baker_b200 import _capi as A
    H, W = 21, 37
    if device:
        import torch
        tsh = torch.from_numpy(sh).cuda()
        tenv = torch.from_numpy(env).cuda()
        torch.cuda.synchronize()
        A.check(gpu_ctx.lib.shb_save_sh_lightmap(gpu_ctx.h, tsh.data_ptr(), tenv.data_ptr(), W, H, 1,
                                                 str(path).encode(), mode))
    else:
        A.check(gpu_ctx.lib.shb_save_sh_lightmap(gpu_ctx.h, sh.ctypes.data, env.ctypes.data, W, H, 0,
                                                 str(path).encode(), mode))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("device", [False, True])
def test_cuda_writer_matches_reference_files(gpu_ctx, mode, device):
    g = gold()
    sh = np.ascontiguousarray(g["sh"])
    env = np.ascontiguousarray(g["env"])
    with tempfile.TemporaryDirectory() as d:
        save(gpu_ctx, sh, env, Path(d) / "lightmap.exr", mode, device)
        written = sorted(p.name for p in Path(d).iterdir())
        assert written == sorted(f + ".exr" for f in FILES[mode])
        for stem in FILES[mode]:
            check_file(Path(d) / (stem + ".exr"), g, f"m{mode}_{stem}")


@pytest.mark.gpu
def test_save_rejects_bad_arguments(gpu_ctx, tmp_path):
    """Empty dimensions, an unknown mode and an unwritable path are errors
    (the reference logs them and returns false)."""
    sh = np.zeros(27, np.float32)
    lib, h = gpu_ctx.lib, gpu_ctx.h
    assert lib.shb_save_sh_lightmap(h, sh.ctypes.data, None, 0, 1, 0, str(tmp_path / "a.exr").encode(), 0) == 1
    assert lib.shb_save_sh_lightmap(h, sh.ctypes.data, None, 1, 1, 0, str(tmp_path / "b.exr").encode(), 7) == 1
    assert lib.shb_save_sh_lightmap(h, sh.ctypes.data, None, 1, 1, 0, str(tmp_path / "no" / "c.exr").encode(), 0) != 0


def _exr(window, rows, comp=0, offsets=None):
    """A minimal single-part scanline OpenEXR file with one FLOAT channel R:
    `rows` is a list of (y, payload bytes) chunks, `window` the dataWindow
    (x0, y0, x1, y1); `offsets` overrides the offset table."""
    import struct

    def attr(name, typ, data):
        return name.encode() + b"\0" + typ.encode() + b"\0" + struct.pack("<i", len(data)) + data

    chlist = b"R\0" + struct.pack("<iB3xii", 2, 0, 1, 1) + b"\0"
    head = b"\x76\x2f\x31\x01\x02\x00\x00\x00" + attr("channels", "chlist", chlist) + \
        attr("compression", "compression", bytes([comp])) + attr("dataWindow", "box2i", struct.pack("<4i", *window)) + b"\0"
    pos = len(head) + 8 * len(rows)
    table, body = [], b""
    for y, payload in rows:
        table.append(pos + len(body))
        body += struct.pack("<ii", y, len(payload)) + payload
    table = offsets if offsets is not None else table
    return head + b"".join(struct.pack("<Q", t) for t in table) + body


def _load(path):
    from sh_baker_b200 import _capi as A
    lib = A.load()
    names = (C.c_char_p * 1)(b"R")
    w, h = C.c_int32(), C.c_int32()
    st = lib.shb_exr_load_channels(str(path).encode(), C.cast(names, C.c_void_p), 1, C.byref(w), C.byref(h), None)
    if st != 0:
        return st, lib.shb_last_error().decode(), None
    out = np.zeros(w.value * h.value, np.float32)
    st = lib.shb_exr_load_channels(str(path).encode(), C.cast(names, C.c_void_p), 1, C.byref(w), C.byref(h),
                                   out.ctypes.data)
    return st, lib.shb_last_error().decode(), out.reshape(h.value, w.value)


def test_reader_rejects_damaged_files(tmp_path):
    """shb_exr_load_channels (host code, no GPU) on crafted files: a good
    one reads back; a dataWindow whose width overflows int32, an offset
    table entry near 2^64 (offset + 8 wraps) and a ZIP chunk too small to
    inflate to its lines are SHB_ERR_INVALID_ARG, refused before any read
    or allocation they would drive."""
    vals = np.arange(6, dtype=np.float32).reshape(2, 3) + 0.5
    p = tmp_path / "good.exr"
    p.write_bytes(_exr((0, 0, 2, 1), [(0, vals[0].tobytes()), (1, vals[1].tobytes())]))
    st, msg, got = _load(p)
    assert st == 0, msg
    np.testing.assert_array_equal(got, vals)
    cases = {
        "wide": (_exr((-2 ** 31, 0, 39, 0), [(0, b"")]), "larger than 2^31 - 1"),
        "offset": (_exr((0, 0, 2, 1), [(0, vals[0].tobytes()), (1, vals[1].tobytes())],
                        offsets=[2 ** 64 - 7, 2 ** 64 - 7]), "chunk offset"),
        "inflate": (_exr((0, 0, 99999, 15), [(0, b"\x78\x9c" + bytes(8))], comp=3), "chunk size"),
    }
    for name, (data, what) in cases.items():
        q = tmp_path / f"{name}.exr"
        q.write_bytes(data)
        st, msg, _ = _load(q)
        assert st == 1 and what in msg, (name, st, msg)
