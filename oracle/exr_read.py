"""Minimal OpenEXR reader for the files of SaveSHLightMap (scanline,
single part, NO or ZIP compression, HALF/FLOAT channels).

TEST INFRASTRUCTURE ONLY: the checker of the CUDA EXR writer, pinned against
the reference's own EXR library (tinyexr, oracle/_ref) in tests.  Follows the
OpenEXR file layout: magic + version, attributes up to a null byte, a chunk
offset table, then per chunk (y, size, data).  ZIP chunks are zlib-inflated,
the delta predictor is undone and the two byte halves re-interleaved.
"""
from __future__ import annotations

import struct
import zlib
from dataclasses import dataclass, field
from typing import Dict, List, Tuple

import numpy as np

PIXEL_BYTES = {0: 4, 1: 2, 2: 4}  # UINT, HALF, FLOAT
LINES_PER_CHUNK = {0: 1, 2: 1, 3: 16}  # NO, ZIPS, ZIP


@dataclass
class ExrFile:
    attributes: List[Tuple[str, str, bytes]]
    channels: List[Tuple[str, int]]  # (name, pixel type) in file order
    width: int
    height: int
    compression: int
    raw: Dict[str, np.ndarray] = field(default_factory=dict)  # name -> (H, W) uint16 / uint32

    def half(self, name: str) -> np.ndarray:
        return self.raw[name].view(np.float16).astype(np.float32)


def _cstr(b: bytes, i: int) -> Tuple[str, int]:
    j = b.index(b"\0", i)
    return b[i:j].decode(), j + 1


def unpredict(data: bytes) -> bytes:
    """Inverse of the ZIP pre-pass: running sum of (byte - 128), then the
    first half of the buffer holds the even bytes and the second the odd."""
    t = np.frombuffer(data, np.uint8).astype(np.int64)
    if t.size == 0:
        return b""
    d = t.copy()
    d[1:] -= 128
    t = (np.cumsum(d) & 0xFF).astype(np.uint8)
    n = t.size
    half = (n + 1) // 2
    out = np.empty(n, np.uint8)
    out[0::2] = t[:half]
    out[1::2] = t[half:]
    return out.tobytes()


def read(path) -> ExrFile:
    b = open(path, "rb").read()
    if b[:4] != b"\x76\x2f\x31\x01":
        raise ValueError("not an OpenEXR file")
    if b[4] != 2 or b[5] & 0x1E:
        raise ValueError("only single-part scanline files")
    i = 8
    attrs = []
    while b[i] != 0:
        name, i = _cstr(b, i)
        typ, i = _cstr(b, i)
        (size,) = struct.unpack_from("<i", b, i)
        i += 4
        attrs.append((name, typ, b[i:i + size]))
        i += size
    i += 1
    a = {n: v for n, _, v in attrs}
    chans = []
    cl, j = a["channels"], 0
    while cl[j] != 0:
        name, j = _cstr(cl, j)
        ptype, _plin, _xs, _ys = struct.unpack_from("<iB3xii", cl, j)
        j += 16
        chans.append((name, ptype))
    x0, y0, x1, y1 = struct.unpack("<4i", a["dataWindow"])
    W, H = x1 - x0 + 1, y1 - y0 + 1
    comp = a["compression"][0]
    lpc = LINES_PER_CHUNK[comp]
    nchunks = (H + lpc - 1) // lpc
    offsets = struct.unpack_from(f"<{nchunks}Q", b, i)
    line_bytes = sum(W * PIXEL_BYTES[t] for _, t in chans)
    planes = {n: np.zeros((H, W), np.uint16 if t == 1 else np.uint32) for n, t in chans}
    for k, off in enumerate(offsets):
        y, size = struct.unpack_from("<ii", b, off)
        data = b[off + 8: off + 8 + size]
        lines = min(lpc, y1 + 1 - y)
        n = line_bytes * lines
        if comp != 0 and size < n:
            data = unpredict(zlib.decompress(data))
        if len(data) != n:
            raise ValueError(f"chunk {k}: {len(data)} bytes, expected {n}")
        p = 0
        for ly in range(lines):
            for name, t in chans:
                nb = W * PIXEL_BYTES[t]
                dt = "<u2" if t == 1 else "<u4"
                planes[name][y - y0 + ly] = np.frombuffer(data, dt, W, p)
                p += nb
    return ExrFile(attrs, chans, W, H, comp, planes)
