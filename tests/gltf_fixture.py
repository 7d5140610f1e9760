"""Writes small glTF 2.0 files for the loader tests: meshes from numpy
arrays, materials, KHR_lights_punctual lights, node transforms, buffers as
a data URI, a .bin file beside the .gltf or a .glb container, and PNG
textures (own minimal encoder)."""
from __future__ import annotations

import base64
import json
import struct
import zlib
from pathlib import Path

import numpy as np


def png_bytes(pixels: np.ndarray, color_type: int = None, palette=None, trns=None) -> bytes:
    """8-bit PNG of (H, W, C) uint8 pixels (C = 1..4), or of (H, W) palette
    indices with `palette` (N, 3) and optional `trns` alphas.  Rows use
    filter types 0..4 in turn so that the decoder meets every filter."""
    if palette is not None:
        idx = np.asarray(pixels, np.uint8)
        H, W = idx.shape
        ct, data = 3, idx.reshape(H, W, 1)
    else:
        data = np.asarray(pixels, np.uint8)
        H, W, C = data.shape
        ct = {1: 0, 2: 4, 3: 2, 4: 6}[C] if color_type is None else color_type
    bpp = data.shape[2]
    raw = bytearray()
    prev = np.zeros(W * bpp, np.int32)
    for y in range(H):
        row = data[y].reshape(-1).astype(np.int32)
        ft = y % 5
        left = np.concatenate([np.zeros(bpp, np.int32), row[:-bpp]])
        upleft = np.concatenate([np.zeros(bpp, np.int32), prev[:-bpp]])
        if ft == 0:
            f = row
        elif ft == 1:
            f = row - left
        elif ft == 2:
            f = row - prev
        elif ft == 3:
            f = row - (left + prev) // 2
        else:
            p = left + prev - upleft
            pa, pb, pc = np.abs(p - left), np.abs(p - prev), np.abs(p - upleft)
            pred = np.where((pa <= pb) & (pa <= pc), left, np.where(pb <= pc, prev, upleft))
            f = row - pred
        raw.append(ft)
        raw += (f & 0xFF).astype(np.uint8).tobytes()
        prev = row

    def chunk(t, d):
        return struct.pack(">I", len(d)) + t + d + struct.pack(">I", zlib.crc32(t + d) & 0xFFFFFFFF)

    out = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", W, H, 8, ct, 0, 0, 0))
    if palette is not None:
        out += chunk(b"PLTE", np.asarray(palette, np.uint8).tobytes())
        if trns is not None:
            out += chunk(b"tRNS", np.asarray(trns, np.uint8).tobytes())
    return out + chunk(b"IDAT", zlib.compress(bytes(raw))) + chunk(b"IEND", b"")


class GltfBuilder:
    def __init__(self):
        self.j = {"asset": {"version": "2.0"}, "scenes": [{"nodes": []}], "scene": 0, "nodes": [], "meshes": [],
                  "accessors": [], "bufferViews": [], "buffers": []}
        self.bin = bytearray()

    def _view(self, data: bytes, stride: int = 0) -> int:
        while len(self.bin) % 4:
            self.bin.append(0)
        v = {"buffer": 0, "byteOffset": len(self.bin), "byteLength": len(data)}
        if stride:
            v["byteStride"] = stride
        self.bin += data
        self.j["bufferViews"].append(v)
        return len(self.j["bufferViews"]) - 1

    def accessor(self, a: np.ndarray, ctype: int = 5126, interleave_pad: int = 0) -> int:
        a = np.asarray(a)
        comps = 1 if a.ndim == 1 else a.shape[1]
        dt = {5126: "<f4", 5125: "<u4", 5123: "<u2", 5121: "u1"}[ctype]
        arr = np.ascontiguousarray(a.astype(dt)).reshape(len(a), comps)
        stride = 0
        if interleave_pad:  # exercise byteStride: pad every element
            elem = arr.itemsize * comps
            padded = np.zeros((len(a), elem + interleave_pad), np.uint8)
            padded[:, :elem] = arr.view(np.uint8).reshape(len(a), elem)
            data, stride = padded.tobytes(), elem + interleave_pad
        else:
            data = arr.tobytes()
        v = self._view(data, stride)
        t = {1: "SCALAR", 2: "VEC2", 3: "VEC3", 4: "VEC4"}[comps]
        self.j["accessors"].append({"bufferView": v, "componentType": ctype, "count": len(a), "type": t})
        return len(self.j["accessors"]) - 1

    def mesh(self, prims) -> int:
        self.j["meshes"].append({"primitives": prims})
        return len(self.j["meshes"]) - 1

    def primitive(self, pos, nrm=None, uv0=None, uv1=None, tan=None, idx=None, material=0, idx_type=5125,
                  pad=0) -> dict:
        attrs = {"POSITION": self.accessor(pos, interleave_pad=pad)}
        if nrm is not None:
            attrs["NORMAL"] = self.accessor(nrm, interleave_pad=pad)
        if uv0 is not None:
            attrs["TEXCOORD_0"] = self.accessor(uv0)
        if uv1 is not None:
            attrs["TEXCOORD_1"] = self.accessor(uv1)
        if tan is not None:
            attrs["TANGENT"] = self.accessor(tan)
        p = {"attributes": attrs}
        if material is not None:
            p["material"] = material
        if idx is not None:
            p["indices"] = self.accessor(np.asarray(idx).reshape(-1), idx_type)
        return p

    def node(self, root=True, **kw) -> int:
        self.j["nodes"].append(kw)
        i = len(self.j["nodes"]) - 1
        if root:
            self.j["scenes"][0]["nodes"].append(i)
        return i

    def material(self, factor=None, emissive_strength=None, texture_png: bytes = None, name="") -> int:
        m = {"name": name, "pbrMetallicRoughness": {}}
        if factor is not None:
            m["pbrMetallicRoughness"]["baseColorFactor"] = list(map(float, factor))
        if texture_png is not None:
            self.j.setdefault("images", []).append(
                {"uri": "data:image/png;base64," + base64.b64encode(texture_png).decode()})
            self.j.setdefault("textures", []).append({"source": len(self.j["images"]) - 1})
            m["pbrMetallicRoughness"]["baseColorTexture"] = {"index": len(self.j["textures"]) - 1}
        if emissive_strength is not None:
            m["extensions"] = {"KHR_materials_emissive_strength": {"emissiveStrength": float(emissive_strength)}}
        self.j.setdefault("materials", []).append(m)
        return len(self.j["materials"]) - 1

    def light(self, **kw) -> int:
        ext = self.j.setdefault("extensions", {}).setdefault("KHR_lights_punctual", {"lights": []})
        ext["lights"].append(kw)
        return len(ext["lights"]) - 1

    def write(self, path: Path, container: str = "data") -> Path:
        """container: "data" (data URI), "bin" (file beside) or "glb"."""
        path = Path(path)
        j = json.loads(json.dumps(self.j))
        data = bytes(self.bin)
        if container == "glb":
            j["buffers"] = [{"byteLength": len(data)}]
            js = json.dumps(j).encode()
            js += b" " * ((4 - len(js) % 4) % 4)
            data += b"\0" * ((4 - len(data) % 4) % 4)
            body = struct.pack("<II", len(js), 0x4E4F534A) + js + struct.pack("<II", len(data), 0x004E4942) + data
            path.write_bytes(b"glTF" + struct.pack("<II", 2, 12 + len(body)) + body)
            return path
        if container == "bin":
            (path.parent / (path.stem + ".bin")).write_bytes(data)
            j["buffers"] = [{"byteLength": len(data), "uri": path.stem + ".bin"}]
        else:
            j["buffers"] = [{"byteLength": len(data),
                             "uri": "data:application/octet-stream;base64," + base64.b64encode(data).decode()}]
        path.write_text(json.dumps(j, indent=1))
        return path


def quad(size=1.0):
    """Unit quad in XY at z=0 facing +Z, UV = lightmap UV = [0,1]^2."""
    s = size / 2
    pos = np.array([[-s, -s, 0], [s, -s, 0], [s, s, 0], [-s, s, 0]], np.float32)
    nrm = np.tile(np.array([[0, 0, 1]], np.float32), (4, 1))
    uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    idx = np.array([0, 1, 2, 0, 2, 3], np.uint32)
    return pos, nrm, uv, idx


ADAM7 = [(0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2)]


def png_encode(samples: np.ndarray, color_type: int, depth: int, interlace: bool = False, palette=None,
               trns: bytes = None) -> bytes:
    """PNG of raw samples (H, W, channels) in [0, 2^depth) at any bit depth
    PNG allows (sub-byte rows packed most significant bit first), optionally
    Adam7-interlaced; each pass is filtered with types 0..4 in turn."""
    samples = np.asarray(samples, np.uint32)
    H, W, ch = samples.shape
    bpp = max(1, ch * depth // 8)

    def pack(row):  # one row of (w, ch) samples -> bytes
        flat = row.reshape(-1)
        if depth == 16:
            return b"".join(int(v).to_bytes(2, "big") for v in flat)
        if depth == 8:
            return bytes(int(v) for v in flat)
        bits = "".join(format(int(v), f"0{depth}b") for v in flat)
        bits += "0" * (-len(bits) % 8)
        return bytes(int(bits[i:i + 8], 2) for i in range(0, len(bits), 8))

    raw = bytearray()
    for x0, y0, dx, dy in (ADAM7 if interlace else [(0, 0, 1, 1)]):
        sub = samples[y0::dy, x0::dx]
        if sub.size == 0:
            continue
        prev = None
        for y, row in enumerate(sub):
            cur = np.frombuffer(pack(row), np.uint8).astype(np.int32)
            up = prev if prev is not None else np.zeros_like(cur)
            left = np.concatenate([np.zeros(bpp, np.int32), cur[:-bpp]])
            upleft = np.concatenate([np.zeros(bpp, np.int32), up[:-bpp]])
            ft = y % 5
            if ft == 0:
                f = cur
            elif ft == 1:
                f = cur - left
            elif ft == 2:
                f = cur - up
            elif ft == 3:
                f = cur - (left + up) // 2
            else:
                p = left + up - upleft
                pa, pb, pc = np.abs(p - left), np.abs(p - up), np.abs(p - upleft)
                f = cur - np.where((pa <= pb) & (pa <= pc), left, np.where(pb <= pc, up, upleft))
            raw.append(ft)
            raw += (f & 0xFF).astype(np.uint8).tobytes()
            prev = cur

    def chunk(t, d):
        return struct.pack(">I", len(d)) + t + d + struct.pack(">I", zlib.crc32(t + d) & 0xFFFFFFFF)

    out = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", W, H, depth, color_type, 0, 0,
                                                            1 if interlace else 0))
    if palette is not None:
        out += chunk(b"PLTE", np.asarray(palette, np.uint8).tobytes())
    if trns is not None:
        out += chunk(b"tRNS", bytes(trns))
    return out + chunk(b"IDAT", zlib.compress(bytes(raw), 9)) + chunk(b"IEND", b"")
