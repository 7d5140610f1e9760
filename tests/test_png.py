"""PNG base-colour textures at every colour type, bit depth and interlace
method PNG allows, through LoadScene (shb_load_gltf).  The reference reads
textures through tinygltf's image loader over stb_image
(src/loader.cpp:415-432); the expected pixels apply stb_image's conversions
to 8-bit RGB(A): 16-bit samples keep their high byte, 1/2/4-bit grey is
scaled to 0..255, palette indices are looked up, and a tRNS colour key on a
grey or RGB image adds an alpha of 0 where the samples equal the key.  The files come from the test encoder
tests/gltf_fixture.png_encode, itself checked against Pillow's decoder
where Pillow's conversions are the same.  Host code only, no GPU."""
import io
import struct
import zlib

import numpy as np
import pytest

from sh_baker_b200 import api
from tests.gltf_fixture import GltfBuilder, png_encode, quad

CHANNELS = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}


def expected(s, ctype, depth, palette=None, trns=None):
    """8-bit RGB or RGBA pixels stb_image returns for raw samples s."""
    s = s.astype(np.int64)
    if depth == 16:
        b8 = s >> 8
    elif ctype == 0 and depth < 8:
        b8 = s * (255 // ((1 << depth) - 1))
    else:
        b8 = s
    H, W = s.shape[:2]
    if ctype == 3:
        pal = np.asarray(palette, np.int64).reshape(-1, 3)
        rgb = pal[s[..., 0]]
        if trns is None:
            return rgb.astype(np.uint8)
        a = np.array([trns[i] if i < len(trns) else 255 for i in s[..., 0].ravel()]).reshape(H, W, 1)
        return np.concatenate([rgb, a], -1).astype(np.uint8)
    if ctype in (0, 4):
        rgb = np.repeat(b8[..., :1], 3, -1)
    else:
        rgb = b8[..., :3]
    if ctype in (4, 6):
        return np.concatenate([rgb, b8[..., -1:]], -1).astype(np.uint8)
    if trns is not None:
        key = [int.from_bytes(bytes(trns[2 * k:2 * k + 2]), "big") for k in range(CHANNELS[ctype])]
        a = np.where(np.all(s == np.array(key), -1, keepdims=True), 0, 255)
        return np.concatenate([rgb, a], -1).astype(np.uint8)
    return rgb.astype(np.uint8)


def cases():
    out = []
    for interlace in (False, True):
        for depth in (1, 2, 4, 8, 16):
            out.append((0, depth, interlace, False))
        for depth in (1, 2, 4, 8):
            out.append((3, depth, interlace, False))
            out.append((3, depth, interlace, True))
        for ctype in (2, 4, 6):
            for depth in (8, 16):
                out.append((ctype, depth, interlace, False))
        for ctype, depth in ((0, 2), (0, 8), (0, 16), (2, 8), (2, 16)):
            out.append((ctype, depth, interlace, True))  # colour key
    return out


def make(ctype, depth, interlace, with_trns, size, seed):
    rng = np.random.default_rng(seed)
    H, W = size
    ch = CHANNELS[ctype]
    top = (1 << depth) if ctype != 3 else min(1 << depth, 7)  # palette of 7 entries
    s = rng.integers(0, top, (H, W, ch))
    palette = trns = None
    if ctype == 3:
        palette = rng.integers(0, 256, (7, 3))
        if with_trns:
            trns = list(rng.integers(0, 256, 4))  # alphas of the first 4 entries only
    elif with_trns:
        key = s[0, 0]  # the first pixel's samples: at least one transparent pixel
        trns = b"".join(int(v).to_bytes(2, "big") for v in key)
    return s, png_encode(s, ctype, depth, interlace, palette, trns), palette, trns


@pytest.mark.parametrize("ctype,depth,interlace,with_trns", cases())
def test_png_forms_decode_like_stb_image(tmp_path, ctype, depth, interlace, with_trns):
    for size, seed in (((13, 11), 1), ((1, 1), 2), ((3, 9), 3), ((17, 33), 4)):
        s, data, palette, trns = make(ctype, depth, interlace, with_trns, size, seed)
        want = expected(s, ctype, depth, palette, trns)
        b = GltfBuilder()
        m = b.material(texture_png=data)
        pos, nrm, uv, idx = quad()
        b.node(mesh=b.mesh([b.primitive(pos, nrm, uv, idx=idx, material=m)]))
        err = []
        sc = api.LoadScene(b.write(tmp_path / "t.gltf"), err)
        assert sc is not None, err
        a = sc.materials[0].albedo
        assert (a.height, a.width, a.channels) == want.shape, (size, want.shape)
        np.testing.assert_array_equal(np.asarray(a.pixel_data).reshape(want.shape), want, err_msg=str(size))


@pytest.mark.parametrize("ctype,depth,interlace,with_trns",
                         [c for c in cases() if c[1] != 16 and not (c[0] == 0 and c[1] < 8 and c[3])])
def test_encoder_agrees_with_pillow(ctype, depth, interlace, with_trns):
    """The test encoder's files, decoded by Pillow, give the expected pixels.
    Left out: 16-bit files (Pillow narrows 16-bit samples by clipping, not
    by their high byte) and the colour key of 1/2/4-bit grey, which Pillow
    does not turn into alpha while stb_image does (it scales key and samples
    alike)."""
    from PIL import Image
    s, data, palette, trns = make(ctype, depth, interlace, with_trns, (13, 11), 1)
    want = expected(s, ctype, depth, palette, trns)
    im = Image.open(io.BytesIO(data))
    assert im.info.get("interlace", 0) == (1 if interlace else 0)
    got = np.asarray(im.convert("RGBA" if want.shape[-1] == 4 else "RGB"))
    np.testing.assert_array_equal(got, want)


def test_bad_depth_for_colour_type_is_rejected(tmp_path):
    s = np.zeros((2, 2, 3), np.uint32)
    data = png_encode(s, 2, 8)
    bad = bytearray(data)
    bad[24] = 4  # IHDR bit depth 4 on an RGB image
    bad[29:33] = struct.pack(">I", zlib.crc32(bytes(bad[12:29])) & 0xFFFFFFFF)
    b = GltfBuilder()
    m = b.material(texture_png=bytes(bad))
    pos, nrm, uv, idx = quad()
    b.node(mesh=b.mesh([b.primitive(pos, nrm, uv, idx=idx, material=m)]))
    err = []
    assert api.LoadScene(b.write(tmp_path / "b.gltf"), err) is None and "bit depth" in err[0], err
