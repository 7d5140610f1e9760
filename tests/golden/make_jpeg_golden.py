"""Generates tests/golden/jpeg_reference.npz: small JPEG files written by
Pillow (libjpeg) and the RGB pixels Pillow decodes from them.  The loader's
own JPEG decoder (sh_baker_b200/csrc/jpeg.cpp) is checked against these.

Cases: 4:4:4, 4:2:2 and 4:2:0 chroma sampling at quality 90, 4:2:0 at
quality 50, 4:2:0 with a restart marker every 3 MCUs, a greyscale file,
and odd sizes (37 x 53, 1 x 1, 17 x 9) so that partial MCUs are cut.
Progressive twins (`prog_<case>`): the same image and settings written as a
progressive file (spectral selection and successive approximation scans),
whose quantised coefficients equal its sequential twin's.

    python tests/golden/make_jpeg_golden.py
"""
from __future__ import annotations

import io
from pathlib import Path

import numpy as np
from PIL import Image


def texture(h: int, w: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w]
    img = np.stack([128 + 100 * np.sin(x / 5.0), 128 + 90 * np.cos(y / 4.0), (x * 3 + y * 2) % 256], -1)
    return np.clip(img + rng.integers(-20, 20, img.shape), 0, 255).astype(np.uint8)


CASES = {
    "s444_q90": (37, 53, dict(subsampling=0, quality=90)),
    "s422_q90": (37, 53, dict(subsampling=1, quality=90)),
    "s420_q90": (37, 53, dict(subsampling=2, quality=90)),
    "s420_q50": (40, 64, dict(subsampling=2, quality=50)),
    "s420_restart": (37, 53, dict(subsampling=2, quality=90, restart_marker_blocks=3)),
    "grey": (23, 31, None),
    "tiny": (1, 1, dict(subsampling=2, quality=90)),
    "odd": (9, 17, dict(subsampling=1, quality=75)),
}
PROGRESSIVE = ["s444_q90", "s422_q90", "s420_q90", "s420_restart", "grey", "odd"]


def main():
    out = {}
    for i, (name, (h, w, kw)) in enumerate(CASES.items()):
        img = texture(h, w, i)
        b = io.BytesIO()
        if kw is None:
            Image.fromarray(img[..., 0]).save(b, "JPEG", quality=90)
        else:
            Image.fromarray(img).save(b, "JPEG", **kw)
        data = b.getvalue()
        out[f"{name}_jpeg"] = np.frombuffer(data, np.uint8)
        out[f"{name}_rgb"] = np.array(Image.open(io.BytesIO(data)).convert("RGB"))
        if name in PROGRESSIVE:
            b = io.BytesIO()
            if kw is None:
                Image.fromarray(img[..., 0]).save(b, "JPEG", quality=90, progressive=True)
            else:
                Image.fromarray(img).save(b, "JPEG", progressive=True, **kw)
            data = b.getvalue()
            assert data[2:].find(b"\xff\xc2") >= 0  # SOF2
            out[f"prog_{name}_jpeg"] = np.frombuffer(data, np.uint8)
            out[f"prog_{name}_rgb"] = np.array(Image.open(io.BytesIO(data)).convert("RGB"))
    path = Path(__file__).parent / "jpeg_reference.npz"
    np.savez_compressed(path, **out)
    print(f"{len(CASES) + len(PROGRESSIVE)} cases -> {path}")


if __name__ == "__main__":
    main()
