"""Image and transfer-function files for the headless renderer.

* PNG (8-bit RGBA, zlib, no dependencies), binary PPM (RGB8) and PFM (float RGB) writers.
  `flip=True` writes the bottom framebuffer row last, like the reference's snapshot
  (stbi_flip_vertically_on_write(true), viewer.cpp:67, and stbi_write_png, viewer.cpp:393-395):
  framebuffer row 0 is the bottom of the image (screen y = (py + jitter) / H grows upward).
* TF files.  The reference stores transfer functions in the `.tf` state format of the
  imgui-transfer-function submodule, which is not part of the checkout, so this project
  defines its own: JSON {"colormap": [[r, g, b, a], ...], "opacityScale": s,
  "range": [lo, hi]} with the same three pieces of state the viewer pushes into the
  renderer (SetXFColormap / SetXFOpacityScale / SetXFRange, viewer.cpp:496-509).
"""
from __future__ import annotations

import json
import struct
import zlib
from typing import Tuple

import numpy as np


def rgba8_to_array(fb: np.ndarray) -> np.ndarray:
    """(H, W) uint32 RGBA8 words (R in the low byte) -> (H, W, 4) uint8."""
    return np.ascontiguousarray(fb).view(np.uint8).reshape(fb.shape[0], fb.shape[1], 4)


def _png_chunk(tag: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)


def write_png(path: str, rgba: np.ndarray, flip: bool = True) -> None:
    """8-bit RGBA PNG of an (H, W, 4) uint8 array or an (H, W) RGBA8 framebuffer."""
    if rgba.ndim == 2:
        rgba = rgba8_to_array(rgba)
    img = rgba[::-1] if flip else rgba
    h, w = img.shape[:2]
    raw = b"".join(b"\x00" + img[y].tobytes() for y in range(h))
    data = (b"\x89PNG\r\n\x1a\n" + _png_chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0))
            + _png_chunk(b"IDAT", zlib.compress(raw, 6)) + _png_chunk(b"IEND", b""))
    with open(path, "wb") as f:
        f.write(data)


def read_png(path: str) -> np.ndarray:
    """Reader for the PNGs written above (8-bit RGBA, filter 0); returns rows as stored."""
    with open(path, "rb") as f:
        data = f.read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, w = 8, b"", 0
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        tag = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        if tag == b"IHDR":
            w, h = struct.unpack(">II", body[:8])
        elif tag == b"IDAT":
            idat += body
        pos += 12 + n
    raw = zlib.decompress(idat)
    stride = 1 + 4 * w
    rows = [np.frombuffer(raw[y * stride + 1:(y + 1) * stride], np.uint8) for y in range(len(raw) // stride)]
    return np.stack(rows).reshape(len(rows), w, 4)


def write_ppm(path: str, rgba: np.ndarray, flip: bool = True) -> None:
    if rgba.ndim == 2:
        rgba = rgba8_to_array(rgba)
    img = rgba[::-1] if flip else rgba
    h, w = img.shape[:2]
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (w, h))
        f.write(np.ascontiguousarray(img[..., :3]).tobytes())


def write_pfm(path: str, accum: np.ndarray) -> None:
    """Linear float RGB of an (H, W, 4) accumulation buffer.  PFM stores rows bottom to
    top, the framebuffer's own row order."""
    h, w = accum.shape[:2]
    with open(path, "wb") as f:
        f.write(b"PF\n%d %d\n-1.0\n" % (w, h))
        f.write(np.ascontiguousarray(accum[..., :3], dtype="<f4").tobytes())


def save_tf(path: str, colormap: np.ndarray, opacity_scale: float = 1.0, rng: Tuple[float, float] = (0.0, 1.0)) -> None:
    cm = np.asarray(colormap, dtype=np.float32).reshape(-1, 4)
    with open(path, "w") as f:
        json.dump({"colormap": cm.tolist(), "opacityScale": float(opacity_scale),
                   "range": [float(rng[0]), float(rng[1])]}, f)


def load_tf(path: str):
    """(colormap (n, 4) float32, opacity scale, (lo, hi)) of a TF file."""
    with open(path) as f:
        d = json.load(f)
    cm = np.asarray(d["colormap"], dtype=np.float32).reshape(-1, 4)
    if cm.shape[0] < 1:
        raise ValueError(f"{path}: empty colormap")
    return cm, float(d.get("opacityScale", 1.0)), tuple(float(x) for x in d.get("range", (0.0, 1.0)))
