"""Headless image output: the RGBA8 buffers of ``Context.tonemap`` written as
binary PPM (P6, alpha dropped), in place of the reference's canvas swap chain
(src/toneMapper.ts, src/main.ts:579-592)."""
from __future__ import annotations

import numpy as np


def write_ppm(path: str, rgba8: np.ndarray) -> None:
    """rgba8: (height, width, 4) uint8, row 0 at the top."""
    a = np.asarray(rgba8)
    if a.dtype != np.uint8 or a.ndim != 3 or a.shape[2] != 4:
        raise ValueError("rgba8 must be a (height, width, 4) uint8 array")
    h, w = a.shape[:2]
    with open(path, "wb") as fh:
        fh.write(f"P6\n{w} {h}\n255\n".encode("ascii"))
        fh.write(np.ascontiguousarray(a[:, :, :3]).tobytes())


def read_ppm(path: str) -> np.ndarray:
    """Inverse of write_ppm: (height, width, 3) uint8."""
    with open(path, "rb") as fh:
        data = fh.read()
    parts = data.split(b"\n", 3)
    if parts[0] != b"P6" or parts[2] != b"255":
        raise ValueError("not a binary 8-bit PPM written by write_ppm")
    w, h = (int(x) for x in parts[1].split())
    return np.frombuffer(parts[3], dtype=np.uint8, count=w * h * 3).reshape(h, w, 3)
