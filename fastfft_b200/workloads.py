"""Seeded synthetic inputs for the correlation workloads (no dataset is published for them).

The 2D search image is N(0,1) noise plus Gaussian blobs (sigma 8 px, amplitude 5) at
seeded positions; templates are N(0,1).  Template-matching images in cryo-EM are of
this size and kind (4096^2 micrographs, 128..512 px templates).
"""
from __future__ import annotations

import numpy as np

SEED_BASE = 20261203


def blob_image(n: int, n_blobs: int = 20, sigma: float = 8.0, amp: float = 5.0, seed: int = SEED_BASE + 2):
    rng = np.random.default_rng(seed)
    img = rng.standard_normal((n, n)).astype(np.float32)
    lo, hi = min(32, n // 4), max(n - 32, 3 * n // 4)
    centres = rng.uniform(lo, hi, size=(n_blobs, 2))
    r = int(np.ceil(4 * sigma))
    yy, xx = np.mgrid[-r: r + 1, -r: r + 1]
    for cy, cx in centres:
        iy, ix = int(np.floor(cy)), int(np.floor(cx))
        g = amp * np.exp(-((yy - (cy - iy)) ** 2 + (xx - (cx - ix)) ** 2) / (2 * sigma * sigma))
        y0, x0 = iy - r, ix - r
        ys = slice(max(y0, 0), min(y0 + 2 * r + 1, n))
        xs = slice(max(x0, 0), min(x0 + 2 * r + 1, n))
        img[ys, xs] += g[ys.start - y0: ys.stop - y0, xs.start - x0: xs.stop - x0].astype(np.float32)
    return img


def padded_pitch(x: int) -> int:
    """FFTW pitch 2*(x/2+1) in real elements (ReturnPaddedMemorySize)."""
    return 2 * ((x + (2 if x % 2 == 0 else 1)) // 2)


def to_padded(a: np.ndarray) -> np.ndarray:
    """(y, x) array -> flat FFTW-padded float32 buffer."""
    y, x = a.shape
    out = np.zeros((y, padded_pitch(x)), np.float32)
    out[:, :x] = a
    return out.reshape(-1)
