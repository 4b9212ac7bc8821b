"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark workloads (no public dataset is used)."""
from __future__ import annotations

import numpy as np


def gradient_noise_image(w: int, h: int, c: int, bits: int, seed: int, sigma: float = 8.0) -> np.ndarray:
    """Per-channel bilinear gradients plus N(0, sigma^2) noise (sigma in 8-bit
    units, scaled to the bit depth), clipped to [0, 2^bits-1]; planar [c,h,w]."""
    rng = np.random.default_rng(seed)
    mx = (1 << bits) - 1
    gx = np.linspace(0.0, 1.0, w)[None, :]
    gy = np.linspace(0.0, 1.0, h)[:, None]
    out = np.empty((c, h, w), np.uint8 if bits <= 8 else np.uint16)
    for k in range(c):
        a, b, off = rng.uniform(0.2, 1.0), rng.uniform(0.2, 1.0), rng.uniform(0.0, 0.2)
        base = mx * (off + (1 - off) * (a * gx + b * gy) / (a + b))
        noise = rng.normal(0.0, sigma * mx / 255.0, (h, w)).astype(np.float32)
        out[k] = np.clip(np.rint(base + noise), 0, mx)
    return out


def radial_noise_image(w: int, h: int, bits: int, seed: int, sigma: float = 40.0) -> np.ndarray:
    """Single-component smooth radial field plus N(0, sigma^2) noise."""
    rng = np.random.default_rng(seed)
    mx = (1 << bits) - 1
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    r = np.hypot(xx - w / 2, yy - h / 2) / (0.5 * np.hypot(w, h))
    base = mx * (0.5 + 0.45 * np.cos(np.pi * r * 3))
    return np.clip(np.rint(base + rng.normal(0, sigma, (h, w))), 0, mx).astype(np.uint16)[None]


def laplacian_block(rng, w: int, h: int, bitplanes: int, zero_frac: float = 0.15) -> np.ndarray:
    """Code-block coefficients: Laplacian magnitudes scaled so the block needs
    about `bitplanes` magnitude bit-planes, with ~zero_frac exact zeros."""
    scale = (1 << max(bitplanes - 1, 0)) / 4.0
    v = np.rint(rng.laplace(0.0, scale, (h, w)))
    v[rng.random((h, w)) < zero_frac] = 0
    lim = (1 << bitplanes) - 1
    return np.clip(v, -lim, lim).astype(np.int32)
