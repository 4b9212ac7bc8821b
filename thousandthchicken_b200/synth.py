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


def c3_geometry(n: int = 200_000, seed: int = 3, min_image: int = 64, max_image: int = 4096) -> dict:
    """Code-block geometry of the batched Tier-1 workload: n blocks, 60%
    64x64, 30% 32x32 and 10% edge blocks with width and height uniform in
    1..64; each with a subband orientation, a magnitude bit-plane count
    uniform in 4..14 (its subband's scale) and a seeded pass count at which
    its codeword is truncated, uniform in 1..3*planes-2.  Blocks are stored
    one after another (block i at element off[i], pitch w[i]) and grouped in
    order into "images" of min_image..max_image blocks for the per-image
    comparison."""
    rng = np.random.default_rng(seed)
    kind = rng.choice(3, size=n, p=[0.6, 0.3, 0.1])
    w = np.where(kind == 0, 64, np.where(kind == 1, 32, rng.integers(1, 65, n))).astype(np.uint16)
    h = np.where(kind == 0, 64, np.where(kind == 1, 32, rng.integers(1, 65, n))).astype(np.uint16)
    nb = rng.integers(4, 15, n).astype(np.uint8)
    orient = rng.integers(0, 4, n).astype(np.uint8)
    max_passes = (1 + (rng.random(n) * (3 * nb.astype(np.int64) - 2)).astype(np.int64)).astype(np.uint8)
    size = w.astype(np.int64) * h.astype(np.int64)
    off = np.concatenate([[0], np.cumsum(size)[:-1]]).astype(np.uint64)
    images, s = [], 0
    while s < n:
        k = int(rng.integers(min_image, max_image + 1))
        images.append((s, min(k, n - s)))
        s += k
    return {"w": w, "h": h, "nb": nb, "orient": orient, "max_passes": max_passes, "off": off,
            "elems": int(size.sum()), "images": images}


def c3_coefficients(geom: dict, device, seed: int = 3, zero_frac: float = 0.15, chunk: int = 1 << 26):
    """The blocks' int32 coefficients on `device` (a torch tensor of
    geom["elems"] values): Laplacian with scale 2^(planes-1)/4 per block,
    rounded, about zero_frac exact zeros, clipped to the block's bit-plane
    count.  Generated in chunks with a seeded torch generator."""
    import torch
    n = len(geom["w"])
    size = torch.from_numpy((geom["w"].astype(np.int64) * geom["h"].astype(np.int64))).to(device)
    nb = torch.from_numpy(geom["nb"].astype(np.int64)).to(device)
    g = torch.Generator(device=device).manual_seed(seed)
    out = torch.empty(geom["elems"], dtype=torch.int32, device=device)
    block_of = torch.repeat_interleave(torch.arange(n, device=device), size)
    for a in range(0, geom["elems"], chunk):
        b = min(a + chunk, geom["elems"])
        planes = nb[block_of[a:b]]
        scale = torch.exp2((planes - 1).to(torch.float32)) / 4.0
        u = torch.rand(b - a, generator=g, device=device) - 0.5
        v = torch.round(-scale * torch.sign(u) * torch.log1p(-2.0 * u.abs().clamp(max=0.4999999)))
        v = torch.where(torch.rand(b - a, generator=g, device=device) < zero_frac, torch.zeros_like(v), v)
        lim = (torch.exp2(planes.to(torch.float32)) - 1.0)
        out[a:b] = torch.maximum(torch.minimum(v, lim), -lim).to(torch.int32)
    return out


def c4_specs(n: int = 256, seed: int = 11, min_side: int = 256, max_side: int = 8192, step: int = 16) -> list:
    """The mixed-size batch: n images with width and height each uniform in
    min_side..max_side (multiples of step), 1 or 3 components, 8- or 12-bit
    samples; even-numbered images lossless (RCT + 5-level 5/3), odd ones
    lossy (ICT + 5-level 9/7, base step 1/64)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        w = int(rng.integers(min_side // step, max_side // step + 1)) * step
        h = int(rng.integers(min_side // step, max_side // step + 1)) * step
        c = int(rng.choice([1, 3]))
        bits = int(rng.choice([8, 12]))
        out.append({"w": w, "h": h, "c": c, "bits": bits, "reversible": i % 2 == 0, "levels": 5,
                    "base_step": 1.0 / 64, "seed": 1000 + i})
    return out


def gradient_noise_image_device(w: int, h: int, c: int, bits: int, seed: int, device, sigma: float = 8.0):
    """The gradient_noise_image family generated on a CUDA device with a
    seeded torch generator: per-channel bilinear gradients plus N(0, sigma^2)
    noise (sigma in 8-bit units, scaled to the bit depth), rounded and
    clipped; [c, h, w] uint8 (bits <= 8) or int16 holding the unsigned
    samples.  The same seed gives the same image on the same device."""
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    mx = float((1 << bits) - 1)
    gx = torch.linspace(0.0, 1.0, w, device=device)[None, :]
    gy = torch.linspace(0.0, 1.0, h, device=device)[:, None]
    out = torch.empty((c, h, w), dtype=torch.uint8 if bits <= 8 else torch.int16, device=device)
    for k in range(c):
        a, b, off = (torch.rand(3, generator=g, device=device) * torch.tensor([0.8, 0.8, 0.2], device=device) +
                     torch.tensor([0.2, 0.2, 0.0], device=device)).tolist()
        base = mx * (off + (1 - off) * (a * gx + b * gy) / (a + b))
        noise = torch.randn((h, w), generator=g, device=device) * (sigma * mx / 255.0)
        out[k] = torch.clamp(torch.round(base + noise), 0, mx).to(out.dtype)
    return out
