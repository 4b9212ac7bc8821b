"""Batched Tier-1 over code-blocks from many images (the 200,000-block
workload): the blocks' codewords are produced on the GPU by the Tier-1
encoder, each truncated at its own pass count, and decoded either in one
persistent launch over every block (a work queue sorted longest-first by
passes x area) or with one launch per image, as a decoder that handles one
image at a time would.

Replaces, for this workload, the reference's one-work-item-per-block
g_decode (coefficient_coder.cl:778-819) launched per tile in groups of four
(CoefficientCoder.cpp:240-246).
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from .codec import DESC_DTYPE, ENC_DESC_DTYPE, sort_order
from .stages import CoefficientCoder, T1Encoder, _dev_bytes, _ptr

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None


class BlockBatch:
    """Code-blocks laid out one after another in one int32 buffer (block i
    at element off[i], pitch w[i]), encoded on the device with their seeded
    pass counts, ready to decode.  mb is the magnitude bit-plane count of
    every block's band; cap bounds one codeword."""

    def __init__(self, ctx, geom: dict, coef, mb: int = 16, cap: int = 16384):
        self.ctx = ctx
        self.geom = geom
        self.n = n = len(geom["w"])
        self.cap = cap
        dev = torch.device("cuda", ctx.device)
        enc = np.zeros(n, ENC_DESC_DTYPE)
        enc["in_off"] = geom["off"]
        enc["in_pitch"] = geom["w"]
        enc["inv_step"] = 1.0
        enc["w"], enc["h"] = geom["w"], geom["h"]
        enc["orient"] = geom["orient"]
        enc["mb"] = mb
        enc["max_passes"] = geom["max_passes"]
        self.pool, res = T1Encoder(ctx).encode_device(enc, coef, cap)
        self.results = res
        desc = np.zeros(n, DESC_DTYPE)
        desc["seg_off"] = np.arange(n, dtype=np.uint64) * np.uint64(cap)
        desc["seg_len"] = res["len"]
        desc["out_off"] = geom["off"]
        desc["out_pitch"] = geom["w"]
        desc["step"] = 1.0
        desc["w"], desc["h"] = geom["w"], geom["h"]
        desc["passes"] = res["passes"]
        desc["mb"] = mb
        desc["zero_bitplanes"] = res["zero_bitplanes"]
        desc["orient"] = geom["orient"]
        self.desc = desc
        self.codeword_bytes = int(res["len"].astype(np.int64).sum())
        self.d_desc = _dev_bytes(desc, dev)
        self.d_order = torch.from_numpy(sort_order(desc).view(np.int32)).to(dev)
        self.image_orders = [torch.from_numpy(sort_order(desc[s:s + k]).view(np.int32)).to(dev)
                             for s, k in geom["images"]]
        self.out = torch.zeros(max(geom["elems"], 1), dtype=torch.int32, device=dev)
        nbp = desc["mb"].astype(np.int32) - desc["zero_bitplanes"].astype(np.int32)
        self.max_bitplanes = int(max(1, nbp[desc["passes"] > 0].max())) if (desc["passes"] > 0).any() else 1
        self.coder = CoefficientCoder(ctx)

    def decode_batched(self):
        """Every block in one persistent launch (recon_r 0: the truncated
        values themselves).  Stream-ordered on the context's stream."""
        self.coder.decode(self.d_desc, self.pool, self.out, self.n, self.d_order, raw=False, recon_r=0.0,
                          max_bitplanes=self.max_bitplanes)

    def decode_per_image(self):
        """One launch per image over that image's blocks."""
        lib = L.lib()
        base = _ptr(self.d_desc)
        for (s, k), order in zip(self.geom["images"], self.image_orders):
            self.ctx.check(lib.tc_t1_decode(self.ctx.handle, base + s * DESC_DTYPE.itemsize, _ptr(order), k,
                                            _ptr(self.pool), self.pool.numel(), _ptr(self.out), self.out.numel(),
                                            L.TC_T1_OUT_DEQUANT, 0.0, self.max_bitplanes), "tc_t1_decode")

    def close(self):
        self.pool = self.out = self.d_desc = self.d_order = None
        self.image_orders = []
