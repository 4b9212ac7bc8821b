"""Shared builders for the GPU parity tests (no GPU needed to import)."""
import numpy as np

import oracle as O
from thousandthchicken_b200 import codec
from thousandthchicken_b200.synth import laplacian_block

SLOT = 64 * 64


def make_blocks(seed, n, mix="uneven", truncate=True, irreversible=False, mb=16):
    """n encoded code-blocks, each decoded into its own 64x64 slot of the
    output; returns (desc, pool, list of (coef, seg, passes, numbps))."""
    rng = np.random.default_rng(seed)
    desc = np.zeros(n, codec.DESC_DTYPE)
    segs = []
    blocks = []
    off = 0
    for i in range(n):
        r = rng.random()
        if mix == "uneven":
            if r < 0.6:
                w = h = 64
            elif r < 0.9:
                w = h = 32
            else:
                w, h = int(rng.integers(1, 65)), int(rng.integers(1, 65))
        else:
            w = h = 64
        orient = int(rng.integers(0, 4))
        coef = laplacian_block(rng, w, h, bitplanes=int(rng.integers(4, 15)))
        seg, total, zbp = codec.t1_encode_block(coef, orient, mb)
        passes = total
        if truncate and total > 1:
            passes = int(rng.integers(1, total + 1))
            seg, passes, zbp = codec.t1_encode_block(coef, orient, mb, passes)
        d = desc[i]
        d["seg_off"] = off
        d["seg_len"] = len(seg)
        d["w"], d["h"] = w, h
        d["passes"] = passes
        d["mb"] = mb
        d["zero_bitplanes"] = zbp
        d["orient"] = orient
        d["out_off"] = i * SLOT
        d["out_pitch"] = 64
        d["step"] = float(rng.uniform(0.01, 4.0)) if irreversible else 1.0
        d["flags"] = 1 if irreversible else 0
        segs.append(seg)
        off += len(seg)
        blocks.append((coef, seg, passes, mb - zbp))
    pool = np.frombuffer(b"".join(segs) + b"\0" * 16, np.uint8).copy()
    return desc, pool, blocks


def oracle_slots(desc, pool, mode, r=0.5):
    """Decode every block with the oracle into the same slot layout."""
    n = len(desc)
    if mode == "raw":
        out = np.zeros((n, 64, 64), np.uint32)
    elif mode == "int":
        out = np.zeros((n, 64, 64), np.int32)
    else:
        out = np.zeros((n, 64, 64), np.float32)
    for i, d in enumerate(desc):
        w, h = int(d["w"]), int(d["h"])
        seg = pool[int(d["seg_off"]): int(d["seg_off"]) + int(d["seg_len"])].tobytes()
        numbps = int(d["mb"]) - int(d["zero_bitplanes"])
        if mode == "raw":
            out[i, :h, :w] = O.t1_decode_raw(seg, w, h, int(d["orient"]), int(d["mb"]), int(d["zero_bitplanes"]),
                                             int(d["passes"]))
            continue
        q, u = O.t1_decode(seg, w, h, int(d["orient"]), max(numbps, 0), int(d["passes"]) if numbps > 0 else 0)
        if mode == "int":
            out[i, :h, :w] = O.dequant_int(q, u, r)
        else:
            out[i, :h, :w] = O.dequant_float(q, u, r, float(d["step"]))
    return out


def oracle_mallat(cs, r=0.5):
    """Oracle Tier-1 + dequantisation of a whole codestream into Mallat
    planes [ncomp, h, w] (int32 or float32)."""
    info, desc, pool = codec.parse(cs)
    W, H, C = info["width"], info["height"], info["ncomp"]
    rev = info["reversible"]
    out = np.zeros((C, H, W), np.int32 if rev else np.float32)
    flat = out.reshape(-1)
    for d in desc:
        w, h = int(d["w"]), int(d["h"])
        seg = pool[int(d["seg_off"]): int(d["seg_off"]) + int(d["seg_len"])].tobytes()
        numbps = int(d["mb"]) - int(d["zero_bitplanes"])
        q, u = O.t1_decode(seg, w, h, int(d["orient"]), max(numbps, 0), int(d["passes"]) if numbps > 0 else 0)
        v = O.dequant_int(q, u, r) if rev else O.dequant_float(q, u, r, float(d["step"]))
        for y in range(h):
            o = int(d["out_off"]) + y * int(d["out_pitch"])
            flat[o: o + w] = v[y]
    return out, info


def pil_j2k(img, **kw):
    """OpenJPEG (through Pillow) codestream of a planar uint8/uint16 image."""
    import io
    from PIL import Image
    a = np.moveaxis(img, 0, -1) if img.shape[0] == 3 else img[0]
    buf = io.BytesIO()
    Image.fromarray(a).save(buf, "JPEG2000", no_jp2=True, **kw)
    return buf.getvalue()


def openjpeg_decode(cs):
    """OpenJPEG's own decode of a codestream, planar."""
    import io
    from PIL import Image
    a = np.asarray(Image.open(io.BytesIO(cs)))
    return np.moveaxis(a, -1, 0) if a.ndim == 3 else a[None]


def oracle_decode_tiled(cs, r=0.5):
    """Oracle decode of a (possibly tiled) codestream: each tile's
    descriptors, rebased to the tile's own planes, through the oracle's
    whole-tile decode, placed at the tile's position.  Returns (info, uint16
    [ncomp, height, width])."""
    info, desc, pool = codec.parse(cs)
    W, H, C = info["width"], info["height"], info["ncomp"]
    out = np.zeros((C, H, W), np.int16 if info["is_signed"] else np.uint16)
    bounds = [t[4] for t in info["tiles"]] + [C * W * H]
    for k, (x0, y0, w, h, co) in enumerate(info["tiles"]):
        sel = (desc["out_off"] >= bounds[k]) & (desc["out_off"] < bounds[k + 1])
        d = desc[sel].copy()
        d["out_off"] -= np.uint64(co)
        out[:, y0:y0 + h, x0:x0 + w] = O.decode_tile(d, pool, w, h, C, info["bits"], info["levels"],
                                                     bool(info["reversible"]), bool(info["mct"]), r=r,
                                                     signed=bool(info["is_signed"]))
    return info, out


def oracle_decode_components(cs, r=0.5):
    """Oracle decode of a single-tile codestream whose components may be
    subsampled (no colour transform across them): each component's
    descriptors through the oracle's one-component decode.  Returns (info,
    list of [h, w] planes)."""
    info, desc, pool = codec.parse(cs)
    sizes = info["comp_sizes"]
    bounds = np.cumsum([0] + [h * w for h, w in sizes])
    planes = []
    for c, (h, w) in enumerate(sizes):
        sel = (desc["out_off"] >= bounds[c]) & (desc["out_off"] < bounds[c + 1])
        d = desc[sel].copy()
        d["out_off"] -= np.uint64(bounds[c])
        planes.append(O.decode_tile(d, pool, w, h, 1, info["bits"], info["levels"], bool(info["reversible"]), False,
                                    r=r, signed=bool(info["is_signed"]))[0])
    return info, planes
