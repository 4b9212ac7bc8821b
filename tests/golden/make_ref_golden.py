"""Generate golden vectors from the reference's own kernels run on the CPU.

The reference's OpenCL C (coefficient_coder.cl, preprocess_*.cl,
quantizer_lossless_inverse.cl, dwt_f53.cl, dwt_r53.cl) is compiled as host code by
oracle/ref_shim/Makefile into oracle/_ref/ and driven by oracle/ref.py.
Tier-1 vectors use the build with the state-update helpers passing their
register by reference (defects D1/D2 fixed); each codeword is followed by
one 0xFF byte, which an ISO decoder treats exactly like the end of the data
but which the reference needs to consume the codeword's real last byte (its
bytein stops one byte early).  Blocks one column wide are excluded (the
reference's window scan leaves the block when width == 1).

Run from the repository root: ``python tests/golden/make_ref_golden.py
[fixture ...]`` (every fixture when none is named).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import ref as R  # noqa: E402
from thousandthchicken_b200 import codec  # noqa: E402
from thousandthchicken_b200.synth import laplacian_block  # noqa: E402


def t1_vectors(seed=123, n=160, mb=14):
    rng = np.random.default_rng(seed)
    segs, meta = [], []
    for i in range(n):
        kind = i % 4
        if kind == 0:
            w = h = 64
        elif kind == 1:
            w = h = 32
        else:
            w, h = int(rng.integers(2, 65)), int(rng.integers(1, 65))
        orient = int(rng.integers(0, 4))
        coef = laplacian_block(rng, w, h, bitplanes=int(rng.integers(1, 14)))
        seg, passes, zbp = codec.t1_encode_block(coef, orient, mb)
        segs.append(seg)
        meta.append((w, h, orient, mb, zbp, passes))
    blocks = [(s + b"\xff", m[0], m[1], m[2], m[3], m[3] - m[4]) for s, m in zip(segs, meta)]
    raw, skipped = R.t1_decode(blocks, patched=True)
    assert skipped == 0
    raw_unpatched, _ = R.t1_decode(blocks, patched=False)
    off = np.cumsum([0] + [len(s) for s in segs])
    # block regions only, concatenated in block order (row-major per block)
    flat = np.concatenate([raw[i, :m[1], :m[0]].ravel() for i, m in enumerate(meta)])
    unpatched_diff = np.array([int((raw_unpatched[i, :m[1], :m[0]] != raw[i, :m[1], :m[0]]).sum())
                               for i, m in enumerate(meta)], np.int32)
    return dict(pool=np.frombuffer(b"".join(segs), np.uint8), seg_off=off[:-1].astype(np.int64),
                seg_len=np.array([len(s) for s in segs], np.int32), meta=np.array(meta, np.int32),
                ref_raw=flat, unpatched_mismatches=unpatched_diff)


def t1_trunc_vectors(seed=321, n=160, mb=14):
    """Blocks truncated after P whole bit-planes (3P - 2 coding passes, the
    oracle's encoder terminating the codeword there).  The reference kernel
    decodes every plane it is told a block has (significantBits,
    coefficient_coder.cl:797-815) and ignores pass counts (defect D3), so it
    is given significantBits = P: it then decodes exactly those passes and
    writes the P planes as the top planes of a P-plane block.  The stored
    `ref_raw` words are its own output; a decoder of the same block with its
    nb coded planes puts them nb - P bits higher."""
    import oracle as O
    rng = np.random.default_rng(seed)
    segs, meta = [], []
    while len(meta) < n:
        i = len(meta)
        kind = i % 4
        if kind == 0:
            w = h = 64
        elif kind == 1:
            w = h = 32
        else:
            w, h = int(rng.integers(2, 65)), int(rng.integers(1, 65))
        orient = int(rng.integers(0, 4))
        coef = laplacian_block(rng, w, h, bitplanes=int(rng.integers(2, 14)))
        _, _, nb = O.t1_encode(coef, orient, 0)
        if nb < 2:
            continue
        planes = int(rng.integers(1, nb))
        seg, passes, nb2 = O.t1_encode(coef, orient, 3 * planes - 2)
        assert passes == 3 * planes - 2 and nb2 == nb
        segs.append(seg)
        meta.append((w, h, orient, mb, mb - nb, passes, planes))
    blocks = [(s + b"\xff", m[0], m[1], m[2], m[3], m[6]) for s, m in zip(segs, meta)]
    raw, skipped = R.t1_decode(blocks, patched=True)
    assert skipped == 0
    off = np.cumsum([0] + [len(s) for s in segs])
    flat = np.concatenate([raw[i, :m[1], :m[0]].ravel() for i, m in enumerate(meta)])
    return dict(pool=np.frombuffer(b"".join(segs), np.uint8), seg_off=off[:-1].astype(np.int64),
                seg_len=np.array([len(s) for s in segs], np.int32), meta=np.array(meta, np.int32), ref_raw=flat)


def colour_vectors(seed=7):
    rng = np.random.default_rng(seed)
    out = {}
    for bits in (8, 12):
        img = rng.integers(0, 1 << bits, (3, 40, 56)).astype(np.int32)
        out[f"rgb{bits}"] = img
        out[f"rct{bits}"] = np.stack(R.rct(list(img), bits))
        out[f"rct_inv{bits}"] = np.stack(R.rct_inverse(list(out[f"rct{bits}"]), bits))
        out[f"ict{bits}"] = np.stack(R.ict(list(img), bits))
        out[f"dc{bits}"] = R.dc_shift(img[0], bits)
        out[f"dc_inv{bits}"] = R.dc_shift_inverse(out[f"dc{bits}"], bits)
        ycc = rng.integers(-(1 << (bits - 1)), 1 << (bits - 1), (3, 40, 56)).astype(np.int32)
        out[f"ycc{bits}"] = ycc
        out[f"ict_inv{bits}"] = np.stack(R.ict_inverse(list(ycc), bits))
    return out


# widths that are multiples of the kernels' window (64 columns below 480, 128
# below 960, 192 from there): at other widths the kernels read local memory
# that no work-item wrote
DWT_SIZES = [(64, 64), (128, 61), (192, 66), (256, 40), (512, 24), (960, 16)]


def dwt53_vectors(seed=11):
    """One level of the reference's 5/3 kernels (dwt_f53.cl / dwt_r53.cl,
    truncating division) per size; the window width follows the image width
    as DWTForward53::dwt chooses it (64, 128 or 192 columns).  The reverse
    runs on the oracle's forward coefficients (truncating mode, packed)."""
    import oracle as O
    rng = np.random.default_rng(seed)
    out = {}
    for w, h in DWT_SIZES:
        x = rng.integers(-128, 128, (h, w)).astype(np.int32)
        k = f"{w}x{h}"
        out[f"x_{k}"] = x
        out[f"fwd_{k}"] = R.dwt53_forward(x, 1)
        rev_in = R.mallat_to_packed(O.fdwt53(x, 1, rounding=1), 1)
        out[f"revin_{k}"] = rev_in
        out[f"rev_{k}"] = R.dwt53_reverse(rev_in, w, h, 1)
    return out


FIXTURES = {"ref_t1_blocks": t1_vectors, "ref_t1_trunc": t1_trunc_vectors, "ref_colour": colour_vectors,
            "ref_dwt53": dwt53_vectors}


def main(names=None):
    """Write the named fixtures (all when none are named)."""
    if not R.build() or not R.dwt_available():
        raise SystemExit("oracle/_ref could not be built (reference sources missing)")
    for name in names or FIXTURES:
        np.savez_compressed(HERE / f"{name}.npz", **FIXTURES[name]())
        print(f"written {name}.npz")


if __name__ == "__main__":
    main(sys.argv[1:])
