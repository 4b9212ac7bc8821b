"""Generate the golden fixtures of this directory.

Codestreams are written by OpenJPEG 2.5 (through Pillow's JPEG 2000 plugin),
an encoder independent of this project; the expected outputs are the
original images (lossless streams) and OpenJPEG's own decode of each stream.
Run from the repository root: ``python tests/golden/make_golden.py``.
The fixtures are committed; tests only read them.
"""
from __future__ import annotations

import io
import json
from pathlib import Path

import numpy as np
from PIL import Image, features

HERE = Path(__file__).resolve().parent


def synth(w, h, c, bits, seed):
    """Per-channel bilinear gradient plus Gaussian noise (sigma 8), clipped."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    mx = (1 << bits) - 1
    out = []
    for k in range(c):
        a, b = rng.uniform(0.2, 1.0, 2)
        base = mx * (a * xx / max(w - 1, 1) + b * yy / max(h - 1, 1)) / (a + b)
        out.append(base + rng.normal(0, 8 * (mx / 255.0), (h, w)))
    return np.clip(np.rint(out), 0, mx).astype(np.uint8 if bits <= 8 else np.uint16)


def to_pil(img, bits):
    if img.shape[0] == 3:
        return Image.fromarray(np.moveaxis(img, 0, -1), "RGB")
    if bits > 8:
        return Image.fromarray(img[0].astype(np.uint16))
    return Image.fromarray(img[0], "L")


def from_pil(im):
    a = np.asarray(im)
    return np.moveaxis(a, -1, 0) if a.ndim == 3 else a[None]


CASES = [
    # name, w, h, comps, bits, levels, irreversible, layers, progression, seed
    ("opj_rev_rgb_257x131", 257, 131, 3, 8, 5, False, None, "LRCP", 1),
    ("opj_rev_gray_100x60", 100, 60, 1, 8, 3, False, None, "LRCP", 2),
    ("opj_rev_gray16_96x80", 96, 80, 1, 16, 4, False, None, "LRCP", 3),
    ("opj_rev_rgb_33x17_l4", 33, 17, 3, 8, 4, False, None, "RLCP", 4),
    ("opj_irr_rgb_256x256", 256, 256, 3, 8, 5, True, None, "LRCP", 5),
    ("opj_irr_gray_190x77", 190, 77, 1, 8, 4, True, None, "RPCL", 6),
    ("opj_layers_irr_rgb_256x192", 256, 192, 3, 8, 5, True, [40, 20, 10], "LRCP", 7),
    ("opj_layers_rev_gray_128x128", 128, 128, 1, 8, 3, False, [8, 4], "RPCL", 8),
    ("opj_layers_irr_rgb_128x96_cprl", 128, 96, 3, 8, 3, True, [10, 5], "CPRL", 9),
]


def main():
    meta = {"openjpeg": features.version("jpg_2000"), "cases": {}}
    for name, w, h, c, bits, levels, irr, layers, prog, seed in CASES:
        img = synth(w, h, c, bits, seed)
        kw = dict(irreversible=irr, num_resolutions=levels + 1, codeblock_size=(64, 64), no_jp2=True,
                  progression=prog)
        if layers:
            kw.update(quality_mode="rates", quality_layers=layers)
        buf = io.BytesIO()
        to_pil(img, bits).save(buf, "JPEG2000", **kw)
        cs = buf.getvalue()
        dec = from_pil(Image.open(io.BytesIO(cs)))
        (HERE / f"{name}.j2k").write_bytes(cs)
        np.savez_compressed(HERE / f"{name}.npz", original=img, openjpeg=dec.astype(img.dtype))
        meta["cases"][name] = dict(w=w, h=h, comps=c, bits=bits, levels=levels, irreversible=irr,
                                   layers=layers, progression=prog, seed=seed, bytes=len(cs),
                                   openjpeg_equals_original=bool(np.array_equal(dec, img)))
        print(name, len(cs), "bytes")
    (HERE / "golden.json").write_text(json.dumps(meta, indent=1) + "\n")


if __name__ == "__main__":
    main()
