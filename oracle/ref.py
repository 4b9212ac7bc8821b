"""ctypes wrapper of oracle/_ref: the reference's own OpenCL C kernels
compiled as host code through oracle/ref_shim (TEST INFRASTRUCTURE ONLY).
Built from the reference tree by ``make -C oracle/ref_shim`` when it is
present; the built libraries travel with the repository snapshot."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
# the reference project's source directory (TC_REFERENCE_TREE overrides)
REF_TREE = Path(os.environ.get("TC_REFERENCE_TREE", "/root/reference/ThousandthChicken"))
_libs: dict = {}


def build() -> bool:
    """Build oracle/_ref from the reference sources if they are present."""
    if REF_TREE.exists():
        subprocess.run(["make", "-s", "-C", str(HERE / "ref_shim"), f"REF={REF_TREE}"], check=True)
    return available()


def available() -> bool:
    return all((OUT / n).exists() for n in ("libref_t1.so", "libref_t1_patched.so", "libref_pre.so"))


def dwt_available() -> bool:
    return all((OUT / n).exists() for n in ("libref_dwt53f.so", "libref_dwt53r.so"))


def _lib(name):
    if name not in _libs:
        _libs[name] = C.CDLL(str(OUT / name))
    return _libs[name]


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def t1_decode(blocks, patched=True, threads=0):
    """blocks: list of (seg bytes, w, h, orient, mb, sigbits).  Runs the
    reference g_decode (one work-item per block).  Returns uint32
    [n, 64, 64] in the reference's sign-magnitude layout and the count of
    blocks skipped for exceeding the 16 KiB slot."""
    L = _lib("libref_t1_patched.so" if patched else "libref_t1.so")
    n = len(blocks)
    keep = [np.frombuffer(bytes(b[0]) or b"\0", np.uint8) for b in blocks]
    segs = (C.c_void_p * n)(*[k.ctypes.data for k in keep])
    arr = lambda i: np.array([b[i] for b in blocks], np.int32)
    lens = np.array([len(b[0]) for b in blocks], np.int32)
    # orientation class of the reference: LL/LH -> 0, HL -> 1, HH -> 2
    cls = np.array([{0: 0, 2: 0, 1: 1, 3: 2}[b[3]] for b in blocks], np.int32)
    w, h, mb, sb = arr(1), arr(2), arr(4), arr(5)
    out = np.zeros((n, 64, 64), np.int32)
    skipped = L.ref_t1_decode(C.c_int(n), segs, _p(lens), _p(w), _p(h), _p(cls), _p(mb), _p(sb), _p(out),
                              C.c_int(threads))
    return out.view(np.uint32), skipped


def rct(planes, bits):
    p = [np.ascontiguousarray(x, np.int32).copy() for x in planes]
    _lib("libref_pre.so").ref_rct(*map(_p, p), C.c_int(p[0].size), C.c_int(bits - 1))
    return p


def rct_inverse(planes, bits):
    p = [np.ascontiguousarray(x, np.int32).copy() for x in planes]
    _lib("libref_pre.so").ref_rct_inverse(*map(_p, p), C.c_int(p[0].size), C.c_int(bits - 1), 0, (1 << bits) - 1)
    return p


def ict(planes, bits):
    p = [np.ascontiguousarray(x, np.int32).copy() for x in planes]
    _lib("libref_pre.so").ref_ict(*map(_p, p), C.c_int(p[0].size), C.c_int(bits - 1))
    return p


def ict_inverse(planes, bits):
    p = [np.ascontiguousarray(x, np.int32).copy() for x in planes]
    _lib("libref_pre.so").ref_ict_inverse(*map(_p, p), C.c_int(p[0].size), C.c_int(bits - 1), 0, (1 << bits) - 1)
    return p


def dc_shift(x, bits):
    a = np.ascontiguousarray(x, np.int32).copy()
    _lib("libref_pre.so").ref_dc_shift(_p(a), C.c_int(a.size), C.c_int(bits - 1))
    return a


def dc_shift_inverse(x, bits):
    a = np.ascontiguousarray(x, np.int32).copy()
    _lib("libref_pre.so").ref_dc_shift_inverse(_p(a), C.c_int(a.size), C.c_int(bits - 1), 0, (1 << bits) - 1)
    return a


def dequant_lossless(block, shift):
    a = np.ascontiguousarray(block, np.int32)
    out = np.zeros_like(a)
    _lib("libref_pre.so").ref_dequant_lossless(_p(a), _p(out), a.shape[1], a.shape[0], C.c_int(shift))
    return out


# ---- the reference's 5/3 DWT kernels (dwt_f53.cl / dwt_r53.cl) ------------------
# Their layout is band-packed (DWTKernel.cpp:127-154, dwt_io.cl:207-245): a
# level of an sx x sy image stores LL, HL, LH and HH one after another, each
# packed with its own width, and the next level replaces the LL block.


def _level(name, src, dst, sx, sy):
    fn = getattr(_lib("libref_dwt53f.so" if name == "f" else "libref_dwt53r.so"),
                 "ref_dwt53_forward_level" if name == "f" else "ref_dwt53_reverse_level")
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int]
    fn(_p(src), _p(dst), sx, sy)


def dwt53_forward(x, levels):
    """DWTForward53::dwt (DWTForward53.cpp:20-43) with copyLLBandToSrc between
    levels, on an int32 [h, w] image: the band-packed coefficients."""
    h, w = x.shape
    src = np.ascontiguousarray(x, np.int32).reshape(-1).copy()
    dst = np.zeros_like(src)
    sx, sy = w, h
    for lvl in range(levels):
        _level("f", src, dst, sx, sy)
        llx, lly = (sx + 1) // 2, (sy + 1) // 2
        if lvl + 1 < levels:
            src[: llx * lly] = dst[: llx * lly]
        sx, sy = llx, lly
    return dst


def dwt53_reverse(c, w, h, levels):
    """DWTReverse53::dwt (DWTReverse53.cpp:23-43): the deepest level first,
    each level's output copied back over the next level's LL block."""
    src = np.ascontiguousarray(c, np.int32).reshape(-1).copy()
    dst = np.zeros_like(src)
    sizes = [(w, h)]
    for _ in range(levels - 1):
        sizes.append(((sizes[-1][0] + 1) // 2, (sizes[-1][1] + 1) // 2))
    for i in range(levels - 1, -1, -1):
        sx, sy = sizes[i]
        if i < levels - 1:   # copyLLBandToSrc: the deeper level's output is this level's LL block
            llx, lly = sizes[i + 1]
            src[: llx * lly] = dst[: llx * lly]
        _level("r", src, dst, sx, sy)
    return dst.reshape(h, w)


def _band_offsets(sx, sy):
    llx, lly, hx, hy = (sx + 1) // 2, (sy + 1) // 2, sx // 2, sy // 2
    return {"LL": (0, llx, lly), "HL": (llx * lly, hx, lly), "LH": (lly * sx, llx, hy),
            "HH": (llx * lly + (sx * sy) // 2, hx, hy)}


def mallat_to_packed(m, levels):
    """Mallat-layout coefficients [h, w] -> the reference's band-packed layout."""
    h, w = m.shape
    out = np.zeros(w * h, np.int32)
    sx, sy = w, h
    for lvl in range(levels):
        llx, lly = (sx + 1) // 2, (sy + 1) // 2
        bo = _band_offsets(sx, sy)
        for name, (x0, y0) in (("HL", (llx, 0)), ("LH", (0, lly)), ("HH", (llx, lly))):
            off, bw, bh = bo[name]
            out[off: off + bw * bh] = m[y0: y0 + bh, x0: x0 + bw].reshape(-1)
        if lvl + 1 == levels:
            out[: llx * lly] = m[:lly, :llx].reshape(-1)
        sx, sy = llx, lly
    return out


def packed_to_mallat(p, w, h, levels):
    """The reference's band-packed layout -> Mallat-layout [h, w]."""
    p = np.asarray(p, np.int32).reshape(-1)
    m = np.zeros((h, w), np.int32)
    sx, sy = w, h
    for lvl in range(levels):
        llx, lly = (sx + 1) // 2, (sy + 1) // 2
        bo = _band_offsets(sx, sy)
        for name, (x0, y0) in (("HL", (llx, 0)), ("LH", (0, lly)), ("HH", (llx, lly))):
            off, bw, bh = bo[name]
            m[y0: y0 + bh, x0: x0 + bw] = p[off: off + bw * bh].reshape(bh, bw)
        if lvl + 1 == levels:
            m[:lly, :llx] = p[: llx * lly].reshape(lly, llx)
        sx, sy = llx, lly
    return m


def dwt53_defect_mask(w, h, forward):
    """Samples of one 5/3 level that the reference kernels compute wrongly
    (True), found by running them: the forward kernel's topmost window
    loads image rows 0, 1, 2 where whole-sample symmetric extension needs
    2, 1, 0 (initFDWT53Column, dwt_f53.cl:30-41), which spoils the first two
    rows of LL and HL and the first row of LH and HH (packed layout); the
    reverse kernel gets the last image row wrong when the height is even
    (h x w image layout).  Widths that are not a multiple of the kernels'
    window read local memory that no work-item wrote, so those results are
    undefined; only window-multiple widths are compared."""
    if not forward:
        mk = np.zeros((h, w), bool)
        if h % 2 == 0:   # the last row is a high-pass row only for even heights
            mk[h - 1, :] = True
        return mk
    mk = np.zeros(w * h, bool)
    bo = _band_offsets(w, h)
    for name, rows in (("LL", 2), ("HL", 2), ("LH", 1), ("HH", 1)):
        off, bw, bh = bo[name]
        mk[off: off + min(rows, bh) * bw] = True
    return mk
