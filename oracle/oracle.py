"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: tests, the smoke check and the benchmark's CPU
baseline leg use this module to check the CUDA product path; the product
never imports it.  Each function restates the reference algorithm cited in
oracle/j2k_oracle.h.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SO = HERE / "liboracle.so"

_lib = None


class OrCblk(C.Structure):
    _fields_ = [("seg_off", C.c_uint64), ("seg_len", C.c_uint32), ("w", C.c_uint16), ("h", C.c_uint16),
                ("passes", C.c_uint8), ("mb", C.c_uint8), ("zero_bitplanes", C.c_uint8), ("orient", C.c_uint8),
                ("comp", C.c_uint8), ("flags", C.c_uint8), ("style", C.c_uint8), ("roi", C.c_uint8),
                ("out_x", C.c_uint32), ("out_y", C.c_uint32), ("step", C.c_float)]


def build() -> Path:
    if not SO.exists() or SO.stat().st_mtime < max((HERE / "j2k_oracle.c").stat().st_mtime,
                                                    (HERE / "j2k_oracle.h").stat().st_mtime):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return SO


def lib():
    global _lib
    if _lib is None:
        if not SO.exists():
            build()
        L = C.CDLL(str(SO))
        P = C.c_void_p
        I = C.c_int
        L.or_t1_decode.argtypes = [P, I, I, I, I, I, I, P, P]
        L.or_t1_decode_raw.argtypes = [P, I, I, I, I, I, I, I, P, I]
        L.or_dequant_int.argtypes = [P, P, I, C.c_float, P]
        L.or_dequant_float.argtypes = [P, P, I, C.c_float, C.c_double, P]
        L.or_dequant_raw_int.argtypes = [P, I, I, P]
        for n in ("or_fdwt53", "or_idwt53"):
            getattr(L, n).argtypes = [P, I, I, I, I, I]
        for n in ("or_fdwt97", "or_idwt97"):
            getattr(L, n).argtypes = [P, I, I, I, I]
        L.or_subband_norm.argtypes = [I, I, I]
        L.or_subband_norm.restype = C.c_double
        L.or_rct_forward.argtypes = [P, P, P, C.c_size_t, I]
        L.or_rct_inverse.argtypes = [P, P, P, C.c_size_t, I]
        L.or_ict_forward.argtypes = [P, P, P, P, P, P, C.c_size_t, I]
        L.or_ict_inverse.argtypes = [P, P, P, P, P, P, C.c_size_t, I]
        L.or_dc_forward.argtypes = [P, C.c_size_t, I]
        L.or_dc_inverse_clamp.argtypes = [P, C.c_size_t, I]
        L.or_dc_inverse_float.argtypes = [P, P, C.c_size_t, I]
        L.or_decode_tile.argtypes = [P, I, P, I, I, I, I, I, I, I, C.c_float, I, P]
        L.or_decode_tile_f64.argtypes = [P, I, P, I, I, I, I, I, I, I, C.c_float, I, P, P]
        L.or_t1_encode.argtypes = [P, I, I, I, I, P, I, P, P, P]
        L.or_encode_tile.argtypes = [P, I, I, I, I, I, I, I, C.c_double, I, I, P, P, P, P]
        L.or_encoded_free.argtypes = [P, P]
        L.or_encoded_free.restype = None
        L.or_t1_truncate.argtypes = [P, I, I, I, P]
        L.or_t1_truncate.restype = None
        L.or_t1_truncate_batch.argtypes = [P, P, P, P, P, I, I, P]
        L.or_t1_truncate_batch.restype = None
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def t1_decode(seg: bytes, w: int, h: int, orient: int, numbps: int, passes: int):
    """Returns (q int32[h,w], undecoded uint8[h,w])."""
    q = np.zeros((h, w), np.int32)
    u = np.zeros((h, w), np.uint8)
    buf = np.frombuffer(bytes(seg) or b"\0", np.uint8)
    rc = lib().or_t1_decode(_p(buf), len(seg), w, h, orient, numbps, passes, _p(q), _p(u))
    if rc:
        raise ValueError(f"or_t1_decode failed: {rc}")
    return q, u


def t1_decode_raw(seg: bytes, w: int, h: int, orient: int, mb: int, zbp: int, passes: int):
    out = np.zeros((h, w), np.uint32)
    buf = np.frombuffer(bytes(seg) or b"\0", np.uint8)
    rc = lib().or_t1_decode_raw(_p(buf), len(seg), w, h, orient, mb, zbp, passes, _p(out), w)
    if rc:
        raise ValueError(f"or_t1_decode_raw failed: {rc}")
    return out


def dequant_int(q, u, r=0.0):
    q = np.ascontiguousarray(q, np.int32)
    u = np.ascontiguousarray(u, np.uint8)
    out = np.empty_like(q)
    lib().or_dequant_int(_p(q), _p(u), q.size, r, _p(out))
    return out


def dequant_float(q, u, r, step):
    q = np.ascontiguousarray(q, np.int32)
    u = np.ascontiguousarray(u, np.uint8)
    out = np.empty(q.shape, np.float32)
    lib().or_dequant_float(_p(q), _p(u), q.size, r, step, _p(out))
    return out


def fdwt53(x, levels, rounding=0):
    a = np.ascontiguousarray(x, np.int32).copy()
    h, w = a.shape
    lib().or_fdwt53(_p(a), w, h, w, levels, rounding)
    return a


def idwt53(x, levels, rounding=0):
    a = np.ascontiguousarray(x, np.int32).copy()
    h, w = a.shape
    lib().or_idwt53(_p(a), w, h, w, levels, rounding)
    return a


def fdwt97(x, levels):
    a = np.ascontiguousarray(x, np.float64).copy()
    h, w = a.shape
    lib().or_fdwt97(_p(a), w, h, w, levels)
    return a


def idwt97(x, levels):
    a = np.ascontiguousarray(x, np.float64).copy()
    h, w = a.shape
    lib().or_idwt97(_p(a), w, h, w, levels)
    return a


def subband_norm(wavelet97: bool, level: int, orient: int) -> float:
    return lib().or_subband_norm(1 if wavelet97 else 0, level, orient)


def rct_forward(planes, bits):
    p = [np.ascontiguousarray(c, np.int32).copy() for c in planes[:3]]
    lib().or_rct_forward(_p(p[0]), _p(p[1]), _p(p[2]), p[0].size, bits)
    return p


def rct_inverse(planes, bits):
    p = [np.ascontiguousarray(c, np.int32).copy() for c in planes[:3]]
    lib().or_rct_inverse(_p(p[0]), _p(p[1]), _p(p[2]), p[0].size, bits)
    return p


def ict_forward(planes, bits):
    src = [np.ascontiguousarray(c, np.int32) for c in planes[:3]]
    out = [np.empty(src[0].shape, np.float64) for _ in range(3)]
    lib().or_ict_forward(*map(_p, src), *map(_p, out), src[0].size, bits)
    return out


def ict_inverse(planes, bits):
    src = [np.ascontiguousarray(c, np.float64) for c in planes[:3]]
    out = [np.empty(src[0].shape, np.int32) for _ in range(3)]
    lib().or_ict_inverse(*map(_p, src), *map(_p, out), src[0].size, bits)
    return out


def dc_forward(x, bits):
    a = np.ascontiguousarray(x, np.int32).copy()
    lib().or_dc_forward(_p(a), a.size, bits)
    return a


def dc_inverse_clamp(x, bits):
    a = np.ascontiguousarray(x, np.int32).copy()
    lib().or_dc_inverse_clamp(_p(a), a.size, bits)
    return a


def dc_inverse_float(x, bits):
    a = np.ascontiguousarray(x, np.float64)
    out = np.empty(a.shape, np.int32)
    lib().or_dc_inverse_float(_p(a), _p(out), a.size, bits)
    return out


def decode_tile(cblks, pool: np.ndarray, w, h, ncomp, bits, levels, reversible, mct, r=0.5, threads=0,
                signed=False):
    """Whole-tile decode from parsed code-block descriptors (numpy structured
    rows with the tc_cblk_desc fields of one image).  Returns uint16
    [ncomp, h, w], or int16 for signed samples (no DC level shift)."""
    arr = cblk_array(cblks, w, h)
    return decode_cblks(arr, len(cblks), pool, w, h, ncomp, bits, levels, reversible, mct, r, threads, signed)[0]


def decode_cblks(arr, n, pool, w, h, ncomp, bits, levels, reversible, mct, r=0.5, threads=0, signed=False,
                 f64=False):
    """or_decode_tile(_f64) over an OrCblk array.  Returns (samples, FP64
    samples before rounding or None): uint16 [ncomp, h, w] (int16 when
    signed) and, with f64 on an irreversible tile, float64 [ncomp, h, w]."""
    out = np.zeros((ncomp, h, w), np.uint16)
    ff = np.zeros((ncomp, h, w), np.float64) if f64 and not reversible else None
    pool = np.ascontiguousarray(pool, np.uint8)
    rc = lib().or_decode_tile_f64(arr, n, _p(pool), w, h, ncomp, bits | (0x100 if signed else 0), levels,
                                  int(reversible), int(mct), r, threads, _p(out),
                                  _p(ff) if ff is not None else None)
    if rc:
        raise ValueError(f"or_decode_tile failed: {rc}")
    return (out.view(np.int16) if signed else out), ff


def cblk_array(cblks, w, h):
    """OrCblk array from numpy rows with the tc_cblk_desc fields."""
    n = len(cblks)
    arr = (OrCblk * max(n, 1))()
    plane = w * h
    for i, d in enumerate(cblks):
        c = arr[i]
        off = int(d["out_off"])
        comp, rem = divmod(off, plane)
        oy, ox = divmod(rem, w)
        c.seg_off = int(d["seg_off"])
        c.seg_len = int(d["seg_len"])
        c.w, c.h = int(d["w"]), int(d["h"])
        c.passes, c.mb, c.zero_bitplanes, c.orient = (int(d["passes"]), int(d["mb"]), int(d["zero_bitplanes"]),
                                                      int(d["orient"]))
        c.comp = comp
        if "style" in (d.dtype.names or ()):
            c.style = int(d["style"])
        if "roi_shift" in (d.dtype.names or ()):
            c.roi = int(d["roi_shift"])
        c.out_x, c.out_y = ox, oy
        c.step = float(d["step"])
    return arr


def t1_encode(coef, orient: int, passes: int = 0):
    """Encode one code-block (ISO C.2 / D.3 encoder); returns (codeword
    bytes, passes kept, coded bit-planes)."""
    coef = np.ascontiguousarray(coef, np.int32)
    h, w = coef.shape
    cap = 16 * w * h + 1024
    out = np.empty(cap, np.uint8)
    n, np_, nb = C.c_int(0), C.c_int(0), C.c_int(0)
    rc = lib().or_t1_encode(_p(coef), w, h, orient, passes, _p(out), cap, C.byref(n), C.byref(np_), C.byref(nb))
    if rc:
        raise ValueError(f"or_t1_encode failed: {rc}")
    return out[:n.value].tobytes(), np_.value, nb.value


def t1_truncate(coef, passes: int):
    """The coefficients a decoder reconstructs from the first `passes`
    coding passes (ISO D.3 pass membership, no MQ coding)."""
    coef = np.ascontiguousarray(coef, np.int32)
    h, w = coef.shape
    out = np.empty_like(coef)
    lib().or_t1_truncate(_p(coef), w, h, passes, _p(out))
    return out


def t1_truncate_batch(coef, off, w, h, passes, threads=0):
    """t1_truncate over blocks stored one after another in a flat int32
    array (block i at element off[i], pitch w[i])."""
    coef = np.ascontiguousarray(coef, np.int32)
    off = np.ascontiguousarray(off, np.uint64)
    w = np.ascontiguousarray(w, np.uint16)
    h = np.ascontiguousarray(h, np.uint16)
    passes = np.ascontiguousarray(passes, np.uint8)
    out = np.empty_like(coef)
    lib().or_t1_truncate_batch(_p(coef), _p(off), _p(w), _p(h), _p(passes), len(off), threads, _p(out))
    return out


class EncodedTile:
    """The oracle's own encode of a tile: OrCblk descriptors and their pool."""

    def __init__(self, arr, n, pool, w, h, ncomp, bits, levels, reversible, mct):
        self.arr, self.n, self.pool = arr, n, pool
        self.w, self.h, self.ncomp, self.bits = w, h, ncomp, bits
        self.levels, self.reversible, self.mct = levels, reversible, mct

    def decode(self, r=0.5, threads=0, f64=False):
        return decode_cblks(self.arr, self.n, self.pool, self.w, self.h, self.ncomp, self.bits, self.levels,
                            self.reversible, self.mct, r, threads, False, f64)

    def blocks(self):
        """{(comp, out_x, out_y): (codeword bytes, w, h, passes, numbps, orient, step)}"""
        out = {}
        for i in range(self.n):
            c = self.arr[i]
            seg = self.pool[c.seg_off:c.seg_off + c.seg_len].tobytes()
            out[(c.comp, c.out_x, c.out_y)] = (seg, c.w, c.h, c.passes, c.mb - c.zero_bitplanes, c.orient, c.step)
        return out


def encode_tile(img, bits, levels, reversible, mct, base_step=1.0 / 128, cblk=64, threads=0) -> EncodedTile:
    """or_encode_tile on planar unsigned samples [ncomp, h, w]."""
    a = np.ascontiguousarray(img, np.uint16)
    if a.ndim == 2:
        a = a[None]
    ncomp, h, w = a.shape
    pc, n, pp, pl = C.c_void_p(), C.c_int(0), C.c_void_p(), C.c_size_t(0)
    rc = lib().or_encode_tile(_p(a), w, h, ncomp, bits, levels, int(reversible), int(mct), base_step, cblk, threads,
                              C.byref(pc), C.byref(n), C.byref(pp), C.byref(pl))
    if rc:
        raise ValueError(f"or_encode_tile failed: {rc}")
    try:
        arr = (OrCblk * max(n.value, 1))()
        if n.value:
            C.memmove(arr, pc, C.sizeof(OrCblk) * n.value)
        pool = np.empty(max(pl.value, 16), np.uint8)
        if pl.value:
            C.memmove(pool.ctypes.data, pp, pl.value)
    finally:
        lib().or_encoded_free(pc, pp)
    return EncodedTile(arr, n.value, pool, w, h, ncomp, bits, levels, reversible, mct)
