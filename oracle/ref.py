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
