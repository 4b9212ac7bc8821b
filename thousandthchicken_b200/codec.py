"""Host-side codestream helpers over libtc_j2k: header reading, Tier-2 parsing
into code-block descriptors, and the harness encoder.  No GPU is needed for
anything in this module."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

# numpy view of tc_cblk_desc (include/tc_j2k.h)
DESC_DTYPE = np.dtype([("seg_off", "<u8"), ("out_off", "<u8"), ("seg_len", "<u4"), ("out_pitch", "<u4"),
                       ("step", "<f4"), ("w", "<u2"), ("h", "<u2"), ("passes", "u1"), ("mb", "u1"),
                       ("zero_bitplanes", "u1"), ("orient", "u1"), ("flags", "u1"), ("style", "u1"),
                       ("roi_shift", "u1"), ("reserved", "u1", (1,))])
assert DESC_DTYPE.itemsize == 40

INFO_FIELDS = ("width", "height", "ncomp", "bits", "is_signed", "levels", "reversible", "mct", "cblk_w",
               "cblk_h", "layers", "progression", "guard_bits", "quant_style", "ncblk", "ntiles")


def _info_dict(info: L.ImageInfo) -> dict:
    d = {k: int(getattr(info, k)) for k in INFO_FIELDS}
    n = d["ncomp"]
    d["subsampling"] = [(int(info.comp_dx[c]), int(info.comp_dy[c])) for c in range(n)]
    d["comp_sizes"] = [(-(-d["height"] // dy), -(-d["width"] // dx)) for dx, dy in d["subsampling"]]
    return d


def _buf(data) -> np.ndarray:
    return np.frombuffer(bytes(data), np.uint8) if not isinstance(data, np.ndarray) else \
        np.ascontiguousarray(data, np.uint8)


def read_header(cs) -> dict:
    a = _buf(cs)
    info = L.ImageInfo()
    L.check(L.lib().tc_j2k_read_header(a.ctypes.data, a.size, C.byref(info)), what="tc_j2k_read_header")
    return _info_dict(info)


# tc_t1_enc_desc / tc_t1_enc_result (tc_j2k.h)
ENC_DESC_DTYPE = np.dtype([("in_off", "<u8"), ("in_pitch", "<u4"), ("inv_step", "<f4"), ("w", "<u2"), ("h", "<u2"),
                           ("orient", "u1"), ("mb", "u1"), ("flags", "u1"), ("max_passes", "u1")])
ENC_RESULT_DTYPE = np.dtype([("len", "<u4"), ("passes", "<u4"), ("zero_bitplanes", "<u4"), ("status", "<u4")])
assert ENC_DESC_DTYPE.itemsize == 24 and ENC_RESULT_DTYPE.itemsize == 16


def parse(cs):
    """Parse a codestream: returns (info dict, descriptor array, segment pool).
    info["tiles"] lists each tile as (x0, y0, w, h, coef_off): its region of
    the image and the element offset of its planes in the tile-major
    coefficient arena the descriptors' out_off address."""
    a = _buf(cs)
    out = C.POINTER(L.Parsed)()
    L.check(L.lib().tc_j2k_parse(a.ctypes.data, a.size, C.byref(out)), what="tc_j2k_parse")
    try:
        p = out.contents
        info = _info_dict(p.info)
        info["tiles"] = [(t.x0, t.y0, t.w, t.h, t.coef_off) for t in p.tiles[:info["ntiles"]]]
        info["pool_is_cs"] = int(p.pool_is_cs)  # segments read in place from the codestream
        n = info["ncblk"]
        desc = np.empty(n, DESC_DTYPE)
        if n:
            C.memmove(desc.ctypes.data, p.desc, n * DESC_DTYPE.itemsize)
        if p.pool_is_cs:
            pool = a.copy()
        else:
            pool = np.empty(p.pool_len, np.uint8)
            if p.pool_len:
                C.memmove(pool.ctypes.data, p.pool, p.pool_len)
    finally:
        L.lib().tc_j2k_parsed_free(out)
    return info, desc, pool


# Code-block style bits (COD / COC SPcod, ISO Table A.19).
CBLK_STYLE_BYPASS, CBLK_STYLE_RESET, CBLK_STYLE_TERMALL = 0x01, 0x02, 0x04
CBLK_STYLE_VSC, CBLK_STYLE_PTERM, CBLK_STYLE_SEGSYM = 0x08, 0x10, 0x20


def _encode_params(planes, bits, levels, reversible, mct, cblk_log2, base_step, guard_bits, progression, threads,
                   comp_cblk_log2, comp_step_scale, comp_subsampling=None):
    if comp_subsampling:
        # a list of component planes of their own sizes: ceil(w/dx) x ceil(h/dy)
        comps = [np.asarray(a) for a in planes]
        signed = comps[0].dtype.kind == "i"
        dt = (np.int8 if bits <= 8 else np.int16) if signed else (np.uint8 if bits <= 8 else np.uint16)
        ncomp = len(comps)
        dxy = list(comp_subsampling) + [(1, 1)] * (ncomp - len(comp_subsampling))
        # the image size: a component at 1:1, else what the first one implies
        full = [i for i, (a, b) in enumerate(dxy) if a == 1 and b == 1]
        if full:
            h, w = comps[full[0]].shape
        else:
            h, w = comps[0].shape[0] * dxy[0][1], comps[0].shape[1] * dxy[0][0]
        for a, (dx, dy) in zip(comps, dxy):
            if a.shape != (-(-h // dy), -(-w // dx)):
                raise ValueError(f"component of shape {a.shape} does not match {w}x{h} at {dx}x{dy}")
        planes = np.concatenate([np.ascontiguousarray(a, dt).reshape(-1) for a in comps])
    else:
        signed = np.asarray(planes).dtype.kind == "i"
        if signed:
            planes = np.ascontiguousarray(planes, np.int8 if bits <= 8 else np.int16)
        else:
            planes = np.ascontiguousarray(planes, np.uint8 if bits <= 8 else np.uint16)
        if planes.ndim == 2:
            planes = planes[None]
        ncomp, h, w = planes.shape
        dxy = [(1, 1)] * ncomp
    p = L.EncodeParams(width=w, height=h, ncomp=ncomp, bits=bits, levels=levels, reversible=int(reversible),
                       mct=int(mct), cblk_log2=cblk_log2, base_step=base_step, guard_bits=guard_bits,
                       progression=progression, threads=threads, is_signed=int(signed))
    for c, v in enumerate(comp_cblk_log2 or []):
        p.comp_cblk_log2[c] = int(v)
    for c, v in enumerate(comp_step_scale or []):
        p.comp_step_scale[c] = float(v)
    for c, (dx, dy) in enumerate(dxy):
        p.comp_dx[c], p.comp_dy[c] = int(dx), int(dy)
    return planes, p


def encode_gpu(ctx, planes: np.ndarray, bits: int, levels: int = 5, reversible: bool = True, mct: bool = True,
               cblk_log2: int = 6, base_step: float = 1.0 / 128, guard_bits: int = 0, progression: int = 0,
               comp_cblk_log2=None, comp_step_scale=None, layers: int = 1, packed_headers: int = 0) -> bytes:
    """The encoder on the GPU (tc_encode_j2k_gpu): colour transform, DWT,
    quantisation and Tier-1 as kernels on ctx's device, packets on the
    host.  Same parameters as encode (code-block style 0, no region of
    interest); lossless output is byte-identical."""
    planes, p = _encode_params(planes, bits, levels, reversible, mct, cblk_log2, base_step, guard_bits, progression,
                               0, comp_cblk_log2, comp_step_scale)
    p.layers = int(layers)
    p.packed_headers = int(packed_headers)
    cap = planes.nbytes * 3 + 65536
    out = np.empty(cap, np.uint8)
    n = C.c_size_t(0)
    ctx.check(L.lib().tc_encode_j2k_gpu(ctx.handle, C.byref(p), planes.ctypes.data, out.ctypes.data, cap,
                                        C.byref(n)), "tc_encode_j2k_gpu")
    return out[: n.value].tobytes()


def encode(planes: np.ndarray, bits: int, levels: int = 5, reversible: bool = True, mct: bool = True,
           cblk_log2: int = 6, base_step: float = 1.0 / 128, guard_bits: int = 0, progression: int = 0,
           threads: int = 0, comp_cblk_log2=None, comp_step_scale=None, comp_subsampling=None,
           cblk_style: int = 0, layers: int = 1, packed_headers: int = 0, roi=None) -> bytes:
    """Harness encoder: planar samples [ncomp, h, w] -> codestream; signed
    integer arrays (int8 / int16) give signed components (no DC shift).
    comp_cblk_log2 / comp_step_scale: per-component code-block size exponent
    and irreversible step multiplier (0 = the image-wide value), written as
    COC / QCC marker segments.  comp_subsampling: per component (dx, dy);
    planes is then a list of component arrays of ceil(h/dy) x ceil(w/dx).
    cblk_style: code-block style bits (CBLK_STYLE_*) for every component.
    layers: quality layers; each block's passes are split evenly over them
    (all layers together give the whole codeword).
    packed_headers: 0 packet headers in the packets, 1 in PPT marker
    segments, 2 in PPM marker segments.
    roi: (x0, y0, x1, y1), a region of interest in image samples coded with
    the maxshift method (RGN)."""
    planes, p = _encode_params(planes, bits, levels, reversible, mct, cblk_log2, base_step, guard_bits, progression,
                               threads, comp_cblk_log2, comp_step_scale, comp_subsampling)
    p.cblk_style = int(cblk_style)
    p.layers = int(layers)
    p.packed_headers = int(packed_headers)
    if roi is not None:
        p.roi_x0, p.roi_y0, p.roi_x1, p.roi_y1 = (int(v) for v in roi)
    cap = planes.nbytes * 3 + 65536
    out = np.empty(cap, np.uint8)
    n = C.c_size_t(0)
    L.check(L.lib().tc_encode_j2k(C.byref(p), planes.ctypes.data, out.ctypes.data, cap, C.byref(n)),
            what="tc_encode_j2k")
    return out[: n.value].tobytes()


def t1_encode_block(coef: np.ndarray, orient: int, mb: int, passes: int = 0):
    """Encode one code-block; returns (codeword bytes, passes, zero_bitplanes)."""
    coef = np.ascontiguousarray(coef, np.int32)
    h, w = coef.shape
    cap = 16 * w * h + 1024
    out = np.empty(cap, np.uint8)
    n, np_, zb = C.c_int(0), C.c_int(0), C.c_int(0)
    L.check(L.lib().tc_t1_encode_block(coef.ctypes.data, w, h, orient, mb, passes, out.ctypes.data, cap,
                                       C.byref(n), C.byref(np_), C.byref(zb)), what="tc_t1_encode_block")
    return out[: n.value].tobytes(), np_.value, zb.value


def sort_order(desc: np.ndarray) -> np.ndarray:
    desc = np.ascontiguousarray(desc, DESC_DTYPE)
    order = np.empty(len(desc), np.uint32)
    L.check(L.lib().tc_t1_sort_order(desc.ctypes.data, len(desc), order.ctypes.data), what="tc_t1_sort_order")
    return order
