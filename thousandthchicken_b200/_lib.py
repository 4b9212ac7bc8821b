"""ctypes binding of libtc_j2k.so (the C ABI declared in include/tc_j2k.h).

The library is loaded from the package directory.  There is no CPU fallback:
if the library is missing, every entry point raises ``LibraryMissing``.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libtc_j2k.so"

TC_OK = 0
TC_E_ARG = -1
TC_E_OOM = -2
TC_E_CODESTREAM = -3
TC_E_DEVICE = -4
TC_E_TIMEOUT = -5
TC_E_UNSUPPORTED = -6
TC_E_NOFILE = -7

TC_U8, TC_U16, TC_INT32, TC_FLOAT32 = 1, 2, 3, 4
TC_CBLK_IRREVERSIBLE = 1
TC_T1_OUT_DEQUANT, TC_T1_OUT_RAW, TC_T1_STYLED = 0, 1, 0x10
TC_ROUND_FLOOR, TC_ROUND_TRUNC = 0, 1
TC_COLOR_DC, TC_COLOR_RCT, TC_COLOR_ICT = 0, 1, 2
TC_DWT_CPASYNC, TC_DWT_TMA = 0, 1


class LibraryMissing(RuntimeError):
    pass


class TCError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"{status} ({_status_name(status)}): {msg}")


def _status_name(s: int) -> str:
    return {0: "ok", -1: "invalid argument", -2: "out of memory", -3: "malformed codestream",
            -4: "CUDA error", -5: "device wait timed out", -6: "unsupported codestream feature",
            -7: "file not found"}.get(s, "unknown")


class CblkDesc(C.Structure):
    """tc_cblk_desc (include/tc_j2k.h); 40 bytes."""
    _fields_ = [("seg_off", C.c_uint64), ("out_off", C.c_uint64), ("seg_len", C.c_uint32),
                ("out_pitch", C.c_uint32), ("step", C.c_float), ("w", C.c_uint16), ("h", C.c_uint16),
                ("passes", C.c_uint8), ("mb", C.c_uint8), ("zero_bitplanes", C.c_uint8),
                ("orient", C.c_uint8), ("flags", C.c_uint8), ("style", C.c_uint8), ("roi_shift", C.c_uint8),
                ("reserved", C.c_uint8 * 1)]


class ImageInfo(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("width", "height", "ncomp", "bits", "is_signed", "levels",
                                        "reversible", "mct", "cblk_w", "cblk_h", "layers", "progression",
                                        "guard_bits", "quant_style")] + \
               [("ncblk", C.c_uint32), ("ntiles", C.c_uint32), ("comp_dx", C.c_uint8 * 4),
                ("comp_dy", C.c_uint8 * 4)]


class TileInfo(C.Structure):
    _fields_ = [("x0", C.c_int32), ("y0", C.c_int32), ("w", C.c_int32), ("h", C.c_int32),
                ("coef_off", C.c_uint64)]


class Parsed(C.Structure):
    _fields_ = [("info", ImageInfo), ("desc", C.POINTER(CblkDesc)), ("pool", C.POINTER(C.c_uint8)),
                ("pool_len", C.c_uint64), ("pool_is_cs", C.c_int32), ("reserved", C.c_int32),
                ("tiles", C.POINTER(TileInfo))]


class EncodeParams(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("ncomp", C.c_int32), ("bits", C.c_int32),
                ("levels", C.c_int32), ("reversible", C.c_int32), ("mct", C.c_int32),
                ("cblk_log2", C.c_int32), ("base_step", C.c_double), ("guard_bits", C.c_int32),
                ("progression", C.c_int32), ("threads", C.c_int32), ("is_signed", C.c_int32),
                ("comp_cblk_log2", C.c_int32 * 4), ("comp_step_scale", C.c_double * 4),
                ("comp_dx", C.c_int32 * 4), ("comp_dy", C.c_int32 * 4), ("cblk_style", C.c_int32),
                ("layers", C.c_int32), ("packed_headers", C.c_int32), ("roi_x0", C.c_int32),
                ("roi_y0", C.c_int32), ("roi_x1", C.c_int32), ("roi_y1", C.c_int32)]


assert C.sizeof(CblkDesc) == 40


_VP = C.c_void_p
_I = C.c_int
_PROTOS = {
    "tc_version": (_I, []),
    "tc_status_string": (C.c_char_p, [_I]),
    "tc_ctx_create": (_I, [_I, _VP, C.POINTER(_VP)]),
    "tc_ctx_destroy": (_I, [_VP]),
    "tc_ctx_synchronize": (_I, [_VP]),
    "tc_ctx_last_error": (C.c_char_p, [_VP]),
    "tc_ctx_launch_count": (C.c_uint64, [_VP]),
    "tc_ctx_set_t1_group": (_I, [_VP, _I]),
    "tc_ctx_t1_group": (_I, [_VP]),
    "tc_ctx_set_dwt_variant": (_I, [_VP, _I]),
    "tc_ctx_dwt_variant": (_I, [_VP]),
    "tc_ctx_pool_bytes": (_I, [_VP, C.POINTER(C.c_size_t)]),
    "tc_ctx_trim": (_I, [_VP]),
    "tc_ctx_stream": (_VP, [_VP]),
    "tc_t1_decode": (_I, [_VP, _VP, _VP, _I, _VP, C.c_uint64, _VP, C.c_uint64, _I, C.c_float, _I]),
    "tc_t1_sort_order": (_I, [_VP, _I, _VP]),
    "tc_dequantize_raw": (_I, [_VP, _VP, _I, _VP, _VP, C.c_uint64, C.c_float]),
    "tc_dwt_forward53": (_I, [_VP, _VP, _I, _VP, _I, _I, _I, _I, _I]),
    "tc_dwt_forward97": (_I, [_VP, _VP, _I, _VP, _I, _I, _I, _I]),
    "tc_dwt_reverse53": (_I, [_VP, _VP, _I, _VP, _I, _I, _I, _I, _I]),
    "tc_dwt_reverse97": (_I, [_VP, _VP, _I, _VP, _I, _I, _I, _I]),
    "tc_dwt_reverse97_static": (_I, [_VP, _I, _VP, _I, _I, _I, _I, _VP]),
    "tc_color_inverse": (_I, [_VP, _I, _I, _VP, _I, _I, _VP, _I, _I, _I, _I, _I]),
    "tc_color_forward": (_I, [_VP, _I, _I, _VP, _I, _I, _VP, _I, _I, _I, _I, _I]),
    "tc_j2k_read_header": (_I, [_VP, C.c_size_t, C.POINTER(ImageInfo)]),
    "tc_j2k_parse": (_I, [_VP, C.c_size_t, C.POINTER(C.POINTER(Parsed))]),
    "tc_j2k_parsed_free": (None, [C.POINTER(Parsed)]),
    "tc_decode_j2k": (_I, [_VP, _VP, C.c_size_t, _VP, C.c_size_t, C.POINTER(ImageInfo)]),
    "tc_decode_j2k_file": (_I, [_VP, C.c_char_p, _VP, C.c_size_t, C.POINTER(ImageInfo)]),
    "tc_plan_create": (_I, [_VP, _VP, _VP, _I, C.POINTER(_VP)]),
    "tc_plan_destroy": (_I, [_VP]),
    "tc_plan_rebuild": (_I, [_VP, _VP, _VP, _I]),
    "tc_plan_rebuild_parsed": (_I, [_VP, _VP, _I]),
    "tc_plan_output_bytes": (_I, [_VP, _I, C.POINTER(C.c_size_t)]),
    "tc_plan_image_info": (_I, [_VP, _I, C.POINTER(ImageInfo)]),
    "tc_plan_execute": (_I, [_VP, _VP]),
    "tc_plan_set_profiling": (_I, [_VP, _I]),
    "tc_plan_set_graph": (_I, [_VP, _I]),
    "tc_plan_device_bytes": (_I, [_VP, C.POINTER(C.c_size_t)]),
    "tc_plan_graph_stats": (_I, [_VP, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "tc_plan_stage_ms": (_I, [_VP, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "tc_encode_j2k": (_I, [C.POINTER(EncodeParams), _VP, _VP, C.c_size_t, C.POINTER(C.c_size_t)]),
    "tc_t1_encode_block": (_I, [_VP, _I, _I, _I, _I, _I, _VP, _I, C.POINTER(_I), C.POINTER(_I),
                                C.POINTER(_I)]),
    "tc_t1_encode": (_I, [_VP, _VP, _I, _VP, _VP, C.c_uint32, _VP]),
    "tc_encode_j2k_gpu": (_I, [_VP, C.POINTER(EncodeParams), _VP, _VP, C.c_size_t, C.POINTER(C.c_size_t)]),
}

_lib = None


def lib():
    """Load libtc_j2k.so once; raise LibraryMissing when it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("TC_J2K_LIB", LIB_PATH))
    if not path.exists():
        raise LibraryMissing(f"{path} is not built: run `python -m thousandthchicken_b200.build`")
    L = C.CDLL(str(path))
    for name, (res, args) in _PROTOS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status: int, ctx=None, what: str = "") -> None:
    if status != TC_OK:
        msg = what
        if ctx:
            detail = lib().tc_ctx_last_error(ctx)
            if detail:
                msg = f"{what}: {detail.decode(errors='replace')}"
        raise TCError(status, msg)


def exported_symbols():
    return sorted(_PROTOS)
