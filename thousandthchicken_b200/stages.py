"""The reference's device-stage classes over libtc_j2k.

Names and call shapes follow kgmoore/ThousandthChicken:
``CoefficientCoder.decode_tile`` (CoefficientCoder.h:37-48),
``Quantizer.dequantize_tile`` (Quantizer.h:9-17), ``DWTForward53/97`` and
``DWTReverse53/97.run(in, out, sizeX, sizeY, levels)`` (DWTKernel.h:11-13),
``DWT.iwt`` (DWT.h:14-18), ``Preprocessor.color_decoder_lossless /
color_decoder_lossy / idc_level_shifting`` (Preprocessor.h:22-24) and
``Decoder.decode`` (Decoder.h:18-20).  Device buffers are torch CUDA tensors
(plain device memory); every call is ordered on the context's CUDA stream.
Errors raise TCError instead of returning cl_int codes; there is no CPU
fallback.
"""
from __future__ import annotations

import ctypes as C
import weakref
from pathlib import Path

import numpy as np

from . import _lib as L
from .codec import DESC_DTYPE, parse

try:
    import torch
except ImportError:  # pragma: no cover - torch is part of the image
    torch = None


def _ptr(t) -> int:
    return int(t.data_ptr())


class Context:
    """A tc_ctx bound to one CUDA device and (by default) torch's current
    stream on it.  Replaces KernelInitInfoBase{cmd_queue, buildOptions}."""

    def __init__(self, device: int = 0, stream=None):
        if torch is None or not torch.cuda.is_available():
            raise L.LibraryMissing("a CUDA device is required (no CPU fallback)")
        self.device = device
        with torch.cuda.device(device):
            self.stream = stream if stream is not None else torch.cuda.current_stream(device)
        h = C.c_void_p()
        L.check(L.lib().tc_ctx_create(device, C.c_void_p(self.stream.cuda_stream), C.byref(h)),
                what="tc_ctx_create")
        self.handle = h
        self._plans = weakref.WeakSet()

    def close(self):
        if getattr(self, "handle", None):
            for plan in list(getattr(self, "_plans", ())):
                plan.close()
            L.lib().tc_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        L.check(L.lib().tc_ctx_synchronize(self.handle), self.handle, "tc_ctx_synchronize")

    @property
    def launches(self) -> int:
        return int(L.lib().tc_ctx_launch_count(self.handle))

    def check(self, status: int, what: str):
        L.check(status, self.handle, what)


# code-block style bits that change decoding (all but PTERM)
STYLE_DECODE_BITS = 0x2F


def _dev_bytes(arr: np.ndarray, device) -> "torch.Tensor":
    return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8).reshape(-1)).to(device, non_blocking=False)


class CoefficientCoder:
    """Tier-1 EBCOT/MQ decoding of code-blocks (CoefficientCoder.cpp:62-252),
    one warp per code-block in one persistent launch, with the inverse
    quantiser fused into the store unless raw output is asked for."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def decode(self, desc_dev, pool_dev, out, n: int, order_dev=None, raw: bool = False,
               recon_r: float = 0.5, max_bitplanes: int = 0, styled: bool = False):
        """Low-level: descriptors, pool, order and out are device tensors.
        styled: the descriptors may carry code-block styles (decoded by the
        style-capable kernel; without it such blocks are reported as errors)."""
        mode = (L.TC_T1_OUT_RAW if raw else L.TC_T1_OUT_DEQUANT) | (L.TC_T1_STYLED if styled else 0)
        self.ctx.check(L.lib().tc_t1_decode(self.ctx.handle, _ptr(desc_dev),
                                            _ptr(order_dev) if order_dev is not None else None, n,
                                            _ptr(pool_dev), pool_dev.numel(), _ptr(out),
                                            out.numel() * out.element_size() // 4, mode, recon_r, max_bitplanes),
                       "tc_t1_decode")

    def decode_blocks(self, desc: np.ndarray, pool: np.ndarray, out_elems: int, raw: bool = False,
                      recon_r: float = 0.5, sort: bool = True, dtype=None):
        """Host convenience: upload descriptors and pool, decode into a new
        device tensor of out_elems 4-byte elements (int32, float32 or uint32
        raw words), and return it."""
        dev = torch.device("cuda", self.ctx.device)
        desc = np.ascontiguousarray(desc, DESC_DTYPE)
        d_desc = _dev_bytes(desc, dev)
        d_pool = _dev_bytes(pool if len(pool) else np.zeros(16, np.uint8), dev)
        d_order = None
        if sort and len(desc):
            from .codec import sort_order
            d_order = torch.from_numpy(sort_order(desc).view(np.int32)).to(dev)
        if dtype is None:
            dtype = torch.int32 if raw or not (len(desc) and desc["flags"][0] & 1) else torch.float32
        out = torch.zeros(max(out_elems, 1), dtype=dtype, device=dev)
        nb = desc["mb"].astype(np.int32) - desc["zero_bitplanes"].astype(np.int32)
        maxb = int(np.clip(nb[desc["passes"] > 0], 0, 31).max()) if (desc["passes"] > 0).any() else 1
        styled = bool(len(desc) and (desc["style"] & STYLE_DECODE_BITS).any())
        self.decode(d_desc, d_pool, out, len(desc), d_order, raw, recon_r, max(maxb, 1), styled)
        self.ctx.synchronize()
        return out

    def decode_tile(self, cs: bytes, raw: bool = False, recon_r: float = 0.5):
        """Parse a codestream and decode all its code-blocks into Mallat
        planes [ncomp, h, w] (int32 lossless / float32 lossy, or raw words)."""
        info, desc, pool = parse(cs)
        n = info["ncomp"] * info["width"] * info["height"]
        dtype = torch.int32 if (raw or info["reversible"]) else torch.float32
        out = self.decode_blocks(desc, pool, n, raw=raw, recon_r=recon_r, dtype=dtype)
        return out.view(info["ncomp"], info["height"], info["width"]), info


class T1Encoder:
    """GPU Tier-1 encoder (tc_t1_encode): code-blocks of a device plane set
    -> codewords, bit-exact with the host encoder (codec.t1_encode_block)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def encode(self, desc: np.ndarray, planes, cap: int = 0):
        """desc: ENC_DESC_DTYPE rows addressing `planes` (a device tensor of
        int32 quantised coefficients, or float32 with TC_CBLK_IRREVERSIBLE).
        Returns a list of (codeword bytes, passes, zero_bitplanes)."""
        from .codec import ENC_DESC_DTYPE, ENC_RESULT_DTYPE
        dev = torch.device("cuda", self.ctx.device)
        desc = np.ascontiguousarray(desc, ENC_DESC_DTYPE)
        n = len(desc)
        if n == 0:
            return []
        if cap <= 0:
            cap = int(max(4096, 8 * int(desc["w"].max()) * int(desc["h"].max())))
        d_desc = _dev_bytes(desc, dev)
        out = torch.empty(n * cap, dtype=torch.uint8, device=dev)
        res = torch.empty(n * ENC_RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        self.ctx.check(L.lib().tc_t1_encode(self.ctx.handle, _ptr(d_desc), n, _ptr(planes), _ptr(out), cap,
                                            _ptr(res)), "tc_t1_encode")
        self.ctx.synchronize()
        r = res.cpu().numpy().view(ENC_RESULT_DTYPE)
        if (r["status"] != 0).any():
            bad = int(np.nonzero(r["status"])[0][0])
            raise L.TCError(L.TC_E_ARG, f"tc_t1_encode: block {bad} status {int(r['status'][bad])}")
        data = out.cpu().numpy()
        return [(data[i * cap:i * cap + int(r["len"][i])].tobytes(), int(r["passes"][i]), int(r["zero_bitplanes"][i]))
                for i in range(n)]

    def encode_device(self, desc: np.ndarray, planes, cap: int):
        """Encode on the device and keep the codewords there: returns (a
        uint8 device tensor holding block i's codeword at i * cap, the
        ENC_RESULT_DTYPE results on the host).  desc may set max_passes per
        block to truncate its codeword."""
        from .codec import ENC_DESC_DTYPE, ENC_RESULT_DTYPE
        dev = torch.device("cuda", self.ctx.device)
        desc = np.ascontiguousarray(desc, ENC_DESC_DTYPE)
        n = len(desc)
        d_desc = _dev_bytes(desc, dev)
        out = torch.empty(max(n, 1) * cap, dtype=torch.uint8, device=dev)
        res = torch.empty(max(n, 1) * ENC_RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        self.ctx.check(L.lib().tc_t1_encode(self.ctx.handle, _ptr(d_desc), n, _ptr(planes), _ptr(out), cap,
                                            _ptr(res)), "tc_t1_encode")
        self.ctx.synchronize()
        r = res.cpu().numpy().view(ENC_RESULT_DTYPE)[:n].copy()
        if (r["status"] != 0).any():
            bad = int(np.nonzero(r["status"])[0][0])
            raise L.TCError(L.TC_E_ARG, f"tc_t1_encode: block {bad} status {int(r['status'][bad])}")
        return out, r


class Quantizer:
    """Standalone inverse quantiser over raw Tier-1 words
    (Quantizer::dequantize_tile, Quantizer.cpp:181-216)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def dequantize(self, desc_dev, n: int, raw, out, recon_r: float = 0.5):
        elems = min(raw.numel() * raw.element_size(), out.numel() * out.element_size()) // 4
        self.ctx.check(L.lib().tc_dequantize_raw(self.ctx.handle, _ptr(desc_dev), n, _ptr(raw), _ptr(out),
                                                 elems, recon_r), "tc_dequantize_raw")


class _DWTKernel:
    wavelet = 0
    forward = False

    def __init__(self, ctx: Context, rounding: int = L.TC_ROUND_FLOOR):
        self.ctx = ctx
        self.rounding = rounding

    def run(self, inp, out, size_x: int, size_y: int, levels: int, in_pitch: int | None = None,
            out_pitch: int | None = None):
        """DWTKernel<T>::run(in, out, sizeX, sizeY, levels) on device tensors
        (Mallat layout on the transformed side)."""
        ip = in_pitch or size_x
        op = out_pitch or size_x
        fn = {(0, True): "tc_dwt_forward53", (1, True): "tc_dwt_forward97",
              (0, False): "tc_dwt_reverse53", (1, False): "tc_dwt_reverse97"}[(self.wavelet, self.forward)]
        args = [self.ctx.handle, _ptr(inp), ip, _ptr(out), op, size_x, size_y, levels]
        if self.wavelet == 0:
            args.append(self.rounding)
        self.ctx.check(getattr(L.lib(), fn)(*args), fn)
        return out


class DWTForward53(_DWTKernel):
    wavelet, forward = 0, True


class DWTForward97(_DWTKernel):
    wavelet, forward = 1, True


class DWTReverse53(_DWTKernel):
    wavelet, forward = 0, False


class DWTReverse97(_DWTKernel):
    wavelet, forward = 1, False


class DWT:
    """DWT::iwt (DWT.cpp:57-114): reverse transform of every component."""

    def __init__(self, ctx: Context):
        self.r53 = DWTReverse53(ctx)
        self.r97 = DWTReverse97(ctx)

    def iwt(self, planes, levels: int, reversible: bool):
        out = torch.empty_like(planes)
        k = self.r53 if reversible else self.r97
        for c in range(planes.shape[0]):
            k.run(planes[c], out[c], planes.shape[2], planes.shape[1], levels)
        return out


def _type_code(t):
    """Sample-type code of a tensor (16-bit samples may be int16 or uint16)."""
    if t.dtype == torch.uint8:
        return L.TC_U8
    if t.dtype == torch.int16 or t.dtype == getattr(torch, "uint16", None):
        return L.TC_U16
    if t.dtype == torch.int32:
        return L.TC_INT32
    if t.dtype == torch.float32:
        return L.TC_FLOAT32
    raise TypeError(f"unsupported dtype {t.dtype}")


class Preprocessor:
    """Colour transforms and DC level shift (Preprocessor.cpp:44-306)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def _inverse(self, kind, planes, out, bits):
        n = len(planes)
        ins = (C.c_void_p * 4)(*[_ptr(p) for p in planes])
        outs = (C.c_void_p * 4)(*[_ptr(o) for o in out])
        h, w = planes[0].shape
        self.ctx.check(L.lib().tc_color_inverse(self.ctx.handle, kind, n, ins, _type_code(planes[0]), w, outs,
                                                _type_code(out[0]), w, w, h, bits), "tc_color_inverse")
        return out

    def _forward(self, kind, planes, out, bits):
        n = len(planes)
        ins = (C.c_void_p * 4)(*[_ptr(p) for p in planes])
        outs = (C.c_void_p * 4)(*[_ptr(o) for o in out])
        h, w = planes[0].shape
        self.ctx.check(L.lib().tc_color_forward(self.ctx.handle, kind, n, ins, _type_code(planes[0]), w, outs,
                                                _type_code(out[0]), w, w, h, bits), "tc_color_forward")
        return out

    def color_decoder_lossless(self, planes, out, bits: int):
        """Inverse RCT + DC shift + clamp (tcr_kernel)."""
        return self._inverse(L.TC_COLOR_RCT, planes, out, bits)

    def color_decoder_lossy(self, planes, out, bits: int):
        """Inverse ICT (ISO G.2) + DC shift + round + clamp (tci_kernel)."""
        return self._inverse(L.TC_COLOR_ICT, planes, out, bits)

    def idc_level_shifting(self, planes, out, bits: int):
        """DC shift + clamp per component (idc_level_shift_kernel)."""
        return self._inverse(L.TC_COLOR_DC, planes, out, bits)

    def color_coder_lossless(self, planes, out, bits: int):
        """Forward DC shift + RCT (rct_kernel)."""
        return self._forward(L.TC_COLOR_RCT, planes, out, bits)

    def color_coder_lossy(self, planes, out, bits: int):
        """Forward DC shift + ICT (ict_kernel)."""
        return self._forward(L.TC_COLOR_ICT, planes, out, bits)

    def dc_level_shifting(self, planes, out, bits: int):
        """Forward DC shift (fdc_level_shift_kernel)."""
        return self._forward(L.TC_COLOR_DC, planes, out, bits)


class Plan:
    """Device-resident decode of one or more codestreams: parsed and uploaded
    once, executed many times (batched Tier-1 and DWT launches)."""

    def __init__(self, ctx: Context, codestreams):
        self.ctx = ctx
        self._bufs = [np.frombuffer(bytes(c), np.uint8) for c in codestreams]
        n = len(self._bufs)
        ptrs = (C.c_void_p * n)(*[b.ctypes.data for b in self._bufs])
        lens = (C.c_size_t * n)(*[b.size for b in self._bufs])
        h = C.c_void_p()
        ctx.check(L.lib().tc_plan_create(ctx.handle, ptrs, lens, n, C.byref(h)), "tc_plan_create")
        self.handle = h
        ctx._plans.add(self)  # destroyed before the context (a plan uses its context's stream and pool)
        self._read_infos(n)

    def _read_infos(self, n):
        from .codec import _info_dict
        self.infos = []
        self.out_bytes = []
        for i in range(n):
            info = L.ImageInfo()
            L.check(L.lib().tc_plan_image_info(self.handle, i, C.byref(info)))
            self.infos.append(_info_dict(info))
            nb = C.c_size_t(0)
            L.check(L.lib().tc_plan_output_bytes(self.handle, i, C.byref(nb)))
            self.out_bytes.append(nb.value)

    def alloc_outputs(self):
        dev = torch.device("cuda", self.ctx.device)
        outs = []
        for info in self.infos:
            if info["bits"] <= 8:
                dt = torch.int8 if info["is_signed"] else torch.uint8
            else:
                dt = torch.int16  # 16-bit samples, unsigned ones read back as uint16
            sizes = info["comp_sizes"]
            if len(set(sizes)) > 1:  # subsampled components: one flat planar buffer (split_components)
                outs.append(torch.empty(sum(h * w for h, w in sizes), dtype=dt, device=dev))
            else:
                outs.append(torch.empty((info["ncomp"], info["height"], info["width"]), dtype=dt, device=dev))
        return outs

    def execute(self, outs):
        ptrs = (C.c_void_p * len(outs))(*[_ptr(o) for o in outs])
        self.ctx.check(L.lib().tc_plan_execute(self.handle, ptrs), "tc_plan_execute")
        return outs

    def set_graph(self, on: bool = True):
        """Replay execute as captured CUDA graphs, one per shape bucket (new
        outputs replay the same graph)."""
        L.check(L.lib().tc_plan_set_graph(self.handle, int(on)), self.ctx.handle, "tc_plan_set_graph")

    def graph_stats(self) -> dict:
        """{"captures", "updates", "replays"} of graph mode."""
        a, b, c = C.c_uint64(0), C.c_uint64(0), C.c_uint64(0)
        L.check(L.lib().tc_plan_graph_stats(self.handle, C.byref(a), C.byref(b), C.byref(c)), self.ctx.handle,
                "tc_plan_graph_stats")
        return {"captures": a.value, "updates": b.value, "replays": c.value}

    def rebuild(self, codestreams):
        """Re-parse for new codestreams, keeping the device buffers (and, in
        graph mode, the cached graphs of earlier shape buckets)."""
        self._bufs = [np.frombuffer(bytes(c), np.uint8) for c in codestreams]
        n = len(self._bufs)
        ptrs = (C.c_void_p * n)(*[b.ctypes.data for b in self._bufs])
        lens = (C.c_size_t * n)(*[b.size for b in self._bufs])
        self.ctx.check(L.lib().tc_plan_rebuild(self.handle, ptrs, lens, n), "tc_plan_rebuild")
        self._read_infos(n)

    def set_profiling(self, on: bool = True):
        L.check(L.lib().tc_plan_set_profiling(self.handle, int(on)), self.ctx.handle, "tc_plan_set_profiling")

    def stage_ms(self):
        """(Tier-1 ms, DWT+colour ms) of the last execute (profiling on)."""
        a, b = C.c_float(0), C.c_float(0)
        L.check(L.lib().tc_plan_stage_ms(self.handle, C.byref(a), C.byref(b)), self.ctx.handle, "tc_plan_stage_ms")
        return a.value, b.value

    def close(self):
        if getattr(self, "handle", None):
            L.lib().tc_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def split_components(flat, sizes):
    """Views of a planar output whose components have their own sizes
    (subsampled components): one [h, w] array per component."""
    views, off = [], 0
    for h, w in sizes:
        views.append(flat[off:off + h * w].reshape(h, w))
        off += h * w
    return views


class Decoder:
    """Decoder::decode (Decoder.cpp:94-217): codestream in host memory (or a
    file) -> planar samples in host memory."""

    def __init__(self, ctx: Context | None = None):
        self.ctx = ctx or Context()

    def decode(self, cs, out: np.ndarray | None = None):
        """cs: bytes, a path, or a uint8 array (read in place: a codestream in
        pinned memory is uploaded while it is parsed).  out: optional
        [ncomp, height, width] array to fill (pinned memory gives the fastest
        read-back)."""
        if isinstance(cs, (str, Path)):
            cs = Path(cs).read_bytes()
        if isinstance(cs, np.ndarray):
            buf = np.ascontiguousarray(cs.reshape(-1).view(np.uint8))
        else:
            buf = np.frombuffer(cs, np.uint8)
        hdr = L.ImageInfo()
        self.ctx.check(L.lib().tc_j2k_read_header(buf.ctypes.data, buf.size, C.byref(hdr)), "tc_j2k_read_header")
        if hdr.is_signed:
            dt = np.int8 if hdr.bits <= 8 else np.int16
        else:
            dt = np.uint8 if hdr.bits <= 8 else np.uint16
        from .codec import _info_dict
        sizes = _info_dict(hdr)["comp_sizes"]
        if len(set(sizes)) > 1:
            # subsampled components: planar at their own sizes, returned as a list
            flat = np.empty(sum(h * w for h, w in sizes), dt) if out is None else out.reshape(-1)
            self.ctx.check(L.lib().tc_decode_j2k(self.ctx.handle, buf.ctypes.data, buf.size, flat.ctypes.data,
                                                 flat.nbytes, None), "tc_decode_j2k")
            return split_components(flat, sizes)
        shape = (hdr.ncomp, hdr.height, hdr.width)
        if out is None:
            out = np.empty(shape, dt)
        info = L.ImageInfo()
        self.ctx.check(L.lib().tc_decode_j2k(self.ctx.handle, buf.ctypes.data, buf.size, out.ctypes.data,
                                             out.nbytes, C.byref(info)), "tc_decode_j2k")
        return out

    def decode_to_file(self, cs, path):
        """Decode and write the samples as PNM (.pgm/.ppm) or PGX (.pgx, one
        file per component); returns the written paths."""
        from .imageio import write_image
        out = self.decode(cs)
        hdr = L.ImageInfo()
        buf = np.frombuffer(cs, np.uint8) if not isinstance(cs, (str, Path)) else \
            np.frombuffer(Path(cs).read_bytes(), np.uint8)
        self.ctx.check(L.lib().tc_j2k_read_header(buf.ctypes.data, buf.size, C.byref(hdr)), "tc_j2k_read_header")
        return write_image(path, out, hdr.bits, bool(hdr.is_signed))

    def plan(self, codestreams) -> Plan:
        return Plan(self.ctx, codestreams)
