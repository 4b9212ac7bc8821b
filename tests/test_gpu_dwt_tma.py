"""The fused last reverse 9/7 level with TMA-staged subband tiles
(dwt_tma.cu) against the cp.async-staged kernel: whole lossy decodes of
three-component images whose last level qualifies for tensor copies give
the same samples bit for bit with either staging, and stay within 1 of the
FP64 oracle.  Sizes cover one tile, border tiles on every side, partial
tiles and the 4096^2 workload size."""
import numpy as np
import pytest

import oracle as O
from conftest import synth_image
from thousandthchicken_b200 import _lib as L
from thousandthchicken_b200 import codec

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SIZES = [(16, 16, 2), (200, 72, 3), (264, 136, 4), (1032, 520, 5), (2000, 1000, 6), (4096, 4096, 6)]


@pytest.mark.parametrize("w,h,levels", SIZES, ids=[f"{w}x{h}" for w, h, _ in SIZES])
@pytest.mark.parametrize("bits", [8, 12])
def test_tma_staging_equals_cp_async_staging(gpu_ctx, w, h, levels, bits):
    from thousandthchicken_b200.stages import Decoder
    if w * h > 4 << 20 and bits == 12:
        pytest.skip("one bit depth is enough at full size")
    img = synth_image(w, h, 3, bits, seed=w + h + bits)
    cs = codec.encode(img, bits, levels=levels, reversible=False, mct=True, base_step=1 / 128)
    dec = Decoder(gpu_ctx)
    outs = {}
    try:
        for variant in (L.TC_DWT_CPASYNC, L.TC_DWT_TMA):
            assert L.lib().tc_ctx_set_dwt_variant(gpu_ctx.handle, variant) == L.TC_OK
            outs[variant] = dec.decode(cs).copy()
    finally:
        L.lib().tc_ctx_set_dwt_variant(gpu_ctx.handle, L.TC_DWT_TMA)
    np.testing.assert_array_equal(outs[L.TC_DWT_TMA], outs[L.TC_DWT_CPASYNC])
    if w * h <= 1 << 20:
        info, desc, pool = codec.parse(cs)
        want = O.decode_tile(desc, pool, w, h, 3, bits, levels, False, True, r=0.5)
        d = np.abs(outs[L.TC_DWT_TMA].astype(np.int64) - want.astype(np.int64))
        assert d.max() <= 1 and (d > 0).mean() < 2e-3
