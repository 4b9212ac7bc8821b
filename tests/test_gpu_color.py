"""Colour transform / DC shift kernels against the CPU oracle."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _pre(ctx):
    from thousandthchicken_b200.stages import Preprocessor
    return Preprocessor(ctx)


@pytest.mark.parametrize("bits", [8, 12, 16])
def test_rct_forward_and_inverse_bit_exact(gpu_ctx, bits):
    rng = np.random.default_rng(bits)
    h, w = 77, 129
    img = rng.integers(0, 1 << bits, (3, h, w)).astype(np.int32)
    d_in = [torch.from_numpy(img[c]).cuda() for c in range(3)]
    d_yuv = [torch.empty((h, w), dtype=torch.int32, device="cuda") for _ in range(3)]
    _pre(gpu_ctx).color_coder_lossless(d_in, d_yuv, bits)
    want = O.rct_forward([img[0], img[1], img[2]], bits)
    for c in range(3):
        np.testing.assert_array_equal(d_yuv[c].cpu().numpy(), want[c])
    out_dt = torch.uint8 if bits <= 8 else torch.int16
    d_out = [torch.empty((h, w), dtype=out_dt, device="cuda") for _ in range(3)]
    _pre(gpu_ctx).color_decoder_lossless(d_yuv, d_out, bits)
    for c in range(3):
        got = d_out[c].cpu().numpy().astype(np.int64) & 0xFFFF
        np.testing.assert_array_equal(got, img[c])


def test_ict_inverse_within_one_lsb(gpu_ctx):
    rng = np.random.default_rng(3)
    h, w = 64, 200
    ycc = [rng.uniform(-140, 140, (h, w)) for _ in range(3)]
    want = O.ict_inverse(ycc, 8)
    d_in = [torch.from_numpy(p.astype(np.float32)).cuda() for p in ycc]
    d_out = [torch.empty((h, w), dtype=torch.uint8, device="cuda") for _ in range(3)]
    _pre(gpu_ctx).color_decoder_lossy(d_in, d_out, 8)
    for c in range(3):
        d = np.abs(d_out[c].cpu().numpy().astype(int) - want[c])
        assert d.max() <= 1
        assert (d > 0).mean() < 0.01


def test_ict_forward_matches_fp64(gpu_ctx):
    rng = np.random.default_rng(4)
    img = rng.integers(0, 256, (3, 50, 60)).astype(np.int32)
    want = O.ict_forward([img[0], img[1], img[2]], 8)
    d_in = [torch.from_numpy(img[c]).cuda() for c in range(3)]
    d_out = [torch.empty((50, 60), dtype=torch.float32, device="cuda") for _ in range(3)]
    _pre(gpu_ctx).color_coder_lossy(d_in, d_out, 8)
    for c in range(3):
        assert np.abs(d_out[c].cpu().numpy() - want[c]).max() < 1e-3


def test_dc_shift_round_trip_and_clamp(gpu_ctx):
    rng = np.random.default_rng(5)
    x = rng.integers(-200, 200, (1, 33, 47)).astype(np.int32)
    d_in = [torch.from_numpy(x[0]).cuda()]
    d_out = [torch.empty((33, 47), dtype=torch.uint8, device="cuda")]
    _pre(gpu_ctx).idc_level_shifting(d_in, d_out, 8)
    np.testing.assert_array_equal(d_out[0].cpu().numpy(), O.dc_inverse_clamp(x[0], 8))
