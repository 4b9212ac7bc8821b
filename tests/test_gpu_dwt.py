"""DWT CUDA kernels against the CPU oracle: 5/3 bit-exact (ISO floor and
the reference's truncating rounding), 9/7 within a stated fp32 tolerance of
the FP64 oracle."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SIZES = [(1, 1, 1), (1, 9, 2), (9, 1, 2), (2, 3, 1), (5, 7, 3), (3, 5, 5), (64, 64, 3), (127, 65, 4),
         (300, 257, 5), (1024, 768, 6), (4096, 64, 3), (130, 1030, 7)]

# fp32 lifting over several levels against the FP64 oracle: absolute error
# bound for samples of 8-bit range (|x| <= 255).
TOL97 = 0.02


def _dev(a, dt):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype=dt)


def _rand(w, h, seed, lo=-255, hi=256):
    return np.random.default_rng(seed).integers(lo, hi, (h, w)).astype(np.int32)


@pytest.mark.parametrize("rounding", [0, 1])
@pytest.mark.parametrize("w,h,levels", SIZES)
def test_53_forward_reverse_bit_exact(gpu_ctx, w, h, levels, rounding):
    from thousandthchicken_b200.stages import DWTForward53, DWTReverse53
    x = _rand(w, h, w * 31 + h)
    want_f = O.fdwt53(x, levels, rounding)
    got_f = torch.empty((h, w), dtype=torch.int32, device="cuda")
    DWTForward53(gpu_ctx, rounding).run(_dev(x, torch.int32), got_f, w, h, levels)
    np.testing.assert_array_equal(got_f.cpu().numpy(), want_f)
    want_r = O.idwt53(want_f, levels, rounding)
    np.testing.assert_array_equal(want_r, x)
    got_r = torch.empty((h, w), dtype=torch.int32, device="cuda")
    DWTReverse53(gpu_ctx, rounding).run(_dev(want_f, torch.int32), got_r, w, h, levels)
    np.testing.assert_array_equal(got_r.cpu().numpy(), x)


@pytest.mark.parametrize("w,h,levels", SIZES)
def test_97_forward_reverse_within_tolerance(gpu_ctx, w, h, levels, record_property):
    from thousandthchicken_b200.stages import DWTForward97, DWTReverse97
    x = _rand(w, h, w * 17 + h, -128, 128).astype(np.float64)
    want_f = O.fdwt97(x, levels)
    got_f = torch.empty((h, w), dtype=torch.float32, device="cuda")
    DWTForward97(gpu_ctx).run(_dev(x, torch.float32), got_f, w, h, levels)
    err_f = np.abs(got_f.cpu().numpy().astype(np.float64) - want_f).max()
    scale = max(1.0, np.abs(want_f).max() / 256.0)
    assert err_f <= TOL97 * scale, err_f
    got_r = torch.empty((h, w), dtype=torch.float32, device="cuda")
    DWTReverse97(gpu_ctx).run(_dev(want_f, torch.float32), got_r, w, h, levels)
    err_r = np.abs(got_r.cpu().numpy().astype(np.float64) - x).max()
    record_property("forward_max_abs_vs_fp64", float(err_f))
    record_property("reverse_max_abs_vs_fp64", float(err_r))
    assert err_r <= TOL97, err_r


def test_reverse_does_not_modify_input(gpu_ctx):
    from thousandthchicken_b200.stages import DWTReverse53
    x = O.fdwt53(_rand(200, 120, 5), 4)
    d = _dev(x, torch.int32)
    out = torch.empty_like(d)
    DWTReverse53(gpu_ctx).run(d, out, 200, 120, 4)
    np.testing.assert_array_equal(d.cpu().numpy(), x)


def test_pitched_planes(gpu_ctx):
    from thousandthchicken_b200.stages import DWTForward53
    w, h, p = 100, 70, 128
    x = _rand(w, h, 9)
    big = np.zeros((h, p), np.int32)
    big[:, :w] = x
    out = torch.zeros((h, p), dtype=torch.int32, device="cuda")
    DWTForward53(gpu_ctx).run(_dev(big, torch.int32), out, w, h, 3, in_pitch=p, out_pitch=p)
    np.testing.assert_array_equal(out.cpu().numpy()[:, :w], O.fdwt53(x, 3))
