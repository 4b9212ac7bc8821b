"""The CUDA path against golden vectors produced by the reference's own
kernels (tests/golden/make_ref_golden.py): Tier-1 raw output, RCT and DC
shift bit-exact."""
import numpy as np
import pytest

from conftest import GOLDEN
from thousandthchicken_b200 import codec

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_gpu_t1_equals_reference_kernel(gpu_ctx):
    from thousandthchicken_b200.stages import CoefficientCoder
    z = np.load(GOLDEN / "ref_t1_blocks.npz")
    meta = z["meta"]
    n = len(meta)
    desc = np.zeros(n, codec.DESC_DTYPE)
    desc["seg_off"] = z["seg_off"]
    desc["seg_len"] = z["seg_len"]
    desc["w"], desc["h"], desc["orient"], desc["mb"] = meta[:, 0], meta[:, 1], meta[:, 2], meta[:, 3]
    desc["zero_bitplanes"], desc["passes"] = meta[:, 4], meta[:, 5]
    desc["out_off"] = np.arange(n) * 4096
    desc["out_pitch"] = 64
    got = CoefficientCoder(gpu_ctx).decode_blocks(desc, z["pool"], n * 4096, raw=True).cpu().numpy()
    got = got.view(np.uint32).reshape(n, 64, 64)
    flat, pos = z["ref_raw"], 0
    for i, (w, h, *_rest) in enumerate(meta):
        np.testing.assert_array_equal(got[i, :h, :w], flat[pos: pos + w * h].reshape(h, w), err_msg=f"block {i}")
        pos += w * h


def test_gpu_t1_truncated_equals_reference_kernel(gpu_ctx):
    """Blocks truncated after P whole bit-planes, in one launch: the GPU's raw
    words equal the reference kernel's output for a P-plane block moved up by
    the planes left undecoded (tests/golden/make_ref_golden.py,
    t1_trunc_vectors)."""
    from test_reference_golden import ref_planes_to_coded
    from thousandthchicken_b200.stages import CoefficientCoder
    z = np.load(GOLDEN / "ref_t1_trunc.npz")
    meta = z["meta"]
    n = len(meta)
    desc = np.zeros(n, codec.DESC_DTYPE)
    desc["seg_off"] = z["seg_off"]
    desc["seg_len"] = z["seg_len"]
    desc["w"], desc["h"], desc["orient"], desc["mb"] = meta[:, 0], meta[:, 1], meta[:, 2], meta[:, 3]
    desc["zero_bitplanes"], desc["passes"] = meta[:, 4], meta[:, 5]
    desc["out_off"] = np.arange(n) * 4096
    desc["out_pitch"] = 64
    got = CoefficientCoder(gpu_ctx).decode_blocks(desc, z["pool"], n * 4096, raw=True).cpu().numpy()
    got = got.view(np.uint32).reshape(n, 64, 64)
    flat, pos = z["ref_raw"], 0
    for i, (w, h, _o, mb, zbp, _p, planes) in enumerate(meta):
        ref = flat[pos: pos + w * h].reshape(h, w)
        np.testing.assert_array_equal(got[i, :h, :w], ref_planes_to_coded(ref, int(planes), int(mb - zbp)),
                                      err_msg=f"block {i}")
        pos += w * h


@pytest.mark.parametrize("bits", [8, 12])
def test_gpu_colour_equals_reference_kernels(gpu_ctx, bits):
    from thousandthchicken_b200.stages import Preprocessor
    z = np.load(GOLDEN / "ref_colour.npz")
    img = z[f"rgb{bits}"]
    h, w = img.shape[1:]
    pre = Preprocessor(gpu_ctx)
    d_in = [torch.from_numpy(img[c].copy()).cuda() for c in range(3)]
    d_out = [torch.empty((h, w), dtype=torch.int32, device="cuda") for _ in range(3)]
    pre.color_coder_lossless(d_in, d_out, bits)
    np.testing.assert_array_equal(np.stack([o.cpu().numpy() for o in d_out]), z[f"rct{bits}"])
    d_ict = [torch.empty((h, w), dtype=torch.int32, device="cuda") for _ in range(3)]
    pre.color_coder_lossy(d_in, d_ict, bits)
    d = np.abs(np.stack([o.cpu().numpy() for o in d_ict]).astype(np.int64) - z[f"ict{bits}"])
    assert d.max() <= 1 and (d > 0).mean() < 1e-3
    d_back = [torch.empty((h, w), dtype=torch.int32, device="cuda") for _ in range(3)]
    pre.color_decoder_lossless(d_out, d_back, bits)
    np.testing.assert_array_equal(np.stack([o.cpu().numpy() for o in d_back]), z[f"rct_inv{bits}"])
    d1 = [torch.from_numpy(z[f"dc{bits}"].copy()).cuda()]
    o1 = [torch.empty((h, w), dtype=torch.int32, device="cuda")]
    pre.idc_level_shifting(d1, o1, bits)
    np.testing.assert_array_equal(o1[0].cpu().numpy(), z[f"dc_inv{bits}"])


def test_gpu_53_trunc_equals_reference_kernels(gpu_ctx):
    """tc_dwt_forward53 / tc_dwt_reverse53 in truncating mode (TC_ROUND_TRUNC)
    against one level of the reference's own dwt_f53.cl / dwt_r53.cl run on
    the CPU (tests/golden/ref_dwt53.npz): bit-exact on every sample outside
    the rows those kernels get wrong (D24, D25)."""
    import ref as R
    from thousandthchicken_b200 import _lib as L
    from thousandthchicken_b200.stages import DWTForward53, DWTReverse53
    z = np.load(GOLDEN / "ref_dwt53.npz")
    fw = DWTForward53(gpu_ctx, rounding=L.TC_ROUND_TRUNC)
    rv = DWTReverse53(gpu_ctx, rounding=L.TC_ROUND_TRUNC)
    n = 0
    for k in sorted({f[2:] for f in z.files if f.startswith("x_")}):
        w, h = map(int, k.split("x"))
        x = torch.from_numpy(z[f"x_{k}"]).cuda()
        out = torch.empty_like(x)
        fw.run(x, out, w, h, 1)
        got = R.mallat_to_packed(out.cpu().numpy(), 1)
        mk = R.dwt53_defect_mask(w, h, True)
        np.testing.assert_array_equal(got[~mk], z[f"fwd_{k}"][~mk], err_msg=f"{w}x{h} forward")
        coef = torch.from_numpy(R.packed_to_mallat(z[f"revin_{k}"], w, h, 1)).cuda()
        back = torch.empty_like(coef)
        rv.run(coef, back, w, h, 1)
        mr = R.dwt53_defect_mask(w, h, False)
        np.testing.assert_array_equal(back.cpu().numpy()[~mr], z[f"rev_{k}"][~mr], err_msg=f"{w}x{h} reverse")
        n += 1
    gpu_ctx.synchronize()
    assert n >= 6
