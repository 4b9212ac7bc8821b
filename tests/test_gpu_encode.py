"""The encoder on the GPU (tc_encode_j2k_gpu): forward colour transform,
forward DWT, quantisation and Tier-1 as kernels, packets on the host.  The
host encoder (tc_encode_j2k) is the oracle: lossless streams are
byte-identical; lossy ones decode to the same quality and in OpenJPEG."""
import numpy as np
import pytest

from conftest import synth_image
from thousandthchicken_b200 import codec

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("w,h,c,bits,levels,kw", [
    (300, 200, 3, 8, 5, {}),
    (257, 131, 3, 8, 4, dict(cblk_log2=5)),
    (96, 80, 1, 12, 3, {}),
    (1, 1, 1, 8, 0, {}),
    (45, 1, 3, 8, 2, {}),
    (200, 120, 3, 8, 4, dict(comp_cblk_log2=[0, 4, 5])),
    (200, 120, 3, 8, 4, dict(layers=4, progression=2)),
    (160, 96, 3, 8, 3, dict(layers=3, packed_headers=1)),
    (160, 96, 1, 12, 3, dict(layers=2, packed_headers=2, progression=4)),
], ids=["rgb8", "rgb8-cb32", "g12", "1x1", "45x1", "coc", "layers-rpcl", "layers-ppt", "g12-ppm-cprl"])
def test_lossless_gpu_encode_is_byte_identical(gpu_ctx, w, h, c, bits, levels, kw):
    img = synth_image(w, h, c, bits, seed=w + h)
    cpu = codec.encode(img, bits, levels=levels, reversible=True, mct=c == 3, **kw)
    gpu = codec.encode_gpu(gpu_ctx, img, bits, levels=levels, reversible=True, mct=c == 3, **kw)
    assert gpu == cpu


def test_signed_lossless_gpu_encode(gpu_ctx):
    from test_host_codec import _ct_like
    img = _ct_like(120, 150, 16, seed=3)
    cpu = codec.encode(img, 16, levels=4, reversible=True, mct=False)
    assert codec.encode_gpu(gpu_ctx, img, 16, levels=4, reversible=True, mct=False) == cpu


def test_lossy_gpu_encode_decodes_like_the_host_encode(gpu_ctx):
    """fp32 DWT on the GPU against fp64 on the host: a few quantised
    coefficients may differ, the decoded quality does not, and OpenJPEG
    reads the GPU stream."""
    from gpu_helpers import openjpeg_decode
    from thousandthchicken_b200.stages import Decoder
    img = synth_image(512, 384, 3, 8, seed=4)
    cpu = codec.encode(img, 8, levels=5, reversible=False, base_step=1 / 128)
    gpu = codec.encode_gpu(gpu_ctx, img, 8, levels=5, reversible=False, base_step=1 / 128)
    assert abs(len(gpu) - len(cpu)) < 0.01 * len(cpu)
    dec = Decoder(gpu_ctx)

    def psnr(a):
        d = a.astype(np.float64) - img
        return 10 * np.log10(255 ** 2 / np.mean(d * d))
    p_cpu, p_gpu = psnr(dec.decode(cpu)), psnr(dec.decode(gpu))
    assert abs(p_cpu - p_gpu) < 0.05 and p_gpu > 40
    assert abs(psnr(openjpeg_decode(gpu)) - p_gpu) < 0.05
