"""Tier-1 CUDA kernel (one warp per code-block, persistent queue, fused
inverse quantiser) against the CPU oracle: bit-exact for every output mode."""
import numpy as np
import pytest

import oracle as O
from conftest import golden_cases, load_golden
from gpu_helpers import make_blocks, oracle_mallat, oracle_slots
from thousandthchicken_b200 import codec
from thousandthchicken_b200._lib import TC_E_CODESTREAM, TCError

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _coder(ctx):
    from thousandthchicken_b200.stages import CoefficientCoder
    return CoefficientCoder(ctx)


@pytest.mark.parametrize("truncate", [False, True])
def test_t1_raw_output_matches_oracle(gpu_ctx, truncate):
    desc, pool, _ = make_blocks(seed=11 + truncate, n=300, truncate=truncate)
    got = _coder(gpu_ctx).decode_blocks(desc, pool, len(desc) * 4096, raw=True).cpu().numpy()
    want = oracle_slots(desc, pool, "raw").reshape(-1).view(np.int32)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("r", [0.0, 0.5])
def test_t1_dequant_int_matches_oracle(gpu_ctx, r):
    desc, pool, blocks = make_blocks(seed=21, n=300, truncate=True)
    got = _coder(gpu_ctx).decode_blocks(desc, pool, len(desc) * 4096, recon_r=r).cpu().numpy()
    want = oracle_slots(desc, pool, "int", r).reshape(-1)
    np.testing.assert_array_equal(got, want)


def test_t1_full_passes_recover_coefficients(gpu_ctx):
    desc, pool, blocks = make_blocks(seed=31, n=200, truncate=False)
    got = _coder(gpu_ctx).decode_blocks(desc, pool, len(desc) * 4096, recon_r=0.0).cpu().numpy()
    got = got.reshape(len(desc), 64, 64)
    for i, (coef, _, _, _) in enumerate(blocks):
        h, w = coef.shape
        np.testing.assert_array_equal(got[i, :h, :w], coef)


def test_t1_dequant_float_matches_oracle(gpu_ctx):
    desc, pool, _ = make_blocks(seed=41, n=300, truncate=True, irreversible=True)
    got = _coder(gpu_ctx).decode_blocks(desc, pool, len(desc) * 4096, recon_r=0.5,
                                        dtype=torch.float32).cpu().numpy()
    want = oracle_slots(desc, pool, "float", 0.5).reshape(-1)
    np.testing.assert_array_equal(got.view(np.int32), want.view(np.int32))


def test_t1_queue_order_does_not_change_results(gpu_ctx):
    desc, pool, _ = make_blocks(seed=51, n=500, truncate=True)
    c = _coder(gpu_ctx)
    a = c.decode_blocks(desc, pool, len(desc) * 4096, sort=True).cpu().numpy()
    b = c.decode_blocks(desc, pool, len(desc) * 4096, sort=False).cpu().numpy()
    np.testing.assert_array_equal(a, b)


def test_t1_batched_uneven_blocks_large(gpu_ctx):
    """Uneven batch (60% 64x64, 30% 32x32, 10% ragged edges), truncated at
    seeded pass counts, in one persistent launch."""
    desc, pool, blocks = make_blocks(seed=61, n=4000, truncate=True)
    got = _coder(gpu_ctx).decode_blocks(desc, pool, len(desc) * 4096, recon_r=0.0).cpu().numpy()
    want = oracle_slots(desc, pool, "int", 0.0).reshape(-1)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("name,meta", golden_cases(), ids=[n for n, _ in golden_cases()])
def test_t1_openjpeg_streams(gpu_ctx, name, meta):
    cs, _, _ = load_golden(name)
    got, info = _coder(gpu_ctx).decode_tile(cs, recon_r=0.5)
    want, _ = oracle_mallat(cs, 0.5)
    np.testing.assert_array_equal(got.cpu().numpy().view(np.int32), want.view(np.int32))


def test_t1_bad_descriptor_sets_error_word(gpu_ctx):
    desc, pool, _ = make_blocks(seed=71, n=8, truncate=False)
    bad = desc.copy()
    bad["seg_len"][3] = 1 << 30          # codeword past the pool
    with pytest.raises(TCError) as e:
        _coder(gpu_ctx).decode_blocks(bad, pool, len(bad) * 4096, raw=True)
    assert e.value.status == TC_E_CODESTREAM
    bad = desc.copy()
    bad["w"][2] = 0                      # geometry out of range
    with pytest.raises(TCError):
        _coder(gpu_ctx).decode_blocks(bad, pool, len(bad) * 4096, raw=True)
    # the context stays usable
    got = _coder(gpu_ctx).decode_blocks(desc, pool, len(desc) * 4096, raw=True).cpu().numpy()
    np.testing.assert_array_equal(got, oracle_slots(desc, pool, "raw").reshape(-1).view(np.int32))


def test_t1_empty_and_zero_pass_blocks(gpu_ctx):
    desc, pool, _ = make_blocks(seed=81, n=16, truncate=False)
    desc["passes"][::2] = 0
    got = _coder(gpu_ctx).decode_blocks(desc, pool, len(desc) * 4096, recon_r=0.0).cpu().numpy()
    want = oracle_slots(desc, pool, "int", 0.0).reshape(-1)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("lanes", [8, 16, 32])
def test_t1_lane_group_widths_bit_exact(gpu_ctx, lanes):
    """Two or four code-blocks per warp (8/16 lanes each) decode exactly like
    one block per warp."""
    from thousandthchicken_b200 import _lib as L
    desc, pool, _ = make_blocks(seed=91, n=600, truncate=True)
    assert L.lib().tc_ctx_set_t1_group(gpu_ctx.handle, lanes) == 0
    try:
        got = _coder(gpu_ctx).decode_blocks(desc, pool, len(desc) * 4096, recon_r=0.5).cpu().numpy()
        raw = _coder(gpu_ctx).decode_blocks(desc, pool, len(desc) * 4096, raw=True).cpu().numpy()
    finally:
        L.lib().tc_ctx_set_t1_group(gpu_ctx.handle, 32)
    np.testing.assert_array_equal(got, oracle_slots(desc, pool, "int", 0.5).reshape(-1))
    np.testing.assert_array_equal(raw, oracle_slots(desc, pool, "raw").reshape(-1).view(np.int32))


@pytest.mark.parametrize("irreversible", [False, True])
def test_standalone_dequantiser_matches_oracle(gpu_ctx, irreversible):
    """tc_dequantize_raw over raw Tier-1 words (Quantizer::dequantize_tile):
    every block's coefficients with the reconstruction offset of the last
    decoded plane, against the oracle's dequantiser on the same words."""
    from thousandthchicken_b200.stages import Quantizer, _dev_bytes
    desc, pool, _ = make_blocks(seed=171, n=300, truncate=True)
    raw = _coder(gpu_ctx).decode_blocks(desc, pool, len(desc) * 4096, raw=True)
    rng = np.random.default_rng(5)
    if irreversible:
        desc["flags"] = 1
        desc["step"] = rng.uniform(0.01, 4.0, len(desc)).astype(np.float32)
    dt = torch.float32 if irreversible else torch.int32
    out = torch.zeros(len(desc) * 4096, dtype=dt, device="cuda")
    d_desc = _dev_bytes(np.ascontiguousarray(desc, codec.DESC_DTYPE), torch.device("cuda"))
    Quantizer(gpu_ctx).dequantize(d_desc, len(desc), raw, out, 0.5)
    gpu_ctx.synchronize()
    got = out.cpu().numpy().reshape(len(desc), 64, 64)
    words = raw.cpu().numpy().view(np.uint32).reshape(len(desc), 64, 64)
    for i, d in enumerate(desc):
        w, h, mb = int(d["w"]), int(d["h"]), int(d["mb"])
        q = ((words[i, :h, :w] & 0x7FFFFFFF) >> (31 - mb)).astype(np.int32)
        q = np.where(words[i, :h, :w] >> 31, -q, q)
        numbps = mb - int(d["zero_bitplanes"])
        u = max(numbps - 1 - (int(d["passes"]) + 1) // 3, 0) if numbps > 0 and d["passes"] > 0 else 0
        uu = np.full(q.shape, u, np.uint8)
        if irreversible:
            want = O.dequant_float(q, uu, 0.5, float(d["step"]))
            np.testing.assert_array_equal(got[i, :h, :w].view(np.int32), want.view(np.int32))
        else:
            np.testing.assert_array_equal(got[i, :h, :w], O.dequant_int(q, uu, 0.5))


def _enc_blocks(seed, n):
    """n blocks of quantised Laplacian coefficients in 64x64 slots of one
    int32 plane (64 wide), with their encoder descriptors and the host
    encoder's (codeword, passes, zero bit-planes) for each."""
    from thousandthchicken_b200.synth import laplacian_block
    rng = np.random.default_rng(seed)
    plane = np.zeros((n * 64, 64), np.int32)
    desc = np.zeros(n, codec.ENC_DESC_DTYPE)
    want = []
    for i in range(n):
        r = rng.random()
        w, h = (64, 64) if r < 0.5 else ((32, 32) if r < 0.8 else (int(rng.integers(1, 65)), int(rng.integers(1, 65))))
        orient = int(rng.integers(0, 4))
        coef = laplacian_block(rng, w, h, bitplanes=int(rng.integers(1, 15)))
        if rng.random() < 0.05:
            coef[:] = 0  # an empty block
        mb = 16
        plane[i * 64:i * 64 + h, :w] = coef
        d = desc[i]
        d["in_off"], d["in_pitch"], d["w"], d["h"], d["orient"], d["mb"] = i * 64 * 64, 64, w, h, orient, mb
        seg, passes, zbp = codec.t1_encode_block(coef, orient, mb)
        want.append((seg, passes, zbp))
    return desc, plane, want


def test_gpu_encoder_matches_host_encoder(gpu_ctx):
    """The GPU Tier-1 encoder (one warp per block, flag-word contexts,
    register MQ encoder) writes, block for block, the host encoder's
    codeword, pass count and zero bit-planes; and the GPU decoder reads the
    GPU codewords back to the coefficients."""
    from thousandthchicken_b200.stages import T1Encoder
    desc, plane, want = _enc_blocks(seed=41, n=400)
    got = T1Encoder(gpu_ctx).encode(desc, torch.from_numpy(plane.reshape(-1)).cuda())
    for i, (g, w_) in enumerate(zip(got, want)):
        assert g[1:] == w_[1:] or (w_[0] == b"" and g[0] == b""), (i, g[1:], w_[1:])
        assert g[0] == w_[0], i
    # decode the GPU codewords with the GPU decoder: the coefficients come back
    ddesc = np.zeros(len(desc), codec.DESC_DTYPE)
    pool, off = [], 0
    for i, (seg, passes, zbp) in enumerate(got):
        d = ddesc[i]
        d["seg_off"], d["seg_len"] = off, len(seg)
        d["w"], d["h"], d["passes"], d["mb"], d["zero_bitplanes"] = desc["w"][i], desc["h"][i], passes, 16, zbp
        d["orient"], d["out_off"], d["out_pitch"], d["step"] = desc["orient"][i], i * 4096, 64, 1.0
        pool.append(seg)
        off += len(seg)
    pool = np.frombuffer(b"".join(pool) + b"\0" * 16, np.uint8).copy()
    back = _coder(gpu_ctx).decode_blocks(ddesc, pool, len(desc) * 4096, recon_r=0.0).cpu().numpy()
    np.testing.assert_array_equal(back.reshape(-1, 64), plane)


def test_gpu_encoder_flags_a_short_buffer(gpu_ctx):
    from thousandthchicken_b200._lib import TCError
    from thousandthchicken_b200.stages import T1Encoder
    desc, plane, _ = _enc_blocks(seed=42, n=8)
    with pytest.raises(TCError):
        T1Encoder(gpu_ctx).encode(desc, torch.from_numpy(plane.reshape(-1)).cuda(), cap=16)


def test_block_placed_past_the_output_is_skipped_and_reported(gpu_ctx):
    """A caller-built descriptor whose block would run past the output
    (out_off + (h-1)*out_pitch + w > out_elems) is skipped before any write
    and reported; the other blocks decode as usual and the memory after the
    output is untouched.  The same for the standalone dequantiser."""
    from thousandthchicken_b200.stages import CoefficientCoder, Quantizer, _dev_bytes
    desc, pool, _ = make_blocks(seed=61, n=24, mix="full", truncate=False)
    n = len(desc)
    elems = n * 4096
    dev = torch.device("cuda")
    want = _coder(gpu_ctx).decode_blocks(desc, pool, elems, recon_r=0.0).cpu().numpy()
    bad = desc.copy()
    bad["out_off"][5] = elems - 64 * 3          # three rows left, the block has 64
    guard = 0x5A5A5A5A
    buf = torch.full((elems + 8192,), guard, dtype=torch.int32, device=dev)
    out = buf[:elems]
    out[: n * 4096].zero_()
    cc = CoefficientCoder(gpu_ctx)
    d_desc = _dev_bytes(np.ascontiguousarray(bad, codec.DESC_DTYPE), dev)
    d_pool = _dev_bytes(pool, dev)
    cc.decode(d_desc, d_pool, out, n, None, raw=False, recon_r=0.0, max_bitplanes=16)
    with pytest.raises(TCError) as ei:
        gpu_ctx.synchronize()
    assert ei.value.status == TC_E_CODESTREAM and "past the output" in str(ei.value)
    got = buf.cpu().numpy()
    assert (got[elems:] == guard).all()
    keep = np.ones(elems, bool)
    keep[5 * 4096: 6 * 4096] = False    # block 5's own slot stays as it was (zero)
    np.testing.assert_array_equal(got[:elems][keep], want[keep])
    assert (got[5 * 4096: 6 * 4096] == 0).all()
    # the standalone dequantiser over raw words
    raw = _coder(gpu_ctx).decode_blocks(desc, pool, elems, raw=True)
    buf2 = torch.full((elems + 8192,), guard, dtype=torch.int32, device=dev)
    Quantizer(gpu_ctx).dequantize(d_desc, n, raw, buf2[:elems], 0.0)
    with pytest.raises(TCError):
        gpu_ctx.synchronize()
    assert (buf2[elems:].cpu().numpy() == guard).all()
    gpu_ctx.synchronize()   # the error word was cleared by the report
