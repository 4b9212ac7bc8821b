"""The oracle against golden vectors produced by the reference's own
kernels (compiled as host code from its OpenCL C, tests/golden/
make_ref_golden.py): Tier-1 bit-exact (with the reference's D1/D2 state
bugs fixed), RCT and DC shift bit-exact, and the reference's defective
paths (unpatched Tier-1, inverse ICT) shown to differ."""
import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN


def t1_fixture():
    return np.load(GOLDEN / "ref_t1_blocks.npz")


def iter_blocks(z):
    pool, off, ln, meta, flat = z["pool"], z["seg_off"], z["seg_len"], z["meta"], z["ref_raw"]
    pos = 0
    for i, (w, h, orient, mb, zbp, passes) in enumerate(meta):
        seg = pool[off[i]: off[i] + ln[i]].tobytes()
        ref = flat[pos: pos + w * h].reshape(h, w)
        pos += w * h
        yield i, seg, int(w), int(h), int(orient), int(mb), int(zbp), int(passes), ref


def test_oracle_t1_equals_reference_kernel():
    z = t1_fixture()
    n = 0
    for i, seg, w, h, orient, mb, zbp, passes, ref in iter_blocks(z):
        got = O.t1_decode_raw(seg, w, h, orient, mb, zbp, passes)
        np.testing.assert_array_equal(got, ref, err_msg=f"block {i}")
        n += 1
    assert n >= 100


def ref_planes_to_coded(ref, planes, nb):
    """The reference's raw words of a block decoded as a `planes`-plane block
    (significantBits = planes) in the layout of a decoder that knows the
    block has nb coded planes and decoded the first `planes`: magnitude bits
    nb - planes higher, sign bit unchanged."""
    ref = ref.astype(np.uint64)
    mag = ((ref & 0x7FFFFFFF) << np.uint64(nb - planes)) & 0x7FFFFFFF
    return (mag | (ref & 0x80000000)).astype(np.uint32)


def test_oracle_t1_truncated_equals_reference_kernel():
    """Blocks truncated after whole bit-planes (3P - 2 passes): the oracle's
    raw decode equals the reference kernel's own output for a P-plane block,
    moved up by the planes left undecoded."""
    z = np.load(GOLDEN / "ref_t1_trunc.npz")
    pool, off, ln, flat = z["pool"], z["seg_off"], z["seg_len"], z["ref_raw"]
    pos = n = 0
    for i, (w, h, orient, mb, zbp, passes, planes) in enumerate(z["meta"]):
        seg = pool[off[i]: off[i] + ln[i]].tobytes()
        ref = flat[pos: pos + w * h].reshape(h, w)
        pos += w * h
        got = O.t1_decode_raw(seg, int(w), int(h), int(orient), int(mb), int(zbp), int(passes))
        np.testing.assert_array_equal(got, ref_planes_to_coded(ref, int(planes), int(mb - zbp)), err_msg=f"block {i}")
        assert (got != 0).any() or not ln[i]
        n += 1
    assert n == 160


def test_unpatched_reference_kernel_is_defective():
    """Defects D1/D2 (state helpers take their register by value): the
    reference kernel as written decodes wrong coefficients."""
    z = t1_fixture()
    coded = z["meta"][:, 5] > 0
    assert (z["unpatched_mismatches"][coded] > 0).mean() > 0.9


def test_reference_colour_kernels_match_oracle():
    z = np.load(GOLDEN / "ref_colour.npz")
    for bits in (8, 12):
        img = z[f"rgb{bits}"]
        np.testing.assert_array_equal(np.stack(O.rct_forward(list(img), bits)), z[f"rct{bits}"])
        np.testing.assert_array_equal(np.stack(O.rct_inverse(list(z[f"rct{bits}"]), bits)), z[f"rct_inv{bits}"])
        np.testing.assert_array_equal(z[f"rct_inv{bits}"], img)
        np.testing.assert_array_equal(O.dc_forward(img[0], bits), z[f"dc{bits}"])
        np.testing.assert_array_equal(O.dc_inverse_clamp(z[f"dc{bits}"], bits), z[f"dc_inv{bits}"])
        # forward ICT: the reference rounds to int (convert_int_sat_rte); the
        # oracle keeps FP64 -> equal after rounding except at exact halves
        ict = np.stack(O.ict_forward(list(img), bits))
        d = np.abs(np.rint(ict) - z[f"ict{bits}"])
        assert d.max() <= 1 and (d > 0).mean() < 1e-3


def test_reference_inverse_ict_deviates_from_iso():
    """Defect D9: the reference's inverse ICT uses analogue-YUV constants and
    truncates before rounding; it does not invert the ISO forward ICT."""
    z = np.load(GOLDEN / "ref_colour.npz")
    ycc = z["ycc8"].astype(np.float64)
    iso = np.stack(O.ict_inverse(list(ycc), 8))
    assert np.abs(iso - z["ict_inv8"]).max() > 2


def test_live_reference_kernels_when_built():
    import ref as R
    if not R.available():
        pytest.skip("oracle/_ref not built (reference tree absent)")
    from thousandthchicken_b200 import codec
    from thousandthchicken_b200.synth import laplacian_block
    rng = np.random.default_rng(5)
    blocks, truth = [], []
    for i in range(120):
        w, h = int(rng.integers(2, 65)), int(rng.integers(1, 65))
        orient = int(rng.integers(0, 4))
        coef = laplacian_block(rng, w, h, int(rng.integers(1, 14)))
        seg, passes, zbp = codec.t1_encode_block(coef, orient, 15)
        blocks.append((seg + b"\xff", w, h, orient, 15, 15 - zbp))
        truth.append((seg, zbp, passes))
    raw, _ = R.t1_decode(blocks, patched=True)
    for i, (b, (seg, zbp, passes)) in enumerate(zip(blocks, truth)):
        want = O.t1_decode_raw(seg, b[1], b[2], b[3], 15, zbp, passes)
        np.testing.assert_array_equal(raw[i, :b[2], :b[1]], want)


def _dwt_cases():
    import ref as R
    z = np.load(GOLDEN / "ref_dwt53.npz")
    for k in sorted({f[2:] for f in z.files if f.startswith("x_")}):
        w, h = map(int, k.split("x"))
        yield w, h, z[f"x_{k}"], z[f"fwd_{k}"], z[f"revin_{k}"], z[f"rev_{k}"], R


def test_oracle_53_trunc_equals_reference_kernels():
    """One level of the reference's own 5/3 kernels (dwt_f53.cl, dwt_r53.cl;
    truncating division, defect D13) against the oracle's truncating mode:
    equal on every sample outside the rows the kernels get wrong (D24: the
    forward kernel's top rows; D25: the reverse kernel's last row at even
    heights), and those rows do differ."""
    n = 0
    for w, h, x, fwd, revin, rev, R in _dwt_cases():
        mine = R.mallat_to_packed(O.fdwt53(x, 1, rounding=1), 1)
        mk = R.dwt53_defect_mask(w, h, True)
        np.testing.assert_array_equal(mine[~mk], fwd[~mk], err_msg=f"{w}x{h} forward")
        assert (mine[mk] != fwd[mk]).mean() > 0.9
        back = O.idwt53(R.packed_to_mallat(revin, w, h, 1), 1, rounding=1)
        mr = R.dwt53_defect_mask(w, h, False)
        np.testing.assert_array_equal(back[~mr], rev[~mr], err_msg=f"{w}x{h} reverse")
        np.testing.assert_array_equal(back, x)   # the oracle's own round trip is exact
        if h % 2 == 0:
            assert (back[mr] != rev[mr]).mean() > 0.9
        n += 1
    assert n >= 6


def test_packed_layout_round_trip():
    import ref as R
    rng = np.random.default_rng(3)
    for w, h, lv in [(64, 64, 3), (97, 61, 4), (33, 17, 2)]:
        m = rng.integers(-100, 100, (h, w)).astype(np.int32)
        np.testing.assert_array_equal(R.packed_to_mallat(R.mallat_to_packed(m, lv), w, h, lv), m)


def test_live_reference_53_kernels_match_oracle():
    """With oracle/_ref built: the reference kernels on a fresh 512 x 64
    image (window 128), forward and reverse, against the oracle."""
    import ref as R
    if not R.dwt_available():
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(99)
    w, h = 512, 64
    x = rng.integers(-255, 256, (h, w)).astype(np.int32)
    mine = R.mallat_to_packed(O.fdwt53(x, 1, rounding=1), 1)
    mk = R.dwt53_defect_mask(w, h, True)
    np.testing.assert_array_equal(R.dwt53_forward(x, 1)[~mk], mine[~mk])
    mr = R.dwt53_defect_mask(w, h, False)
    np.testing.assert_array_equal(R.dwt53_reverse(mine, w, h, 1)[~mr], x[~mr])
