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
