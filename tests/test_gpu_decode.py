"""Whole-image decode on the GPU (Tier-1 + fused dequantiser, reverse DWT,
fused inverse colour / DC shift) against OpenJPEG's decode, the oracle and
the original samples."""
import numpy as np
import pytest

import oracle as O
from conftest import golden_cases, load_golden, synth_image
from test_host_codec import (COC_QCC, LAYERED, LAYERED_IDS, PACKED, PRECINCTS, ROI, ROI_IDS, SIGNED, STYLE_IDS, STYLES,
                             SUBSAMPLED, TILED)
from thousandthchicken_b200 import codec

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _decoder(ctx):
    from thousandthchicken_b200.stages import Decoder
    return Decoder(ctx)


def _oracle(cs, r=0.5):
    info, desc, pool = codec.parse(cs)
    return O.decode_tile(desc, pool, info["width"], info["height"], info["ncomp"], info["bits"], info["levels"],
                         info["reversible"], info["mct"], r=r), info


@pytest.mark.parametrize("name,meta", golden_cases(), ids=[n for n, _ in golden_cases()])
def test_decode_openjpeg_streams(gpu_ctx, name, meta):
    cs, original, opj = load_golden(name)
    got = _decoder(gpu_ctx).decode(cs).astype(np.int64)
    if not meta["irreversible"]:
        np.testing.assert_array_equal(got, opj.astype(np.int64))
    else:
        d = np.abs(got - opj.astype(np.int64))
        assert d.max() <= 1
        want, _ = _oracle(cs)
        d2 = np.abs(got - want.astype(np.int64))
        assert d2.max() <= 1
        assert (d2 > 0).mean() < 0.005


@pytest.mark.parametrize("w,h,c,bits,levels", [(512, 512, 3, 8, 5), (333, 217, 3, 12, 4), (64, 64, 1, 16, 3),
                                               (1, 1, 1, 8, 0), (17, 3, 3, 8, 2), (1000, 40, 1, 8, 5)])
def test_lossless_round_trip(gpu_ctx, w, h, c, bits, levels):
    img = synth_image(w, h, c, bits, seed=w + h)
    cs = codec.encode(img, bits, levels=levels, reversible=True, mct=c >= 3)
    got = _decoder(gpu_ctx).decode(cs)
    np.testing.assert_array_equal(got, img)


@pytest.mark.parametrize("w,h,levels", [(1024, 1024, 6), (515, 300, 5)])
def test_lossy_decode_vs_oracle(gpu_ctx, w, h, levels, record_property):
    """Against the oracle's rounded samples: within 1 LSB on < 0.2% of
    samples.  Against its unrounded FP64 samples (9/7, ICT and dequantisation
    in FP64, clamped to the sample range): the GPU's rounded fp32 result is at
    most 0.5 LSB + 0.01 away (rounding plus fp32 error) with PSNR above 55 dB;
    both figures are recorded with the test."""
    img = synth_image(w, h, 3, 8, seed=7)
    cs = codec.encode(img, 8, levels=levels, reversible=False, mct=True, base_step=1 / 128)
    got = _decoder(gpu_ctx).decode(cs).astype(np.int64)
    _, desc, pool = codec.parse(cs)
    want, f64 = O.decode_cblks(O.cblk_array(desc, w, h), len(desc), pool, w, h, 3, 8, levels, False, True, r=0.5,
                               f64=True)
    d = np.abs(got - want.astype(np.int64))
    assert d.max() <= 1, d.max()
    assert (d > 0).mean() < 0.002
    e = np.abs(got.astype(np.float64) - np.clip(f64, 0.0, 255.0))
    psnr64 = 10 * np.log10(255 ** 2 / max(float(np.mean(e * e)), 1e-12))
    record_property("max_abs_vs_fp64", float(e.max()))
    record_property("psnr_vs_fp64_db", float(psnr64))
    assert e.max() <= 0.51, e.max()
    assert psnr64 > 55, psnr64
    mse = np.mean((got - img.astype(np.int64)) ** 2)
    assert 10 * np.log10(255 ** 2 / mse) > 40


def _smooth_image(w, h, seed):
    """12-bit gradients plus +-2 noise: the detail bands code in a few
    bit-planes, the low band in about twelve."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w]
    base = np.stack([x * 3800 // w, y * 3800 // h, (x + y) * 1900 // (w + h)])
    return (base + 100 + rng.integers(-2, 3, (3, h, w))).astype(np.uint16)


def test_few_deep_blocks_ride_with_bulk(gpu_ctx):
    """A handful of blocks with more than 8 coded bit-planes among hundreds
    with fewer: the deep ones are decoded inside the 8-bit launch by the
    heavy decoders.  Lossless, so the output must equal the input."""
    from thousandthchicken_b200.stages import Plan
    img = _smooth_image(1024, 768, 11)
    cs = codec.encode(img, 12, levels=5, reversible=True, mct=True)
    _, desc, _ = codec.parse(cs)
    nb = desc["mb"].astype(int) - desc["zero_bitplanes"].astype(int)
    n16 = int(((nb > 8) & (nb <= 16)).sum())
    assert int((nb <= 8).sum()) > 100 and 0 < n16 <= 64, (n16, np.bincount(nb))
    np.testing.assert_array_equal(_decoder(gpu_ctx).decode(cs), img)
    plan = Plan(gpu_ctx, [cs, cs])
    outs = plan.execute(plan.alloc_outputs())
    gpu_ctx.synchronize()
    for o in outs:
        np.testing.assert_array_equal(o.cpu().numpy().view(np.uint16), img)
    plan.close()


def test_shallow_minority_joins_deep_launch(gpu_ctx):
    """A 12-bit noisy image: mostly blocks with 9-16 coded bit-planes and a
    minority with at most 8, which the 16-bit launch decodes too."""
    img = synth_image(700, 500, 3, 12, seed=21)
    cs = codec.encode(img, 12, levels=5, reversible=True, mct=True)
    _, desc, _ = codec.parse(cs)
    nb = desc["mb"].astype(int) - desc["zero_bitplanes"].astype(int)
    n8, n16 = int((nb <= 8).sum()), int(((nb > 8) & (nb <= 16)).sum())
    assert 0 < n8 and 2 * n8 <= n16, (n8, n16)
    np.testing.assert_array_equal(_decoder(gpu_ctx).decode(cs), img)


def test_batched_levels_of_mixed_depth_equal_single_decodes(gpu_ctx):
    """One plan over images with 0-6 levels, both wavelets, 1 and 3
    components, 8- and 12-bit samples: their DWT levels share launches step
    by step (image i runs its level L_i - t at step t) and must give the
    single-image results bit for bit."""
    from thousandthchicken_b200.stages import Plan
    spec = [(300, 200, 3, 8, 5, True), (64, 48, 1, 12, 0, True), (517, 211, 3, 8, 6, False),
            (33, 129, 1, 8, 1, False), (256, 256, 3, 12, 4, True), (140, 90, 3, 8, 2, False),
            (96, 300, 1, 12, 4, False)]
    streams = [codec.encode(synth_image(w, h, c, b, 30 + i), b, levels=lv, reversible=rev, mct=c == 3,
                            base_step=1 / 64)
               for i, (w, h, c, b, lv, rev) in enumerate(spec)]
    plan = Plan(gpu_ctx, streams)
    outs = plan.alloc_outputs()
    for _ in range(2):  # the second run reuses the uploaded job table
        for o in outs:
            o.zero_()
        plan.execute(outs)
        gpu_ctx.synchronize()
        dec = _decoder(gpu_ctx)
        for s_, o in zip(streams, outs):
            single = dec.decode(s_)
            got = o.cpu().numpy()
            if single.dtype == np.uint16:
                got = got.view(np.uint16)
            np.testing.assert_array_equal(got, single)
    plan.close()


def test_batched_plan_equals_single_decodes(gpu_ctx):
    from thousandthchicken_b200.stages import Plan
    streams = [codec.encode(synth_image(300, 200, 3, 8, 1), 8, levels=5, reversible=True),
               codec.encode(synth_image(128, 256, 1, 12, 2), 12, levels=4, reversible=True, mct=False),
               codec.encode(synth_image(400, 120, 3, 8, 3), 8, levels=5, reversible=False, base_step=1 / 64)]
    plan = Plan(gpu_ctx, streams)
    outs = plan.execute(plan.alloc_outputs())
    gpu_ctx.synchronize()
    dec = _decoder(gpu_ctx)
    for s, o in zip(streams, outs):
        single = dec.decode(s)
        got = o.cpu().numpy()
        if single.dtype == np.uint16:
            got = got.view(np.uint16)
        np.testing.assert_array_equal(got, single)


def test_graphs_per_shape_bucket(gpu_ctx):
    """Graph mode: new outputs replay the bucket's graph (the output
    pointers sit in the DWT job table); a rebuild with the same images
    replays it too; a batch of another shape captures or updates a graph;
    a single-image plan takes the same path.  Every result equals the
    plain decode."""
    from thousandthchicken_b200.stages import Plan
    a = [codec.encode(synth_image(300, 200, 3, 8, 5), 8, levels=5, reversible=True),
         codec.encode(synth_image(200, 180, 3, 8, 6), 8, levels=4, reversible=False, base_step=1 / 64)]
    b = [codec.encode(synth_image(160, 96, 1, 12, 7), 12, levels=3, reversible=True, mct=False),
         codec.encode(synth_image(250, 130, 3, 8, 8), 8, levels=5, reversible=False, base_step=1 / 64)]
    dec = _decoder(gpu_ctx)

    def check(plan, streams, outs):
        gpu_ctx.synchronize()
        for s_, o in zip(streams, outs):
            single = dec.decode(s_)
            got = o.cpu().numpy()
            if single.dtype == np.uint16:
                got = got.view(np.uint16)
            np.testing.assert_array_equal(got, single)

    plan = Plan(gpu_ctx, a)
    plan.set_graph(True)
    o1, o2 = plan.alloc_outputs(), plan.alloc_outputs()
    plan.execute(o1)
    check(plan, a, o1)
    assert plan.graph_stats()["captures"] == 1
    for outs in (o2, o1, o2):   # other outputs: the same graph
        for o in outs:
            o.zero_()
        plan.execute(outs)
        check(plan, a, outs)
    assert plan.graph_stats() == {"captures": 1, "updates": 0, "replays": 3}
    plan.rebuild(a)             # same images, same buffers: replayed
    plan.execute(o2)
    check(plan, a, o2)
    assert plan.graph_stats()["replays"] == 4
    plan.rebuild(b)             # another shape
    ob = plan.alloc_outputs()
    plan.execute(ob)
    check(plan, b, ob)
    plan.execute(ob)
    check(plan, b, ob)
    st = plan.graph_stats()
    assert st["captures"] + st["updates"] == 2 and st["replays"] == 5
    plan.close()
    single = Plan(gpu_ctx, a[1:])
    single.set_graph(True)
    for _ in range(2):
        outs = single.alloc_outputs()
        single.execute(outs)
        check(single, a[1:], outs)
    assert single.graph_stats() == {"captures": 1, "updates": 0, "replays": 1}
    single.close()


def test_decode_file_and_errors(gpu_ctx, tmp_path):
    from thousandthchicken_b200._lib import TCError
    img = synth_image(80, 60, 3, 8, seed=4)
    cs = codec.encode(img, 8, levels=3)
    p = tmp_path / "x.j2k"
    p.write_bytes(cs)
    np.testing.assert_array_equal(_decoder(gpu_ctx).decode(p), img)
    with pytest.raises(TCError):
        _decoder(gpu_ctx).decode(cs[: len(cs) // 3])
    np.testing.assert_array_equal(_decoder(gpu_ctx).decode(cs), img)


def test_graph_replay_and_autotune(gpu_ctx):
    from thousandthchicken_b200 import _lib as L
    from thousandthchicken_b200.autotune import tune_plan
    from thousandthchicken_b200.stages import Plan
    streams = [codec.encode(synth_image(300, 200, 3, 8, 5), 8, levels=5, reversible=True),
               codec.encode(synth_image(200, 180, 3, 8, 6), 8, levels=4, reversible=False, base_step=1 / 64)]
    plan = Plan(gpu_ctx, streams)
    outs = plan.alloc_outputs()
    plan.execute(outs)
    gpu_ctx.synchronize()
    want = [o.cpu().numpy().copy() for o in outs]
    for lanes in (8, 16, 32):
        L.lib().tc_ctx_set_t1_group(gpu_ctx.handle, lanes)
        for o in outs:
            o.zero_()
        plan.execute(outs)
        gpu_ctx.synchronize()
        for o, w in zip(outs, want):
            np.testing.assert_array_equal(o.cpu().numpy(), w)
    L.lib().tc_ctx_set_t1_group(gpu_ctx.handle, 32)
    plan.set_graph(True)
    n0 = gpu_ctx.launches
    for _ in range(3):
        for o in outs:
            o.zero_()
        plan.execute(outs)
        gpu_ctx.synchronize()
        for o, w in zip(outs, want):
            np.testing.assert_array_equal(o.cpu().numpy(), w)
    assert gpu_ctx.launches > n0
    plan.set_graph(False)
    res = tune_plan(plan, outs, trials=1, use_cache=False)
    assert res["lanes"] in (8, 16, 32) and res["dwt"] in ("tma", "cp.async")
    L.lib().tc_ctx_set_t1_group(gpu_ctx.handle, 32)
    L.lib().tc_ctx_set_dwt_variant(gpu_ctx.handle, L.TC_DWT_TMA)
    plan.close()


@pytest.mark.parametrize("size", [(264, 136), (2048, 1024)])
def test_autotuned_choices_decode_like_the_defaults(gpu_ctx, size, tmp_path, monkeypatch):
    """The tuner's choices (Tier-1 lane width, last-level DWT staging) for a
    single lossy RGB image: the tuned decode equals the default decode bit
    for bit, and the cache returns the same choice without searching."""
    from thousandthchicken_b200 import _lib as L
    from thousandthchicken_b200 import autotune
    from thousandthchicken_b200.stages import Plan
    monkeypatch.setattr(autotune, "CACHE", tmp_path / "tune.json")
    w, h = size
    cs = codec.encode(synth_image(w, h, 3, 8, seed=w), 8, levels=5, reversible=False, base_step=1 / 128)
    plan = Plan(gpu_ctx, [cs])
    outs = plan.alloc_outputs()
    plan.execute(outs)
    gpu_ctx.synchronize()
    want = outs[0].cpu().numpy().copy()
    try:
        res = autotune.tune_plan(plan, outs, trials=1)
        assert not res["cached"] and set(res["dwt_ms"]) == {"tma", "cp.async"}
        outs[0].zero_()
        plan.execute(outs)
        gpu_ctx.synchronize()
        np.testing.assert_array_equal(outs[0].cpu().numpy(), want)
        again = autotune.tune_plan(plan, outs)
        assert again["cached"] and (again["lanes"], again["dwt"]) == (res["lanes"], res["dwt"])
    finally:
        L.lib().tc_ctx_set_t1_group(gpu_ctx.handle, 32)
        L.lib().tc_ctx_set_dwt_variant(gpu_ctx.handle, L.TC_DWT_TMA)
        plan.close()


def test_jp2_files_decode(gpu_ctx, tmp_path):
    """JP2 files (the reference's Decoder::decode parses their boxes): one
    written by OpenJPEG through Pillow, losslessly, and the harness's own
    codestream in a JP2 container, from memory and from a .jp2 file."""
    import io
    from PIL import Image
    from test_host_codec import _jp2
    img = synth_image(301, 199, 3, 8, seed=9)
    buf = io.BytesIO()
    Image.fromarray(np.moveaxis(img, 0, -1)).save(buf, format="JPEG2000")
    np.testing.assert_array_equal(_decoder(gpu_ctx).decode(buf.getvalue()), img)
    cs = codec.encode(img, 8, levels=4, reversible=False, base_step=1 / 128)
    jp2 = _jp2(cs, 301, 199, 3, 8)
    p = tmp_path / "x.jp2"
    p.write_bytes(jp2)
    want = _decoder(gpu_ctx).decode(cs)
    np.testing.assert_array_equal(_decoder(gpu_ctx).decode(jp2), want)
    np.testing.assert_array_equal(_decoder(gpu_ctx).decode(p), want)


def _tiled_ids(kw):
    return "-".join(f"{k}={v}" for k, v in kw.items())


@pytest.mark.parametrize("kw", TILED, ids=_tiled_ids)
def test_tiled_streams_decode(gpu_ctx, kw):
    """Tiled OpenJPEG streams (the reference's Decoder::decode loops over
    tiles, Decoder.cpp:127-197): each tile's levels run in the batched
    reverse-DWT launches and its last level writes the tile's region of the
    image.  Lossless: the original; lossy: within 1 LSB of the oracle's
    tile-by-tile decode."""
    from gpu_helpers import oracle_decode_tiled, pil_j2k
    img = synth_image(600, 400, 3, 8, seed=3)
    cs = pil_j2k(img, **kw)
    got = _decoder(gpu_ctx).decode(cs).astype(np.int64)
    _, want = oracle_decode_tiled(cs)
    if kw.get("irreversible"):
        d = np.abs(got - want.astype(np.int64))
        assert d.max() <= 1
        assert (d > 0).mean() < 0.005
    else:
        np.testing.assert_array_equal(got, img)


def test_tiled_and_untiled_images_in_one_plan(gpu_ctx):
    """Tiled and untiled images of both wavelets, 8- and 16-bit, in one plan,
    run twice (the second reuses the job table) and replayed as a graph:
    each output equals the image's own single decode."""
    from gpu_helpers import openjpeg_decode, pil_j2k
    from thousandthchicken_b200.stages import Plan
    g16 = synth_image(300, 260, 1, 16, seed=21)
    streams = [pil_j2k(synth_image(520, 300, 3, 8, seed=20), tile_size=(128, 128)),
               codec.encode(synth_image(400, 120, 3, 8, 22), 8, levels=5, reversible=False, base_step=1 / 64),
               pil_j2k(g16, tile_size=(256, 64), num_resolutions=5),
               pil_j2k(synth_image(333, 257, 3, 8, seed=23), tile_size=(64, 128), irreversible=True),
               codec.encode(synth_image(96, 80, 1, 8, 24), 8, levels=3, reversible=True, mct=False)]
    dec = _decoder(gpu_ctx)
    singles = [dec.decode(s) for s in streams]
    # Pillow's 16-bit tile writer does not hand OpenJPEG the input samples of
    # every tile, so the stream's own content is OpenJPEG's decode of it
    np.testing.assert_array_equal(singles[2], openjpeg_decode(streams[2]))
    np.testing.assert_array_equal(singles[0], synth_image(520, 300, 3, 8, seed=20))
    plan = Plan(gpu_ctx, streams)
    outs = plan.alloc_outputs()
    for graph in (False, False, True, True):
        plan.set_graph(graph)
        for o in outs:
            o.zero_()
        plan.execute(outs)
        gpu_ctx.synchronize()
        for single, o in zip(singles, outs):
            got = o.cpu().numpy()
            if single.dtype == np.uint16:
                got = got.view(np.uint16)
            np.testing.assert_array_equal(got.reshape(single.shape), single)
    plan.close()


@pytest.mark.parametrize("kw", [PRECINCTS[3], PRECINCTS[5], PRECINCTS[7]], ids=_tiled_ids)
def test_precinct_streams_decode(gpu_ctx, kw):
    """Precinct-partitioned streams (code-blocks as small as 2x2 at the
    lowest resolutions) through the GPU: lossless equals the original, lossy
    within 1 LSB of the oracle."""
    from gpu_helpers import oracle_decode_tiled, pil_j2k
    img = synth_image(600, 400, 3, 8, seed=3)
    cs = pil_j2k(img, **kw)
    got = _decoder(gpu_ctx).decode(cs).astype(np.int64)
    if kw.get("irreversible"):
        _, want = oracle_decode_tiled(cs)
        d = np.abs(got - want.astype(np.int64))
        assert d.max() <= 1
        assert (d > 0).mean() < 0.005
    else:
        np.testing.assert_array_equal(got, img)


@pytest.mark.parametrize("kw", COC_QCC, ids=["coc-rev", "qcc-irr", "coc-qcc-irr"])
def test_coc_qcc_streams_decode(gpu_ctx, kw):
    """Per-component code-block sizes and steps (COC / QCC, in the main or
    the tile-part header) through the GPU: lossless equals the original,
    lossy within 1 LSB of the oracle."""
    from gpu_helpers import oracle_decode_tiled
    from test_host_codec import _move_to_tile_header
    img = synth_image(300, 200, 3, 8, seed=5)
    cs = codec.encode(img, 8, levels=4, **kw)
    for s in (cs, _move_to_tile_header(cs)):
        got = _decoder(gpu_ctx).decode(s).astype(np.int64)
        if kw["reversible"]:
            np.testing.assert_array_equal(got, img)
        else:
            _, want = oracle_decode_tiled(s)
            d = np.abs(got - want.astype(np.int64))
            assert d.max() <= 1
            assert (d > 0).mean() < 0.005


def test_digital_cinema_4k_decode(gpu_ctx):
    """OpenJPEG's 4K digital-cinema profile (CPRL with a POC, six
    tile-parts, precincts, 32x32 code-blocks) through the GPU: within 1 LSB
    of the oracle."""
    import io
    from PIL import Image
    from gpu_helpers import oracle_decode_tiled
    img = synth_image(4096, 2160, 3, 8, seed=10)
    buf = io.BytesIO()
    Image.fromarray(np.moveaxis(img, 0, -1)).save(buf, "JPEG2000", cinema_mode="cinema4k-24", no_jp2=True)
    cs = buf.getvalue()
    got = _decoder(gpu_ctx).decode(cs).astype(np.int64)
    _, want = oracle_decode_tiled(cs)
    d = np.abs(got - want.astype(np.int64))
    assert d.max() <= 1
    assert (d > 0).mean() < 0.005


def test_decode_to_pnm_and_pgx(gpu_ctx, tmp_path):
    """Decoder.decode_to_file writes what decode returns: a PPM that Pillow
    reads as the original (lossless) and one PGX per component."""
    from PIL import Image
    from thousandthchicken_b200.imageio import read_pgx
    img = synth_image(120, 90, 3, 8, seed=12)
    cs = codec.encode(img, 8, levels=3)
    dec = _decoder(gpu_ctx)
    (ppm,) = dec.decode_to_file(cs, tmp_path / "o.ppm")
    np.testing.assert_array_equal(np.moveaxis(np.asarray(Image.open(ppm)), -1, 0), img)
    paths = dec.decode_to_file(cs, tmp_path / "o.pgx")
    for c, p in enumerate(paths):
        plane, bits, signed = read_pgx(p)
        np.testing.assert_array_equal(plane, img[c])


@pytest.mark.parametrize("bits,comps,kw", SIGNED, ids=["s12-53", "s16-53", "s8-rct", "s12-97"])
def test_signed_samples_decode(gpu_ctx, bits, comps, kw):
    """Signed components through the GPU (no DC shift, signed clamp, int8 /
    int16 output), alone and in a plan with an unsigned image: lossless
    equals the original, lossy within 1 of the oracle."""
    from gpu_helpers import oracle_decode_tiled
    from test_host_codec import _ct_like
    from thousandthchicken_b200.stages import Plan
    img = _ct_like(120, 150, bits, seed=bits) if comps == 1 else \
        np.random.default_rng(5).integers(-128, 128, (3, 40, 50)).astype(np.int8)
    cs = codec.encode(img, bits, levels=4, **kw)
    got = _decoder(gpu_ctx).decode(cs)
    assert got.dtype == (np.int8 if bits <= 8 else np.int16)
    _, want = oracle_decode_tiled(cs)
    if kw["reversible"]:
        np.testing.assert_array_equal(got, img)
    else:
        d = np.abs(got.astype(np.int64) - want.astype(np.int64))
        assert d.max() <= 1 and (d > 0).mean() < 0.005
    other = codec.encode(synth_image(64, 48, comps, bits, seed=1), bits, levels=3, **kw)
    plan = Plan(gpu_ctx, [cs, other])
    outs = plan.execute(plan.alloc_outputs())
    gpu_ctx.synchronize()
    g0 = outs[0].cpu().numpy()
    np.testing.assert_array_equal(g0.view(np.int16) if bits > 8 else g0, got)
    plan.close()


@pytest.mark.parametrize("w,h,bits,dxy,kw", SUBSAMPLED, ids=["420", "422-97-odd", "g12-pcrl", "cprl-odd-factors"])
def test_subsampled_components_decode(gpu_ctx, w, h, bits, dxy, kw):
    """Subsampled components through the GPU: one reverse DWT unit per
    component at its own size, each written to its own plane of the planar
    output; alone (Decoder.decode returns one array per component) and in a
    plan beside an image without subsampling.  Lossless: the original
    components; lossy: within 1 of the oracle."""
    from gpu_helpers import oracle_decode_components
    from test_host_codec import _subsampled
    from thousandthchicken_b200.stages import Plan, split_components
    comps = _subsampled(w, h, bits, dxy, seed=w)
    cs = codec.encode(comps, bits, levels=3, mct=False, comp_subsampling=dxy, **kw)
    got = _decoder(gpu_ctx).decode(cs)
    _, want = oracle_decode_components(cs)
    for g, c_, o in zip(got, comps, want):
        if kw["reversible"]:
            np.testing.assert_array_equal(g, c_)
        else:
            d = np.abs(g.astype(np.int64) - o.astype(np.int64))
            assert d.max() <= 1 and (d > 0).mean() < 0.01
    other = codec.encode(synth_image(64, 48, 3, bits, seed=1), bits, levels=3, reversible=True)
    plan = Plan(gpu_ctx, [other, cs])
    outs = plan.execute(plan.alloc_outputs())
    gpu_ctx.synchronize()
    flat = outs[1].cpu().numpy()
    if bits > 8:
        flat = flat.view(np.uint16)
    for g, p_ in zip(got, split_components(flat, plan.infos[1]["comp_sizes"])):
        np.testing.assert_array_equal(p_, g)
    plan.close()


@pytest.mark.parametrize("style,bits,kw", STYLES, ids=STYLE_IDS)
def test_code_block_styles_decode(gpu_ctx, style, bits, kw):
    """Code-block styles through the GPU: the styled blocks run in the
    style-capable Tier-1 launch (terminated segments from the pool's length
    tables, raw bypass passes, context resets, vertically causal contexts,
    segmentation symbols).  Lossless: the original; lossy: within 1 of the
    oracle."""
    from gpu_helpers import oracle_decode_tiled
    from test_host_codec import styled_stream
    img, cs = styled_stream(style, bits, kw)
    got = _decoder(gpu_ctx).decode(cs)
    if kw["reversible"]:
        np.testing.assert_array_equal(got, img)
    else:
        _, want = oracle_decode_tiled(cs)
        d = np.abs(got.astype(np.int64) - want.astype(np.int64))
        assert d.max() <= 1 and (d > 0).mean() < 0.01


def test_styled_and_plain_streams_in_one_plan(gpu_ctx):
    """A plan over a styled stream and a style-0 one: the styled blocks form
    a class of their own after the three bit-plane classes; both images
    come out as their single decodes."""
    from test_host_codec import styled_stream
    from thousandthchicken_b200.stages import Plan
    img_a, a = styled_stream(0x3F, 8, dict(reversible=True))
    img_b = synth_image(96, 80, 3, 8, seed=4)
    b = codec.encode(img_b, 8, levels=3, reversible=True)
    plan = Plan(gpu_ctx, [a, b])
    outs = plan.execute(plan.alloc_outputs())
    gpu_ctx.synchronize()
    np.testing.assert_array_equal(outs[0].cpu().numpy(), img_a)
    np.testing.assert_array_equal(outs[1].cpu().numpy(), img_b)
    plan.close()


def test_styled_blocks_in_a_style0_launch_are_errors(gpu_ctx):
    """tc_t1_decode without TC_T1_STYLED leaves styled blocks undecoded and
    reports them at the next synchronize; with it they decode like the
    oracle's Tier-1."""
    from test_host_codec import styled_stream
    from thousandthchicken_b200._lib import TCError
    from thousandthchicken_b200.stages import CoefficientCoder, _dev_bytes
    import torch
    img, cs = styled_stream(codec.CBLK_STYLE_BYPASS | codec.CBLK_STYLE_TERMALL, 8, dict(reversible=True))
    coder = CoefficientCoder(gpu_ctx)
    info, desc, pool = codec.parse(cs)
    dev = torch.device("cuda")
    n = info["ncomp"] * info["width"] * info["height"]
    out = torch.zeros(n, dtype=torch.int32, device=dev)
    d_desc, d_pool = _dev_bytes(desc, dev), _dev_bytes(pool, dev)
    coder.decode(d_desc, d_pool, out, len(desc), styled=False)
    with pytest.raises(TCError):
        gpu_ctx.synchronize()
    gpu_ctx.synchronize()  # the error word was cleared
    got, _ = coder.decode_tile(cs)
    plain_cs = codec.encode(img, 8, levels=3, cblk_log2=5, reversible=True)
    want, _ = coder.decode_tile(plain_cs)
    np.testing.assert_array_equal(got.cpu().numpy(), want.cpu().numpy())


@pytest.mark.parametrize("style,prog,layers", LAYERED, ids=LAYERED_IDS)
def test_layered_streams_decode(gpu_ctx, style, prog, layers):
    """Harness-encoded quality layers in every progression order, with and
    without code-block styles: the blocks' contributions gathered across
    layers (a bypass segment cut by a layer boundary included) decode on the
    GPU to the original."""
    img = synth_image(133, 91, 3, 8, seed=style + prog + layers)
    cs = codec.encode(img, 8, levels=3, cblk_log2=5, reversible=True, cblk_style=style, progression=prog,
                      layers=layers)
    np.testing.assert_array_equal(_decoder(gpu_ctx).decode(cs), img)


@pytest.mark.parametrize("where,style,prog,layers", PACKED,
                         ids=[f"{'ppt' if w == 1 else 'ppm'}-style{s:#x}-prog{p}-{n}layers" for w, s, p, n in PACKED])
def test_packed_packet_headers_decode(gpu_ctx, where, style, prog, layers):
    """PPT / PPM streams decode on the GPU to the original."""
    img = synth_image(133, 91, 3, 8, seed=where + prog)
    cs = codec.encode(img, 8, levels=3, cblk_log2=5, reversible=True, cblk_style=style, progression=prog,
                      layers=layers, packed_headers=where)
    np.testing.assert_array_equal(_decoder(gpu_ctx).decode(cs), img)


@pytest.mark.parametrize("bits,comps,roi,kw", ROI, ids=ROI_IDS)
def test_roi_maxshift_decode(gpu_ctx, bits, comps, roi, kw):
    """ROI maxshift streams on the GPU: the Tier-1 epilogue shifts region
    magnitudes back down; lossless equals the original, lossy is within 1
    of the oracle."""
    from gpu_helpers import oracle_decode_tiled
    img = synth_image(133, 91, comps, bits, seed=bits + comps)
    cs = codec.encode(img, bits, levels=3, cblk_log2=5, mct=comps == 3, roi=roi, **kw)
    got = _decoder(gpu_ctx).decode(cs)
    if kw["reversible"]:
        np.testing.assert_array_equal(got, img)
    else:
        _, want = oracle_decode_tiled(cs)
        d = np.abs(got.astype(np.int64) - want.astype(np.int64))
        assert d.max() <= 1 and (d > 0).mean() < 0.01


def test_large_image_round_trip(gpu_ctx):
    """A 16384 x 16384 x 3 lossless image (3.2 GB of coefficients, byte
    offsets past 2^31, 196,608 code-blocks, 112k DWT tiles in the last
    level): GPU encode, then GPU decode, gives back the original."""
    rng = np.random.default_rng(16384)
    n = 16384
    y = (np.arange(n, dtype=np.int32) * 7)[:, None]
    x = (np.arange(n, dtype=np.int32) * 3)[None, :]
    base = ((x + y) & 255).astype(np.uint8)
    img = np.stack([base, base[::-1], base[:, ::-1]])
    img[:, ::97, ::89] = rng.integers(0, 256, img[:, ::97, ::89].shape, dtype=np.uint8)
    cs = codec.encode_gpu(gpu_ctx, img, 8, levels=6, reversible=True, mct=True)
    got = _decoder(gpu_ctx).decode(cs)
    assert np.array_equal(got, img)


def test_styled_deep_blocks_ride_in_the_bulk_launch(gpu_ctx):
    """A styled lossy image whose blocks mostly code 4 bit-planes, with a few
    deep low-band blocks: those ride in the styled 8-bit launch with 16-bit
    state (heavy queue); within 1 of the oracle."""
    from gpu_helpers import oracle_decode_tiled
    from thousandthchicken_b200.synth import gradient_noise_image
    img = gradient_noise_image(1024, 1024, 3, 8, seed=1024)
    cs = codec.encode(img, 8, levels=6, reversible=False, mct=True, base_step=1 / 128,
                      cblk_style=codec.CBLK_STYLE_BYPASS | codec.CBLK_STYLE_TERMALL)
    info, desc, _ = codec.parse(cs)
    nb = np.where(desc["passes"] > 0, desc["mb"].astype(int) - desc["zero_bitplanes"].astype(int), 0)
    deep = int(((nb > 8) & (nb <= 16)).sum())
    # the heavy queue takes at most one deep block per SM (kMaxHeavy = 148 in
    # t1_decode.cu); more would go to a separate 16-bit launch
    assert 0 < deep <= 148 and 8 * deep <= int((nb <= 8).sum()) and nb.max() <= 16
    got = _decoder(gpu_ctx).decode(cs).astype(np.int64)
    _, want = oracle_decode_tiled(cs)
    d = np.abs(got - want.astype(np.int64))
    assert d.max() <= 1 and (d > 0).mean() < 0.002
