"""Host-side code (no GPU): the harness encoder, the Tier-2 parser and the
Tier-1 oracle round trips, and the error behaviour of the parser."""
import io

import numpy as np
import pytest

import oracle as O
from conftest import synth_image
from thousandthchicken_b200 import codec
from thousandthchicken_b200._lib import TCError, TC_E_CODESTREAM, TC_E_UNSUPPORTED
from thousandthchicken_b200.synth import laplacian_block


@pytest.mark.parametrize("w,h,c,bits,levels", [(64, 64, 1, 8, 2), (97, 53, 3, 8, 3), (512, 512, 3, 8, 5),
                                               (130, 70, 3, 12, 4), (1, 1, 1, 8, 0), (1, 37, 1, 8, 3),
                                               (45, 1, 3, 8, 2), (3, 2, 3, 16, 1), (200, 9, 1, 16, 3)])
def test_lossless_round_trip_through_oracle(w, h, c, bits, levels):
    img = synth_image(w, h, c, bits, seed=w * 7 + h)
    cs = codec.encode(img, bits, levels=levels, reversible=True, mct=c >= 3)
    info, desc, pool = codec.parse(cs)
    assert info["ncblk"] == len(desc)
    out = O.decode_tile(desc, pool, w, h, c, bits, levels, True, info["mct"])
    np.testing.assert_array_equal(out, img)


def test_config0_round_trip_512x512_rgb():
    """The CPU-runnable round trip: 512x512x3 8-bit, DC shift, RCT, 5-level
    5/3, lossless quantiser, inverse RCT, inverse DC shift -> identical."""
    img = synth_image(512, 512, 3, 8, seed=0)
    cs = codec.encode(img, 8, levels=5, reversible=True, mct=True)
    info, desc, pool = codec.parse(cs)
    out = O.decode_tile(desc, pool, 512, 512, 3, 8, 5, True, True)
    np.testing.assert_array_equal(out, img)


@pytest.mark.parametrize("orient", [0, 1, 2, 3])
@pytest.mark.parametrize("w,h", [(64, 64), (32, 32), (1, 1), (64, 1), (1, 64), (17, 45), (63, 5)])
def test_t1_block_truncation(orient, w, h):
    """Encode one block, keep a random number of passes, decode with the
    oracle: the result equals the coefficients truncated to the decoded
    bit-planes of each pass."""
    rng = np.random.default_rng(orient * 1000 + w * 64 + h)
    coef = laplacian_block(rng, w, h, bitplanes=int(rng.integers(1, 14)))
    mb = 14
    seg, total, zbp = codec.t1_encode_block(coef, orient, mb)
    numbps = mb - zbp
    if total == 0:
        assert not coef.any()
        return
    assert total == 3 * numbps - 2
    q, u = O.t1_decode(seg, w, h, orient, numbps, total)
    np.testing.assert_array_equal(q, coef)
    for passes in sorted(set(rng.integers(1, total + 1, 4).tolist()) | {1, total}):
        seg_k, got, _ = codec.t1_encode_block(coef, orient, mb, passes)
        assert got == passes
        q, u = O.t1_decode(seg_k, w, h, orient, numbps, passes)
        # every decoded magnitude is a prefix of the true magnitude
        mag = np.abs(coef)
        assert np.all((np.abs(q) >> u) << u == np.abs(q))
        assert np.all((mag >> u) == np.abs(q) >> u)
        assert np.all(np.sign(q)[q != 0] == np.sign(coef)[q != 0])


def test_parser_rejects_corrupt_streams():
    img = synth_image(64, 48, 3, 8, seed=3)
    cs = codec.encode(img, 8, levels=3)
    with pytest.raises(TCError) as e:
        codec.parse(cs[:40])
    assert e.value.status in (TC_E_CODESTREAM,)
    with pytest.raises(TCError):
        codec.parse(b"\x00\x01" + cs[2:])
    # truncated packet data: the code-block lengths run past the tile-part
    with pytest.raises(TCError) as e:
        codec.parse(cs[: len(cs) // 2])
    assert e.value.status == TC_E_CODESTREAM
    # random corruption never crashes the parser
    rng = np.random.default_rng(0)
    for _ in range(200):
        b = bytearray(cs)
        for _k in range(4):
            b[int(rng.integers(0, len(b)))] = int(rng.integers(0, 256))
        try:
            codec.parse(bytes(b))
        except TCError as ex:
            assert ex.status in (TC_E_CODESTREAM, TC_E_UNSUPPORTED, -1)


def test_header_fields():
    img = synth_image(300, 200, 3, 12, seed=9)
    cs = codec.encode(img, 12, levels=4, reversible=False, mct=True, base_step=1 / 64)
    h = codec.read_header(cs)
    assert (h["width"], h["height"], h["ncomp"], h["bits"], h["levels"], h["reversible"], h["mct"]) == \
        (300, 200, 3, 12, 4, 0, 1)
    assert h["quant_style"] == 2


def test_our_encoder_decodes_in_openjpeg():
    PIL = pytest.importorskip("PIL.Image")
    img = synth_image(96, 80, 3, 8, seed=11)
    cs = codec.encode(img, 8, levels=4, reversible=True, mct=True)
    dec = np.moveaxis(np.asarray(PIL.open(io.BytesIO(cs))), -1, 0)
    np.testing.assert_array_equal(dec, img)


def test_sort_order_longest_first():
    d = np.zeros(5, codec.DESC_DTYPE)
    d["w"] = d["h"] = 64
    d["passes"] = [1, 7, 3, 7, 0]
    d["seg_len"] = [10, 5, 3, 50, 0]
    assert codec.sort_order(d).tolist() == [3, 1, 2, 0, 4]


# ---- JP2 file format (Decoder::decode reads .jp2 through jp2_parse_boxes) ----

def _box(t: bytes, body: bytes, form: str = "short") -> bytes:
    import struct
    if form == "xl":  # LBox = 1, 8-byte length follows
        return struct.pack(">I4sQ", 1, t, 16 + len(body)) + body
    if form == "eof":  # LBox = 0, the box runs to the end of the file
        return struct.pack(">I4s", 0, t) + body
    return struct.pack(">I4s", 8 + len(body), t) + body


def _jp2(cs: bytes, w: int, h: int, nc: int, bits: int, form: str = "short", ihdr_w: int | None = None) -> bytes:
    import struct
    sig = _box(b"jP  ", bytes.fromhex("0d0a870a"))
    ftyp = _box(b"ftyp", b"jp2 " + struct.pack(">I", 0) + b"jp2 ")
    ihdr = _box(b"ihdr", struct.pack(">IIHBBBB", h, ihdr_w if ihdr_w is not None else w, nc, bits - 1, 7, 0, 0))
    colr = _box(b"colr", struct.pack(">BBBI", 1, 0, 0, 16 if nc >= 3 else 17))
    return sig + ftyp + _box(b"jp2h", ihdr + colr) + _box(b"xml ", b"<x/>") + _box(b"jp2c", cs, form)


@pytest.mark.parametrize("form", ["short", "xl", "eof"])
def test_jp2_file_parses_like_its_codestream(form):
    img = synth_image(90, 70, 3, 8, seed=3)
    cs = codec.encode(img, 8, levels=3)
    jp2 = _jp2(cs, 90, 70, 3, 8, form)
    off = len(jp2) - len(cs)
    info_a, desc_a, pool_a = codec.parse(cs)
    info_b, desc_b, pool_b = codec.parse(jp2)
    assert info_a == info_b
    assert codec.read_header(jp2) == codec.read_header(cs)
    np.testing.assert_array_equal(desc_b["seg_off"], desc_a["seg_off"] + off)
    for name in desc_a.dtype.names:
        if name != "seg_off":
            np.testing.assert_array_equal(desc_a[name], desc_b[name])
    for da, db in zip(desc_a, desc_b):
        a, b = int(da["seg_off"]), int(db["seg_off"])
        assert bytes(pool_a[a:a + da["seg_len"]]) == bytes(pool_b[b:b + db["seg_len"]])


def test_jp2_written_by_openjpeg_parses():
    import io
    from PIL import Image
    img = synth_image(52, 40, 3, 8, seed=4)
    buf = io.BytesIO()
    Image.fromarray(np.moveaxis(img, 0, -1)).save(buf, format="JPEG2000")
    data = buf.getvalue()
    assert data[4:8] == b"jP  "
    info = codec.read_header(data)
    assert (info["width"], info["height"], info["ncomp"]) == (52, 40, 3)
    _, desc, _ = codec.parse(data)
    assert len(desc) > 0


@pytest.mark.parametrize("case", ["no_jp2c", "truncated", "ihdr_mismatch", "no_ftyp", "garbage"])
def test_bad_jp2_files_are_rejected(case):
    img = synth_image(40, 30, 1, 8, seed=5)
    cs = codec.encode(img, 8, levels=2, mct=False)
    good = _jp2(cs, 40, 30, 1, 8)
    data = {"no_jp2c": good[: len(good) - len(cs) - 8],
            "truncated": good[: len(good) - len(cs) // 2 - 4] + b"\x00" * 3,
            "ihdr_mismatch": _jp2(cs, 40, 30, 1, 8, ihdr_w=41),
            "no_ftyp": good.replace(b"ftyp", b"ftyq", 1),
            "garbage": b"\x00\x01\x02\x03" * 8}[case]
    with pytest.raises(TCError):
        codec.parse(data)


TILED = [  # OpenJPEG encoder options: tile grids, image and tile offsets, progressions
    dict(tile_size=(256, 256)),
    dict(tile_size=(128, 256), num_resolutions=4),
    dict(tile_size=(256, 128), progression="RPCL"),
    dict(tile_size=(96, 160)),  # tiles whose subbands start inside a code-block
    dict(tile_size=(256, 256), offset=(32, 64)),
    dict(tile_size=(192, 96), offset=(64, 32), irreversible=True),
    dict(tile_size=(512, 512), irreversible=True, quality_mode="rates", quality_layers=[20, 5]),
]


@pytest.mark.parametrize("kw", TILED, ids=lambda kw: "-".join(f"{k}={v}" for k, v in kw.items()))
def test_tiled_streams_through_oracle(kw):
    """Tiled codestreams written by OpenJPEG: the parser's tile grid (ISO B.3,
    the reference's init_tiles, codestream_image.c:256-270) partitions the
    image, each tile's coefficients are a tile-major arena, and the oracle
    decodes each tile to the original (lossless) or within 1 LSB of
    OpenJPEG's own decode (lossy)."""
    pytest.importorskip("PIL.Image")
    from gpu_helpers import oracle_decode_tiled, openjpeg_decode, pil_j2k
    img = synth_image(600, 400, 3, 8, seed=3)
    cs = pil_j2k(img, **kw)
    info, out = oracle_decode_tiled(cs)
    tiles = info["tiles"]
    assert info["ntiles"] == len(tiles) > 1
    cover = np.zeros((400, 600), np.int32)
    off = 0
    for x0, y0, w, h, co in tiles:
        cover[y0:y0 + h, x0:x0 + w] += 1
        assert co == off
        off += 3 * w * h
    assert (cover == 1).all()
    if kw.get("irreversible"):
        assert np.abs(out.astype(np.int64) - openjpeg_decode(cs)).max() <= 1
    else:
        np.testing.assert_array_equal(out, img)


def test_tile_origins_off_the_dwt_grid_are_unsupported():
    """Tiles whose origin is not a multiple of 2^levels would need odd-origin
    lifting: refused as unsupported, by the header reader too."""
    pytest.importorskip("PIL.Image")
    from gpu_helpers import pil_j2k
    cs = pil_j2k(synth_image(300, 200, 1, 8, seed=4), tile_size=(100, 100))
    for fn in (codec.parse, codec.read_header):
        with pytest.raises(TCError) as ei:
            fn(cs)
        assert ei.value.status == TC_E_UNSUPPORTED


def test_tiled_16bit_stream_matches_openjpeg():
    """A 16-bit single-component tiled stream with ragged edge tiles decodes
    through the oracle exactly as OpenJPEG decodes it."""
    pytest.importorskip("PIL.Image")
    from gpu_helpers import oracle_decode_tiled, openjpeg_decode, pil_j2k
    cs = pil_j2k(synth_image(300, 260, 1, 16, seed=21), tile_size=(256, 64), num_resolutions=5)
    info, out = oracle_decode_tiled(cs)
    assert info["ntiles"] == 10 and info["bits"] == 16
    np.testing.assert_array_equal(out, openjpeg_decode(cs))


PRECINCTS = [  # OpenJPEG encoder options with precinct partitions (several precincts per resolution)
    dict(codeblock_size=(32, 32), precinct_size=(64, 64), progression="LRCP"),
    dict(codeblock_size=(32, 32), precinct_size=(64, 64), progression="RLCP"),
    dict(codeblock_size=(32, 32), precinct_size=(64, 64), progression="RPCL"),
    dict(codeblock_size=(32, 32), precinct_size=(64, 64), progression="PCRL"),
    dict(codeblock_size=(32, 32), precinct_size=(64, 64), progression="CPRL"),
    dict(codeblock_size=(16, 16), precinct_size=(128, 32), progression="PCRL", irreversible=True),
    dict(codeblock_size=(32, 32), precinct_size=(64, 64), tile_size=(256, 256), progression="CPRL"),
    dict(codeblock_size=(32, 32), precinct_size=(128, 128), tile_size=(192, 96), offset=(64, 32),
         progression="RPCL", quality_mode="rates", quality_layers=[20, 5], irreversible=True),
    dict(codeblock_size=(64, 64), precinct_size=(256, 256), num_resolutions=7, progression="PCRL"),
]


@pytest.mark.parametrize("kw", PRECINCTS, ids=lambda kw: "-".join(f"{k}={v}" for k, v in kw.items()))
def test_precinct_streams_through_oracle(kw):
    """Precinct partitions (ISO B.6): packets per precinct in all five
    progression orders, the position-driven ones (RPCL, PCRL, CPRL) visiting
    each precinct at its first reference-grid position (B.12.1.3-B.12.1.5),
    code-blocks capped to the precinct size (B.7), one tag-tree pair per
    precinct and band.  The reference reads one precinct per resolution
    (codestream.c:373-376); lossless decodes equal the original, lossy ones
    OpenJPEG's decode within 1 LSB."""
    pytest.importorskip("PIL.Image")
    from gpu_helpers import oracle_decode_tiled, openjpeg_decode, pil_j2k
    img = synth_image(600, 400, 3, 8, seed=3)
    cs = pil_j2k(img, **kw)
    info, out = oracle_decode_tiled(cs)
    if kw.get("irreversible"):
        assert np.abs(out.astype(np.int64) - openjpeg_decode(cs)).max() <= 1
    else:
        np.testing.assert_array_equal(out, img)


def _main_header_markers(cs):
    """(marker, offset, length) of the main header's marker segments."""
    out, pos = [], 2
    while True:
        m = int.from_bytes(cs[pos:pos + 2], "big")
        if m == 0xFF90:
            return out, pos
        n = int.from_bytes(cs[pos + 2:pos + 4], "big")
        out.append((m, pos, n + 2))
        pos += n + 2


def _move_to_tile_header(cs, markers=(0xFF53, 0xFF5D)):
    """The same codestream with the main header's COC/QCC segments moved
    into the single tile-part's header (Psot grown to match)."""
    segs, sot = _main_header_markers(cs)
    moved = b"".join(cs[o:o + n] for m, o, n in segs if m in markers)
    main = cs[:2] + b"".join(cs[o:o + n] for m, o, n in segs if m not in markers)
    psot = int.from_bytes(cs[sot + 6:sot + 10], "big")
    sot_seg = bytearray(cs[sot:sot + 12])
    sot_seg[6:10] = (psot + len(moved)).to_bytes(4, "big")
    return main + bytes(sot_seg) + moved + cs[sot + 12:]


COC_QCC = [  # harness-encoder options written as COC / QCC marker segments
    dict(reversible=True, comp_cblk_log2=[0, 4, 5]),
    dict(reversible=False, comp_step_scale=[1, 4, 0.5]),
    dict(reversible=False, comp_cblk_log2=[5, 0, 3], comp_step_scale=[0, 2, 2]),
]


@pytest.mark.parametrize("kw", COC_QCC, ids=["coc-rev", "qcc-irr", "coc-qcc-irr"])
def test_coc_qcc_streams_through_oracle(kw):
    """Per-component code-block sizes (COC) and step sizes (QCC), in the main
    header and moved into the tile-part header (ISO A.6 precedence: tile
    COC/QCC > tile COD/QCD > main COC/QCC > main COD/QCD).  The reference
    reads COD/QCD only and stubs COC/QCC (codestream.c:137-140).  OpenJPEG
    decodes the same streams; lossless equals the original, lossy agrees
    with OpenJPEG within 1 LSB."""
    pytest.importorskip("PIL.Image")
    from gpu_helpers import oracle_decode_tiled, openjpeg_decode
    img = synth_image(300, 200, 3, 8, seed=5)
    cs = codec.encode(img, 8, levels=4, **kw)
    segs, _ = _main_header_markers(cs)
    kinds = {m for m, _, _ in segs}
    assert (0xFF53 in kinds) == bool(kw.get("comp_cblk_log2"))
    assert (0xFF5D in kinds) == bool(kw.get("comp_step_scale"))
    info, out = oracle_decode_tiled(cs)
    if kw["reversible"]:
        np.testing.assert_array_equal(out, img)
    else:
        assert np.abs(out.astype(np.int64) - openjpeg_decode(cs)).max() <= 1
    moved = _move_to_tile_header(cs)
    assert moved != cs and len(moved) == len(cs)
    info2, out2 = oracle_decode_tiled(moved)
    np.testing.assert_array_equal(out2, out)
    _, d1, _ = codec.parse(cs)
    _, d2, _ = codec.parse(moved)
    for f in ("w", "h", "mb", "zero_bitplanes", "passes", "step", "out_off", "seg_len"):
        np.testing.assert_array_equal(d1[f], d2[f])


def test_component_levels_must_agree():
    """A COC that changes a component's decomposition levels is refused as
    unsupported (the fused colour level needs one geometry per image)."""
    img = synth_image(64, 48, 3, 8, seed=6)
    cs = bytearray(codec.encode(img, 8, levels=3, reversible=True, comp_cblk_log2=[0, 5, 0]))
    segs, _ = _main_header_markers(bytes(cs))
    (_, off, _), = [s for s in segs if s[0] == 0xFF53]
    cs[off + 6] = 2  # SPcoc levels: 3 -> 2
    with pytest.raises(TCError) as ei:
        codec.parse(bytes(cs))
    assert ei.value.status == TC_E_UNSUPPORTED


def _with_main_marker(cs, marker, body):
    """The codestream with one more main-header marker segment before the
    first SOT."""
    _, sot = _main_header_markers(cs)
    return cs[:sot] + marker.to_bytes(2, "big") + (len(body) + 2).to_bytes(2, "big") + body + cs[sot:]


def _poc(*entries):
    """POC body (ISO A.6.6) for fewer than 257 components: (RSpoc, CSpoc,
    LYEpoc, REpoc, CEpoc, Ppoc) per progression volume."""
    return b"".join(bytes([rs, cs]) + lye.to_bytes(2, "big") + bytes([re, ce, p]) for rs, cs, lye, re, ce, p in entries)


@pytest.mark.parametrize("prog,vols", [
    ("LRCP", [(0, 0, 1, 6, 3, 0), (0, 0, 3, 6, 3, 0)]),            # layer 0 first, then the rest
    ("RPCL", [(0, 0, 3, 2, 3, 2), (2, 0, 3, 6, 3, 2)]),            # resolutions 0-1, then 2-5
    # resolution 3 in two volumes by layer, the second skipping what the first read
    ("RLCP", [(0, 0, 3, 3, 3, 1), (3, 0, 2, 4, 3, 1), (3, 0, 3, 4, 3, 1), (4, 0, 3, 6, 3, 1)]),
], ids=["lrcp-by-layer", "rpcl-by-resolution", "rlcp-four-volumes"])
def test_poc_volumes(prog, vols):
    """Progression order changes (POC, ISO A.6.6): volumes that restate the
    stream's own order in pieces give the same descriptors as the plain
    stream, each packet read once at the first volume that reaches it (the
    reference reads one order from COD)."""
    pytest.importorskip("PIL.Image")
    from gpu_helpers import pil_j2k
    img = synth_image(300, 200, 3, 8, seed=7)
    cs = pil_j2k(img, num_resolutions=6, progression=prog, irreversible=True, quality_mode="rates",
                 quality_layers=[40, 20, 10], codeblock_size=(32, 32), precinct_size=(64, 64))
    with_poc = _with_main_marker(cs, 0xFF5F, _poc(*vols))
    _, d1, p1 = codec.parse(cs)
    _, d2, p2 = codec.parse(with_poc)
    for f in ("w", "h", "mb", "zero_bitplanes", "passes", "step", "out_off", "seg_len"):
        np.testing.assert_array_equal(d1[f], d2[f])
    np.testing.assert_array_equal(p1, p2)  # multi-layer: gathered pools, byte for byte


def test_bad_poc_entries_are_rejected():
    """A volume whose resolution or component range is empty, or whose
    progression is out of range, is a malformed codestream."""
    pytest.importorskip("PIL.Image")
    from gpu_helpers import pil_j2k
    cs = pil_j2k(synth_image(64, 64, 1, 8, seed=8), num_resolutions=3)
    for entry in [(2, 0, 1, 1, 1, 0), (0, 1, 1, 3, 1, 0), (0, 0, 1, 3, 1, 5)]:
        with pytest.raises(TCError) as ei:
            codec.parse(_with_main_marker(cs, 0xFF5F, _poc(entry)))
        assert ei.value.status == TC_E_CODESTREAM


@pytest.mark.parametrize("mode", ["cinema2k-24", "cinema4k-24"])
def test_digital_cinema_profiles(mode):
    """OpenJPEG's digital-cinema profiles: 2K (CPRL, one tile-part per
    component, precincts) and 4K (CPRL with a POC in the first of six
    tile-parts) decode within 1 LSB of OpenJPEG."""
    pytest.importorskip("PIL.Image")
    from gpu_helpers import oracle_decode_tiled, openjpeg_decode
    import io
    from PIL import Image
    w, h = (4096, 2160) if mode.startswith("cinema4k") else (2048, 1080)
    img = synth_image(w, h, 3, 8, seed=10)
    buf = io.BytesIO()
    Image.fromarray(np.moveaxis(img, 0, -1)).save(buf, "JPEG2000", cinema_mode=mode, no_jp2=True)
    cs = buf.getvalue()
    info, out = oracle_decode_tiled(cs)
    assert info["progression"] == 4
    assert np.abs(out.astype(np.int64) - openjpeg_decode(cs)).max() <= 1


def test_pnm_and_pgx_writers_round_trip(tmp_path):
    """The output writers: PGM/PPM (8 and 12 bit) and PGX (unsigned and
    signed) read back identically, and Pillow reads the 8-bit PNM files."""
    from PIL import Image
    from thousandthchicken_b200.imageio import read_pgx, read_pnm, write_image
    rgb = synth_image(37, 21, 3, 8, seed=1)
    g12 = synth_image(40, 30, 1, 12, seed=2)
    for planes, bits, name in [(rgb, 8, "a.ppm"), (g12, 12, "b.pgm"), (rgb[:1], 8, "c.pgm")]:
        (p,) = write_image(tmp_path / name, planes, bits)
        back, b2 = read_pnm(p)
        np.testing.assert_array_equal(back, planes)
        assert b2 == bits
        if bits == 8:  # (Pillow rescales deeper PGMs to 16 bits)
            pil = np.asarray(Image.open(p))
            np.testing.assert_array_equal(pil[None] if pil.ndim == 2 else np.moveaxis(pil, -1, 0), planes)
    s16 = (synth_image(20, 10, 2, 16, seed=3).astype(np.int32) - 32768).astype(np.int16)
    for planes, bits, signed in [(rgb, 8, False), (s16, 16, True)]:
        paths = write_image(tmp_path / "x.pgx", planes, bits, signed)
        assert len(paths) == planes.shape[0]
        for c, p in enumerate(paths):
            plane, b2, sg = read_pgx(p)
            np.testing.assert_array_equal(plane, planes[c])
            assert (b2, sg) == (bits, signed)


def _ct_like(h, w, bits, seed):
    """A signed single-component image like a CT slice: a smooth field
    around zero plus noise, clipped to the signed range of `bits`."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    lo, hi = -(1 << (bits - 1)), (1 << (bits - 1)) - 1
    v = np.sin(xx / 15.0) * hi * 0.4 + (yy / h - 0.5) * hi * 0.5 + rng.normal(0, hi / 60, (h, w))
    return np.clip(np.rint(v), lo, hi).astype(np.int8 if bits <= 8 else np.int16)[None]


SIGNED = [  # (bits, components, harness-encoder options)
    (12, 1, dict(reversible=True, mct=False)),
    (16, 1, dict(reversible=True, mct=False)),
    (8, 3, dict(reversible=True, mct=True)),
    (12, 1, dict(reversible=False, mct=False, base_step=1 / 256)),
]


@pytest.mark.parametrize("bits,comps,kw", SIGNED, ids=["s12-53", "s16-53", "s8-rct", "s12-97"])
def test_signed_samples_through_oracle(bits, comps, kw):
    """Signed components (Ssiz bit 7): no DC level shift (ISO G.1.2 shifts
    unsigned ones only), two's complement samples clamped to the signed
    range.  Lossless streams give back the original; OpenJPEG decodes the
    8- and 16-bit ones to the same values (Pillow presents them offset by
    2^(bits-1))."""
    img = _ct_like(120, 150, bits, seed=bits) if comps == 1 else \
        np.random.default_rng(5).integers(-128, 128, (3, 40, 50)).astype(np.int8)
    cs = codec.encode(img, bits, levels=4, **kw)
    from gpu_helpers import oracle_decode_tiled, openjpeg_decode
    info, out = oracle_decode_tiled(cs)
    assert info["is_signed"] == 1 and out.dtype == np.int16
    if kw["reversible"]:
        np.testing.assert_array_equal(out, img.astype(np.int16))
        if bits in (8, 16):
            opj = openjpeg_decode(cs).astype(np.int64) - (1 << (bits - 1))
            np.testing.assert_array_equal(opj, img.astype(np.int64))
    else:
        assert np.abs(out.astype(np.int64) - img).max() <= 64


def _subsampled(w, h, bits, dxy, seed):
    """Components of a w x h image subsampled by dxy[c] = (dx, dy)."""
    full = synth_image(w, h, len(dxy), bits, seed=seed)
    return [full[c, ::dy, ::dx] for c, (dx, dy) in enumerate(dxy)]


SUBSAMPLED = [  # (w, h, bits, per-component (dx, dy), harness options)
    (200, 120, 8, [(1, 1), (2, 2), (2, 2)], dict(reversible=True)),                  # 4:2:0
    (201, 121, 8, [(1, 1), (2, 1), (2, 1)], dict(reversible=False, base_step=1 / 256)),  # 4:2:2, odd sizes
    (150, 98, 12, [(1, 1), (2, 2)], dict(reversible=True, progression=3)),          # PCRL
    (97, 63, 8, [(1, 1), (4, 2), (3, 3)], dict(reversible=True, progression=4)),    # CPRL, odd factors
]


@pytest.mark.parametrize("w,h,bits,dxy,kw", SUBSAMPLED, ids=["420", "422-97-odd", "g12-pcrl", "cprl-odd-factors"])
def test_subsampled_components_through_oracle(w, h, bits, dxy, kw):
    """Subsampled components (SIZ XRsiz / YRsiz, ISO B.2): each component
    on its own ceil(w/dx) x ceil(h/dy) grid, with its own subband geometry
    and its precincts visited at reference-grid positions scaled by its
    subsampling (ISO B.12.1.3).  Lossless streams give back every
    component; OpenJPEG reads the 4:2:0 one as YCbCr, within 1 of the same
    conversion of the original components."""
    comps = _subsampled(w, h, bits, dxy, seed=w)
    cs = codec.encode(comps, bits, levels=3, mct=False, comp_subsampling=dxy, **kw)
    from gpu_helpers import oracle_decode_components
    info, planes = oracle_decode_components(cs)
    assert info["subsampling"] == dxy
    assert [p.shape for p in planes] == [c.shape for c in comps]
    for p_, c_ in zip(planes, comps):
        if kw["reversible"]:
            np.testing.assert_array_equal(p_, c_)
        else:
            assert np.abs(p_.astype(np.int64) - c_).max() <= 8
    if dxy == [(1, 1), (2, 2), (2, 2)]:
        import io
        from PIL import Image
        rgb = np.asarray(Image.open(io.BytesIO(cs))).astype(np.float64)
        up = [np.repeat(np.repeat(c_.astype(np.float64), 2, 0), 2, 1)[:h, :w] - 128 for c_ in comps[1:]]
        y = comps[0].astype(np.float64)
        want = np.stack([y + 1.402 * up[1], y - 0.344136 * up[0] - 0.714136 * up[1], y + 1.772 * up[0]], -1)
        assert np.abs(rgb - np.clip(np.rint(want), 0, 255)).max() <= 1


def test_subsampled_tiles_are_unsupported():
    comps = _subsampled(128, 128, 8, [(1, 1), (2, 2)], seed=2)
    cs = codec.encode(comps, 8, levels=2, mct=False, comp_subsampling=[(1, 1), (2, 2)])
    # rewrite SIZ for 64x64 tiles: XTsiz / YTsiz at bytes 22-29 from the marker
    b = bytearray(cs)
    i = bytes(b).index(b"\xff\x51")
    b[i + 22:i + 26] = (64).to_bytes(4, "big")
    b[i + 26:i + 30] = (64).to_bytes(4, "big")
    with pytest.raises(TCError) as ei:
        codec.read_header(bytes(b))
    assert ei.value.status == TC_E_UNSUPPORTED


STYLES = [  # (code-block style bits, bits, harness options)
    (codec.CBLK_STYLE_BYPASS, 8, dict(reversible=True)),
    (codec.CBLK_STYLE_RESET, 8, dict(reversible=True)),
    (codec.CBLK_STYLE_TERMALL, 8, dict(reversible=True)),
    (codec.CBLK_STYLE_VSC, 8, dict(reversible=True)),
    (codec.CBLK_STYLE_PTERM, 8, dict(reversible=True)),
    (codec.CBLK_STYLE_SEGSYM, 8, dict(reversible=True)),
    (0x3F, 8, dict(reversible=True)),
    (codec.CBLK_STYLE_BYPASS | codec.CBLK_STYLE_TERMALL, 12, dict(reversible=True, cblk_log2=4)),
    (codec.CBLK_STYLE_BYPASS | codec.CBLK_STYLE_VSC, 16, dict(reversible=True)),
    (codec.CBLK_STYLE_RESET | codec.CBLK_STYLE_SEGSYM, 8, dict(reversible=False, base_step=1 / 512)),
    (0x3F, 12, dict(reversible=False, base_step=1 / 1024)),
]
STYLE_IDS = ["bypass", "reset", "termall", "vsc", "pterm", "segsym", "all", "bypass-termall-12",
             "bypass-vsc-16", "reset-segsym-97", "all-97-12"]


def styled_stream(style, bits, kw, w=133, h=91):
    c = 3 if bits == 8 else 1  # OpenJPEG through Pillow: 16-bit samples as one component
    img = synth_image(w, h, c, bits, seed=style + bits)
    opts = dict(levels=3, cblk_log2=5, mct=c >= 3)
    opts.update(kw)
    return img, codec.encode(img, bits, cblk_style=style, **opts)


@pytest.mark.parametrize("style,bits,kw", STYLES, ids=STYLE_IDS)
def test_code_block_styles_through_oracle(style, bits, kw):
    """Code-block styles (SPcod, ISO Table A.19; D.4-D.7): bypass (raw
    significance and refinement passes from the 11th pass on), context
    reset, termination on every pass, vertically causal contexts,
    predictable termination and segmentation symbols, alone and combined.
    OpenJPEG decodes the harness encoder's streams to the original
    (lossless); the parser's terminated segments and the oracle's modes give
    the original too, and within 1 of OpenJPEG for 9/7."""
    from gpu_helpers import oracle_decode_tiled, openjpeg_decode
    img, cs = styled_stream(style, bits, kw)
    info, desc, pool = codec.parse(cs)
    assert (desc["style"] == style).all()
    _, out = oracle_decode_tiled(cs)
    if kw["reversible"]:
        np.testing.assert_array_equal(out, img)
        if bits in (8, 16):
            np.testing.assert_array_equal(openjpeg_decode(cs), img)
    elif bits == 8:
        assert np.abs(out.astype(np.int64) - openjpeg_decode(cs)).max() <= 1


def test_terminated_segments_have_a_length_table():
    """With TERMALL every pass is a codeword segment of its own: the block's
    pool entry starts (4-byte aligned) with one uint32 length per pass, the
    codeword after it, and the lengths add up to seg_len."""
    img, cs = styled_stream(codec.CBLK_STYLE_TERMALL, 8, dict(reversible=True))
    info, desc, pool = codec.parse(cs)
    assert info["pool_is_cs"] == 0
    coded = desc[desc["passes"] > 0]
    assert len(coded) > 10
    for d in coded:
        off, n = int(d["seg_off"]), int(d["passes"])
        assert off % 4 == 0
        lens = np.frombuffer(pool[off: off + 4 * n].tobytes(), "<u4")
        assert lens.sum() == d["seg_len"]
    # bypass alone: segments of 10, then 2 and 1 passes
    img, cs = styled_stream(codec.CBLK_STYLE_BYPASS, 16, dict(reversible=True))
    _, desc, pool = codec.parse(cs)
    deep = desc[desc["passes"] >= 14][0]
    p = int(deep["passes"])
    # passes 0-9 form one segment; from pass 10 on, {SPP, MRP} and {CUP}
    n = 1 + len({(t - 10) // 3 * 2 + ((t - 10) % 3 == 2) for t in range(10, p)})
    assert O.lib().or_pass_segments(int(deep["style"]), p) == n
    off = int(deep["seg_off"])
    assert np.frombuffer(pool[off: off + 4 * n].tobytes(), "<u4").sum() == deep["seg_len"]


def test_unknown_style_bits_are_rejected():
    img, cs = styled_stream(0, 8, dict(reversible=True))
    i = cs.find(b"\xff\x52")
    bad = bytearray(cs)
    bad[i + 2 + 2 + 1 + 1 + 2 + 1 + 1 + 2] = 0x40  # SPcod code-block style
    with pytest.raises(TCError) as e:
        codec.parse(bytes(bad))
    assert e.value.status == TC_E_UNSUPPORTED
    with pytest.raises(TCError):
        codec.encode(img, 8, cblk_style=0x40)


LAYERED = [  # (code-block style, progression, layers)
    (0, 0, 3), (0, 2, 5), (codec.CBLK_STYLE_BYPASS, 0, 7), (codec.CBLK_STYLE_BYPASS, 1, 3),
    (codec.CBLK_STYLE_BYPASS, 3, 4), (codec.CBLK_STYLE_BYPASS | codec.CBLK_STYLE_TERMALL, 2, 3),
    (codec.CBLK_STYLE_TERMALL, 4, 6), (0x3F, 1, 5), (codec.CBLK_STYLE_RESET, 3, 2),
]
LAYERED_IDS = [f"style{s:#x}-prog{p}-{n}layers" for s, p, n in LAYERED]


@pytest.mark.parametrize("style,prog,layers", LAYERED, ids=LAYERED_IDS)
def test_layered_streams_through_oracle(style, prog, layers):
    """Quality layers from the harness encoder, every progression order:
    each block's passes are spread over the layers, so blocks join in later
    layers (inclusion tag trees across layers), Lblock grows across
    contributions, and a bypass block's first ten-pass segment, cut by layer
    boundaries, continues in the next layer's packet. OpenJPEG and the
    parser + oracle both give back the original."""
    from gpu_helpers import oracle_decode_tiled, openjpeg_decode
    img = synth_image(133, 91, 3, 8, seed=style + prog + layers)
    cs = codec.encode(img, 8, levels=3, cblk_log2=5, reversible=True, cblk_style=style, progression=prog,
                      layers=layers)
    info, _, _ = codec.parse(cs)
    assert info["layers"] == layers
    np.testing.assert_array_equal(openjpeg_decode(cs), img)
    _, out = oracle_decode_tiled(cs)
    np.testing.assert_array_equal(out, img)


def _header_markers(cs):
    """Marker codes of the main header and of the first tile-part header."""
    main, tile, i = [], [], 2
    while i + 4 <= len(cs):
        m = int.from_bytes(cs[i:i + 2], "big")
        if m == 0xFF90:  # SOT: the tile-part header follows its 10-byte segment
            i += 12
            while i + 2 <= len(cs):
                m = int.from_bytes(cs[i:i + 2], "big")
                if m == 0xFF93:
                    return main, tile
                tile.append(m)
                i += 2 + int.from_bytes(cs[i + 2:i + 4], "big")
            break
        main.append(m)
        i += 2 + int.from_bytes(cs[i + 2:i + 4], "big")
    return main, tile


PACKED = [  # (PPT 1 / PPM 2, code-block style, progression, layers)
    (1, 0, 0, 1), (1, codec.CBLK_STYLE_BYPASS, 1, 4), (1, 0x3F, 4, 2),
    (2, 0, 2, 3), (2, codec.CBLK_STYLE_BYPASS | codec.CBLK_STYLE_TERMALL, 3, 5),
]


@pytest.mark.parametrize("where,style,prog,layers", PACKED,
                         ids=[f"{'ppt' if w == 1 else 'ppm'}-style{s:#x}-prog{p}-{n}layers" for w, s, p, n in PACKED])
def test_packed_packet_headers_through_oracle(where, style, prog, layers):
    """Packet headers packed into PPT (tile-part header) or PPM (main
    header, with each tile-part's Nppm) marker segments, ISO A.7.4-A.7.5:
    the parser reads the headers from the packed stream and the bodies from
    the tile-part; OpenJPEG and the oracle give back the original."""
    from gpu_helpers import oracle_decode_tiled, openjpeg_decode
    img = synth_image(133, 91, 3, 8, seed=where + prog)
    cs = codec.encode(img, 8, levels=3, cblk_log2=5, reversible=True, cblk_style=style, progression=prog,
                      layers=layers, packed_headers=where)
    main, tile = _header_markers(cs)
    assert (0xFF61 in tile) == (where == 1) and (0xFF60 in main) == (where == 2)
    np.testing.assert_array_equal(openjpeg_decode(cs), img)
    _, out = oracle_decode_tiled(cs)
    np.testing.assert_array_equal(out, img)


@pytest.mark.parametrize("where", [1, 2], ids=["ppt", "ppm"])
def test_packed_headers_over_several_marker_segments(where):
    """Headers longer than one marker segment (65532 bytes) continue in the
    next PPT / PPM segment (Zppt / Zppm incrementing)."""
    from gpu_helpers import oracle_decode_tiled
    img = synth_image(700, 500, 3, 8, seed=9)
    cs = codec.encode(img, 8, levels=5, cblk_log2=2, reversible=True, layers=12, packed_headers=where)
    main, tile = _header_markers(cs)
    assert (tile if where == 1 else main).count(0xFF61 if where == 1 else 0xFF60) >= 2
    _, out = oracle_decode_tiled(cs)
    np.testing.assert_array_equal(out, img)


ROI = [  # (bits, components, region, harness options)
    (8, 3, (30, 20, 90, 60), dict(reversible=True)),
    (8, 3, (0, 0, 40, 91), dict(reversible=True, layers=3, progression=2)),
    (12, 1, (10, 10, 70, 70), dict(reversible=True, cblk_style=0x01)),
    (8, 3, (50, 10, 133, 50), dict(reversible=False, base_step=1 / 256)),
]
ROI_IDS = ["rgb-53", "rgb-53-layers-rpcl", "g12-bypass", "rgb-97"]


@pytest.mark.parametrize("bits,comps,roi,kw", ROI, ids=ROI_IDS)
def test_roi_maxshift_through_oracle(bits, comps, roi, kw):
    """Region of interest with the maxshift method (RGN, ISO Annex H): the
    region's coefficients are shifted above every background bit-plane, the
    bands code s more bit-planes, and a decoded magnitude >= 2^s is shifted
    back down.  Lossless streams give back the original through the parser +
    oracle and (8-bit) through OpenJPEG; the 9/7 stream stays within the
    quantiser's error."""
    from gpu_helpers import oracle_decode_tiled, openjpeg_decode
    img = synth_image(133, 91, comps, bits, seed=bits + comps)
    cs = codec.encode(img, bits, levels=3, cblk_log2=5, mct=comps == 3, roi=roi, **kw)
    main, _ = _header_markers(cs)
    assert 0xFF5E in main
    info, desc, pool = codec.parse(cs)
    assert (desc["roi_shift"] > 0).all()
    _, out = oracle_decode_tiled(cs)
    if kw["reversible"]:
        np.testing.assert_array_equal(out, img)
        if bits == 8:
            np.testing.assert_array_equal(openjpeg_decode(cs), img)
    else:
        err = out.astype(np.int64) - img
        assert np.abs(err).max() <= 4 and 10 * np.log10(255 ** 2 / np.mean(err ** 2)) > 45


def test_crg_marker_is_read_past():
    """A CRG marker segment (component registration, ISO A.9.1: a display
    offset per component) changes no decoded sample."""
    from gpu_helpers import oracle_decode_tiled
    img = synth_image(64, 48, 3, 8, seed=2)
    cs = codec.encode(img, 8, levels=2, reversible=True)
    i = cs.find(b"\xff\x90")  # before SOT
    crg = b"\xff\x63" + (2 + 4 * 3).to_bytes(2, "big") + b"".join(
        (0).to_bytes(2, "big") + (32768).to_bytes(2, "big") for _ in range(3))
    _, out = oracle_decode_tiled(cs[:i] + crg + cs[i:])
    np.testing.assert_array_equal(out, img)
