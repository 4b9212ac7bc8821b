"""Malformed input (no GPU): seeded mutations of valid codestreams (styled,
layered, subsampled, OpenJPEG-written, tiled JP2) must parse or be rejected
with an error, never crash; and the same mutations through a sanitizer build
of the host parser must raise no AddressSanitizer / UBSan report."""
import io
import shutil
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN, ROOT, synth_image
from thousandthchicken_b200 import codec
from thousandthchicken_b200._lib import TCError


def _bases():
    img = synth_image(67, 45, 3, 8, seed=1)
    bases = [
        codec.encode(img, 8, levels=3, cblk_log2=4, reversible=True),
        codec.encode(img, 8, levels=3, cblk_log2=4, reversible=True, cblk_style=0x3F, layers=3, progression=2),
        codec.encode(img, 8, levels=2, cblk_log2=3, reversible=False, cblk_style=0x05, layers=4, progression=4),
        codec.encode(img, 8, levels=2, cblk_log2=4, reversible=True, cblk_style=0x01, layers=5, progression=1),
        codec.encode([img[0], img[1][::2, ::2]], 8, levels=2, mct=False, comp_subsampling=[(1, 1), (2, 2)]),
        codec.encode(img, 8, levels=2, cblk_log2=4, reversible=True, layers=3, packed_headers=1),
        codec.encode(img, 8, levels=2, cblk_log2=4, reversible=True, cblk_style=0x01, layers=2, packed_headers=2),
        codec.encode(img, 8, levels=2, cblk_log2=4, reversible=True, roi=(10, 5, 40, 30)),
    ]
    bases += [p.read_bytes() for p in sorted(GOLDEN.glob("*.j2k"))[:4]]
    from PIL import Image
    buf = io.BytesIO()
    Image.fromarray(np.moveaxis(img, 0, -1)).save(buf, "JPEG2000", quality_layers=[40, 10], irreversible=True,
                                                  tile_size=(32, 32))
    bases.append(buf.getvalue())
    return bases


def _mutations(seed, n):
    """n mutated streams: random bytes, truncation, header bit flips, and
    inserted or deleted byte runs."""
    rng = np.random.default_rng(seed)
    bases = _bases()
    for i in range(n):
        b = bytearray(bases[i % len(bases)])
        kind = rng.integers(0, 4)
        if kind == 0:
            for _ in range(rng.integers(1, 6)):
                b[rng.integers(0, len(b))] = rng.integers(0, 256)
        elif kind == 1:
            b = b[: rng.integers(2, len(b))]
        elif kind == 2:
            for _ in range(rng.integers(1, 4)):
                p = rng.integers(0, min(200, len(b)))
                b[p] ^= 1 << rng.integers(0, 8)
        else:
            p = rng.integers(0, len(b))
            if rng.integers(0, 2):
                b[p:p] = bytes(rng.integers(0, 256, rng.integers(1, 9)).astype(np.uint8))
            else:
                del b[p: p + rng.integers(1, 9)]
        yield bytes(b)


def _check_descriptors(info, desc, pool):
    """What the Tier-1 kernels are handed stays inside its buffers: block
    geometry and pass counts in range, every codeword (and segment table)
    inside the pool, every block inside the coefficient arena."""
    arena = sum(h * w for h, w in info["comp_sizes"])
    for d in desc:
        w, h, mb, zb, passes = int(d["w"]), int(d["h"]), int(d["mb"]), int(d["zero_bitplanes"]), int(d["passes"])
        assert 1 <= w <= 64 and 1 <= h <= 64 and 1 <= mb <= 31 and zb <= mb
        assert int(d["out_off"]) + (h - 1) * int(d["out_pitch"]) + w <= arena
        if passes == 0:
            continue
        assert passes <= 3 * (mb - zb) - 2
        off, n = int(d["seg_off"]), int(d["seg_len"])
        if int(d["style"]) & (codec.CBLK_STYLE_BYPASS | codec.CBLK_STYLE_TERMALL):
            nseg = O.lib().or_pass_segments(int(d["style"]), passes)
            assert off % 4 == 0 and off + 4 * nseg + n <= len(pool)
            assert np.frombuffer(pool[off: off + 4 * nseg].tobytes(), "<u4").sum() == n
        else:
            assert off + n <= len(pool)


def test_mutated_streams_parse_or_fail_cleanly():
    parsed = rejected = 0
    for b in _mutations(7, 1500):
        try:
            info, desc, pool = codec.parse(b)
        except TCError:
            rejected += 1
            continue
        parsed += 1
        _check_descriptors(info, desc, pool)
    assert parsed > 100 and rejected > 100


def test_parser_under_sanitizers(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    exe = tmp_path / "parse_fuzz"
    csrc = ROOT / "thousandthchicken_b200" / "csrc"
    build = subprocess.run([gxx, "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined",
                            "-fno-sanitize-recover=undefined", f"-I{ROOT / 'include'}", f"-I{csrc}",
                            str(csrc / "j2k_host.cpp"), str(Path(__file__).parent / "parse_fuzz_harness.cpp"),
                            "-o", str(exe), "-lpthread"], capture_output=True, text=True)
    if build.returncode != 0:
        pytest.skip("sanitizer runtime unavailable: " + build.stderr[-200:])
    data = b"".join(struct.pack("<I", len(b)) + b for b in _mutations(11, 3000))
    run = subprocess.run([str(exe)], input=data, capture_output=True, timeout=600)
    report = run.stderr.decode(errors="replace")
    assert run.returncode == 0, report[-2000:]
    assert "AddressSanitizer" not in report and "runtime error" not in report, report[-2000:]
    assert b"of 3000" in run.stdout
