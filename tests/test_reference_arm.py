"""The benchmark's reference arm and the oracle encoder it codes its input
with.  The arm must decode the workload image itself without loading the
product library, so the oracle carries its own encoder (ISO C.2 MQ coder,
ISO D.3 passes, FP64 forward DWT); these tests pin that encoder to the
harness encoder byte for byte, and run the arm on a small image."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O
from conftest import ROOT
from thousandthchicken_b200 import codec
from thousandthchicken_b200.synth import gradient_noise_image, laplacian_block


def test_oracle_block_encoder_matches_harness_encoder():
    """Random Laplacian blocks of every size, all passes and truncated:
    the oracle's codewords equal the harness encoder's."""
    rng = np.random.default_rng(7)
    for _ in range(200):
        w, h, nb = int(rng.integers(1, 65)), int(rng.integers(1, 65)), int(rng.integers(1, 15))
        blk = laplacian_block(rng, w, h, nb)
        orient = int(rng.integers(0, 4))
        for passes in (0, int(rng.integers(1, 3 * nb))):
            a = O.t1_encode(blk, orient, passes)
            b = codec.t1_encode_block(blk, orient, 31, passes)
            assert a[0] == b[0] and a[1] == b[1]


@pytest.mark.parametrize("reversible", [True, False])
@pytest.mark.parametrize("w,h,levels", [(300, 200, 5), (257, 131, 3), (64, 64, 6)])
def test_oracle_tile_encoder_matches_harness_codestream(reversible, w, h, levels):
    """The oracle's tile encode gives the same code-blocks (codeword, passes,
    bit-planes, step) as the harness codestream parsed back."""
    img = gradient_noise_image(w, h, 3, 8, seed=w + h)
    et = O.encode_tile(img, 8, levels, reversible, True, 1 / 128)
    info, desc, pool = codec.parse(codec.encode(img, 8, levels=levels, reversible=reversible, mct=True,
                                                base_step=1 / 128))
    mine = et.blocks()
    assert et.n == len(desc)
    for d in desc:
        comp, rem = divmod(int(d["out_off"]), w * h)
        y, x = divmod(rem, w)
        seg, bw, bh, passes, numbps, orient, step = mine[(comp, x, y)]
        assert seg == pool[int(d["seg_off"]):int(d["seg_off"]) + int(d["seg_len"])].tobytes()
        assert (bw, bh, passes, orient) == (d["w"], d["h"], d["passes"], d["orient"])
        if passes:
            assert numbps == int(d["mb"]) - int(d["zero_bitplanes"])
        if not reversible:
            assert step == pytest.approx(float(d["step"]), rel=0, abs=0)
    out, f64 = et.decode(f64=not reversible)
    if reversible:
        np.testing.assert_array_equal(out, img)
    else:
        assert np.abs(out.astype(int) - img).max() <= 16
        assert np.abs(np.clip(f64, 0, 255) - out).max() <= 0.5 + 1e-9


def test_reference_arm_runs_without_the_product_library():
    """bench.py --impl reference on a small image: one JSON line, the oracle
    port timed, and no library of the package mapped in the process."""
    env = dict(os.environ, PYTHONPATH=str(ROOT))
    res = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--size", "256",
                          "--steps", "1", "--warmup", "1"], capture_output=True, text=True, env=env, timeout=600)
    assert res.returncode == 0, res.stderr
    line = json.loads(res.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["config"]["width"] == 256 and line["config"]["code_blocks"] > 0
    assert line["cpu_baseline"]["kind"] == "port"
    assert not any("libtc_j2k" in m for m in line["repo_libraries_mapped"])
    assert line["psnr_db"] > 38
