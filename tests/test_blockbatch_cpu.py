"""The batched Tier-1 workload's generator and the oracle's truncation rule
(CPU): block-size shares, bit-plane and pass-count ranges, and the rule
against the oracle's own decode of truncated codewords."""
import numpy as np

import oracle as O
from thousandthchicken_b200.synth import c3_geometry, laplacian_block


def test_geometry_follows_the_workload_distribution():
    g = c3_geometry(200_000, seed=3)
    w, h = g["w"].astype(int), g["h"].astype(int)
    full = (w == 64) & (h == 64)
    half = (w == 32) & (h == 32)
    assert abs(full.mean() - 0.6) < 0.01 and abs(half.mean() - 0.3) < 0.01
    assert w.min() >= 1 and h.min() >= 1 and w.max() <= 64
    assert g["nb"].min() == 4 and g["nb"].max() == 14
    mp = g["max_passes"].astype(int)
    assert mp.min() >= 1 and (mp <= 3 * g["nb"].astype(int) - 2).all()
    assert sum(k for _, k in g["images"]) == 200_000
    assert g["elems"] == int((w * h).sum()) and g["off"][1] == w[0] * h[0]


def test_truncation_rule_equals_oracle_decode():
    rng = np.random.default_rng(9)
    n = 0
    for _ in range(600):
        w, h, nb = int(rng.integers(1, 65)), int(rng.integers(1, 65)), int(rng.integers(1, 15))
        blk = laplacian_block(rng, w, h, nb)
        orient = int(rng.integers(0, 4))
        _, total, numbps = O.t1_encode(blk, orient, 0)
        if numbps == 0:
            continue
        k = int(rng.integers(1, total + 1))
        seg, kept, _ = O.t1_encode(blk, orient, k)
        q, _ = O.t1_decode(seg, w, h, orient, numbps, kept)
        np.testing.assert_array_equal(O.t1_truncate(blk, k), q)
        n += 1
    assert n > 500
