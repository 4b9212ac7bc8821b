"""CPU checks of the Tier-1 decoder's table and bit tricks against plain
restatements of the rules they encode (no GPU needed):

* the MQ probability tables in t1_common.cuh equal the oracle's ISO Table
  C.2, and the decoder's whole-word context entries (Tables::mqd: Qe, the
  entries after an MPS and after an LPS, the MPS) walk the same state
  machine as ISO C.3.2 (NMPS keeps the MPS; NLPS switches it where SWITCH
  is set);
* the significance-propagation candidate test of a stripe column, written
  bit-parallel in t1_decode.cu, equals the row-by-row rule (a row not yet
  significant with a significant neighbour) for every significance pattern
  of the 3x6 neighbourhood and every stripe height.
"""
import re
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
T1_COMMON = ROOT / "thousandthchicken_b200" / "csrc" / "t1_common.cuh"
T1_DECODE = ROOT / "thousandthchicken_b200" / "csrc" / "t1_decode.cu"
ORACLE_C = ROOT / "oracle" / "j2k_oracle.c"


def _c_array(text, name):
    m = re.search(name + r"\[\d*\]\s*=\s*\{([^}]*)\}", text)
    assert m, name
    return [int(v, 0) for v in m.group(1).replace("\n", " ").split(",") if v.strip()]


def _tables():
    k = T1_COMMON.read_text()
    o = ORACLE_C.read_text()
    return (_c_array(k, "c_qe"), _c_array(k, "c_nmps"), _c_array(k, "c_nlps"),
            _c_array(o, "kQe"), _c_array(o, "kNMPS"), _c_array(o, "kNLPS"), _c_array(o, "kSWITCH"))


def test_kernel_mq_tables_equal_iso_table_c2():
    qe, nmps, nlps, oqe, onmps, onlps, osw = _tables()
    assert len(qe) == len(oqe) == 47
    assert qe == oqe and nmps == onmps and nlps == onlps
    # the kernel marks the switch states by index (build_tables)
    assert [i for i, s in enumerate(osw) if s] == [0, 6, 14]


def _mqd(qe, nmps, nlps):
    """Tables::mqd as build_tables fills it."""
    out = [0] * 96
    for i in range(94):
        st, mps = i >> 1, i & 1
        sw = 1 if st in (0, 6, 14) else 0
        out[i] = (qe[st] << 16) | ((2 * nlps[st] + (mps ^ sw)) << 7) | (2 * nmps[st] + mps)
    return out


def test_whole_word_successors_walk_iso_state_machine():
    qe, nmps, nlps, _, _, _, osw = _tables()
    mqd = _mqd(qe, nmps, nlps)
    src = T1_DECODE.read_text()
    # the decoder picks the successor entry exactly this way
    assert "tbl[d != mps ? (w >> 7) & 127u : w & 127u]" in src
    for st in range(47):
        for mps in (0, 1):
            w = mqd[2 * st + mps]
            assert w >> 16 == qe[st] and (w & 1) == mps
            after_mps = mqd[w & 127]
            assert after_mps >> 16 == qe[nmps[st]] and (after_mps & 1) == mps
            assert after_mps == mqd[2 * nmps[st] + mps]
            after_lps = mqd[(w >> 7) & 127]
            assert after_lps == mqd[2 * nlps[st] + (mps ^ osw[st])]
            assert (after_lps & 1) == mps ^ osw[st]
    # the initial states (ISO Table D.7) with MPS 0
    assert mqd[2 * 4] >> 16 == qe[4] and mqd[2 * 46] >> 16 == qe[46] and mqd[2 * 3] >> 16 == qe[3]


def test_bit_parallel_spp_candidate_test_equals_row_rule():
    assert "(f | (f >> 1) | (f >> 2)) & 0x9249u" in T1_DECODE.read_text()
    f = np.arange(1 << 18, dtype=np.uint32)
    # pi / sigma' / sign bits above bit 17 must not matter
    f = f | (np.random.default_rng(5).integers(0, 1 << 14, f.size, dtype=np.uint32) << np.uint32(18))
    g = (f | (f >> 1) | (f >> 2)) & np.uint32(0x9249)
    for rows in range(1, 5):
        fast = ((g | (g >> 3) | (g >> 6)) & ~(f >> 4) & np.uint32(0x249 >> (3 * (4 - rows)))) != 0
        slow = np.zeros(f.size, bool)
        for k in range(rows):
            self_sig = (f >> np.uint32(3 * k + 4)) & 1
            nbr = (f >> np.uint32(3 * k)) & np.uint32(0x1EF)
            slow |= (self_sig == 0) & (nbr != 0)
        np.testing.assert_array_equal(fast, slow, err_msg=f"rows={rows}")
