"""The CPU oracle against the golden fixtures written by OpenJPEG (an
independent conformant codec).  These pin the oracle's Tier-1, dequantiser,
DWT and colour restatements, and the product's Tier-2 parser."""
import numpy as np
import pytest

import oracle as O
from conftest import golden_cases, load_golden
from thousandthchicken_b200 import codec


@pytest.mark.parametrize("name,meta", golden_cases(), ids=[n for n, _ in golden_cases()])
def test_oracle_decodes_openjpeg_stream(name, meta):
    cs, original, opj = load_golden(name)
    info, desc, pool = codec.parse(cs)
    assert (info["width"], info["height"], info["ncomp"], info["bits"]) == (meta["w"], meta["h"], meta["comps"],
                                                                            meta["bits"])
    assert info["levels"] == meta["levels"] and info["reversible"] == (not meta["irreversible"])
    out = O.decode_tile(desc, pool, info["width"], info["height"], info["ncomp"], info["bits"], info["levels"],
                        info["reversible"], info["mct"], r=0.5)
    if info["reversible"]:
        # lossless (or reversible truncated with mid-point reconstruction):
        # bit-exact with OpenJPEG's own decode
        np.testing.assert_array_equal(out, opj)
        if meta["openjpeg_equals_original"]:
            np.testing.assert_array_equal(out, original)
    else:
        d = np.abs(out.astype(np.int64) - opj.astype(np.int64))
        assert d.max() <= 1, f"max |oracle - openjpeg| = {d.max()}"
        assert (d > 0).mean() < 0.005


def test_golden_fixtures_present():
    assert len(golden_cases()) >= 8
