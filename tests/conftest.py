import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def built():
    """Make sure the product library and the oracle are built (CPU-only
    compilation; nvcc cross-compiles sm_100a without a GPU)."""
    from thousandthchicken_b200 import build as B
    import oracle as O
    B.build()
    O.build()
    return True


def golden_cases():
    meta = json.loads((GOLDEN / "golden.json").read_text())
    return sorted(meta["cases"].items())


def load_golden(name):
    cs = (GOLDEN / f"{name}.j2k").read_bytes()
    z = np.load(GOLDEN / f"{name}.npz")
    return cs, z["original"], z["openjpeg"]


def synth_image(w, h, c, bits, seed, sigma=8.0):
    """Per-channel bilinear gradients plus Gaussian noise, clipped (the
    synthetic image family of the benchmark workloads)."""
    from thousandthchicken_b200.synth import gradient_noise_image
    return gradient_noise_image(w, h, c, bits, seed, sigma)


@pytest.fixture(scope="session")
def gpu_ctx():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from thousandthchicken_b200.stages import Context
    ctx = Context(0)
    yield ctx
    ctx.close()
