"""The allocation-free reverse 9/7 entry point, tc_dwt_reverse97_static.

Some callers cannot allocate device memory: code under stream capture that
must not allocate, hosts whose memory manager owns every device allocation,
real-time paths that cannot afford cudaMalloc and cudaFree.  This entry point
serves them: its intermediate plane lives in a fixed 16 MiB device array
inside the library.

The test calls it through the C ABI twice in a row, on different shapes; the
second call finds the first call's leftovers in the shared array.  Each
result is checked against tc_dwt_reverse97 and against the FP64 oracle,
within the 9/7 tolerance of the other DWT tests.  The file is collected last
so that a run stopping at the first failure has already run every other test;
it passes both alone in a fresh process and after the other tests."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from thousandthchicken_b200 import _lib as L

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOL97 = 0.02  # the 9/7 bound of test_gpu_dwt.py (8-bit-range samples)


def _mallat(w, h, levels, seed):
    x = np.random.default_rng(seed).integers(-128, 128, (h, w)).astype(np.float64)
    return torch.from_numpy(O.fdwt97(x, levels).astype(np.float32)).cuda(), x


def _call_static(inp, out, w, h, levels):
    stream = torch.cuda.current_stream().cuda_stream
    return L.lib().tc_dwt_reverse97_static(inp.data_ptr(), w, out.data_ptr(), w, w, h, levels, C.c_void_p(stream))


def test_static_scratch_reverse97_matches_context_entry_point():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from thousandthchicken_b200.stages import Context, DWTReverse97
    ctx = Context(0)
    reference_path = DWTReverse97(ctx)
    for w, h, levels, seed in [(1000, 700, 5, 1), (515, 333, 6, 2)]:  # two calls in a row
        inp, x = _mallat(w, h, levels, seed)
        want = torch.empty((h, w), dtype=torch.float32, device="cuda")
        reference_path.run(inp, want, w, h, levels)
        got = torch.full((h, w), float("nan"), dtype=torch.float32, device="cuda")
        assert _call_static(inp, got, w, h, levels) == L.TC_OK
        torch.cuda.synchronize()
        g, r = got.cpu().numpy().astype(np.float64), want.cpu().numpy().astype(np.float64)
        assert np.abs(g - r).max() <= TOL97
        assert np.abs(g - x).max() <= TOL97
    ctx.close()


def test_static_scratch_largest_plane_that_fits():
    """4096 x 4096: the first-level low band (2048 x 2048) is exactly the
    array's 4 Mi samples, which the size check must accept; same result as
    the context entry point (random Mallat coefficients, both on the GPU)."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from thousandthchicken_b200.stages import Context, DWTReverse97
    ctx = Context(0)
    n, levels = 4096, 3
    g = torch.Generator(device="cuda").manual_seed(4096)
    inp = torch.randn((n, n), generator=g, device="cuda") * 40
    want = torch.empty_like(inp)
    DWTReverse97(ctx).run(inp, want, n, n, levels)
    got = torch.full_like(inp, float("nan"))
    assert _call_static(inp, got, n, n, levels) == L.TC_OK
    torch.cuda.synchronize()
    assert float((got - want).abs().max()) <= TOL97
    ctx.close()


def test_static_scratch_rejects_planes_beyond_the_array():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    inp = torch.empty(1, dtype=torch.float32, device="cuda")
    out = torch.empty(1, dtype=torch.float32, device="cuda")
    # first-level low band 2049 x 2048 samples, one row over
    # TC_DWT97_STATIC_SCRATCH_ELEMS (4 Mi)
    w, h = 4098, 4096
    rc = L.lib().tc_dwt_reverse97_static(inp.data_ptr(), w, out.data_ptr(), w, w, h, 3, None)
    assert rc == L.TC_E_ARG
