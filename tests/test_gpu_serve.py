"""The continuous-batching server: every request's result is identical
whether it is decoded alone or in a mix, batches respect the memory budget,
and plans reuse their buffers across batches (tc_plan_rebuild)."""
import numpy as np
import pytest

from conftest import synth_image
from thousandthchicken_b200 import codec

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _streams():
    out = []
    specs = [(300, 200, 3, 8, True), (128, 256, 1, 12, True), (400, 120, 3, 8, False), (64, 64, 1, 8, False),
             (513, 97, 3, 12, False), (250, 250, 1, 16, True)]
    for i, (w, h, c, bits, rev) in enumerate(specs):
        img = synth_image(w, h, c, bits, seed=40 + i)
        out.append(codec.encode(img, bits, levels=4, reversible=rev, mct=c == 3, base_step=1 / 64))
    return out


def test_results_identical_alone_and_in_the_mix(gpu_ctx):
    from thousandthchicken_b200.serve import Request, Server
    from thousandthchicken_b200.stages import Decoder
    streams = _streams()
    alone = [Decoder(gpu_ctx).decode(s) for s in streams]
    server = Server(0, budget_bytes=1 << 30, max_batch=4, inflight=2)
    reqs = [Request(i, s, arrival=0.0) for i, s in enumerate(streams * 3)]
    done, wall = server.run(reqs, realtime=False, keep_outputs=True)
    server.close()
    assert len(done) == len(reqs)
    for r in done:
        np.testing.assert_array_equal(r.output, alone[r.rid % len(streams)])
        assert r.done >= r.arrival


def test_budget_limits_batches(gpu_ctx):
    from thousandthchicken_b200.serve import Request, Server, request_device_bytes
    streams = _streams()
    reqs = [Request(i, s, arrival=0.0) for i, s in enumerate(streams)]
    biggest = max(request_device_bytes(codec.read_header(s), len(s)) for s in streams)
    server = Server(0, budget_bytes=biggest, max_batch=8, inflight=2)
    done, _ = server.run(reqs, realtime=False)
    server.close()
    assert len(done) == len(reqs) and not any(r.error for r in done)
    assert server.stats["peak_admitted_bytes"] <= biggest
    # a request above the whole budget fails alone, with an error
    big = int(np.argmax([request_device_bytes(codec.read_header(s), len(s)) for s in streams]))
    server = Server(0, budget_bytes=biggest - 1)
    done, _ = server.run([Request(0, streams[big], 0.0)], realtime=False)
    server.close()
    assert done[0].error and "budget" in done[0].error


def test_corrupt_request_fails_alone_on_the_gpu(gpu_ctx):
    """One truncated codestream among good ones: one error, the others
    decode to the same samples as alone."""
    from thousandthchicken_b200.serve import Request, Server
    from thousandthchicken_b200.stages import Decoder
    streams = _streams()
    alone = [Decoder(gpu_ctx).decode(s) for s in streams]
    bad = streams[2][: len(streams[2]) // 2]
    reqs = [Request(i, s, 0.0) for i, s in enumerate(streams)] + [Request(77, bad, 0.0)]
    server = Server(0, budget_bytes=1 << 30, max_batch=4, inflight=2)
    done, _ = server.run(reqs, realtime=False, keep_outputs=True)
    server.close()
    assert [r.rid for r in done if r.error] == [77]
    for r in done:
        if r.rid != 77:
            np.testing.assert_array_equal(r.output, alone[r.rid])


def test_poisson_arrivals_report_latency(gpu_ctx):
    from thousandthchicken_b200.serve import Request, Server, latency_stats, poisson_arrivals
    streams = _streams()
    arr = poisson_arrivals(24, rate_per_s=400.0, seed=3)
    reqs = [Request(i, streams[i % len(streams)], float(a)) for i, a in enumerate(arr)]
    server = Server(0, budget_bytes=1 << 30, max_batch=8)
    done, wall = server.run(reqs, realtime=True)
    server.close()
    st = latency_stats(done)
    assert st["p50_ms"] > 0 and st["p99_ms"] >= st["p50_ms"]
