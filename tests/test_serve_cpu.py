"""The serving loop's admission, failure isolation and latency accounting
against a CPU fake of its GPU executor (no device): a malformed codestream
or a batch the device flags fails only its own request, the budget is never
exceeded and is released by finished and failed requests alike, latency is
measured from arrival, and an overloaded run can stop admitting."""
import time

import numpy as np
import pytest

from conftest import synth_image
from thousandthchicken_b200 import codec
from thousandthchicken_b200.serve import Request, Server, latency_stats, poisson_arrivals, request_device_bytes


class FakeSlot:
    """Executes a batch by waiting `latency_s` per request; a batch holding
    a request of `flagged` fails as a device error would."""

    def __init__(self, latency_s=0.002, flagged=(), launch_fails=(), watch=None):
        self.latency_s = latency_s
        self.flagged = set(flagged)
        self.launch_fails = set(launch_fails)
        self.batch = []
        self.t_end = 0.0
        self.watch = watch if watch is not None else {}
        self.watch.setdefault("batches", [])
        self.plan = None        # a plan's buffers: grow-only, by at least half again
        self.held = 0

    def launch(self, batch, keep_outputs):
        for r in batch:
            r.parsed.result()            # a bad parse surfaces here, as in the GPU slot
        if any(r.rid in self.launch_fails for r in batch):
            raise RuntimeError("plan build failed")
        self.batch = list(batch)
        need = sum(r.device_bytes for r in batch)
        if self.plan is None:
            self.plan, self.held = object(), need
        elif need > self.held:
            self.held = max(need, int(1.5 * self.held))
        self.watch["batches"].append([r.rid for r in batch])
        self.t_end = time.perf_counter() + self.latency_s * len(batch)

    def busy(self):
        return bool(self.batch)

    def poll(self, now_fn):
        if not self.batch or time.perf_counter() < self.t_end:
            return []
        done, self.batch = self.batch, []
        if any(r.rid in self.flagged for r in done):
            raise RuntimeError("device error word: bad code-block data")
        t = now_fn()
        for r in done:
            r.done = t
        return done

    def device_bytes(self):
        return self.held

    def shrink(self):
        self.plan, self.held = None, 0

    def close(self):
        pass


def _streams(n=8):
    out = []
    for i in range(n):
        w, h = 64 + 16 * i, 48 + 8 * i
        out.append(codec.encode(synth_image(w, h, 3 if i % 2 else 1, 8, seed=i), 8, levels=3,
                                reversible=i % 3 != 0, mct=i % 2 == 1, base_step=1 / 64))
    return out


def _server(budget=1 << 30, max_batch=4, inflight=2, **kw):
    watch = {}
    return Server(budget_bytes=budget, max_batch=max_batch, inflight=inflight,
                  slot_factory=lambda i: FakeSlot(watch=watch, **kw)), watch


def test_malformed_codestream_fails_alone():
    streams = _streams()
    bad = streams[3][: len(streams[3]) // 2]          # header intact, packets cut
    reqs = [Request(i, s, 0.0) for i, s in enumerate(streams)] + [Request(99, bad, 0.0)]
    reqs.append(Request(98, b"\x00\x01garbage", 0.0))  # no codestream at all
    srv, _ = _server()
    done, _ = srv.run(reqs, realtime=False)
    srv.close()
    errs = {r.rid for r in done if r.error}
    assert errs == {98, 99}
    assert sorted(r.rid for r in done if not r.error) == list(range(len(streams)))
    assert srv.stats["failed"] == 2


def test_flagged_batch_is_split_and_only_the_bad_request_fails():
    streams = _streams()
    reqs = [Request(i, s, 0.0) for i, s in enumerate(streams)]
    srv, watch = _server(flagged={5}, launch_fails={2})
    done, _ = srv.run(reqs, realtime=False)
    srv.close()
    assert {r.rid for r in done if r.error} == {2, 5}
    assert sorted(r.rid for r in done) == list(range(len(streams)))
    assert [5] in watch["batches"] and [2] not in watch["batches"]   # 5 re-ran alone; 2 failed at launch alone


def test_budget_bounds_requests_in_flight_and_is_released():
    streams = _streams()
    sizes = [request_device_bytes(codec.read_header(s), len(s)) for s in streams]
    budget = max(sizes) + min(sizes)
    reqs = [Request(i, s, 0.0) for i, s in enumerate(streams)]
    reqs.append(Request(50, streams[0], 0.0))
    srv, watch = _server(budget=budget, max_batch=8)
    done, _ = srv.run(reqs, realtime=False)
    srv.close()
    assert len(done) == len(reqs) and not any(r.error for r in done)
    assert srv.stats["peak_admitted_bytes"] <= budget
    assert srv.stats["peak_device_bytes"] <= budget
    for b in watch["batches"]:
        assert sum(sizes[i % len(streams)] if i < 50 else sizes[0] for i in b) <= budget
    # a request larger than the whole budget fails without blocking the others
    srv, _ = _server(budget=min(sizes))
    small = int(np.argmin(sizes))
    done, _ = srv.run([Request(0, streams[int(np.argmax(sizes))], 0.0), Request(1, streams[small], 0.0)],
                      realtime=False)
    srv.close()
    assert [r.rid for r in done if r.error] == [0] and [r.rid for r in done if not r.error] == [1]


def test_latency_from_arrival_with_injected_latency():
    streams = _streams()
    arr = poisson_arrivals(24, rate_per_s=200.0, seed=1)
    reqs = [Request(i, streams[i % len(streams)], float(a)) for i, a in enumerate(arr)]
    srv, _ = _server(latency_s=0.004, max_batch=2, inflight=2)
    done, wall = srv.run(reqs, realtime=True)
    srv.close()
    assert len(done) == 24 and all(r.done >= r.arrival for r in done)
    st = latency_stats(done)
    assert st["p50_ms"] >= 4.0 * 0.9 and st["p99_ms"] >= st["p50_ms"]
    assert wall >= float(arr[-1])


def test_overloaded_run_stops_admitting():
    streams = _streams()
    arr = poisson_arrivals(400, rate_per_s=4000.0, seed=2)
    reqs = [Request(i, streams[i % len(streams)], float(a)) for i, a in enumerate(arr)]
    srv, _ = _server(latency_s=0.01, max_batch=1, inflight=1)
    done, wall = srv.run(reqs, realtime=True, stop_backlog_s=0.05)
    srv.close()
    assert srv.stats["unserved"] > 0 and len(done) + srv.stats["unserved"] == len(reqs)
    assert wall < 400 * 0.01


def test_batch_sample_cap():
    streams = _streams()
    sizes = {i: codec.read_header(s) for i, s in enumerate(streams)}
    cap = max(v["width"] * v["height"] * v["ncomp"] for v in sizes.values())
    watch = {}
    srv = Server(budget_bytes=1 << 30, max_batch=8, inflight=1, max_batch_samples=cap,
                 slot_factory=lambda i: FakeSlot(watch=watch))
    done, _ = srv.run([Request(i, s, 0.0) for i, s in enumerate(streams)], realtime=False)
    srv.close()
    assert len(done) == len(streams)
    for b in watch["batches"]:
        assert len(b) == 1 or sum(sizes[i]["width"] * sizes[i]["height"] * sizes[i]["ncomp"] for i in b) <= cap
    assert any(len(b) > 1 for b in watch["batches"])
