"""Continuous-batching decode server over the C ABI.

Requests (codestreams) arrive over time.  The server admits them against a
device-memory budget and a per-batch cap, merges every admitted request into
one batch plan (one Tier-1 work-queue launch over all their code-blocks, then
their DWT levels), and keeps up to `inflight` batches on the GPU at once, each
on its own CUDA stream with its own resident plan buffers (`tc_plan_rebuild`
reuses them).  While batches run, newly arrived requests are admitted into the
next free slot, so arrivals overlap with decoding.  Each request's latency is
its completion time minus its arrival time.

Each request's codestream is parsed (Tier-2: packet headers, segment
gathering, descriptors) on a worker thread as soon as it is admitted, while
earlier batches decode; a batch is then built from the parsed requests with
`tc_plan_rebuild_parsed`, which only lays out and uploads.

Results are deterministic per code-block, so a request decoded in a mix is
bit-identical to the same request decoded alone.
"""
from __future__ import annotations

import ctypes as C
import os
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .codec import read_header

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None


@dataclass
class Request:
    rid: int
    cs: bytes
    arrival: float                      # seconds, on the server clock
    info: dict = field(default_factory=dict)
    device_bytes: int = 0
    done: float = -1.0
    output: object = None               # numpy array when keep_outputs
    parsed: object = None               # future of the tc_j2k_parse result


def _parse(cs: bytes):
    """tc_j2k_parse on a worker thread (the call runs without the GIL); the
    result points into `cs`, which the request keeps alive."""
    buf = np.frombuffer(cs, np.uint8)
    out = C.POINTER(L.Parsed)()
    L.check(L.lib().tc_j2k_parse(buf.ctypes.data, buf.size, C.byref(out)), what="tc_j2k_parse")
    return out


def _free_parsed(r):
    if r.parsed is not None:
        try:
            p = r.parsed.result()
        except Exception:  # noqa: BLE001 - a failed parse holds nothing
            p = None
        if p:
            L.lib().tc_j2k_parsed_free(p)
        r.parsed = None


def request_device_bytes(info: dict, cs_len: int) -> int:
    """Device memory a request occupies while in flight: codestream copy,
    descriptors, coefficient planes, DWT scratch and output samples."""
    w, h, c = info["width"], info["height"], info["ncomp"]
    coef = 4 * w * h * c
    scratch = 2 * 4 * ((w + 1) // 2) * ((h + 1) // 2) * c
    out = (1 if info["bits"] <= 8 else 2) * w * h * c
    ncblk = ((w + 63) // 64) * ((h + 63) // 64) * c * 2
    return cs_len + coef + scratch + out + 44 * ncblk


class _Slot:
    def __init__(self, server, device):
        self.stream = torch.cuda.Stream(device)
        from .stages import Context
        self.ctx = Context(device, self.stream)
        self.plan = None
        self.outs = None
        self.batch = []
        self.event = None
        self.keep = []

    def launch(self, batch, keep_outputs):
        lib = L.lib()
        try:
            if self.plan is None:
                bufs = [np.frombuffer(r.cs, np.uint8) for r in batch]
                ptrs = (C.c_void_p * len(bufs))(*[b.ctypes.data for b in bufs])
                lens = (C.c_size_t * len(bufs))(*[b.size for b in bufs])
                h = C.c_void_p()
                self.ctx.check(lib.tc_plan_create(self.ctx.handle, ptrs, lens, len(bufs), C.byref(h)),
                               "tc_plan_create")
                self.plan = h
            else:
                parsed = [r.parsed.result() for r in batch]
                arr = (C.POINTER(L.Parsed) * len(parsed))(*parsed)
                self.ctx.check(lib.tc_plan_rebuild_parsed(self.plan, arr, len(parsed)), "tc_plan_rebuild_parsed")
        finally:
            for r in batch:
                _free_parsed(r)
        dev = torch.device("cuda", self.ctx.device)
        self.outs = []
        for r in batch:
            i = r.info
            dt = torch.uint8 if i["bits"] <= 8 else torch.int16
            self.outs.append(torch.empty((i["ncomp"], i["height"], i["width"]), dtype=dt, device=dev))
        optrs = (C.c_void_p * len(self.outs))(*[o.data_ptr() for o in self.outs])
        with torch.cuda.stream(self.stream):
            self.ctx.check(lib.tc_plan_execute(self.plan, optrs), "tc_plan_execute")
            self.event = torch.cuda.Event()
            self.event.record(self.stream)
        self.batch = batch
        self.keep = keep_outputs

    def busy(self) -> bool:
        return bool(self.batch)

    def poll(self, now_fn):
        if not self.batch or not self.event.query():
            return []
        t = now_fn()
        self.ctx.synchronize()  # reads the device error word
        done = self.batch
        for r, o in zip(done, self.outs):
            r.done = t
            if self.keep:
                a = o.cpu().numpy()
                if r.info["bits"] > 8:
                    a = a.view(np.int16 if r.info.get("is_signed") else np.uint16)
                r.output = a
        self.batch = []
        self.outs = None
        return done

    def close(self):
        if self.plan is not None:
            L.lib().tc_plan_destroy(self.plan)
            self.plan = None
        self.ctx.close()


class Server:
    """Continuous-batching decoder.  `budget_bytes` bounds the device memory
    of the requests in flight; `max_batch` bounds a batch's request count."""

    def __init__(self, device: int = 0, budget_bytes: int = 40 << 30, max_batch: int = 32, inflight: int = 2):
        if torch is None or not torch.cuda.is_available():
            raise L.LibraryMissing("a CUDA device is required (no CPU fallback)")
        self.budget = budget_bytes
        self.max_batch = max_batch
        self.slots = [_Slot(self, device) for _ in range(inflight)]
        self.parser = ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1)))

    def close(self):
        for s in self.slots:
            s.close()
        self.parser.shutdown(wait=True)

    def run(self, requests, realtime: bool = True, keep_outputs: bool = False):
        """Serve `requests` (Request objects with arrival times in seconds
        from the start).  With realtime, a request becomes visible only once
        the clock passes its arrival; otherwise all are visible at once.
        Returns (requests with done times, wall seconds)."""
        for r in requests:
            if not r.info:
                r.info = read_header(r.cs)
                r.device_bytes = request_device_bytes(r.info, len(r.cs))
            if r.device_bytes > self.budget:
                raise ValueError(f"request {r.rid} needs {r.device_bytes} B, above the budget")
        pending = sorted(requests, key=lambda r: r.arrival)
        t0 = time.perf_counter()
        now = (lambda: time.perf_counter() - t0) if realtime else (lambda: time.perf_counter() - t0)
        if not realtime:
            for r in pending:
                r.arrival = 0.0
        queue, finished = [], []
        nxt = 0
        in_flight_bytes = 0
        while len(finished) < len(requests):
            t = now()
            while nxt < len(pending) and pending[nxt].arrival <= t:
                r = pending[nxt]
                r.parsed = self.parser.submit(_parse, r.cs)  # Tier-2 overlaps the decodes in flight
                queue.append(r)
                nxt += 1
            for s in self.slots:
                for r in s.poll(now):
                    in_flight_bytes -= r.device_bytes
                    finished.append(r)
            for s in self.slots:
                if s.busy() or not queue:
                    continue
                batch = []
                while queue and len(batch) < self.max_batch and \
                        in_flight_bytes + queue[0].device_bytes <= self.budget:
                    r = queue.pop(0)
                    batch.append(r)
                    in_flight_bytes += r.device_bytes
                if batch:
                    s.launch(batch, keep_outputs)
            if not any(s.busy() for s in self.slots) and not queue and nxt < len(pending):
                # idle until the next arrival
                wait = pending[nxt].arrival - now()
                if wait > 0:
                    time.sleep(min(wait, 0.001))
        return finished, now()


def poisson_arrivals(n: int, rate_per_s: float, seed: int = 0):
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_per_s, n))


def latency_stats(reqs):
    lat = np.array([(r.done - r.arrival) * 1000.0 for r in reqs])
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean())}
