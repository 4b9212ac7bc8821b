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
gathering, descriptors) on a worker thread as soon as it arrives, while
earlier batches decode; a batch is then built from the parsed requests with
`tc_plan_rebuild_parsed`, which only lays out and uploads.

Failures stay with their request.  A request whose header or codestream does
not parse, or whose estimated device memory is above the whole budget,
finishes at once with `error` set and never holds budget.  A batch that fails
on the device (a kernel flagged bad code-block data) is split: each of its
requests is run again alone, and only the ones that fail alone finish with an
error.  Budget is released whenever a request finishes, failed or not.

The GPU side of a slot is an executor object (`_Slot` by default); tests pass
a CPU fake through `slot_factory` to drive admission, failures and latency
without a device.

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
    error: str | None = None            # set when the request failed
    alone: bool = False                 # re-run alone after its batch failed


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
    """One batch in flight on its own CUDA stream and resident plan."""

    def __init__(self, device):
        self.stream = torch.cuda.Stream(device)
        from .stages import Context
        self.ctx = Context(device, self.stream)
        self.plan = None
        self.outs = None
        self.batch = []
        self.event = None
        self.keep = []

    def launch(self, batch, keep_outputs):
        """Build the slot's plan for `batch` and start its decode; raises on
        a host-side failure (a request that does not parse)."""
        lib = L.lib()
        self.batch = []
        try:
            parsed = [r.parsed.result() for r in batch]
            arr = (C.POINTER(L.Parsed) * len(parsed))(*parsed)
            if self.plan is None:
                bufs = [np.frombuffer(r.cs, np.uint8) for r in batch]
                ptrs = (C.c_void_p * len(bufs))(*[b.ctypes.data for b in bufs])
                lens = (C.c_size_t * len(bufs))(*[b.size for b in bufs])
                h = C.c_void_p()
                self.ctx.check(lib.tc_plan_create(self.ctx.handle, ptrs, lens, len(bufs), C.byref(h)),
                               "tc_plan_create")
                self.plan = h
            else:
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
        """The finished batch's requests, or []; raises when the device
        flagged the batch (the slot is free again either way)."""
        if not self.batch or not self.event.query():
            return []
        t = now_fn()
        done = self.batch
        self.batch = []
        try:
            self.ctx.synchronize()  # reads and clears the device error word
            for r, o in zip(done, self.outs):
                r.done = t
                if self.keep:
                    a = o.cpu().numpy()
                    if r.info["bits"] > 8:
                        a = a.view(np.int16 if r.info.get("is_signed") else np.uint16)
                    r.output = a
        finally:
            self.outs = None
        return done

    def device_bytes(self) -> int:
        """Device memory the slot holds now: what its context's memory pool
        reserves (its plan's buffers and blocks kept for regrowth) and its
        batch's outputs."""
        b = C.c_size_t(0)
        L.check(L.lib().tc_ctx_pool_bytes(self.ctx.handle, C.byref(b)), self.ctx.handle, "tc_ctx_pool_bytes")
        return b.value + sum(o.numel() * o.element_size() for o in self.outs or [])

    def shrink(self):
        """Give the slot's device memory back (idle slots only): destroy its
        plan and return the pool's blocks; the next batch builds a new plan."""
        if self.plan is not None:
            L.lib().tc_plan_destroy(self.plan)
            self.plan = None
        L.check(L.lib().tc_ctx_trim(self.ctx.handle), self.ctx.handle, "tc_ctx_trim")

    def close(self):
        if self.plan is not None:
            L.lib().tc_plan_destroy(self.plan)
            self.plan = None
        self.ctx.close()


class Server:
    """Continuous-batching decoder.  `budget_bytes` bounds the estimated
    device memory of the requests in flight; `max_batch` bounds a batch's
    request count.  `slot_factory(i)` makes the executor of slot i (default:
    a GPU slot on `device`)."""

    def __init__(self, device: int = 0, budget_bytes: int = 40 << 30, max_batch: int = 32, inflight: int = 2,
                 slot_factory=None, max_batch_samples: int = 0):
        if slot_factory is None:
            if torch is None or not torch.cuda.is_available():
                raise L.LibraryMissing("a CUDA device is required (no CPU fallback)")
            slot_factory = lambda i: _Slot(device)  # noqa: E731
        self.budget = budget_bytes
        self.max_batch = max_batch
        # samples (width x height x components) per batch, 0: no cap.  Large
        # images fill the GPU alone; batching pays for small ones, and a cap
        # keeps a batch's decode, and so its requests' latency, short.
        self.max_batch_samples = max_batch_samples
        self.slots = [slot_factory(i) for i in range(inflight)]
        self.parser = ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1)))
        self.stats = {}

    def close(self):
        for s in self.slots:
            s.close()
        self.parser.shutdown(wait=True)

    def run(self, requests, realtime: bool = True, keep_outputs: bool = False, stop_backlog_s: float = 0.0):
        """Serve `requests` (Request objects with arrival times in seconds
        from the start).  With realtime, a request becomes visible only once
        the clock passes its arrival; otherwise all are visible at once.
        stop_backlog_s > 0 ends an overloaded run early: once the oldest
        waiting request has waited that long, no further arrivals are
        admitted, waiting requests are dropped and the run finishes the
        batches in flight (the dropped and unarrived requests are left
        unserved, done < 0, and not returned).  Returns (finished requests, wall seconds);
        failed requests are among them with `error` set.  self.stats then
        holds the peak admitted and measured device bytes and the counts of
        failed and unserved requests."""
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731
        finished = []

        def fail(r, msg):
            r.error = msg
            r.done = now()
            _free_parsed(r)
            finished.append(r)

        pending = []
        for r in sorted(requests, key=lambda r: r.arrival):
            if not realtime:
                r.arrival = 0.0
            r.error, r.done, r.alone = None, -1.0, False
            pending.append(r)
        queue, retry = [], []
        nxt = 0
        in_flight_bytes = 0
        peak_admitted = peak_measured = 0
        stopped = False
        unserved = []
        while True:
            t = now()
            while not stopped and nxt < len(pending) and pending[nxt].arrival <= t:
                r = pending[nxt]
                nxt += 1
                try:
                    if not r.info:
                        r.info = read_header(r.cs)
                        r.device_bytes = request_device_bytes(r.info, len(r.cs))
                except Exception as ex:  # noqa: BLE001 - a bad header fails its request only
                    fail(r, f"header: {ex}")
                    continue
                if r.device_bytes > self.budget:
                    fail(r, f"needs {r.device_bytes} B of device memory, above the budget")
                    continue
                r.parsed = self.parser.submit(_parse, r.cs)  # Tier-2 overlaps the decodes in flight
                queue.append(r)
            if stop_backlog_s > 0 and not stopped and queue and t - queue[0].arrival > stop_backlog_s:
                stopped = True          # overloaded: stop admitting, finish the batches in flight
                unserved = pending[nxt:] + queue
                for r in queue:
                    _free_parsed(r)
                queue = []
                nxt = len(pending)
            for s in self.slots:
                batch = s.batch if s.busy() else []
                try:
                    done = s.poll(now)
                except Exception as ex:  # noqa: BLE001 - the device flagged this batch
                    for r in batch:
                        in_flight_bytes -= r.device_bytes
                        if len(batch) == 1 or r.alone:
                            fail(r, f"decode: {ex}")
                        else:
                            r.alone = True
                            r.parsed = self.parser.submit(_parse, r.cs)
                            retry.append(r)
                    continue
                for r in done:
                    in_flight_bytes -= r.device_bytes
                    finished.append(r)
            for s in self.slots:
                if s.busy():
                    continue
                src = retry if retry else queue
                if not src:
                    continue
                # Measured memory: the other slots hold `others`, so this slot
                # may hold `room`.  A slot with a plan grows its buffers by up
                # to half again to fit a batch; a fresh one allocates exactly.
                # An idle slot that keeps more than the head request leaves
                # room for gives its memory back, then the other idle ones.
                head = src[0].device_bytes
                others = sum(x.device_bytes() for x in self.slots if x is not s)

                def fits(n, s=s, others=others):
                    held = n if s.plan is None else max(s.device_bytes(), 1.5 * n)
                    return held <= self.budget - others

                if not fits(head):
                    s.shrink()
                    if self.budget - others < head:
                        for x in self.slots:
                            if x is not s and not x.busy():
                                x.shrink()
                        others = sum(x.device_bytes() for x in self.slots if x is not s)
                batch = []
                need = samples = 0
                cap = self.max_batch_samples or float("inf")
                while src and len(batch) < (1 if src is retry else self.max_batch) and \
                        in_flight_bytes + src[0].device_bytes <= self.budget and \
                        fits(need + src[0].device_bytes, s, others) and \
                        (not batch or samples + _samples(src[0]) <= cap):
                    r = src[0]
                    if r.parsed is not None and r.parsed.done() and r.parsed.exception() is not None:
                        src.pop(0)
                        fail(r, f"parse: {r.parsed.exception()}")
                        continue
                    src.pop(0)
                    batch.append(r)
                    need += r.device_bytes
                    samples += _samples(r)
                    in_flight_bytes += r.device_bytes
                if not batch:
                    continue
                peak_admitted = max(peak_admitted, in_flight_bytes)
                try:
                    s.launch(batch, keep_outputs)
                except Exception as ex:  # noqa: BLE001 - host-side failure of the batch
                    for r in batch:
                        in_flight_bytes -= r.device_bytes
                        if len(batch) == 1 or r.alone:
                            fail(r, f"launch: {ex}")
                        else:
                            r.alone = True
                            r.parsed = self.parser.submit(_parse, r.cs)
                            retry.append(r)
                    continue
                peak_measured = max(peak_measured, sum(x.device_bytes() for x in self.slots))
            if nxt >= len(pending) and not queue and not retry and not any(s.busy() for s in self.slots):
                break
            if not any(s.busy() for s in self.slots) and not queue and not retry and nxt < len(pending):
                wait = pending[nxt].arrival - now()   # idle until the next arrival
                if wait > 0:
                    time.sleep(min(wait, 0.001))
            elif any(s.busy() for s in self.slots):
                time.sleep(0)
        wall = now()
        self.stats = {"peak_admitted_bytes": int(peak_admitted), "peak_device_bytes": int(peak_measured),
                      "failed": sum(1 for r in finished if r.error), "unserved": len(unserved),
                      "stopped_at_s": round(wall, 3) if stopped else None}
        return finished, wall


def _samples(r) -> int:
    i = r.info
    return i["width"] * i["height"] * i["ncomp"]


def poisson_arrivals(n: int, rate_per_s: float, seed: int = 0):
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_per_s, n))


def latency_stats(reqs):
    ok = [r for r in reqs if r.error is None and r.done >= 0]
    if not ok:
        return {"p50_ms": float("nan"), "p99_ms": float("nan"), "mean_ms": float("nan")}
    lat = np.array([(r.done - r.arrival) * 1000.0 for r in ok])
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean())}
