"""Autotuner for the decode's launch shapes, per GPU and shape bucket.

Two choices are tuned, each on the plan's own work with CUDA events on its
stream (tc_plan_stage_ms):

  * the Tier-1 lane-group width: 32 lanes per code-block (one warp per
    block, eight per CTA), 16 (two blocks per warp) or 8 (four per warp,
    decoded in lock-step); uniform blocks keep the groups of a warp in step,
    ragged ones make them diverge;
  * the staging of the fused last reverse 9/7 level: 2-D tensor copies (TMA)
    into persistent CTAs, or one 4-byte asynchronous copy per sample into a
    CTA per tile; large levels favour the first, small ones can favour the
    second (fewer tiles than the persistent grid, tensor-map set-up per
    launch).

The reference picks its DWT window by image width (DWTReverse53.cpp:36-42,
DWTReverse97.cpp:37-43: 192, 128 or 64 columns); here the choice is
measured.  `tune_plan` times the candidates, sets the winners on the plan's
context and caches them in a JSON file keyed by GPU and bucket (image size
class, code-block count class, image count class, wavelet mix, component
count), so later plans of the same kind of batch skip the search.  Results
do not depend on the choices (every candidate decodes bit for bit the
same).
"""
from __future__ import annotations

import json
import math
import os
from pathlib import Path

from . import _lib as L

WIDTHS = (32, 16, 8)
DWT_VARIANTS = {"tma": L.TC_DWT_TMA, "cp.async": L.TC_DWT_CPASYNC}
CACHE = Path(os.environ.get("TC_J2K_TUNE_CACHE", Path(__file__).resolve().parent / "tune_cache.json"))


def _load():
    try:
        return json.loads(CACHE.read_text())
    except (OSError, ValueError):
        return {}


def _store(d):
    try:
        CACHE.write_text(json.dumps(d, indent=1, sort_keys=True) + "\n")
    except OSError:
        pass


def bucket(plan) -> str:
    """Shape bucket: largest image (power-of-two pixel class), code-block
    count, image count, wavelet mix and component counts."""
    n = sum(i["ncblk"] for i in plan.infos)
    kinds = {i["reversible"] for i in plan.infos}
    kind = "mixed" if len(kinds) > 1 else ("lossless" if 1 in kinds else "lossy")
    px = max(i["width"] * i["height"] for i in plan.infos)
    comps = "/".join(str(c) for c in sorted({i["ncomp"] for i in plan.infos}))
    return (f"px2^{int(math.log2(max(px, 1)))}|cblk2^{int(math.log2(max(n, 1)))}|"
            f"img2^{int(math.log2(len(plan.infos)))}|{kind}|c{comps}")


def _set(ctx, lanes=None, dwt=None):
    if lanes is not None:
        L.check(L.lib().tc_ctx_set_t1_group(ctx.handle, lanes), ctx.handle, "tc_ctx_set_t1_group")
    if dwt is not None:
        L.check(L.lib().tc_ctx_set_dwt_variant(ctx.handle, dwt), ctx.handle, "tc_ctx_set_dwt_variant")


def tune_plan(plan, outs, trials: int = 2, use_cache: bool = True) -> dict:
    """Pick the fastest Tier-1 lane-group width and last-level DWT staging
    for this plan's workload and set them on the plan's context.  Returns
    {"lanes", "dwt", "bucket", "tier1_ms", "dwt_ms", "cached"}."""
    import torch
    ctx = plan.ctx
    b = bucket(plan)
    key = f"{torch.cuda.get_device_name(ctx.device)}|{b}"
    cache = _load() if use_cache else {}
    if key in cache and "dwt" in cache[key]:
        c = cache[key]
        _set(ctx, int(c["lanes"]), DWT_VARIANTS[c["dwt"]])
        return {**c, "bucket": b, "cached": True}

    def timed(stage):
        plan.execute(outs)   # warm-up (first launch of a variant sets its attributes)
        plan.stage_ms()
        best = float("inf")
        for _ in range(trials):
            plan.execute(outs)
            best = min(best, plan.stage_ms()[stage])
        return best

    plan.set_profiling(True)
    try:
        _set(ctx, dwt=L.TC_DWT_TMA)
        t1 = {}
        for g in WIDTHS:
            _set(ctx, lanes=g)
            t1[g] = timed(0)
        lanes = min(t1, key=t1.get)
        _set(ctx, lanes=lanes)
        dw = {}
        for name, v in DWT_VARIANTS.items():
            _set(ctx, dwt=v)
            dw[name] = timed(1)
        dwt = min(dw, key=dw.get)
        _set(ctx, dwt=DWT_VARIANTS[dwt])
    finally:
        plan.set_profiling(False)
    res = {"lanes": lanes, "dwt": dwt, "tier1_ms": {str(k): round(v, 3) for k, v in t1.items()},
           "dwt_ms": {k: round(v, 4) for k, v in dw.items()}}
    if use_cache:
        cache = _load()
        cache[key] = res
        _store(cache)
    return {**res, "bucket": b, "cached": False}


def apply(plan, table: dict | None = None) -> dict | None:
    """Set the cached choices of the plan's bucket on its context (the
    defaults, TMA staging and 32 lanes, when the bucket was never tuned).
    `table` maps buckets to choices (default: the cache file)."""
    import torch
    ctx = plan.ctx
    b = bucket(plan)
    if table is None:
        table = {k.split("|", 1)[1]: v for k, v in _load().items()
                 if k.startswith(torch.cuda.get_device_name(ctx.device) + "|")}
    c = table.get(b)
    if c is None:
        _set(ctx, 32, L.TC_DWT_TMA)
        return None
    _set(ctx, int(c["lanes"]), DWT_VARIANTS[c["dwt"]])
    return c
