"""Autotuner for the Tier-1 launch shape.

The Tier-1 kernel is compiled for three lane-group widths: 32 lanes per
code-block (one warp per block, four warps per CTA), 16 (two blocks per warp)
and 8 (four blocks per warp, decoded in lock-step).  Which one is fastest
depends on the block mix: uniform blocks keep the lane groups of a warp in
step, ragged ones make them diverge.  `tune_plan` times each width on the
plan's own work, sets the winner on the context and caches it in a JSON file
keyed by GPU and workload bucket, so later runs with the same kind of batch
skip the search.
"""
from __future__ import annotations

import json
import math
import os
from pathlib import Path

from . import _lib as L

WIDTHS = (32, 16, 8)
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
    """Workload bucket: code-block count (power-of-two bucket), image count
    bucket and whether lossless / lossy / mixed."""
    n = sum(i["ncblk"] for i in plan.infos)
    kinds = {i["reversible"] for i in plan.infos}
    kind = "mixed" if len(kinds) > 1 else ("lossless" if 1 in kinds else "lossy")
    return f"cblk2^{int(math.log2(max(n, 1)))}|img2^{int(math.log2(len(plan.infos)))}|{kind}"


def tune_plan(plan, outs, trials: int = 2, use_cache: bool = True) -> int:
    """Pick the fastest Tier-1 lane-group width for this plan's workload and
    set it on the plan's context.  Returns the width."""
    import torch
    ctx = plan.ctx
    key = f"{torch.cuda.get_device_name(ctx.device)}|{bucket(plan)}"
    cache = _load() if use_cache else {}
    if key in cache:
        g = int(cache[key]["lanes"])
        L.check(L.lib().tc_ctx_set_t1_group(ctx.handle, g), ctx.handle, "tc_ctx_set_t1_group")
        return g
    times = {}
    plan.set_profiling(True)
    for g in WIDTHS:
        L.check(L.lib().tc_ctx_set_t1_group(ctx.handle, g), ctx.handle, "tc_ctx_set_t1_group")
        plan.execute(outs)  # warm-up (first launch of this variant sets its attributes)
        plan.stage_ms()
        best = float("inf")
        for _ in range(trials):
            plan.execute(outs)
            best = min(best, plan.stage_ms()[0])
        times[g] = best
    plan.set_profiling(False)
    g = min(times, key=times.get)
    L.check(L.lib().tc_ctx_set_t1_group(ctx.handle, g), ctx.handle, "tc_ctx_set_t1_group")
    if use_cache:
        cache = _load()
        cache[key] = {"lanes": g, "tier1_ms": {str(k): round(v, 3) for k, v in times.items()}}
        _store(cache)
    return g
