"""Block-size and member-tile autotuner of the routing kernels.

The sub-step kernels are latency-bound gathers, and their best CTA size
depends on the network (catchment count, share of flooded and levee cells,
members) and on the GPU; with several members, so does the member-tile width
(members of one catchment per thread).  `tune_block_size` measures them
instead of guessing: for every candidate pair it builds the model's plan with
that block size and tile, runs a few sub-steps of the model's current state
through the per-kernel entry points (momentum, limit rate, stage, levee),
timed with CUDA events on the model's stream, restores the state, and keeps
the fastest.

Results can be cached in a JSON file keyed by the GPU name and the network's
shape (catchments, members, floodplain levels, feature bits), so later runs
of the same configuration skip the measurement.
"""
from __future__ import annotations

import json
import os
from typing import Iterable, Optional

import torch

from . import _lib

DEFAULT_CANDIDATES = (64, 128, 192, 256)
DEFAULT_TILES = (1, 2, 4, 8, 16)
_PARTS = (_lib.PART_MOMENTUM, _lib.PART_LIMIT, _lib.PART_STAGE, _lib.PART_LEVEE)


def _cache_key(model) -> str:
    props = torch.cuda.get_device_properties(model.device)
    return (f"{props.name}|N={model.num_catchments}|M={model.num_members}|"
            f"K={model.base.num_flood_levels}|F={model._features() & ~_lib.FEAT_GRAPH}")


def _time_candidate(model, sub_steps: int, repeats: int) -> float:
    """Mean milliseconds of one sub-step (all four kernels) on the model's
    current plan, from the model's current state (restored by the caller)."""
    stream = torch.cuda.current_stream(model.device)
    model.compute_adaptive_time_step()
    n = max(1, min(sub_steps, int(model.sub_step_counts().max().item())))
    for k in range(n):                                   # warm-up pass
        for part in _PARTS:
            model.launch_substep_kernel(k, part)
    best = float("inf")
    for _ in range(repeats):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for k in range(n):
            for part in _PARTS:
                model.launch_substep_kernel(k, part)
        b.record(stream)
        b.synchronize()
        best = min(best, a.elapsed_time(b) / n)
    return best


def tune_block_size(model, candidates: Iterable[int] = DEFAULT_CANDIDATES, sub_steps: int = 6,
                    repeats: int = 3, cache_path: Optional[str] = None,
                    tile_candidates: Optional[Iterable[int]] = None) -> dict:
    """Pick the fastest block size (and member tile) for `model`, leave the
    model's plan built with them and return {"block_size": b, "member_tile":
    w, "ms_per_sub_step": {b: ms} (one member) or {"b/w": ms}, "cached": bool}.
    Tile candidates default to the divisors of the member count in
    DEFAULT_TILES (just 1 for one member).

    The model's state after the call equals its state before the call."""
    M = model.num_members
    tiles = [int(w) for w in (tile_candidates or DEFAULT_TILES) if M % int(w) == 0]
    if M == 1 or not tiles:
        tiles = [1]
    key = _cache_key(model)
    cache = {}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as fh:
            cache = json.load(fh)
    if key in cache:
        b = int(cache[key]["block_size"])
        w = int(cache[key].get("member_tile", 1))
        if b != model.block_size:
            model._rebuild_plan(b)
        if w != model.member_tile:
            model.set_member_tile(w)
        return {"block_size": b, "member_tile": w, "ms_per_sub_step": cache[key]["ms_per_sub_step"],
                "cached": True}

    snapshot = {k: v.clone() for k, v in model.state_tensors().items()}
    original = (model.block_size, model.member_tile)
    times = {}
    try:
        for b in candidates:
            b = int(b)
            if b < 32 or b > 256 or b % 32:
                raise ValueError(f"block size {b} is not a multiple of 32 in [32, 256]")
            model._rebuild_plan(b)
            for w in tiles:
                model.set_member_tile(w)
                times[(b, w)] = _time_candidate(model, sub_steps, repeats)
                for k, v in model.state_tensors().items():
                    v.copy_(snapshot[k])
    except Exception:
        model._rebuild_plan(original[0])
        model.set_member_tile(original[1])
        for k, v in model.state_tensors().items():
            v.copy_(snapshot[k])
        raise
    best_b, best_w = min(times, key=times.get)
    model._rebuild_plan(best_b)
    model.set_member_tile(best_w)
    if torch.device(model.device).type == "cuda":
        torch.cuda.synchronize(model.device)
    shown = ({b: t for (b, _), t in times.items()} if tiles == [1]
             else {f"{b}/{w}": t for (b, w), t in times.items()})
    if cache_path:
        cache[key] = {"block_size": best_b, "member_tile": best_w,
                      "ms_per_sub_step": {str(k): v for k, v in shown.items()}}
        with open(cache_path, "w") as fh:
            json.dump(cache, fh, indent=1, sort_keys=True)
    return {"block_size": best_b, "member_tile": best_w, "ms_per_sub_step": shown, "cached": False}
