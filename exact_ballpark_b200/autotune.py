"""The tiled schedule's autotuner: tile size (rows a tile holds, so worlds a block takes), threads a block (warps a
block runs; each warp takes 32 of the tile's ships at a time through the warp-cooperative orientation step), and the
persistent grid (blocks resident for the whole launch, or one block a tile). Each candidate is timed on the park itself with CUDA events (median of a few ticks,
after one warm-up); the park's state is saved before and restored after, so tuning changes nothing a caller sees.
The winner becomes the park's plan. Worlds larger than a candidate's tile size raise it to the largest world."""

from __future__ import annotations

import statistics

import torch

from .tiles import plan_tiles


def candidates(sm_count: int) -> list:
    out = []
    for cap, block in ((128, 128), (256, 128), (256, 256), (384, 256), (512, 256)):
        for per_sm in (None, 3, 6):
            out.append((cap, block, None if per_sm is None else per_sm * sm_count))
    return out


def autotune(park, ticks: int = 3, cands: list | None = None, verbose: bool = False) -> dict:
    """Time every candidate plan on `park` and keep the fastest; returns {(cap, block, grid): ms} and sets
    park.plan."""
    from .modes import tick_tiled

    if park.plan is None:
        raise ValueError("the park's worlds are not contiguous rows: nothing to tune")
    dev = park.dev
    sm = torch.cuda.get_device_properties(dev).multi_processor_count
    names = park.row_tensors()
    saved = {k: getattr(park, k).clone() for k in names}
    stream = torch.cuda.current_stream(dev)
    results = {}
    best = None
    for cap, block, grid in (cands or candidates(sm)):
        plan = plan_tiles(park.world, cap=cap, block=block, grid=grid)
        if plan is None:
            continue
        if grid is not None and grid > plan.tiles:
            continue
        times = []
        for k in range(ticks + 1):
            for name, v in saved.items():
                getattr(park, name).copy_(v)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            tick_tiled(park, plan)
            b.record(stream)
            b.synchronize()
            if k:
                times.append(a.elapsed_time(b))
        ms = statistics.median(times)
        results[(plan.cap, block, plan.grid)] = ms
        if verbose:
            print(f"cap {plan.cap:5d} block {block:4d} grid {plan.grid:6d}: {ms:.4f} ms")
        if best is None or ms < best[0]:
            best = (ms, plan)
    for name, v in saved.items():
        getattr(park, name).copy_(v)
    park.plan = best[1]
    return results
