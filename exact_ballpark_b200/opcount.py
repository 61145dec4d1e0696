"""The IEEE operations a tick executes, counted on the device by the counting build of the native library
(libebb_count.so: built with EBB_COUNT_OPS, every double and float add, subtract, multiply, divide, square root and
fused multiply-add of the kernels counted by kind). A measurement tool, never the timed path: the counts give the
FLOPs per ship-tick of each workload's algorithm as it runs, the compute side of its roofline.

Run as its own process with EBB_COUNTING=1 (the package then loads the counting build):

    EBB_COUNTING=1 python -m exact_ballpark_b200.opcount flight|partition [--worlds W] [--ticks T]

prints one JSON object: per ship-tick the operations of each kind, the double and float totals, and FLOPs (a fused
multiply-add counted as two, a divide or square root as one).
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os

KINDS = ("dadd", "dsub", "dmul", "ddiv", "dsqrt", "dfma", "fadd", "fsub", "fmul", "fdiv", "fsqrt", "ffma")
UNITS = ("flight", "space", "collide", "combat", "server")


def _counts(reset: bool = True) -> dict:
    from . import _native
    lib = _native.lib()
    out = {k: 0 for k in KINDS}
    for unit in UNITS:
        buf = (ctypes.c_ulonglong * len(KINDS))()
        rc = getattr(lib, "ebb_count_ops_" + unit)(buf, int(reset))
        _native.check(rc, "ebb_count_ops_" + unit)
        for k, v in zip(KINDS, buf):
            out[k] += int(v)
    return out


def per_ship_tick(counts: dict, ship_ticks: int) -> dict:
    d = sum(counts[k] for k in KINDS[:6])
    f = sum(counts[k] for k in KINDS[6:])
    flops = d + f + counts["dfma"] + counts["ffma"]
    out = {k: counts[k] / ship_ticks for k in KINDS}
    out.update(fp64_ops=d / ship_ticks, fp32_ops=f / ship_ticks, fp64_flops=(d + counts["dfma"]) / ship_ticks,
               fp32_flops=(f + counts["ffma"]) / ship_ticks, flops=flops / ship_ticks, ship_ticks=ship_ticks)
    return out


def count_flight(worlds: int, ticks: int) -> dict:
    """The flight-mode benchmark's worlds (4 ships, dynamical orientation on, the new orbit law), `ticks` ticks of the
    tiled schedule after one uncounted tick."""
    import torch

    from . import VecModesPark, tick_tiled
    from .workloads import flight_worlds
    w = flight_worlds(1, worlds, 4)
    p = VecModesPark(len(w.rows), device="cuda", dynamical_orientation=True, use_new_orbit=True)
    p.load(w.rows)
    w.apply(p)
    tick_tiled(p)
    torch.cuda.synchronize()
    _counts()
    for _ in range(ticks):
        tick_tiled(p)
    torch.cuda.synchronize()
    return per_ship_tick(_counts(), p.n * ticks)


def _sensor_paths(reset: bool = True) -> list:
    from . import _native
    buf = (ctypes.c_ulonglong * 3)()
    _native.check(_native.lib().ebb_count_sensor_paths(buf, int(reset)), "ebb_count_sensor_paths")
    return [int(v) for v in buf]


def count_partition(worlds: int, ticks: int) -> dict:
    """The partition worlds (ragged 1-128 ships, sensors on every ship) with the space layer and the server on top,
    as the benchmark ticks them (the ragged arrangement), `ticks` ticks after the set-up and one uncounted tick."""
    import torch

    from .partition import partition_setup
    from .workloads import partition_worlds
    pw = partition_worlds(11, worlds)
    r = partition_setup(pw, torch.device("cuda"), ragged=True)
    r["graph"].tick()
    torch.cuda.synchronize()
    _counts()
    _sensor_paths()
    for _ in range(ticks):
        r["graph"].tick()
    torch.cuda.synchronize()
    out = per_ship_tick(_counts(), pw.n * ticks)
    checks, skipped, same = _sensor_paths()
    out["sensor_checks"] = checks
    out["sensor_refilings_skipped"] = skipped / max(checks, 1)    # CheckSensor's two re-filings skipped (no trace)
    out["sensor_filing_unchanged"] = same / max(checks, 1)        # of them: the inflated filing the ball's own
    return out


def main() -> None:
    if os.environ.get("EBB_COUNTING") != "1":
        raise SystemExit("run with EBB_COUNTING=1: the counts come from the counting build (libebb_count.so)")
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=("flight", "partition"))
    ap.add_argument("--worlds", type=int, default=4096)
    ap.add_argument("--ticks", type=int, default=10)
    a = ap.parse_args()
    run = {"flight": count_flight, "partition": count_partition}[a.workload]
    print(json.dumps({"workload": a.workload, "worlds": a.worlds, "ticks": a.ticks, **run(a.worlds, a.ticks)}))


if __name__ == "__main__":
    main()
