"""Benchmark of the batched destiny tick on B200: bit-exact ship-ticks/s of the flight-mode park.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--worlds W] [--ships S]

A step is one tick of every world. The workload is the flight-mode park's benchmark shape: `--worlds` (65,536)
worlds of `--ships` (4) ships drawn by exact_ballpark_b200.workloads.flight_worlds (config 0's distributions, each
world its own seed), dynamical orientation on, the new orbit law. Each rank ticks its own worlds (seed = rank + 1):
replicas, weak scaling, no collective on the data path; the timing is the max over ranks.

Timed: W untimed warm-up ticks, then K ticks, each launched as one CUDA-graph replay of the tiled (ragged,
persistent) schedule and timed with CUDA events on the launching stream; L2 is flushed (a 256 MiB write, untimed)
before each step. Beside it the plain schedule (two launches, records in scratch) is timed the same way, and `e2e`
times the same step through the public API from host buffers: every step a pinned host->device copy of the ships'
speed fractions applied by set_speed_fraction (the values they hold, so the flight is unchanged), the tick, and a
device->host copy of every position. `cpu_baseline` is the C++ oracle (a scalar port of the reference's algorithm)
on the host's cores over a bounded sample. `--impl reference` times that CPU port on the whole workload instead (the
reference's own implementation is Python; the port is its compiled restatement), rank 0 only. `serve` runs the
serving loop (continuous batching of arriving episodes, state resident under a byte budget): an open loop at the
configured arrival rate, with p50/p99 step latency, and a saturated closed loop (bench.serve_runs).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests" / "golden"))      # the golden streams' operation codes (space_trace)

METRIC = "bit-exact ship-ticks/s on 1 B200 (ragged batch vs plain); serve p50/p99 latency"
UNIT = "ship-ticks/s"
# Algorithmic bytes a ship-tick reads and writes in the minimal (this package's) layout, dynamical orientation on:
# reads 229 B (pos, vel, goto, last_g 4 x 24; mass, time factor, warp length 3 x 8; radius, max_vel, agility, speed
# fraction, follow range, max_ang_vel, rot_agility 7 x 4; ids, stamp, follow id, owner id, clock 5 x 8; mode,
# follow_ptr 2 x 4; 5 flag bytes; rotation 16, angular velocity 12), writes 274 B (pos, vel, old_pos, old_vel, goto,
# last_g 6 x 24; warp length 8, speed fraction and follow range 2 x 4, mode 4, stamp, follow id, owner id, clock
# 4 x 8, follow_ptr 4, 2 flag bytes; rotation and old rotation 2 x 16, angular velocity, old angular velocity,
# torque 3 x 12, roll 4).
BYTES_PER_SHIP_TICK = 229 + 274
FALLBACK_HBM_GBS = 6650.0


def _peaks() -> tuple:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


class Clocks:
    """nvidia-smi sampled every 100 ms during the timed region (SM clock, throttle reasons)."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        self._wait_lines(1, 5.0)                 # sampling has started before the timed region
        return self

    def _wait_lines(self, k: int, limit: float) -> int:
        until = time.perf_counter() + limit
        n = 0
        while self.proc is not None and time.perf_counter() < until:
            n = len(Path(self.path).read_text().splitlines())
            if n >= k or self.proc.poll() is not None:
                break
            time.sleep(0.01)
        return n

    def __exit__(self, *exc):
        if self.proc is not None:
            self._wait_lines(self._wait_lines(0, 0.0) + 1, 1.0)   # one more sample after the timed region
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if self.proc is None or self.path is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        Path(self.path).unlink(missing_ok=True)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            for k, name in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def cpu_sample(worlds: int, ships: int, warmup: int, steps: int) -> dict:
    """The CPU oracle on every host core over the same tick window as the GPU run (ticks warmup+1 .. warmup+steps of
    the same workload), on `worlds` worlds: ship-ticks/s."""
    from exact_ballpark_b200.workloads import flight_worlds
    from oracle.park import OraclePark
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    w = flight_worlds(1, worlds, ships)
    p = OraclePark(len(w.rows), dynamical_orientation=True, use_new_orbit=True)
    p.load(w.rows)
    w.apply(p)
    for _ in range(warmup):
        p.evolve(threads=threads)
    t0 = time.perf_counter()
    for _ in range(steps):
        p.evolve(threads=threads)
    dt = time.perf_counter() - t0
    return {"value": len(w.rows) * steps / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{worlds} worlds x {ships} ships (seed 1), ticks {warmup + 1}..{warmup + steps} "
                      f"({dt:.1f} s wall, {dt * threads:.0f} core-s), C++ oracle (oracle/flight.cpp), "
                      f"{threads} threads over disjoint worlds"}


def reduce_max(x: float, dist, device) -> float:
    """The largest x over the ranks of the process group (one all-reduce; x itself without a group): the timing of a
    multi-GPU run is its slowest rank's. `device`: where the group's backend reduces (a CUDA device for NCCL, the CPU
    for gloo)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args, rank: int) -> None:
    """The reference arm: the reference's algorithm on the host's cores (the space oracle, oracle/space.cpp, its
    compiled restatement; the reference's own implementation is Python), on the headline's workload and metric, rank 0
    only: a bounded sample of the partition worlds (up to 2,000 worlds spread over the sizes) loaded and ticked W times,
    then K ticks timed; ship-ticks/s over the sample."""
    if rank != 0:
        return
    from exact_ballpark_b200.workloads import partition_worlds
    pw = partition_worlds(11, args.partition_worlds)
    sample = partition_cpu_sample(pw, min(args.partition_worlds, 2000), args.steps, warm=args.warmup)
    value = sample["value"]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": pw.n / value * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64/f32",
            "data": "synthetic (seeded)",
            "config": {"workload": (f"partition worlds: {args.partition_worlds} worlds of 1-128 ships, sensors, "
                                    "bubbles and the partition (the headline's); a bounded sample timed, ms_per_step "
                                    "the whole workload's at the sample's rate"),
                       "worlds_per_rank": args.partition_worlds, "parallelism": "host cores"},
            "cpu_baseline": dict(sample), "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                                                  "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)

def serve_runs(args, dev) -> dict:
    """The serving loop (exact_ballpark_b200.serving) on this GPU: an open loop of episodes arriving as a Poisson
    process (--serve-rate a second, 1-256 ships log-uniform, 10-10,000 ticks log-uniform, flight-mode worlds), state
    admitted under an --serve-budget-gb budget, for --serve-seconds of arrivals; then a saturated closed loop (every
    episode waiting from the start, a 262,144-row budget, two steps in flight) for --serve-steps steps after
    untimed warm-up steps (at least --serve-warmup, and until 90 % of the budget's rows are live). p50/p99 of each step's latency (host wall time from the step's
    start to its tick's completion; with two steps in flight, to when the loop saw it complete), ship-ticks/s over the
    wall time, and the tick launches' own device rate."""
    import torch

    from exact_ballpark_b200.serving import Server, episode_stream, serve
    out = {}
    count = int(args.serve_rate * args.serve_seconds)
    eps = episode_stream(11, count, rate=args.serve_rate)
    with Server(budget_bytes=args.serve_budget_gb * 1e9, device=dev, keep=False) as srv:
        s = serve(srv, eps, realtime=True, max_steps=None if args.serve_all else args.serve_max_steps)
        out["open_loop"] = dict(s, rate_per_s=args.serve_rate, episodes=count, budget_rows=srv.capacity,
                                arrivals_s=args.serve_seconds)
    del srv
    torch.cuda.empty_cache()
    eps = episode_stream(12, 16000, rate=0.0)
    with Server(rows=262144, device=dev, keep=False, depth=2) as srv:
        for ep in eps:
            srv.submit(ep)
        until = time.perf_counter() + 120.0                                 # fill the budget, untimed
        warm = 0
        while time.perf_counter() < until and (warm < args.serve_warmup or srv.live_rows < 0.9 * srv.capacity):
            if srv.step():
                warm += 1
            else:
                time.sleep(0.0001)
        srv.reset_stats()
        s = serve(srv, [], realtime=False, max_steps=args.serve_steps)
        out["saturated"] = dict(s, budget_rows=srv.capacity, episodes_offered=len(eps), depth=2,
                                warmup_steps=warm)
    del srv
    torch.cuda.empty_cache()
    return out


def serve_configurations(dev, episodes: int = 4000, steps: int = 20, warmup: int = 3) -> dict:
    """The serving loop's episodes (1-256 ships, flight modes, dynamical orientation on) run two ways on the same
    GPU, every episode resident: the plain per-configuration kernels (the episodes grouped by their ship count, one
    park a configuration, each ticked by the plain schedule, every park each step) against the ragged batch (every
    episode in one park, packed with no padding, one tiled launch a step in a CUDA graph). Both tick the same worlds;
    their rows are compared bit for bit at the end."""
    import numpy as np
    import torch

    from exact_ballpark_b200 import ModesGraph, VecModesPark, tick_plain
    from exact_ballpark_b200.serving import episode_stream
    from exact_ballpark_b200.workloads import PackedWorlds
    eps = episode_stream(13, episodes, rate=0.0)
    by_size = {}
    for e in eps:
        by_size.setdefault(e.ships, []).append(e)
    parks = []
    for size, group in sorted(by_size.items()):
        pk = PackedWorlds.concat([e.world.packed() for e in group])
        p = VecModesPark(pk.n, device=dev, dynamical_orientation=True, use_new_orbit=True)
        pk.load(p)
        pk.apply(p)
        p.scratch()
        parks.append((size, group, p))
    order = [e for _, group, _ in parks for e in group]          # the ragged park holds the same worlds in this order
    pk = PackedWorlds.concat([e.world.packed() for e in order])
    ragged = VecModesPark(pk.n, device=dev, dynamical_orientation=True, use_new_orbit=True)
    pk.load(ragged)
    pk.apply(ragged)
    graph = ModesGraph(ragged)
    stream = torch.cuda.current_stream(dev)

    def per_configuration():
        for _, _, p in parks:
            tick_plain(p, 256)

    def timed(step, k):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(k):
            step()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b)
    for _ in range(warmup):
        per_configuration()
        graph.tick()
    ms_plain = timed(per_configuration, steps)
    ms_ragged = timed(graph.tick, steps)
    same = True
    at = 0
    for _, _, p in parks:
        for k in ("pos", "vel", "rot", "mode", "clock"):
            same = same and torch.equal(getattr(p, "_" + k)[..., :p.n], getattr(ragged, "_" + k)[..., at:at + p.n])
        at += p.n
    n = pk.n
    return {"episodes": episodes, "ships": n, "configurations": len(parks), "steps": steps,
            "plain_per_configuration": {"ms_per_step": ms_plain / steps, "ship_ticks_per_s": n * steps / (ms_plain / 1e3),
                                        "launches_per_step": 2 * len(parks)},
            "ragged_batch": {"ms_per_step": ms_ragged / steps, "ship_ticks_per_s": n * steps / (ms_ragged / 1e3),
                             "launches_per_step": 1},
            "speedup_ragged_vs_plain": ms_plain / ms_ragged, "bit_identical": bool(same),
            "note": "back-to-back steps on the device (no flush): the serving loop's tick without its host loop, "
                    "against the same episodes grouped by ship count, a plain-schedule park each"}


# Algorithmic bytes of one world-tick of the collision park (4 ships, 4 free spheres, 8 fixed spheres): a free ball
# reads 235 B (position, velocity, goto point 3 x 24; mode, mass, agility, speed fraction, max velocity, decay factor,
# radius, id, level 8 x 8; key, side 2 x 24; 5 flags) and writes 740 B (mLastG, mLastC, old position and velocity,
# position, velocity 6 x 24 plus the damped vertical velocity 8; the collision list 45 x 8 and its count 8, the impact
# record's slots 15 x 8 and its count 8, mLastCollision 8; level 8, key and side 2 x 24 when re-filed); a fixed ball
# is read as a candidate, 150 B (position, velocity, mLastG 3 x 24; decay factor, mass, agility, radius, id, level
# 6 x 8; key, side counted once with the free balls' 0; 5 flags, rounded up).
COLLIDE_BYTES_PER_WORLD_TICK = 8 * (235 + 740) + 8 * 150


def ragged_runs(args, dev) -> dict:
    """The ragged batch against the plain schedule on the same GPU: --ragged-worlds flight-mode worlds of 1-128 ships
    (log-uniform, the ragged benchmark's world sizes; workloads.ragged_flight_worlds), dynamical orientation on, packed
    with no padding. The same --ragged-steps ticks from the same state (saved and restored) through each schedule:
    plain (two launches, records in scratch), tiled (worlds packed greedily in row order, one tile a block) and listed
    worlds packed best fit (ebb_plan_worlds: any worlds in a tile, one tile a block), each tick timed with CUDA events
    after an L2 flush."""
    import torch

    from exact_ballpark_b200 import VecModesPark, tick_plain, tick_tiled, tick_worlds
    from exact_ballpark_b200.tiles import plan_best_fit, plan_tiles
    from exact_ballpark_b200.workloads import ragged_flight_worlds
    w = ragged_flight_worlds(31, args.ragged_worlds)
    n = len(w.rows)
    park = VecModesPark(n, device=dev, dynamical_orientation=True, use_new_orbit=True)
    w.packed().load(park)
    w.apply(park)
    for _ in range(args.warmup):
        tick_plain(park, 256)
    greedy = plan_tiles(park.world, cap=256, block=256)
    best = plan_best_fit(park.world, cap=256, block=256)
    saved = {k: getattr(park, k).clone() for k in park.row_tensors()}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    out = {"workload": f"ragged flight-mode batch: {args.ragged_worlds} worlds of 1-128 ships (log-uniform), {n} "
                       "ships, dynamical orientation on, new orbit law", "ships": n, "worlds": args.ragged_worlds,
           "steps": args.ragged_steps, "tiles_greedy": greedy.tiles, "tiles_best_fit": best.tiles}
    for name, run in (("plain", lambda: tick_plain(park, 256)), ("tiled_greedy", lambda: tick_tiled(park, greedy)),
                      ("worlds_best_fit", lambda: tick_worlds(park, None, best))):
        for k, v in saved.items():
            getattr(park, k).copy_(v)
        total = 0.0
        for _ in range(args.ragged_steps):
            flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            run()
            b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
        per = total / args.ragged_steps
        out[name] = {"ms_per_step": per, "value": n / (per / 1e3), "unit": "ship-ticks/s"}
    out["speedup_best_fit_vs_plain"] = out["plain"]["ms_per_step"] / out["worlds_best_fit"]["ms_per_step"]
    out["speedup_greedy_vs_plain"] = out["plain"]["ms_per_step"] / out["tiled_greedy"]["ms_per_step"]
    return out


def collide_runs(args, dev, statics: bool = False) -> dict:
    """The collision park (exact_ballpark_b200.collide, the gradient method on spheres) at the collision
    benchmark's shape: --collide-worlds worlds of 4 ships, 4 free spheres and 8 fixed spheres
    (workloads.collide_worlds: +-20 km, radii log-uniform 10 m - 5 km, ships GOTO at spheres, re-aimed every 25 ticks
    between timed ticks), warm-up ticks, then --collide-steps ticks each one CUDA-graph replay of the one-launch tick,
    timed with CUDA events (L2 flushed before each). Ship-ticks count the 4 ships a world, as the reference's
    collision benchmark does; world-ticks and ball-ticks beside them."""
    import torch

    from exact_ballpark_b200.collide import CollideGraph, VecCollidePark
    from exact_ballpark_b200.workloads import collide_statics_worlds, collide_worlds
    W = args.collide_worlds
    ticks = args.warmup + args.collide_steps
    if statics:
        w = collide_statics_worlds(22, W, ticks=ticks)
        park = VecCollidePark(W, 8, device=dev, statics=8)
        park.load(w.worlds, w.collidables)
    else:
        w = collide_worlds(21, W, ticks=ticks)
        park = VecCollidePark(W, 16, device=dev)
        park.load(w.worlds)
    graph = CollideGraph(park)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    total = 0.0
    contacts = 0
    for step in range(1, ticks + 1):
        w.apply(park, step)
        flush.fill_(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        graph.tick()
        b.record(stream)
        b.synchronize()
        if step > args.warmup:
            total += a.elapsed_time(b)
            contacts += int(park.hits_n.sum().item())
    park.check()
    per = total / args.collide_steps
    peak, kind = _peaks()
    achieved = COLLIDE_BYTES_PER_WORLD_TICK * W / (per / 1e3) / 1e9
    traffic = None
    tp = ROOT / "profiles" / "collide_tick_traffic.json"
    if tp.exists():
        try:
            traffic = float(json.loads(tp.read_text())["dram_bytes_per_world_tick"]) * W
        except Exception:
            traffic = None
    if statics:
        return {"workload": f"collision park with static collidables: {W} worlds x (4 ships + 4 fixed spheres + 4 "
                            "capsules + 4 oriented boxes), ships GOTO at them re-aimed every 25 ticks",
                "value": 4 * W / (per / 1e3), "unit": "ship-ticks/s", "world_ticks_per_s": W / (per / 1e3),
                "ms_per_step": per, "steps": args.collide_steps, "warmup": args.warmup,
                "contacts_per_tick": contacts / args.collide_steps,
                "reference_published": {"value": 54.3e6, "unit": "ship-ticks/s", "hardware": "GH200",
                                        "config": "contact_slots=8, ships=4, spheres=4, statics=8, kernel, 65,536 "
                                                  "worlds (docs/benchmarks.md)"}}
    return {"workload": f"collision park, gradient method on spheres: {W} worlds x (4 ships + 4 free spheres + 8 "
                        "fixed spheres), ships GOTO at spheres re-aimed every 25 ticks",
            "value": 4 * W / (per / 1e3), "unit": "ship-ticks/s", "world_ticks_per_s": W / (per / 1e3),
            "ball_ticks_per_s": 16 * W / (per / 1e3), "ms_per_step": per, "steps": args.collide_steps,
            "warmup": args.warmup, "contacts_per_tick": contacts / args.collide_steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": kind, "traffic": traffic,
                         "note": f"algorithmic {COLLIDE_BYTES_PER_WORLD_TICK} B/world-tick x {W} worlds over the "
                                 "tick's CUDA-event time; the tick is FP64 latency-bound (divides, square roots, "
                                 "the candidates' sort), not HBM-bound"},
            "reference_published": {"value": 141e6, "unit": "ship-ticks/s", "hardware": "GH200",
                                    "config": "ships=4, spheres=4, statics=0, kernel, 65,536 worlds "
                                              "(docs/benchmarks.md)"}}


# The combat park's algorithmic bytes a row-tick: the flight row's (BYTES_PER_SHIP_TICK) and the combat state it
# reads (exists 1, formation id 8, owner row 8, bubble 8, cloak 8) and writes (contacts 8, dispatch count 8, the
# self-collision byte 1)
COMBAT_BYTES_PER_ROW_TICK = BYTES_PER_SHIP_TICK + (1 + 8 + 8 + 8 + 8) + (8 + 8 + 1)
# The composed park's on top: the collision acceleration (24 written, 24 read by the commit), the filing (level and
# key, side 8 + 48 read; written again by the commit's re-filing: counted once) and the collision list's length
COMPOSED_EXTRA_BYTES_PER_ROW_TICK = 24 + 24 + 56 + 8


def combat_cpu_sample(worlds: int, warmup: int, steps: int, composed: bool = False) -> dict:
    """The CPU oracle of the combat park (oracle/combat_park.py, the C++ sequential tick) or of the composed park
    (oracle/composed_park.py: each massive ball's Gradient at its turn) on every host core, on `worlds` worlds of the
    benchmark's workload over `steps` ticks after `warmup`: ship-ticks/s."""
    from exact_ballpark_b200.workloads import combat_worlds, composed_worlds
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    if composed:
        from oracle.composed_park import OracleComposedPark as Park
        w = composed_worlds(41, worlds)
    else:
        from oracle.combat_park import OracleCombatPark as Park
        w = combat_worlds(31, worlds)
    p = Park(len(w.rows), dynamical_orientation=True, use_new_orbit=True)
    p.load(w.rows)
    w.apply(p)
    for _ in range(warmup):
        p.evolve(threads=threads)
    t0 = time.perf_counter()
    for _ in range(steps):
        p.evolve(threads=threads)
    dt = time.perf_counter() - t0
    shape = "6 ships + 1 sphere + 2 missiles (seed 41)" if composed else "4 ships + 4 missiles (seed 31)"
    return {"value": w.ships * worlds * steps / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{worlds} worlds x ({shape}), ticks {warmup + 1}..{warmup + steps} ({dt:.1f} s wall), C++ "
                      f"oracle (oracle/flight.cpp's {'composed' if composed else 'combat'} tick), {threads} threads "
                      "over disjoint worlds"}


def combat_runs(args, dev, composed: bool = False) -> dict:
    """The combat park (exact_ballpark_b200.combat) at the reference's combat benchmark shape, or the composed park
    (exact_ballpark_b200.composed, combat with collisions) at its composed benchmark shape: --combat-worlds worlds of
    4 ships and 4 missiles (workloads.combat_worlds: the ships following, orbiting or flying to points, half the
    worlds with a formation; each missile added at a random launcher and launched aimed and massive at another ship),
    or of 6 massive ships, 1 fixed sphere and 2 missiles within 5 km (workloads.composed_worlds); warm-up ticks, then
    --combat-steps ticks each one CUDA-graph replay of the tick, timed with CUDA events (L2 flushed before each).
    Ship-ticks count the ships (missiles and spheres excluded), as the reference's benchmarks do."""
    import torch

    from exact_ballpark_b200.combat import CombatGraph, VecCombatPark
    from exact_ballpark_b200.composed import VecComposedPark
    from exact_ballpark_b200.workloads import combat_worlds, composed_worlds
    W = args.combat_worlds
    w = composed_worlds(41, W) if composed else combat_worlds(31, W)
    n = len(w.rows)
    cls = VecComposedPark if composed else VecCombatPark
    park = cls(n, device=dev, dynamical_orientation=True, use_new_orbit=True, block=256)
    park.load(w.rows)
    w.apply(park)
    graph = CombatGraph(park)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    total, events, contacts = 0.0, 0, 0
    for step in range(1, args.warmup + args.combat_steps + 1):
        flush.fill_(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        graph.tick()
        b.record(stream)
        b.synchronize()
        if step > args.warmup:
            total += a.elapsed_time(b)
            events += len(park.events())
            contacts += int(park.hits_n.sum().item())
    park.check()
    per = total / args.combat_steps
    peak, kind = _peaks()
    row_bytes = COMBAT_BYTES_PER_ROW_TICK + (COMPOSED_EXTRA_BYTES_PER_ROW_TICK if composed else 0)
    achieved = row_bytes * n / (per / 1e3) / 1e9
    if composed:
        workload = (f"composed park: {W} worlds x (6 massive ships + 1 fixed sphere + 2 missiles launched aimed and "
                    "massive) within 5 km, the gradient method's collisions between every massive ball, ships follow / "
                    "orbit / goto, half the worlds with a formation, dynamical orientation on")
        published = {"value": 89e6, "unit": "ship-ticks/s", "hardware": "GH200",
                     "config": "do=1, missiles=2, ships=6, spheres=1, graph, 65,536 worlds (docs/benchmarks.md)"}
    else:
        workload = (f"combat park: {W} worlds x (4 ships + 4 missiles launched aimed and massive), ships follow / "
                    "orbit / goto, half the worlds with a formation, dynamical orientation on")
        published = {"value": 92.7e6, "unit": "ship-ticks/s", "hardware": "GH200",
                     "config": "do=1, missiles=4, ships=4, graph, 65,536 worlds (docs/benchmarks.md)"}
    out = {"workload": workload, "value": w.ships * W / (per / 1e3), "unit": "ship-ticks/s",
           "world_ticks_per_s": W / (per / 1e3), "row_ticks_per_s": n / (per / 1e3), "ms_per_step": per,
           "steps": args.combat_steps, "warmup": args.warmup, "events_per_tick": events / args.combat_steps,
           "contacts_per_tick": contacts / args.combat_steps,
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "peak_kind": kind, "traffic": None,
                        "note": f"algorithmic {row_bytes} B/row-tick x {n} rows over the tick's CUDA-event time (a "
                                "graph replay); issue- and latency-bound like the flight tick"},
           "reference_published": published}
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = combat_cpu_sample(256, 3, 20, composed)
    return out


def pipelined(dev, steps: int, send, run, fetch) -> float:
    """Milliseconds for `steps` end-to-end steps through the public API, double-buffered over two streams: step t+1's
    inputs are copied in and step t-1's results copied out on a copy stream while step t's tick runs. send(t, s)
    copies step t's inputs from pinned host memory into device slot s = t % 2 (on the copy stream); run(t, s) takes
    slot s into the tick, runs it and copies its results into device slot s (on the compute stream); fetch(t, s)
    copies result slot s to pinned host memory (on the copy stream). Every step still moves its own bytes each way;
    the CUDA events bracket all the steps, both streams joined at the end."""
    import torch
    comp = torch.cuda.current_stream(dev)
    side = torch.cuda.Stream(device=dev)
    sent = [torch.cuda.Event() for _ in range(2)]          # slot s's inputs are on the device
    taken = [torch.cuda.Event() for _ in range(2)]         # slot s's inputs are in the tick, slot s's results out
    fetched = [torch.cuda.Event() for _ in range(2)]       # slot s's results are on the host
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    start.record(comp)
    side.wait_stream(comp)
    with torch.cuda.stream(side):
        send(0, 0)
        sent[0].record(side)
    for t in range(steps):
        s = t % 2
        if t + 1 < steps:
            with torch.cuda.stream(side):
                if t >= 1:
                    side.wait_event(taken[1 - s])         # the tick of step t - 1 has its inputs
                send(t + 1, 1 - s)
                sent[1 - s].record(side)
        comp.wait_event(sent[s])
        if t >= 2:
            comp.wait_event(fetched[s])                   # step t - 2's results are on the host
        run(t, s)
        taken[s].record(comp)
        with torch.cuda.stream(side):
            side.wait_event(taken[s])
            fetch(t, s)
            fetched[s].record(side)
    comp.wait_stream(side)
    end.record(comp)
    end.synchronize()
    return start.elapsed_time(end)


# Algorithmic bytes of one world's pre-tick on the server kernel at the server benchmark's shape (4 piloted ships, the
# 8 pushes GotoDirection and SetSpeedFraction a ship): per queued call the pushed columns read (mask 1, ball, target,
# n, local flag 4 x 8, floats 32) and the outputs written (queued 1, row, target row, local 3 x 8, route 1) and read
# again by the history and the flags (34); per world the stamps (next stamp read and written, stamp and park time
# written, the first row's clock read: 40), the bubble update's park time (16) and the world's rows and ids (2 x 32);
# per ship the command fields (position read, goto point written 2 x 24; mode read and written 8; speed fraction read
# and written twice 12), the bubble update (interactive, exists, settled 3, cloaked 8, fresh, listed and settled
# written 3) and the route and flags (pilot 8, the two flags 2).
SERVER_BYTES_PER_WORLD_TICK = 8 * (1 + 32 + 32 + 26 + 34) + 40 + 16 + 64 + 4 * (48 + 8 + 12 + 14 + 10)
# (the dead-bubble test fused into the same launch reads interactive and exists again: L1 hits, not counted)


def server_worlds(W: int, seed: int = 7) -> list:
    """The server benchmark's worlds (benchmarks/server_speed.py's shape): W worlds of 4 ships near a centre, every ship
    interactive and piloted, at rest, speed fraction 1, seeded."""
    import random
    r = random.Random(seed)
    rows = []
    for i in range(W * 4):
        if i % 4 == 0:
            centre = [r.uniform(-1e5, 1e5) for _ in range(3)]
        rows.append({"id": i % 4 + 1, "world": i // 4, "time": 0, "mass": 10 ** r.uniform(6.0, 8.0),
                     "radius": r.uniform(20.0, 80.0), "max_vel": r.uniform(100.0, 400.0),
                     "pos": [c + r.uniform(-4e3, 4e3) for c in centre], "vel": [0.0, 0.0, 0.0],
                     "agility": r.uniform(0.3, 1.5), "speed_fraction": 1.0, "free": True, "massive": False,
                     "interactive": True, "cloaked": 0, "bubble": 0, "moribund": False})
    return rows


def server_pushes(W: int, dev) -> list:
    """Per ship k of a world: (kind, mask, ball id, floats) for GotoDirection and SetSpeedFraction, drawn once."""
    import torch
    gen = torch.Generator().manual_seed(11)
    out = []
    for k in range(4):
        d = torch.rand(W, 3, generator=gen, dtype=torch.float64) * 2 - 1
        sf = torch.rand(W, generator=gen, dtype=torch.float64)[:, None]
        mask = torch.ones(W, dtype=torch.bool, device=dev)
        ball = torch.full((W,), k + 1, dtype=torch.int64, device=dev)
        out += [("GotoDirection", mask, ball, d.to(dev)), ("SetSpeedFraction", mask, ball, sf.to(dev))]
    return out


def server_cpu_sample(worlds: int, warmup: int, steps: int) -> dict:
    """The server benchmark's ticks on the host: the C++ flight oracle's park (oracle/park.py, its tick on every core
    over disjoint worlds) with each tick's pilots' calls applied through its commands (GotoDirection and
    SetSpeedFraction for every ship, in queue order); the queue's bookkeeping and routing are index work the oracle
    leaves out. ship-ticks/s on `worlds` worlds."""
    import numpy as np

    from oracle.park import OraclePark
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    rows = server_worlds(worlds)
    park = OraclePark(len(rows))
    park.load(rows)
    pushes = server_pushes(worlds, "cpu")
    n = len(rows)
    calls = []
    for k in range(4):
        mask = np.zeros(n, dtype=bool)
        mask[k::4] = True
        d = pushes[2 * k][3].numpy()
        sf = pushes[2 * k + 1][3].numpy()[:, 0]
        dirs = np.zeros((n, 3))
        dirs[k::4] = d
        fr = np.zeros(n)
        fr[k::4] = sf
        calls.append((mask, dirs, fr))

    def tick():
        for mask, dirs, fr in calls:
            park.goto_direction(mask, dirs)
            park.set_speed_fraction(mask, fr)
        park.evolve(threads=threads)
    for _ in range(warmup):
        tick()
    t0 = time.perf_counter()
    for _ in range(steps):
        tick()
    dt = time.perf_counter() - t0
    return {"value": n * steps / dt, "unit": "ship-ticks/s", "cores": threads, "kind": "port",
            "sample": f"{worlds} worlds x 4 piloted ships, GotoDirection and SetSpeedFraction a ship a tick, "
                      f"{steps} ticks after {warmup} ({dt:.1f} s wall): the C++ flight oracle's park with the calls "
                      f"applied by its commands, its tick on {threads} threads over disjoint worlds"}


def space_runs(args, dev) -> dict:
    """The space layer (exact_ballpark_b200.space: filing, boxes, bubbles, dictionaries, dead rows, the tick's
    re-filings; one thread a world) over the flight park: --space-worlds worlds of 128 slots with ragged ship counts
    (log-uniform 1 to 128, the ragged benchmark's draw: ragged_flight_worlds, follow, orbit and warp, positions in a
    +-50 km cube a world), loaded and filed, then --space-steps ticks of VecSpace.tick after warm-up, each timed with
    CUDA events: the whole tick (DEAD, the park's tick with the dead rows skipped, AFTER_EVOLVE) and the layer's two
    launches alone; the worlds a full table flagged are counted. Not a headline line: the sensors are not in the layer
    yet."""
    import numpy as np
    import torch

    from exact_ballpark_b200 import VecModesPark
    from exact_ballpark_b200.modes import WARP
    from exact_ballpark_b200.space import VecSpace
    from exact_ballpark_b200.workloads import ragged_flight_worlds
    W, N = args.space_worlds, 128
    fw = ragged_flight_worlds(7, W, N)
    sizes = fw.sizes
    n = sum(sizes)
    park = VecModesPark(n, device=dev)
    park.load_columns(fw.packed().cols)
    fw.apply(park)
    slots = np.full((W, N), -1, dtype=np.int64)
    start = 0
    for w, k in enumerate(sizes):
        slots[w, :k] = np.arange(start, start + k)
        start += k
    space = VecSpace(park, slots, boxes=64 * N + 64, entries=16 * N + 64)   # warpers file far from their worlds
    space.load()
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        space.tick()
    ev = lambda: torch.cuda.Event(enable_timing=True)     # noqa: E731
    whole = layer = 0.0
    for _ in range(args.space_steps):
        e = [ev() for _ in range(6)]
        e[0].record(stream)
        dead = space.dead_rows()
        e[1].record(stream)
        warp_proper = ((park._mode == WARP) & (park._effect_stamp >= 0) & park._free & ~park._moribund & ~dead)
        saved = park._moribund.clone()
        park._moribund.logical_or_(dead)
        park.evolve()
        park._moribund.copy_(saved)
        dropped = warp_proper & (park._mode != WARP)
        e[2].record(stream)
        space.after_evolve(dropped)
        e[3].record(stream)
        e[3].synchronize()
        whole += e[0].elapsed_time(e[3])
        layer += e[0].elapsed_time(e[1]) + e[2].elapsed_time(e[3])
    K = args.space_steps
    return {"worlds": W, "slots": N, "ships": n, "steps": K, "ms_per_tick": whole / K,
            "layer_ms_per_tick": layer / K, "ship_ticks_per_s": n * K / (whole * 1e-3),
            "layer_share": layer / whole, "dead_rows_last": int(dead.sum()),
            "flagged_worlds": int((space.st["flags"] != 0).sum()), "boxes_max": int(space.st["box_n"].max())}


def partition_cpu_sample(pw, worlds: int, ticks: int, warm: int = 0) -> dict:
    """The space oracle (oracle/space.cpp: the master's partition, bubbles and sensors over the flight oracle's tick, a
    sequential C++ restatement of the reference's SpaceBallpark) on every host core, one world a task (ctypes releases
    the interpreter's lock): `worlds` worlds of the partition workload spread over its sizes, each loaded (AddBall,
    the sensors) and ticked `warm` times, then `ticks` ticks more, every ship sent to a goto point along its pilot's
    direction each tick; the timed ticks' time is the longer run's less the shorter's. The server layer is not in the
    oracle's tick."""
    from concurrent.futures import ThreadPoolExecutor

    import numpy as np

    import space_trace as sp_trace
    from oracle import space_world
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    pick = np.linspace(0, len(pw.sizes) - 1, worlds).astype(np.int64)
    c = pw.cols
    jobs = []
    for w in pick.tolist():
        s0, k = int(pw.starts[w]), int(pw.sizes[w])
        ops = [sp_trace._op(sp_trace.ADD, j + 1, c["mass"][s0 + j], c["radius"][s0 + j], c["max_vel"][s0 + j], 1.0,
                            1.0, *c["pos"][s0 + j], 0.0, 0.0, 0.0, c["agility"][s0 + j], 1.0, 0.0) for j in range(k)]
        ops += [sp_trace._op(sp_trace.SENSOR, j + 1, pw.sensor_range[s0 + j], 1.0, 0.0, 0.0) for j in range(k)]
        per_tick = [sp_trace._op(sp_trace.GOTO, j + 1, *(c["pos"][s0 + j] + pw.direction[s0 + j] * 1e9))
                    for j in range(k)] + [sp_trace._op(sp_trace.TICK)]
        jobs.append((np.array(ops + per_tick * warm), np.array(ops + per_tick * (warm + ticks)), w + 1))

    def timed(job, which):
        space_world.run_quiet(job[which], seed=job[2])
    with ThreadPoolExecutor(threads) as ex:
        t0 = time.perf_counter()
        list(ex.map(lambda j: timed(j, 0), jobs))
        t_short = time.perf_counter() - t0
        t0 = time.perf_counter()
        list(ex.map(lambda j: timed(j, 1), jobs))
        t_long = time.perf_counter() - t0
    ships = int(pw.sizes[pick].sum())
    dt = max(t_long - t_short, 1e-9)
    return {"value": ships * ticks / dt, "unit": UNIT, "cores": threads, "kind": "port", "seconds": dt,
            "sample": f"{worlds} of the {len(pw.sizes)} worlds ({ships} ships, sizes spread as the workload's), "
                      f"{ticks} ticks each after the load and {warm} ticks ({dt:.2f} s wall of timed ticks), the "
                      f"space oracle (oracle/space.cpp) over the flight oracle's tick, {threads} threads over "
                      "disjoint worlds, no server layer"}


def partition_runs(args, dev) -> dict:
    """The metric's workload: the partition worlds (exact_ballpark_b200.workloads.partition_worlds: --partition-worlds
    ragged worlds of 1 to 128 ships, log-uniform, in 1 to 5 Gaussian blobs, a sensor of 1 to 250 km on every ship)
    with bubbles, the partition and the proximity sensors, the server layer on top (every ship piloted: GotoDirection
    and SetSpeedFraction every tick). Two arrangements of the same worlds on the same GPU, each a captured tick
    replayed --partition-steps times after warm-up, timed with CUDA events (L2 flushed before each step):
    the ragged batch (the layer in size classes, worlds ordered by size; the park's tiled schedule) and the plain
    per-configuration kernels (one 128-slot layout in world order; the park's plain schedule). Both end in the same
    state, compared here bit for bit (the park's rows, each world's event count)."""
    import torch

    from exact_ballpark_b200.partition import partition_setup, tune_partition
    from exact_ballpark_b200.workloads import partition_worlds
    W, K = args.partition_worlds, args.partition_steps
    pw = partition_worlds(11, W)
    n = pw.n
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    out = {}
    runs = {}
    plan = None if args.no_partition_autotune else tune_partition(pw, dev)[0]
    for name, ragged in (("ragged", True), ("plain", False)):
        t0 = time.time()
        r = partition_setup(pw, dev, ragged, warp_class=args.partition_warp_class, plan=plan)
        setup_s = time.time() - t0
        g = r["graph"]
        for _ in range(args.warmup):
            g.tick()
        total = 0.0
        for _ in range(K):
            flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            g.tick()
            b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
        per = total / K
        part = r["part"]
        # one eager tick, each part timed alone: the server's pre-tick, the layers' dead-bubble tests, the park's tick,
        # each layer's re-filings and HandleProximities, the send flags
        parts_ms = {}
        park, srv, q = r["park"], r["server"], r["q"]

        def timed_part(name, fn):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            out_ = fn()
            b.record(stream)
            b.synchronize()
            parts_ms[name] = parts_ms.get(name, 0.0) + a.elapsed_time(b)
            return out_
        if srv is not None:
            timed_part("server_pre_tick", lambda: srv._launch(q, 5))
        dead = timed_part("dead_bubbles", part.dead_rows)
        saved = park._moribund.clone()
        park._moribund.logical_or_(dead)
        timed_part("park_tick", r["park_tick"])
        park._moribund.copy_(saved)
        for layer, _ in part.layers:
            layer.clear_events()
            timed_part(f"after_evolve_{layer.N}", lambda: layer.after_evolve(None))
        if srv is not None:
            timed_part("server_flags", lambda: srv._launch(q, 3))
        park.current_time += 1
        ev = part.event_counts()
        out[name] = {"ms_per_step": per, "ship_ticks_per_s": n / (per / 1e3), "world_ticks_per_s": W / (per / 1e3),
                     "eager_parts_ms": parts_ms,
                     "setup_s": setup_s, "layers": [[layer.N, layer.W] for layer, _ in part.layers],
                     "events_last_tick": int(ev.sum()), "flagged_worlds": int((part.flags() != 0).sum())}
        runs[name] = (r["park"], ev)
        if name == "ragged":
            keep = r
        else:
            del r, g, part
    pr, er = runs["ragged"]
    pp, ep = runs["plain"]
    same = all(torch.equal(getattr(pr, "_" + k), getattr(pp, "_" + k)) for k in ("pos", "vel", "mode", "clock"))
    out["bit_identical"] = bool(same and torch.equal(er, ep))
    out["speedup_ragged_vs_plain"] = out["plain"]["ms_per_step"] / out["ragged"]["ms_per_step"]
    out["workload"] = (f"partition worlds: {W} ragged worlds of 1-128 ships (log-uniform, mean {n / W:.1f}; {n} "
                       "ships) in 1-5 Gaussian blobs (sigma 10 km) a world, a proximity sensor of 1-250 km on every "
                       "ship (period 1 s), bubbles and the partition, the server layer on top (GotoDirection and "
                       "SetSpeedFraction for every ship every tick), dynamical orientation off")
    out["ships"], out["worlds"], out["steps"], out["warmup"] = n, W, K, args.warmup
    del keep
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = partition_cpu_sample(pw, min(W, 400), 5)
    return out


def server_runs(args, dev) -> dict:
    """The server layer (exact_ballpark_b200.server) over the flight park at the reference's server benchmark shape
    (benchmarks/server_speed.py): --server-worlds worlds of 4 ships, each flown by a pilot that sends GotoDirection
    and SetSpeedFraction every tick (8 Actions calls a world a tick, directions and speed fractions drawn once,
    seeded), the flight park without dynamical orientation; a ServerGraph (the server kernel's pre-tick with the
    dead-bubble test, the park's tick, the send flags) replayed --server-steps times after warm-up, timed with CUDA
    events (L2 flushed before each). Then the same three launches eagerly, each timed alone (the shares and the server
    kernel's roofline), and the end-to-end tick: the pushes' floats copied in from pinned host memory, the replay, the
    two send flags of every row copied back."""
    import torch

    from exact_ballpark_b200 import VecModesPark, server
    from exact_ballpark_b200.modes import tick as park_tick
    K, W = 4, args.server_worlds
    rows = server_worlds(W)
    n = len(rows)
    park = VecModesPark(n, device=dev)
    park.load(rows)
    srv = server.VecServer(server.ModesAdapter(park), [x["id"] - 1 for x in rows], kernel="cuda")
    srv.pre_tick()                                                   # the first tick (its additions) eagerly
    srv.evolve()
    srv.post_tick()
    sched = [k for _ in range(K) for k in ("GotoDirection", "SetSpeedFraction")]
    g = server.ServerGraph(srv, sched)
    for j, (kind, mask, ball, f) in enumerate(server_pushes(W, dev)):
        g.inputs[j]["mask"].copy_(mask)
        g.inputs[j]["ball"].copy_(ball)
        g.inputs[j]["f"][:, :f.shape[1]].copy_(f)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        g.tick()
    total = 0.0
    for _ in range(args.server_steps):
        flush.fill_(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        g.tick()
        b.record(stream)
        b.synchronize()
        total += a.elapsed_time(b)
    per = total / args.server_steps
    routed = int((g.out.route == server.BUBBLE).sum().item())
    flags = int(g.out.gets_bubble.sum().item())
    # the same four launches eagerly, each timed alone
    parts = {"pre_tick": lambda: srv._launch(g.q, 5), "park_tick": lambda: park_tick(park, park.block),
             "send_flags": lambda: srv._launch(g.q, 3)}
    times = {k: 0.0 for k in parts}
    for _ in range(args.server_steps):
        flush.fill_(1)
        for k, f in parts.items():
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            f()
            b.record(stream)
            b.synchronize()
            times[k] += a.elapsed_time(b)
        park.current_time += 1
    ms = {k: v / args.server_steps for k, v in times.items()}
    # end to end: the pushes' floats in from pinned host memory, the two flags of every row back, double-buffered
    f_host = torch.empty_like(g.q["f"], device="cpu").pin_memory()
    f_host.copy_(g.q["f"])
    f_slot = [torch.empty_like(g.q["f"]) for _ in range(2)]
    flags_slot = [torch.empty(2, n, dtype=torch.bool, device=dev) for _ in range(2)]
    flags_host = [torch.empty(2, n, dtype=torch.bool).pin_memory() for _ in range(2)]

    def send(t, s):
        f_slot[s].copy_(f_host, non_blocking=True)

    def run(t, s):
        g.q["f"].copy_(f_slot[s])
        out = g.tick()
        flags_slot[s][0].copy_(out.has_character)
        flags_slot[s][1].copy_(out.gets_bubble)

    def fetch(t, s):
        flags_host[s].copy_(flags_slot[s], non_blocking=True)

    pipelined(dev, args.warmup, send, run, fetch)
    e2e = pipelined(dev, args.server_steps, send, run, fetch) / args.server_steps
    srv.check()
    peak, kind = _peaks()
    achieved = SERVER_BYTES_PER_WORLD_TICK * W / (ms["pre_tick"] / 1e3) / 1e9
    return {"workload": (f"server layer over the flight park: {W} worlds x 4 piloted ships, 8 Actions calls a world a "
                         "tick (GotoDirection + SetSpeedFraction a ship), dynamical orientation off; ServerGraph "
                         "(server kernel pre-tick with the dead-bubble test, park tick, send flags)"),
            "value": n / (per / 1e3), "unit": "ship-ticks/s", "world_ticks_per_s": W / (per / 1e3),
            "ms_per_step": per, "steps": args.server_steps, "warmup": args.warmup,
            "launch_ms": ms, "launch_share": {k: v / sum(ms.values()) for k, v in ms.items()},
            "routed_to_bubble_last_tick": routed, "narrowcast_rows_last_tick": flags,
            "roofline": {"bound": "hbm", "kernel": "server_kernel (pre-tick and dead-bubble test, phase 5)",
                         "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": kind, "traffic": None,
                         "note": f"algorithmic {SERVER_BYTES_PER_WORLD_TICK} B/world x {W} worlds over the pre-tick "
                                 "launch's own CUDA-event time (eager, L2 flushed); one thread a world walking its "
                                 "queue: latency-bound"},
            "e2e": {"value": n / (e2e / 1e3), "unit": "ship-ticks/s", "ms_per_step": e2e,
                    "h2d_bytes_per_step": g.q["f"].numel() * 8, "d2h_bytes_per_step": 2 * n,
                    "pipeline": "double-buffered: step t+1's floats in and step t-1's flags out on a copy stream "
                                "during step t's tick; timed over all steps; inputs larger than L2, no flush"},
            "gpu_launches_per_step": 3,
            "reference_published": {"value": 716e6, "unit": "ship-ticks/s", "hardware": "GH200",
                                    "config": "layer=server, mode=server_k_graph, park=modes, 65,536 worlds x 4 "
                                              "(docs/benchmarks.md)"},
            **({} if args.no_cpu_baseline else {"cpu_baseline": server_cpu_sample(16384, 3, 100)})}


def ref_sm100_runs(args, dev) -> dict:
    """The Blackwell bar: the reference's own kernels, built for sm_100 by baseline/ref_sm100.py (the reference's
    build with its flags, sm_100 SASS alone, its PTX read-back not made), driven through the reference's own public
    API on this GPU beside this package's parks, on the same seeded workloads as the sections above: the flight park
    (ModesGraph), the collision park (its kernel, eager: the reference has no graph for it), the combat and composed
    parks (CombatGraph, ComposedGraph) and the server layer (ServerGraph). Per park: --warmup ticks, then
    --ref-steps ticks, this package's tick and the reference's alternating, each timed alone with CUDA events with L2
    flushed before it; after the same ticks both parks' states are compared bit for bit."""
    import torch

    sys.path.insert(0, str(ROOT / "baseline"))
    import ref_sm100
    why = ref_sm100.unavailable()
    if why is not None:
        return {"unavailable": why}
    ref_sm100.install()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    K = args.ref_steps

    def timed(step) -> float:
        flush.fill_(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        step()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b)

    def bits(t):
        t = torch.as_tensor(t).detach().contiguous()
        as_int = {torch.float64: torch.int64, torch.float32: torch.int32}.get(t.dtype)
        return t.view(as_int) if as_int is not None else t

    def race(ships: int, mine, theirs, names, prep=None) -> dict:
        """mine, theirs: (park, tick); prep(park, step) before each tick (step from 1)."""
        (pm, tm), (pr, tr) = mine, theirs
        ms_m = ms_r = 0.0
        for step in range(1, args.warmup + K + 1):
            if prep is not None:
                prep(pm, step)
                prep(pr, step)
            if step <= args.warmup:
                tm()
                tr()
            else:
                ms_m += timed(tm)
                ms_r += timed(tr)
        torch.cuda.synchronize(dev)
        diff = {}
        for nm in names:
            if not (hasattr(pm, nm) and hasattr(pr, nm)):
                continue
            a, b = bits(getattr(pm, nm)), bits(getattr(pr, nm))
            diff[nm] = int((a != b).sum().item()) if a.shape == b.shape else f"{tuple(a.shape)} vs {tuple(b.shape)}"
        ms_m, ms_r = ms_m / K, ms_r / K
        return {"ships": ships, "ms_per_step": ms_m, "ref_sm100_ms_per_step": ms_r,
                "ship_ticks_per_s": ships / (ms_m / 1e3), "ref_sm100_ship_ticks_per_s": ships / (ms_r / 1e3),
                "speedup": ms_r / ms_m, "ticks_compared": args.warmup + K, "bit_differences": diff,
                "bit_identical": all(v == 0 for v in diff.values())}

    def flight():
        from exact_ballpark import vec_modes as RM
        from exact_ballpark import vec_modes_cuda as RMC

        from exact_ballpark_b200 import ModesGraph, VecModesPark
        from exact_ballpark_b200.autotune import autotune
        from exact_ballpark_b200.workloads import flight_worlds
        w = flight_worlds(1, args.worlds, args.ships)
        n = len(w.rows)
        pm, pr = (cls(n, device=dev, dynamical_orientation=True, use_new_orbit=True)
                  for cls in (VecModesPark, RM.VecModesPark))
        for p in (pm, pr):
            p.load(w.rows)
            w.apply(p)
        autotune(pm)
        out = race(n, (pm, ModesGraph(pm).tick), (pr, RMC.ModesGraph(pr).tick),
                   ("pos", "vel", "rot", "ang_vel", "mode", "effect_stamp"))
        out["workload"] = f"flight park: {args.worlds} worlds x {args.ships} ships, dynamical orientation, new orbit"
        return out

    def collide():
        from exact_ballpark import vec_collide as RC

        from exact_ballpark_b200.collide import CollideGraph, VecCollidePark
        from exact_ballpark_b200.workloads import collide_worlds
        W = args.collide_worlds
        w = collide_worlds(21, W, ticks=args.warmup + K)
        pm, pr = VecCollidePark(W, 16, device=dev), RC.VecCollidePark(W, 16, device=dev, kernel="cuda")
        for p in (pm, pr):
            p.load(w.worlds)
        out = race(4 * W, (pm, CollideGraph(pm).tick), (pr, pr.evolve), ("pos", "vel"), prep=w.apply)
        out["workload"] = f"collision park: {W} worlds x (4 ships + 4 free + 8 fixed spheres)"
        return out

    def combat(composed: bool):
        from exact_ballpark import vec_combat as RB
        from exact_ballpark import vec_combat_cuda as RBC
        from exact_ballpark import vec_composed as RP
        from exact_ballpark import vec_composed_cuda as RPC

        from exact_ballpark_b200.combat import CombatGraph, VecCombatPark
        from exact_ballpark_b200.composed import VecComposedPark
        from exact_ballpark_b200.workloads import combat_worlds, composed_worlds
        W = args.combat_worlds
        w = composed_worlds(41, W) if composed else combat_worlds(31, W)
        n = len(w.rows)
        mine = (VecComposedPark if composed else VecCombatPark)(n, device=dev, dynamical_orientation=True,
                                                                 use_new_orbit=True, block=256)
        theirs = (RP.VecComposedPark if composed else RB.VecCombatPark)(n, device=dev, dynamical_orientation=True,
                                                                         use_new_orbit=True)
        for p in (mine, theirs):
            p.load(w.rows)
            w.apply(p)
        graph = (RPC.ComposedGraph if composed else RBC.CombatGraph)(theirs)
        out = race(w.ships * W, (mine, CombatGraph(mine).tick), (theirs, graph.tick),
                   ("pos", "vel", "rot", "mode", "exists"))
        out["workload"] = (f"{'composed' if composed else 'combat'} park: {W} worlds, "
                           f"{w.ships} ships a world (missiles{' and spheres' if composed else ''} not counted)")
        return out

    def server_layer():
        from exact_ballpark import vec_modes as RM
        from exact_ballpark import vec_server as RS

        from exact_ballpark_b200 import VecModesPark, server
        W = args.server_worlds
        rows = server_worlds(W)
        n = len(rows)
        sched = [k for _ in range(4) for k in ("GotoDirection", "SetSpeedFraction")]
        graphs = []
        for cls, mod in ((VecModesPark, server), (RM.VecModesPark, RS)):
            park = cls(n, device=dev)
            park.load(rows)
            srv = mod.VecServer(mod.ModesAdapter(park), [x["id"] - 1 for x in rows], kernel="cuda")
            srv.pre_tick()
            srv.evolve()
            srv.post_tick()
            g = mod.ServerGraph(srv, sched)
            for j, (kind, mask, ball, f) in enumerate(server_pushes(W, dev)):
                g.inputs[j]["mask"].copy_(mask)
                g.inputs[j]["ball"].copy_(ball)
                g.inputs[j]["f"][:, :f.shape[1]].copy_(f)
            graphs.append((park, g.tick))
        out = race(n, graphs[0], graphs[1], ("pos", "vel", "bubble"))
        out["workload"] = f"server layer over the flight park: {W} worlds x 4 pilots, 8 Actions calls a world a tick"
        return out

    def space_server():
        from exact_ballpark import vec_modes as RM
        from exact_ballpark import vec_server_space as RSS
        from exact_ballpark import vec_server_space_cuda as RSC
        from exact_ballpark import vec_space as RV

        from exact_ballpark_b200.partition import partition_setup, tune_partition
        from exact_ballpark_b200.workloads import face_worlds
        W, N = args.ref_space_worlds, 4
        fw = face_worlds(1, W)
        n = fw.n
        plan, tuning = tune_partition(fw, dev)                        # as the headline: measured on the workload
        mine = partition_setup(fw, dev, ragged=True, server_on=True, plan=plan)
        vec = ("pos", "vel")
        rows = [{k: (v[i].tolist() if k in vec else v[i].item()) for k, v in fw.cols.items()} for i in range(n)]
        park = RM.VecModesPark(n, device=dev)
        park.load(rows)
        del rows
        srv = RSC.CudaSpaceServer(RSS.SpaceModesAdapter(park), (fw.cols["id"] - 1).tolist())
        space = srv.space
        code = torch.full((W, N), RV.OP["ADD_SENSOR"], dtype=torch.int64, device=dev)
        f = torch.zeros(W, N, 4, dtype=torch.float64, device=dev)
        f[..., 0] = torch.as_tensor(fw.sensor_range, device=dev).reshape(W, N)
        f[..., 1] = 1.0
        space.tape(code, torch.arange(N, device=dev).expand(W, N).contiguous(), torch.zeros_like(code), f)
        srv.pre_tick()                                               # the first tick (its additions) eagerly
        srv.evolve()
        srv.post_tick()
        g = RSC.SpaceServerGraph(srv, [k for _ in range(N) for k in ("GotoDirection", "SetSpeedFraction")])
        direction = torch.as_tensor(fw.direction, device=dev).reshape(W, N, 3)
        speed = torch.as_tensor(fw.speed, device=dev).reshape(W, N)
        for k in range(N):
            for j, v in ((2 * k, direction[:, k]), (2 * k + 1, speed[:, k:k + 1])):
                g.inputs[j]["mask"].fill_(True)
                g.inputs[j]["ball"].fill_(k + 1)
                g.inputs[j]["f"][:, :v.shape[1]].copy_(v)
        # the reference's event list grows until its consumer clears it (vec_space.py: clear_events); cleared before
        # each of its ticks here, outside the timed region, so that both counts are the last tick's events
        out = race(n, (mine["park"], mine["graph"].tick), (park, g.tick), ("pos", "vel", "mode"),
                   prep=lambda p, step: space.clear_events() if p is park else None)
        out["plan"] = {str(k): list(v) for k, v in plan.items()}
        out["tuning_ms"] = {str(k): v for k, v in tuning.items()}
        ours_ev, theirs_ev = mine["part"].event_counts().to(torch.int64), space.st["evn"].to(torch.int64)
        out["event_counts_differ"] = int((ours_ev != theirs_ev).sum().item())
        out["events_last_tick"] = {"ours": int(ours_ev.sum().item()), "reference": int(theirs_ev.sum().item())}
        out["flagged_worlds_reference"] = int((space.st["flags"] != 0).sum().item())
        out["workload"] = (f"the reference's space benchmark shape with its server (benchmarks/space_speed.py "
                           f"build_server): {W} worlds x 4 piloted ships across a top box's face, a 5 km sensor on "
                           "every ship, GotoDirection and SetSpeedFraction every ship every tick; this package's "
                           "PartitionGraph against the reference's SpaceServerGraph (CudaSpaceServer)")
        return out

    out = {"library": "the reference's kernels, its build for sm_100 (baseline/ref_sm100.py)", "steps": K,
           "warmup": args.warmup, "l2": "flushed before every timed tick",
           "partition_worlds": "not run: the reference's partition layer takes at most 64 slots a world "
                               "(vec_space.py:131), and its fixed box table flags BOXES on worlds whose ships spread "
                               "over 1-5 blobs 1,000 km apart, so the headline's worlds of 1-128 ships are outside "
                               "its domain; the space_server line is its own benchmark's shape"}
    for name, fn in (("flight", flight), ("collide", collide), ("combat", lambda: combat(False)),
                     ("composed", lambda: combat(True)), ("server", server_layer), ("space_server", space_server)):
        try:
            out[name] = fn()
        except Exception as e:                                       # one park's failure is reported, not fatal
            out[name] = {"error": f"{type(e).__name__}: {e}"[:400]}
        torch.cuda.synchronize(dev)
        torch.cuda.empty_cache()
    return out


# Algorithmic bytes of one ship's tick in the partition layer's re-filings and HandleProximities (the layer's
# dominant launches): the ship's filing read and written (level, key, side, active neighbours, its box and top entries:
# 10 x 8 B each way), its position, velocity and old position read (72), its bubble and seq (16), its row, id, mode
# and the park's flags (8 + 8 + 4 + 4), radius and the flight values of the inflated radius (mass, decay factor,
# agility, speed fraction, max velocity: 8 + 8 + 4 x 4 + 4), its sensor's range, period and elapsed time (24, the
# elapsed time written back 8), its proximity flags (4), its sensor list's length and bucket count (8), and each
# candidate a sensing ship meets counted once for the world (its filing, position and radius: 96 + 24 + 4, in the
# ship's own share).
PARTITION_BYTES_PER_SHIP_TICK = 2 * 80 + 72 + 16 + 24 + 36 + 24 + 8 + 4 + 8 + 124


def partition_headline(args, dev, dist, rank: int, world_size: int, barrier, max_over_ranks) -> dict:
    """The metric's own line: the partition worlds (workloads.partition_worlds: --partition-worlds ragged worlds of
    1-128 ships a rank, sensors on every ship, bubbles and the partition, the server layer on top), the ragged batch's
    captured tick (the layer in size classes ordered by size, the large ones a warp a world; the park's tiled schedule)
    timed against the plain per-configuration layout's (one 128-slot layout in world order, a thread a world; the
    park's plain schedule) on the same GPU, both replayed K times after W warm-up ticks, CUDA events on the launching
    stream, L2 flushed before each step, max over ranks; both must end bit-identical. `e2e` runs the ragged tick
    through the public API from host buffers: every step each ship's pilot's GotoDirection and SetSpeedFraction
    arguments copied in from pinned memory and scattered into the server's queue, the tick, and every world's event
    count and every row's two send flags copied back, double-buffered over a copy stream."""
    import torch

    from exact_ballpark_b200.partition import partition_setup, tune_partition
    from exact_ballpark_b200.workloads import partition_worlds
    W, K = args.partition_worlds, args.steps
    pw = partition_worlds(11 + rank, W)
    n = pw.n
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def timed(step, k: int) -> float:
        total = 0.0
        for _ in range(k):
            flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step()
            b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
        return total

    out = {}
    plain = partition_setup(pw, dev, ragged=False)
    for _ in range(args.warmup):
        plain["graph"].tick()
    barrier()
    ms_plain = max_over_ranks(timed(plain["graph"].tick, K))
    plain_park, plain_ev = plain["park"], plain["part"].event_counts()
    plain_state = {k: getattr(plain_park, "_" + k).clone() for k in ("pos", "vel", "mode", "clock")}
    plain_layout = [[layer.N, layer.W, layer.lanes] for layer, _ in plain["part"].layers]
    del plain, plain_park
    torch.cuda.empty_cache()
    plan, tuning = None, None
    if not args.no_partition_autotune:                     # each size class's arrangement, measured (untimed)
        plan, tuning = tune_partition(pw, dev)
    r = partition_setup(pw, dev, ragged=True, warp_class=args.partition_warp_class, plan=plan)
    g, part, park = r["graph"], r["part"], r["park"]
    for _ in range(args.warmup):
        g.tick()
    barrier()
    with Clocks(dev.index or 0) as clk:
        barrier()
        ms_ragged = max_over_ranks(timed(g.tick, K))
        barrier()
    clocks = clk.summary()
    same = all(torch.equal(getattr(park, "_" + k), v) for k, v in plain_state.items())
    same = same and torch.equal(part.event_counts(), plain_ev)
    del plain_state
    # one more tick, eager, each part timed alone (L2 flushed before each): the server's pre-tick, the dead-bubble
    # tests, the park's tick, every layer's re-filings and HandleProximities (the dominant launches), the send flags
    launch_ms, parts_ms = {}, {}
    q, srv = r["q"], r["server"]

    def timed_part(name, fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.fill_(1)
        a.record(stream)
        res = fn()
        b.record(stream)
        b.synchronize()
        parts_ms[name] = a.elapsed_time(b)
        return res
    timed_part("server_pre_tick", lambda: srv._launch(q, 5))
    dead = timed_part("dead_bubbles", part.dead_rows)
    saved = park._moribund.clone()
    park._moribund.logical_or_(dead)
    timed_part("park_tick", r["park_tick"])
    park._moribund.copy_(saved)
    for layer, _ in part.layers:
        layer.clear_events()
        name = f"{layer.N}_slots_{'warp' if layer.lanes == 32 else 'thread'}"
        timed_part(name, lambda: layer.after_evolve(None))
        launch_ms[name] = parts_ms[name]
    timed_part("server_flags", lambda: srv._launch(q, 3))
    park.current_time += 1
    layer_ms = sum(launch_ms.values())
    # e2e: the pilots' arguments in, the events and send flags out
    sizes = torch.as_tensor(pw.sizes, device=dev)
    world = torch.repeat_interleave(torch.arange(W, device=dev), sizes)
    k_in = torch.arange(n, device=dev) - torch.repeat_interleave(torch.as_tensor(pw.starts, device=dev), sizes)
    at_dir, at_sf = (2 * k_in) * W + world, (2 * k_in + 1) * W + world
    qf = q["f"].view(-1, 4)
    cmd_host = torch.empty(n, 4, dtype=torch.float64, pin_memory=True)
    cmd_host[:, :3] = torch.from_numpy(pw.direction)
    cmd_host[:, 3] = torch.from_numpy(pw.speed)
    cmd_slot = [torch.empty(n, 4, dtype=torch.float64, device=dev) for _ in range(2)]
    res_slot = [torch.empty(W * 8 + 2 * n, dtype=torch.uint8, device=dev) for _ in range(2)]
    res_host = [torch.empty(W * 8 + 2 * n, dtype=torch.uint8, pin_memory=True) for _ in range(2)]

    def send(t, s_):
        cmd_slot[s_].copy_(cmd_host, non_blocking=True)

    def run(t, s_):
        qf[at_dir, :3] = cmd_slot[s_][:, :3]
        qf[at_sf, 0] = cmd_slot[s_][:, 3]
        g.tick()
        res_slot[s_][:W * 8].view(torch.int64).copy_(part.event_counts())
        res_slot[s_][W * 8:W * 8 + n].copy_(q["has_character"].view(torch.uint8))
        res_slot[s_][W * 8 + n:].copy_(q["gets_bubble"].view(torch.uint8))

    def fetch(t, s_):
        res_host[s_].copy_(res_slot[s_], non_blocking=True)

    pipelined(dev, 3, send, run, fetch)
    barrier()
    ms_e2e = max_over_ranks(pipelined(dev, K, send, run, fetch))
    total = n * world_size
    peak, peak_kind = _peaks()
    achieved = PARTITION_BYTES_PER_SHIP_TICK * n / (layer_ms / 1e3) / 1e9
    part.check()
    out.update({
        "value": total * K / (ms_ragged / 1e3), "ms_per_step": ms_ragged / K,
        "plain": {"value": total * K / (ms_plain / 1e3), "ms_per_step": ms_plain / K, "layout": plain_layout,
                  "schedule": "the plain per-configuration layout: one 128-slot layer, worlds in their order, a "
                              "thread a world; the park's plain schedule; the same server layer; one CUDA graph"},
        "speedup_ragged_vs_plain": ms_plain / ms_ragged, "bit_identical_ragged_vs_plain": bool(same),
        "ragged_layout": [[layer.N, layer.W, layer.lanes, layer.block] for layer, _ in part.layers],
        "autotune": None if tuning is None else {
            "plan": {str(c): {"lanes": l, "block": b} for c, (l, b) in plan.items()},
            "ms_a_class_a_tick": {f"lanes{l}_block{b}": {str(c): round(v, 3) for c, v in t.items()}
                                  for (l, b), t in tuning.items()},
            "note": "each size class's arrangement (a thread a world in 64- or 128-thread blocks, or a warp a world) "
                    "timed on the workload itself, eager, untimed in the headline; each class takes its fastest"},
        "layer_launch_ms": launch_ms, "layer_share": layer_ms / (ms_ragged / K), "eager_parts_ms": parts_ms,
        "roofline": {"bound": "hbm", "kernel": "the space layer's re-filings and HandleProximities (tape kernels, "
                                                "a launch a size class)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                     "peak_kind": peak_kind,
                     "note": f"algorithmic {PARTITION_BYTES_PER_SHIP_TICK} B/ship-tick x {n} ships over the layer "
                             "launches' summed CUDA-event time (eager, L2 flushed); a sequential program a world "
                             "(dependent loads through the box table and the unordered maps): latency-bound"},
        "e2e": {"value": total * K / (ms_e2e / 1e3), "unit": UNIT, "ms_per_step": ms_e2e / K,
                "h2d_bytes_per_step": n * 32, "d2h_bytes_per_step": W * 8 + 2 * n,
                "pipeline": "double-buffered: step t+1's pilots' arguments in and step t-1's event counts and send "
                            "flags out on a copy stream during step t's tick; timed over all steps; inputs larger "
                            "than L2, no flush"},
        "clocks": clocks, "ships_per_rank": n, "worlds_per_rank": W,
        "events_last_tick": int(part.event_counts().sum()), "flagged_worlds": int((part.flags() != 0).sum()),
        "gpu_launches": K * (2 + 3 + 2 * len(part.layers))})
    del r, g, part, park, q, srv
    torch.cuda.empty_cache()
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = partition_cpu_sample(pw, min(W, 20000), K, warm=args.warmup)
        out["compute"] = compute_roofline(op_counts("partition", 2000, 5), out["value"])
    return out


FP64_PEAK_TFLOPS = 37.0        # B200 FP64 (vector) nominal; no measured FP64 peak on this pool
FP32_PEAK_TFLOPS = 75.0        # B200 FP32 nominal


def compute_roofline(counts: dict | None, ship_ticks_per_s: float) -> dict | None:
    """The counted FLOPs per ship-tick as achieved rates against the FP64 and FP32 pipes' nominal peaks."""
    if not counts or "error" in counts:
        return counts
    out = dict(counts)
    for kind, peak in (("fp64", FP64_PEAK_TFLOPS), ("fp32", FP32_PEAK_TFLOPS)):
        gf = counts[kind + "_flops"] * ship_ticks_per_s / 1e9
        out[kind] = {"achieved": gf / 1e3, "peak": peak, "unit": "TFLOP/s", "frac": gf / 1e3 / peak,
                     "peak_kind": "nominal"}
    return out


def op_counts(workload: str, worlds: int, ticks: int) -> dict | None:
    """FLOPs per ship-tick of a workload, counted by the counting build in a process of its own
    (exact_ballpark_b200.opcount with EBB_COUNTING=1), or None when that build is missing."""
    if not (ROOT / "exact_ballpark_b200" / "libebb_count.so").exists():
        return None
    env = dict(os.environ, EBB_COUNTING="1")
    r = subprocess.run([sys.executable, "-m", "exact_ballpark_b200.opcount", workload, "--worlds", str(worlds),
                        "--ticks", str(ticks)], capture_output=True, text=True, env=env, cwd=str(ROOT), timeout=600)
    if r.returncode != 0:
        return {"error": r.stderr[-300:]}
    return json.loads(r.stdout.strip().splitlines()[-1])


def _config(args, schedule: str) -> dict:
    return {"workload": (f"flight-mode park, dynamical orientation on, new orbit law: {args.worlds} worlds x "
                         f"{args.ships} ships (follow / orbit / warp), per-rank"),
            "worlds_per_rank": args.worlds, "ships_per_world": args.ships, "schedule": schedule,
            "parallelism": f"replicas x{args.gpus}", "l2": "flushed between timed steps (256 MiB write, untimed)"}


def flight_runs(args, dev, rank: int, world_size: int, barrier, max_over_ranks) -> dict:
    """The flight-mode park's benchmark shape (config 0's distributions at --worlds worlds x --ships ships a rank,
    dynamical orientation on): the tiled schedule's CUDA graph (autotuned) against the plain schedule, CUDA events, L2
    flushed before each step, max over ranks; `e2e` through the public API (speed fractions in, positions out,
    double-buffered); the HBM roofline of the tiled launch and the FLOPs per ship-tick."""
    import torch

    from exact_ballpark_b200 import ModesGraph, VecModesPark, tick_plain
    from exact_ballpark_b200.autotune import autotune
    from exact_ballpark_b200.workloads import flight_worlds
    w = flight_worlds(rank + 1, args.worlds, args.ships)
    n = len(w.rows)
    park = VecModesPark(n, device=dev, dynamical_orientation=True, use_new_orbit=True)
    park.load(w.rows)
    w.apply(park)
    plain = VecModesPark(n, device=dev, dynamical_orientation=True, use_new_orbit=True)
    plain.load(w.rows)
    w.apply(plain)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def timed(step, k: int) -> float:
        total = 0.0
        for _ in range(k):
            flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step()
            b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
        return total

    for _ in range(args.warmup):                                     # warm-up ticks
        park.evolve()
        tick_plain(plain, 256)
        plain.current_time += 1
    tuning = autotune(park)                                          # the tiled plan, the park's state unchanged
    plan = park.plan
    graph = ModesGraph(park)
    barrier()
    with Clocks(dev.index or 0) as clk:
        barrier()
        ms_tiled = timed(graph.tick, args.flight_steps)
        barrier()
        ms_plain = timed(lambda: tick_plain(plain, 256), args.flight_steps)
        barrier()
    clocks = clk.summary()
    ms_tiled, ms_plain = max_over_ranks(ms_tiled), max_over_ranks(ms_plain)
    per_tiled, per_plain = ms_tiled / args.flight_steps, ms_plain / args.flight_steps

    # e2e through the public API from host buffers: each step's speed fractions in, each step's positions out,
    # double-buffered over a copy stream
    every = torch.ones(n, dtype=torch.bool, device=dev)
    sf_host = torch.empty(n, dtype=torch.float64, pin_memory=True)
    sf_host.copy_(park.speed_fraction.cpu())
    sf_slot = [torch.empty(n, dtype=torch.float64, device=dev) for _ in range(2)]
    pos_slot = [torch.empty(3, n, dtype=torch.float64, device=dev) for _ in range(2)]
    pos_host = [torch.empty(3, n, dtype=torch.float64, pin_memory=True) for _ in range(2)]

    def send(t, s):
        sf_slot[s].copy_(sf_host, non_blocking=True)

    def run(t, s):
        park.set_speed_fraction(every, sf_slot[s])
        graph.tick()
        pos_slot[s].copy_(park._pos)                                 # the positions as stored: x, y, z planes

    def fetch(t, s):
        pos_host[s].copy_(pos_slot[s], non_blocking=True)

    pipelined(dev, 3, send, run, fetch)
    barrier()
    ms_e2e = max_over_ranks(pipelined(dev, args.flight_steps, send, run, fetch))
    h2d, d2h = n * 8, n * 24

    total_ships = n * world_size
    value = total_ships * args.flight_steps / (ms_tiled / 1e3)
    peak, peak_kind = _peaks()
    achieved = BYTES_PER_SHIP_TICK * n / (per_tiled / 1e3) / 1e9
    traffic = None
    tp = ROOT / "profiles" / "flight_tiled_traffic.json"
    if tp.exists():
        try:
            t = json.loads(tp.read_text())
            traffic = float(t["dram_bytes_per_ship_tick"]) * n
        except Exception:
            traffic = None
    line = {"value": value, "unit": UNIT, "ms_per_step": per_tiled,
            "config": dict(_config(args, "tiled: worlds packed in tiles, one block a tile, records in shared memory, "
                                         "warp-cooperative torque searches, one launch, CUDA graph"),
                           plan={"tile_rows_max": plan.cap, "block": plan.block, "grid": plan.grid, "tiles": plan.tiles,
                                 "candidates_timed": len(tuning)}),
            "plain": {"value": total_ships * args.flight_steps / (ms_plain / 1e3), "ms_per_step": per_plain,
                      "schedule": "plain: records pass + tick, two launches, records in scratch, 256-thread blocks"},
            "speedup_tiled_vs_plain": per_plain / per_tiled,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "peak_kind": peak_kind,
                         "note": (f"algorithmic {BYTES_PER_SHIP_TICK} B/ship-tick x {n} ships per launch over the "
                                  "tiled launch's CUDA-event time; the tick is FP64/FP32 issue- and latency-bound "
                                  "(divides, square roots, libm, divergent torque searches), not HBM-bound")},
            "e2e": {"value": total_ships * args.flight_steps / (ms_e2e / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e / args.flight_steps,
                    "pipeline": "double-buffered: step t+1's speed fractions in and step t-1's positions out on a "
                                "copy stream during step t's tick (SetSpeedFraction, the graph's tick); timed over "
                                "all steps; the park's state (131 MB) larger than L2, no flush"},
            "gpu_launches": 3 * args.flight_steps, "clocks": clocks}
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sample(args.worlds, args.ships, args.warmup, args.flight_steps)
        line["compute"] = compute_roofline(op_counts("flight", 4096, 10), value)
    del graph
    return line


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10, help="timed steps of the headline (the partition worlds' tick)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--flight-steps", type=int, default=200, help="timed steps of the flight-mode section")
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--worlds", type=int, default=65536)
    ap.add_argument("--ships", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-collide", action="store_true")
    ap.add_argument("--no-ragged", action="store_true")
    ap.add_argument("--ragged-worlds", type=int, default=10000)
    ap.add_argument("--ragged-steps", type=int, default=30)
    ap.add_argument("--collide-worlds", type=int, default=65536)
    ap.add_argument("--collide-steps", type=int, default=50)
    ap.add_argument("--no-combat", action="store_true")
    ap.add_argument("--only", choices=("ragged", "collide", "collide_statics", "combat", "composed", "serve", "server",
                                       "space", "partition", "serve_configurations", "ref_sm100"),
                    default=None, help="run one section alone on one GPU and print it (for profiling); the default "
                                       "run prints the headline line with every section")
    ap.add_argument("--combat-worlds", type=int, default=65536)
    ap.add_argument("--combat-steps", type=int, default=50)
    ap.add_argument("--no-server", action="store_true")
    ap.add_argument("--no-ref-sm100", action="store_true",
                    help="skip the reference's own kernels (built for sm_100) timed beside this package's")
    ap.add_argument("--ref-steps", type=int, default=10, help="timed ticks a park of the ref_sm100 section")
    ap.add_argument("--ref-space-worlds", type=int, default=65536,
                    help="worlds of four ships of the ref_sm100 section's space-server line")
    ap.add_argument("--server-worlds", type=int, default=65536)
    ap.add_argument("--server-steps", type=int, default=100)
    ap.add_argument("--space-worlds", type=int, default=20000)
    ap.add_argument("--space-steps", type=int, default=5)
    ap.add_argument("--partition-worlds", type=int, default=100000)
    ap.add_argument("--partition-steps", type=int, default=10)
    ap.add_argument("--no-partition-autotune", action="store_true",
                    help="the ragged batch's arrangement from --partition-warp-class instead of measured per class")
    ap.add_argument("--partition-warp-class", type=int, default=32,
                    help="the ragged batch's size classes from this size up run a warp a world (129: none)")
    ap.add_argument("--serve-rate", type=float, default=2000.0)
    ap.add_argument("--serve-seconds", type=float, default=6.0)
    ap.add_argument("--serve-budget-gb", type=float, default=80.0)
    ap.add_argument("--serve-max-steps", type=int, default=20000)
    ap.add_argument("--serve-all", action="store_true")
    ap.add_argument("--serve-steps", type=int, default=3000)
    ap.add_argument("--serve-warmup", type=int, default=200)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if world_size > 1:
            import torch.distributed as dist
            dist.init_process_group("gloo", init_method="env://")
        run_reference(args, rank)
        if world_size > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch


    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if args.only is not None:
        run = {"ragged": lambda: ragged_runs(args, dev), "collide": lambda: collide_runs(args, dev),
               "collide_statics": lambda: collide_runs(args, dev, statics=True),
               "combat": lambda: combat_runs(args, dev), "composed": lambda: combat_runs(args, dev, composed=True),
               "serve": lambda: serve_runs(args, dev), "server": lambda: server_runs(args, dev),
               "serve_configurations": lambda: serve_configurations(dev),
               "space": lambda: space_runs(args, dev), "partition": lambda: partition_runs(args, dev),
               "ref_sm100": lambda: ref_sm100_runs(args, dev)}[args.only]
        print(json.dumps({"metric": METRIC, "section": args.only, args.only: run()}), flush=True)
        return
    dist = None
    if rank != 0 or world_size > 1:                                   # the sections' CPU baselines: rank 0 at N = 1
        args.no_cpu_baseline = True
    if world_size > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        return reduce_max(x, dist, dev)

    head = partition_headline(args, dev, dist, rank, world_size, barrier, max_over_ranks)
    rest = {k: v for k, v in head.items() if k not in ("value", "ms_per_step", "roofline", "e2e", "clocks",
                                                      "gpu_launches", "cpu_baseline", "compute")}
    line = {"metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world_size, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64/f32", "data": "synthetic (seeded)",
            "config": {"workload": (f"partition worlds (the metric's ragged batch): {args.partition_worlds} worlds a "
                                    "rank of 1-128 ships (log-uniform) in 1-5 Gaussian blobs (sigma 10 km), a "
                                    "proximity sensor of 1-250 km on every ship, bubbles and the spatial partition, "
                                    "the server layer on top (GotoDirection and SetSpeedFraction for every ship every "
                                    "tick), dynamical orientation off; the ragged persistent graph (size classes, "
                                    "the large ones a warp a world) against the plain per-configuration layout"),
                       "worlds_per_rank": args.partition_worlds, "ships_per_rank": head["ships_per_rank"],
                       "max_ships": 128, "parallelism": f"replicas x{world_size}",
                       "l2": "flushed between timed steps (256 MiB write, untimed)"},
            "roofline": head["roofline"], "e2e": head["e2e"], "gpu_launches": head["gpu_launches"],
            "clocks": head["clocks"], "partition": rest}
    if "cpu_baseline" in head:
        line["cpu_baseline"] = head["cpu_baseline"]
    if head.get("compute"):
        line["compute"] = head["compute"]
    line["flight"] = flight_runs(args, dev, rank, world_size, barrier, max_over_ranks)
    if not args.no_ragged:
        line["ragged"] = ragged_runs(args, dev)
    if not args.no_collide:
        line["collide"] = collide_runs(args, dev)
        line["collide_statics"] = collide_runs(args, dev, statics=True)
    if not args.no_combat:
        line["combat"] = combat_runs(args, dev)
        line["composed"] = combat_runs(args, dev, composed=True)
    if not args.no_server:
        line["server"] = server_runs(args, dev)
    if not args.no_ref_sm100 and world_size == 1:
        line["ref_sm100"] = ref_sm100_runs(args, dev)
    if not args.no_serve:
        line["serve"] = serve_runs(args, dev)
        line["serve"]["plain_ship_ticks_per_s"] = line["flight"]["plain"]["value"] / world_size
        line["serve"]["configurations"] = serve_configurations(dev)
    if dist is not None:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
