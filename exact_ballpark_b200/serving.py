"""The serving loop: continuous batching of flight-mode episodes on one GPU.

Episodes (one world each: its ships, their initial commands, and a length in ticks) arrive while others run. The
server keeps every live episode's state resident in one device park (`Server.park`, rows reserved up front from a
state budget in bytes, as a key-value cache is), admits waiting episodes first come first served as rows free up,
and ticks every live episode once a step in ONE launch of the listed-worlds tick (include/ebb.h:
ebb_flight_tick_worlds): the live episodes are a list of row runs anywhere in the park, packed into tiles of whole
worlds, so nothing is copied to close the holes that finished episodes leave.

A step:
1. the episodes staged in the previous step are moved into their rows (ebb_flight_move, one launch);
2. the tile plan of the live episodes is uploaded (only when the set changed) and the tick launched;
3. while the tick runs: the episodes that have had all their ticks are moved out behind it (their final state,
   `results`) and their rows freed; the arrivals are queued, and the waiting episodes that now find rows are staged on
   a side stream: a staging park of their rows, loaded and commanded through the park API exactly as each episode
   alone would be (a park's load and commands act on each world's own rows), to be moved in by the next step.
The step ends when its tick is complete on the device: its latency is the host's wall time from the step's start to
then, and the loop reports p50/p99 over the steps with ship-ticks/s.

Each episode's result is the same, bit for bit, as the episode run alone: the tick computes every world from its own
rows only, each row keeps its own clock, and staging and moves copy state exactly. tests/test_serving.py checks it
against the park and against the oracle.
"""

from __future__ import annotations

import bisect
import ctypes
import math
import random
import statistics
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native
from .modes import _STATE_FIELD, _STORAGE, VecModesPark
from .workloads import FlightWorlds, flight_worlds, ragged_ships

STATE_BYTES_PER_ROW = sum((8 if dt in (torch.float64, torch.int64) else 4 if dt in (torch.float32, torch.int32) else 1)
                          * max(planes, 1) for _, dt, planes in _STORAGE)
# The resident park also keeps four int64 columns a row for the park API's guards (world, cloaked, bubble, refiled)
ROW_BYTES = STATE_BYTES_PER_ROW + 4 * 8


@dataclass
class Episode:
    eid: int
    world: FlightWorlds        # one world: its rows (ids, clock 0) and its initial commands
    ticks: int                 # ticks it runs
    arrival: float = 0.0       # seconds after the loop's start

    @property
    def ships(self) -> int:
        return len(self.world.rows)


def episode_stream(seed: int, count: int, rate: float = 2000.0, max_ships: int = 256, min_ticks: int = 10,
                   max_ticks: int = 10000) -> list:
    """`count` episodes arriving as a Poisson process of `rate` a second: ship counts log-uniform in [1, max_ships],
    lengths log-uniform in [min_ticks, max_ticks] ticks, each world drawn by workloads.flight_worlds from its own seed
    (follow / orbit / warp ships)."""
    r = random.Random(seed)
    t = 0.0
    out = []
    for e in range(count):
        t += r.expovariate(rate) if rate > 0 else 0.0
        ships = ragged_ships(r, max_ships)
        ticks = max(min_ticks, min(max_ticks, int(10.0 ** r.uniform(math.log10(min_ticks), math.log10(max_ticks)))))
        out.append(Episode(e, flight_worlds(seed * 1_000_033 + e, 1, ships), ticks, t))
    return out


class RowSpace:
    """First-fit allocation of row runs in [0, capacity), free runs kept sorted and merged."""

    def __init__(self, capacity: int):
        self.capacity = int(capacity)
        self.starts = [0] if capacity else []
        self.lens = [self.capacity] if capacity else []
        self.used = 0

    def alloc(self, n: int) -> int | None:
        for k, ln in enumerate(self.lens):
            if ln >= n:
                start = self.starts[k]
                if ln == n:
                    del self.starts[k], self.lens[k]
                else:
                    self.starts[k] += n
                    self.lens[k] -= n
                self.used += n
                return start
        return None

    def free(self, start: int, n: int) -> None:
        k = bisect.bisect_left(self.starts, start)
        if k > 0 and self.starts[k - 1] + self.lens[k - 1] > start:
            raise ValueError(f"rows {start}..{start + n} are already free")
        if k < len(self.starts) and start + n > self.starts[k]:
            raise ValueError(f"rows {start}..{start + n} overlap a free run")
        self.starts.insert(k, start)
        self.lens.insert(k, n)
        if k + 1 < len(self.starts) and self.starts[k] + self.lens[k] == self.starts[k + 1]:
            self.lens[k] += self.lens[k + 1]
            del self.starts[k + 1], self.lens[k + 1]
        if k > 0 and self.starts[k - 1] + self.lens[k - 1] == self.starts[k]:
            self.lens[k - 1] += self.lens[k]
            del self.starts[k], self.lens[k]
        self.used -= n


class Rows:
    """Rows of park state in the park's device layout with no park behind them (finished episodes' final states): the
    storage tensors `_<name>`, `field()` in the reference layout, and `state()` for the native calls."""

    def __init__(self, n: int, like: VecModesPark):
        self.n, self.dev = int(n), like.dev
        for name, dt, planes in _STORAGE:
            setattr(self, "_" + name, torch.empty((planes, n) if planes else (n,), dtype=dt, device=like.dev))
        self._like = like
        self._state = None

    def state(self) -> _native.FlightState:
        if self._state is None:
            s = _native.FlightState()
            lk = self._like.state()
            s.n, s.friction, s.dt, s.ffriction, s.fdt = self.n, lk.friction, lk.dt, lk.ffriction, lk.fdt
            s.new_orbit, s.dynamical = lk.new_orbit, lk.dynamical
            for name, _, _ in _STORAGE:
                setattr(s, _STATE_FIELD.get(name, name), getattr(self, "_" + name).data_ptr())
            self._state = s
        return self._state

    def field(self, name: str, start: int = 0, n: int | None = None) -> torch.Tensor:
        """A field of rows [start, start + n) in the reference layout ([n, k] or [n])."""
        n = self.n - start if n is None else n
        t = getattr(self, "_" + name)
        return (t[:, start:start + n].t() if t.dim() == 2 else t[start:start + n])


def move_rows(dst, src, src_rows: torch.Tensor, dst_rows: torch.Tensor, status: torch.Tensor, stream: int) -> None:
    """Every field of src's rows src_rows into dst's rows dst_rows (ebb_flight_move), on `stream`."""
    m = int(src_rows.numel())
    if m == 0:
        return
    rc = _native.lib().ebb_flight_move(ctypes.byref(dst.state()), ctypes.byref(src.state()), src_rows.data_ptr(),
                                       dst_rows.data_ptr(), m, status.data_ptr(), stream, 256)
    _native.check(rc, "ebb_flight_move")


def plan_worlds(starts: np.ndarray, lens: np.ndarray, tile_cap: int) -> tuple:
    """The tile plan of the listed-worlds tick for worlds at rows [starts[k], starts[k] + lens[k]): the worlds in row
    order, binned by their cumulative rows so that no tile exceeds tile_cap rows (a bin of tile_cap - max + 1 rows
    can end in a world of `max` rows). Returns (worlds [2E] int64, tile_worlds [T + 1] int64)."""
    order = np.argsort(starts, kind="stable")
    st, ln = starts[order], lens[order]
    worlds = np.empty(2 * len(st), dtype=np.int64)
    worlds[0::2] = st
    worlds[1::2] = st + ln
    if len(st) == 0:
        return worlds, np.zeros(1, dtype=np.int64)
    biggest = int(ln.max())
    if biggest > tile_cap:
        raise ValueError(f"a world of {biggest} rows does not fit a tile of {tile_cap}")
    span = tile_cap - biggest + 1
    cum = np.concatenate(([0], np.cumsum(ln)[:-1]))
    tile = cum // span
    cuts = np.flatnonzero(np.diff(tile)) + 1
    tile_worlds = np.concatenate(([0], cuts, [len(st)])).astype(np.int64)
    return worlds, tile_worlds


@dataclass
class Live:
    episode: Episode
    start: int
    last_step: int             # the step whose tick is its last


class LiveTable:
    """The live episodes' row runs as numpy columns (swap-removal), for a vectorised tile plan."""

    def __init__(self):
        self.eid = np.zeros(64, dtype=np.int64)
        self.start = np.zeros(64, dtype=np.int64)
        self.len = np.zeros(64, dtype=np.int64)
        self.count = 0
        self.where: dict = {}

    def add(self, eid: int, start: int, n: int) -> None:
        if self.count == len(self.eid):
            for k in ("eid", "start", "len"):
                a = getattr(self, k)
                setattr(self, k, np.concatenate([a, np.zeros_like(a)]))
        k = self.count
        self.eid[k], self.start[k], self.len[k] = eid, start, n
        self.where[eid] = k
        self.count += 1

    def remove(self, eid: int) -> None:
        k = self.where.pop(eid)
        last = self.count - 1
        if k != last:
            self.eid[k], self.start[k], self.len[k] = self.eid[last], self.start[last], self.len[last]
            self.where[int(self.eid[k])] = k
        self.count = last


@dataclass
class Result:
    eid: int
    rows: Rows
    start: int
    n: int
    ticks: int

    def field(self, name: str) -> torch.Tensor:
        return self.rows.field(name, self.start, self.n)


@dataclass
class StepStats:
    latency_ms: list = field(default_factory=list)     # host wall time from a step's start to its tick's completion
    rows: list = field(default_factory=list)           # ship-ticks of each step
    admitted: int = 0
    retired: int = 0
    wall_s: float = 0.0

    def summary(self) -> dict:
        lat = sorted(self.latency_ms)
        q = lambda p: lat[min(len(lat) - 1, int(math.ceil(p * len(lat))) - 1)] if lat else float("nan")
        total = sum(self.rows)
        return {"steps": len(lat), "p50_ms": q(0.50), "p99_ms": q(0.99), "mean_ms": statistics.fmean(lat) if lat
                else float("nan"), "ship_ticks": total, "ship_ticks_per_s": total / self.wall_s if self.wall_s else
                float("nan"), "admitted": self.admitted, "retired": self.retired}


class Server:
    """The continuous-batching loop (module docstring). `budget_bytes` of device state caps the resident rows
    (ROW_BYTES a row; `rows` overrides it); `tile_cap` rows a tile of the listed-worlds tick, the largest episode at
    most; `keep` keeps each finished episode's final state in `results`."""

    def __init__(self, budget_bytes: float = 80e9, rows: int | None = None, dynamical: bool = True,
                 new_orbit: bool = True, tile_cap: int = 512, block: int = 256, grid: int | None = None,
                 device="cuda", keep: bool = True, max_ships: int = 256):
        capacity = int(rows) if rows is not None else int(budget_bytes // ROW_BYTES)
        if capacity <= 0:
            raise ValueError("the state budget holds no row")
        if max_ships > tile_cap:
            raise ValueError("an episode must fit one tile")
        self.park = VecModesPark(capacity, device=device, dynamical_orientation=dynamical, use_new_orbit=new_orbit)
        self.dev = self.park.dev
        self.capacity = capacity
        self.space = RowSpace(capacity)
        self.waiting: deque = deque()
        self.live: dict = {}
        self.results: dict = {}
        self.keep = keep
        self.max_ships = max_ships
        self.tile_cap, self.block = int(tile_cap), int(block)
        self.grid = grid
        self.status = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.side = torch.cuda.Stream(device=self.dev)
        self.staged = None                       # (staging park, src rows, dst rows, event, [(episode, start)])
        self._plan = None                        # (worlds, tile_worlds, tiles) on the device
        self._dirty = True
        self.table = LiveTable()
        self.ends: dict = {}                     # step -> eids whose last tick it is
        self.live_rows = 0
        self.step_no = 0
        self.stats = StepStats()
        self.done_event = torch.cuda.Event()
        self.sm = torch.cuda.get_device_properties(self.dev).multi_processor_count

    # ---- requests ----
    def submit(self, episode: Episode) -> None:
        if episode.ships > self.max_ships:
            raise ValueError(f"episode {episode.eid}: {episode.ships} ships, more than {self.max_ships}")
        self.waiting.append(episode)

    def _stage(self) -> None:
        """Admit waiting episodes first come first served while rows are free, and stage them on the side stream."""
        batch = []
        while self.waiting:
            ep = self.waiting[0]
            start = self.space.alloc(ep.ships)
            if start is None:
                break
            self.waiting.popleft()
            batch.append((ep, start))
        if not batch:
            return
        fw = FlightWorlds.concat([ep.world for ep, _ in batch])
        with torch.cuda.stream(self.side):        # staging touches no resident row: it overlaps the tick
            stage = VecModesPark(len(fw.rows), device=self.dev, dynamical_orientation=self.park.dynamical_orientation,
                                 use_new_orbit=self.park.use_new_orbit)
            stage.load(fw.rows)
            fw.apply(stage)
            dst = np.concatenate([np.arange(s, s + ep.ships, dtype=np.int64) for ep, s in batch])
            src_rows = torch.arange(len(fw.rows), dtype=torch.int64, device=self.dev)
            dst_rows = torch.from_numpy(dst).pin_memory().to(self.dev, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.side)
        self.staged = (stage, src_rows, dst_rows, ev, batch)

    def _move_in(self) -> None:
        if self.staged is None:
            return
        stage, src_rows, dst_rows, ev, batch = self.staged
        main = torch.cuda.current_stream(self.dev)
        main.wait_event(ev)
        for t in (src_rows, dst_rows):
            t.record_stream(main)
        for name, _, _ in _STORAGE:
            getattr(stage, "_" + name).record_stream(main)
        move_rows(self.park, stage, src_rows, dst_rows, self.status, main.cuda_stream)
        for ep, start in batch:
            last = self.step_no + ep.ticks - 1
            self.live[ep.eid] = Live(ep, start, last)
            self.ends.setdefault(last, []).append(ep.eid)
            self.table.add(ep.eid, start, ep.ships)
            self.live_rows += ep.ships
        self.stats.admitted += len(batch)
        self.staged = None
        self._dirty = True

    def _upload_plan(self) -> None:
        if not self._dirty:
            return
        c = self.table.count
        worlds, tile_worlds = plan_worlds(self.table.start[:c], self.table.len[:c], self.tile_cap)
        up = lambda a: torch.from_numpy(a).pin_memory().to(self.dev, non_blocking=True)
        self._plan = (up(worlds), up(tile_worlds), len(tile_worlds) - 1)
        self._dirty = False

    def _tick(self) -> int:
        worlds, tile_worlds, tiles = self._plan
        if tiles <= 0:
            return 0
        grid = tiles if self.grid is None else min(tiles, self.grid)
        rc = _native.lib().ebb_flight_tick_worlds(
            ctypes.byref(self.park.state()), worlds.data_ptr(), tile_worlds.data_ptr(), tiles, self.tile_cap, None,
            self.status.data_ptr(), torch.cuda.current_stream(self.dev).cuda_stream, self.block, grid)
        _native.check(rc, "ebb_flight_tick_worlds")
        return self.live_rows

    def _retire(self) -> None:
        done = [self.live[e] for e in self.ends.pop(self.step_no, ())]
        if not done:
            return
        main = torch.cuda.current_stream(self.dev)
        total = sum(lv.episode.ships for lv in done)
        if self.keep:
            out = Rows(total, self.park)
            src = np.concatenate([np.arange(lv.start, lv.start + lv.episode.ships, dtype=np.int64) for lv in done])
            src_rows = torch.from_numpy(src).pin_memory().to(self.dev, non_blocking=True)
            dst_rows = torch.arange(total, dtype=torch.int64, device=self.dev)
            move_rows(out, self.park, src_rows, dst_rows, self.status, main.cuda_stream)
            off = 0
            for lv in done:
                self.results[lv.episode.eid] = Result(lv.episode.eid, out, off, lv.episode.ships, lv.episode.ticks)
                off += lv.episode.ships
        for lv in done:
            del self.live[lv.episode.eid]
            self.table.remove(lv.episode.eid)
            self.space.free(lv.start, lv.episode.ships)
            self.live_rows -= lv.episode.ships
        self.stats.retired += len(done)
        self._dirty = True

    # ---- the loop ----
    def step(self, arrivals=()) -> int:
        """One step (module docstring); returns the ship-ticks it ran. `arrivals` are submitted first."""
        t0 = time.perf_counter()
        with torch.cuda.device(self.dev):
            self._move_in()
            self._upload_plan()
            ran = self._tick()
            for ep in arrivals:
                self.submit(ep)
            self._retire()
            self._stage()
            self.done_event.record(torch.cuda.current_stream(self.dev))
            self.done_event.synchronize()
        self.stats.latency_ms.append((time.perf_counter() - t0) * 1e3)
        self.stats.rows.append(ran)
        self.step_no += 1
        return ran

    def idle(self) -> bool:
        return not self.live and not self.waiting and self.staged is None

    def check(self) -> None:
        """The device's status bits (a follow pointer leaving its world, a malformed tile, a bad move) as an error."""
        st = int(self.status.item())
        if st:
            raise RuntimeError(f"serving status {st:#x}: 1 a target outside its world, 2 a malformed tile, "
                               "4 a row or pointer outside a park in a move")


def serve(server: Server, episodes: list, realtime: bool = True, max_steps: int | None = None) -> dict:
    """Run `episodes` through `server` until every one has finished (or max_steps): with `realtime`, each arrives at
    its `arrival` second of wall time after the start (an open loop); otherwise all wait from the start (a saturated,
    closed loop). Returns the step statistics' summary."""
    pending = deque(sorted(episodes, key=lambda e: e.arrival)) if realtime else deque()
    if not realtime:
        for ep in episodes:
            server.submit(ep)
    t0 = time.perf_counter()
    steps = 0
    while pending or not server.idle():
        now = time.perf_counter() - t0
        arrivals = []
        while pending and pending[0].arrival <= now:
            arrivals.append(pending.popleft())
        if server.idle() and not arrivals and pending:
            time.sleep(max(0.0, min(pending[0].arrival - now, 0.001)))
            continue
        server.step(arrivals)
        steps += 1
        if max_steps is not None and steps >= max_steps:
            break
    server.stats.wall_s += time.perf_counter() - t0
    server.check()
    return server.stats.summary()
