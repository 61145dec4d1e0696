"""The serving loop: continuous batching of flight-mode episodes on one GPU.

Episodes (one world each: its ships, their initial commands, and a length in ticks) arrive while others run. The
server keeps every live episode's state resident in one device park (`Server.park`, rows reserved up front from a
state budget in bytes, as a key-value cache is), admits waiting episodes first come first served as rows free up,
and ticks every live episode once a step in ONE launch of the listed-worlds tick (include/ebb.h:
ebb_flight_tick_worlds): the live episodes are a list of row runs anywhere in the park, packed into tiles of whole
worlds, so nothing is copied to close the holes that finished episodes leave.

Staging runs on a thread of its own and a side stream: each batch of submitted episodes becomes a staging park of
their rows, loaded and commanded through the park API exactly as each episode alone would be (a park's load and
commands act on each world's own rows), while the GPU ticks. A step then:
1. admits staged episodes first come first served into free rows (ebb_flight_move, one launch a staged batch);
2. uploads the tile plan of the live episodes (when the set changed; ebb_plan_worlds packs them) and launches the
   tick;
3. moves out, behind the tick, the episodes that have had all their ticks (their final state, `results`) and frees
   their rows for the next step's admissions.
The step ends when its tick is complete on the device: its latency is the host's wall time from the step's start to
then, and the loop reports p50/p99 over the steps with ship-ticks/s.

Each episode's result is the same, bit for bit, as the episode run alone: the tick computes every world from its own
rows only, each row keeps its own clock, and staging and moves copy state exactly. tests/test_gpu_serving.py checks
it against the park and against the oracle.
"""

from __future__ import annotations

import bisect
import ctypes
import math
import random
import statistics
import sys
import threading
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native
from .modes import _STATE_FIELD, _STORAGE, VecModesPark
from .workloads import FlightWorlds, PackedWorlds, flight_worlds, ragged_ships

STATE_BYTES_PER_ROW = sum((8 if dt in (torch.float64, torch.int64) else 4 if dt in (torch.float32, torch.int32) else 1)
                          * max(planes, 1) for _, dt, planes in _STORAGE)
# How long the staging thread may hold the interpreter while the loop waits for it (Python's default is 5 ms)
SWITCH_INTERVAL_S = 2e-4
# The resident park also keeps four int64 columns a row for the park API's guards (world, cloaked, bubble, refiled)
ROW_BYTES = STATE_BYTES_PER_ROW + 4 * 8


@dataclass
class Episode:
    eid: int
    world: FlightWorlds        # one world: its rows (ids, clock 0) and its initial commands (`packed()` columns)
    ticks: int                 # ticks it runs
    arrival: float = 0.0       # seconds after the loop's start

    @property
    def ships(self) -> int:
        return len(self.world.rows)


def episode_stream(seed: int, count: int, rate: float = 2000.0, max_ships: int = 256, min_ticks: int = 10,
                   max_ticks: int = 10000, min_ships: int = 1) -> list:
    """`count` episodes arriving as a Poisson process of `rate` a second: ship counts log-uniform in [1, max_ships]
    (redrawn up to min_ships when a floor is given: uniform in [min_ships, max_ships]), lengths log-uniform in
    [min_ticks, max_ticks] ticks, each world drawn by workloads.flight_worlds from its own seed (follow / orbit / warp
    ships)."""
    r = random.Random(seed)
    t = 0.0
    out = []
    for e in range(count):
        t += r.expovariate(rate) if rate > 0 else 0.0
        ships = ragged_ships(r, max_ships) if min_ships <= 1 else r.randint(min_ships, max_ships)
        ticks = max(min_ticks, min(max_ticks, int(10.0 ** r.uniform(math.log10(min_ticks), math.log10(max_ticks)))))
        world = flight_worlds(seed * 1_000_033 + e, 1, ships)
        world.packed()                           # the request in columns, made by the client before it arrives
        out.append(Episode(e, world, ticks, t))
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


class Uploads:
    """int64 arrays copied host to device without an allocation a copy: two pinned host buffers used in turn (each
    reused only after the event of its previous copy) and one device buffer, both grown when an array outgrows them.
    Copies run on the given stream, so a device buffer is rewritten only after the work queued before it."""

    def __init__(self, dev, capacity: int = 4096):
        self.dev = dev
        self._grow(capacity)

    def _grow(self, capacity: int) -> None:
        self.capacity = int(capacity)
        self.host = [torch.empty(self.capacity, dtype=torch.int64, pin_memory=True) for _ in range(2)]
        self.views = [h.numpy() for h in self.host]
        self.done = [None, None]
        self.device = torch.empty(self.capacity, dtype=torch.int64, device=self.dev)
        self.turn = 0

    def buffer(self, n: int) -> np.ndarray:
        """A pinned host array of at least n entries, free to write (its previous copy has finished)."""
        if n > self.capacity:
            self._grow(max(n, 2 * self.capacity))
        self.turn ^= 1
        if self.done[self.turn] is not None:
            self.done[self.turn].synchronize()
        return self.views[self.turn]

    def send(self, n: int, stream) -> torch.Tensor:
        """The first n entries of the buffer just written, on the device (queued on `stream`)."""
        dst = self.device[:n]
        dst.copy_(self.host[self.turn][:n], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(stream)
        self.done[self.turn] = ev
        return dst

    def put(self, a: np.ndarray, stream) -> torch.Tensor:
        buf = self.buffer(len(a))
        buf[:len(a)] = a
        return self.send(len(a), stream)


def plan_worlds(starts: np.ndarray, lens: np.ndarray, tile_cap: int, worlds: np.ndarray | None = None,
                tile_worlds: np.ndarray | None = None) -> tuple:
    """The tile plan of the listed-worlds tick for worlds at rows [starts[k], starts[k] + lens[k]): best-fit
    decreasing packing into tiles of at most tile_cap rows, in the native library (include/ebb.h:
    ebb_plan_worlds), into `worlds` and `tile_worlds` when given (contiguous int64 arrays of at least 2E and E + 1
    entries). Returns (worlds [2 x listed] int64, tile_worlds [T + 1] int64) views."""
    starts = np.ascontiguousarray(starts, dtype=np.int64)
    lens = np.ascontiguousarray(lens, dtype=np.int64)
    e = len(starts)
    worlds = np.empty(2 * e, dtype=np.int64) if worlds is None else worlds
    tile_worlds = np.empty(e + 1, dtype=np.int64) if tile_worlds is None else tile_worlds
    if len(worlds) < 2 * e or len(tile_worlds) < e + 1:
        raise ValueError("plan arrays too short")
    if e and int(lens.max()) > tile_cap:
        raise ValueError(f"a world of {int(lens.max())} rows does not fit a tile of {tile_cap}")
    tiles = _native.lib().ebb_plan_worlds(starts.ctypes.data, lens.ctypes.data, e, int(tile_cap), worlds.ctypes.data,
                                          tile_worlds.ctypes.data)
    if tiles < 0:
        _native.check(int(tiles), "ebb_plan_worlds")
    listed = int(tile_worlds[tiles]) if tiles else 0
    return worlds[:2 * listed], tile_worlds[:tiles + 1]


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
    tick_ms: list = field(default_factory=list)        # the tick launch's device time (CUDA events)
    rows: list = field(default_factory=list)           # ship-ticks of each step
    admitted: int = 0
    retired: int = 0
    wall_s: float = 0.0

    def summary(self) -> dict:
        lat = sorted(self.latency_ms)
        q = lambda p: lat[min(len(lat) - 1, int(math.ceil(p * len(lat))) - 1)] if lat else float("nan")
        total = sum(self.rows)
        tick = sum(self.tick_ms)
        return {"steps": len(lat), "p50_ms": q(0.50), "p99_ms": q(0.99), "mean_ms": statistics.fmean(lat) if lat
                else float("nan"), "ship_ticks": total, "ship_ticks_per_s": total / self.wall_s if self.wall_s else
                float("nan"), "tick_ship_ticks_per_s": total / (tick * 1e-3) if tick else float("nan"),
                "mean_rows": total / len(lat) if lat else 0.0, "admitted": self.admitted, "retired": self.retired}


@dataclass
class Staged:
    """A batch of episodes staged together: their staging park, each episode's first row in it, and the event after
    which the park is complete on the device. `next` is the first episode not yet admitted."""
    park: VecModesPark
    episodes: list
    offsets: list
    event: torch.cuda.Event
    rows: int
    next: int = 0


class Server:
    """The continuous-batching loop (module docstring). `budget_bytes` of device state caps the resident rows
    (ROW_BYTES a row; `rows` overrides it); `tile_cap` rows a tile of the listed-worlds tick, at least the largest
    episode; `stage_rows` caps the rows staged ahead of admission, `stage_batch` the rows of one staging park; `depth`
    steps may be in flight on the device; `keep` keeps each finished episode's final state in `results`. Staging runs
    on a thread of its own (`close()` ends it)."""

    def __init__(self, budget_bytes: float = 80e9, rows: int | None = None, dynamical: bool = True,
                 new_orbit: bool = True, tile_cap: int = 256, block: int = 256, grid: int | None = None,
                 device="cuda", keep: bool = True, max_ships: int = 256, stage_rows: int | None = None,
                 stage_batch: int = 8192, depth: int = 1):
        capacity = int(rows) if rows is not None else int(budget_bytes // ROW_BYTES)
        if capacity <= 0:
            raise ValueError("the state budget holds no row")
        if max_ships > tile_cap:
            raise ValueError("an episode must fit one tile")
        self.park = VecModesPark(capacity, device=device, dynamical_orientation=dynamical, use_new_orbit=new_orbit)
        self.dev = self.park.dev
        self.capacity = capacity
        self.space = RowSpace(capacity)
        self.live: dict = {}
        self.results: dict = {}
        self.keep = keep
        self.max_ships = max_ships
        self.tile_cap, self.block = int(tile_cap), int(block)
        self.grid = grid
        self.status = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self._plan = None                        # (worlds, tile_worlds, tiles) on the device
        self._dirty = True
        self.table = LiveTable()
        self.ends: dict = {}                     # step -> eids whose last tick it is
        self.live_rows = 0
        self.step_no = 0
        self.stats = StepStats()
        self.up_worlds, self.up_tiles = Uploads(self.dev), Uploads(self.dev)
        self.up_src, self.up_dst = Uploads(self.dev), Uploads(self.dev)
        self.depth = max(1, int(depth))
        self.inflight: deque = deque()           # (host start, (tick start, tick end, step end) events, ship-ticks)
        self._events: list = []
        # staging: episodes in `inbox` are staged by the thread into `ready` batches, at most stage_rows rows ahead
        self.stage_rows = int(stage_rows) if stage_rows is not None else max(max_ships, min(capacity, 1 << 16))
        self.stage_batch = max(int(stage_batch), max_ships)           # rows a staging batch takes at most
        self.side = torch.cuda.Stream(device=self.dev)
        self.inbox: deque = deque()
        self.ready: deque = deque()
        self.pending = 0                         # submitted, not yet admitted
        self.staged_rows = 0
        self._cv = threading.Condition()
        self._error = None
        self._stop = False
        self._thread = threading.Thread(target=self._stager, name="episode-stager", daemon=True)
        self._thread.start()

    # ---- requests and staging ----
    def submit(self, episode: Episode) -> None:
        if episode.ships > self.max_ships:
            raise ValueError(f"episode {episode.eid}: {episode.ships} ships, more than {self.max_ships}")
        with self._cv:
            self.inbox.append(episode)
            self.pending += 1
            self._cv.notify_all()

    def _stager(self) -> None:
        try:
            torch.cuda.set_device(self.dev)
            while True:
                with self._cv:
                    while not self._stop and not (self.inbox and
                                                  self.staged_rows + self.inbox[0].ships <= self.stage_rows):
                        self._cv.wait()
                    if self._stop:
                        return
                    batch, rows = [], 0
                    while (self.inbox and self.staged_rows + rows + self.inbox[0].ships <= self.stage_rows
                           and rows + self.inbox[0].ships <= self.stage_batch):
                        ep = self.inbox.popleft()
                        batch.append(ep)
                        rows += ep.ships
                    self.staged_rows += rows
                staged = self._stage(batch, rows)
                with self._cv:
                    self.ready.append(staged)
        except BaseException as exc:                                  # surfaced by the next step
            self._error = exc

    def _stage(self, batch: list, rows: int) -> Staged:
        """A staging park of the batch's worlds, loaded and commanded through the park API on the side stream (each
        world as it would be alone)."""
        pw = PackedWorlds.concat([ep.world.packed() for ep in batch])
        offsets = np.concatenate(([0], np.cumsum([ep.ships for ep in batch])[:-1])).astype(np.int64).tolist()
        with torch.cuda.stream(self.side):
            stage = VecModesPark(rows, device=self.dev, dynamical_orientation=self.park.dynamical_orientation,
                                 use_new_orbit=self.park.use_new_orbit)
            pw.load(stage)
            pw.apply(stage)
            ev = torch.cuda.Event()
            ev.record(self.side)
        return Staged(stage, batch, offsets, ev, rows)

    def _admit(self) -> None:
        """Staged episodes into free rows, first come first served: one move a staged batch."""
        main = torch.cuda.current_stream(self.dev)
        while True:
            with self._cv:
                if not self.ready:
                    return
                b = self.ready[0]
            take = []
            while b.next < len(b.episodes):
                ep = b.episodes[b.next]
                start = self.space.alloc(ep.ships)
                if start is None:
                    break
                take.append((ep, b.offsets[b.next], start))
                b.next += 1
            if take:
                src = np.concatenate([np.arange(o, o + ep.ships, dtype=np.int64) for ep, o, _ in take])
                dst = np.concatenate([np.arange(st, st + ep.ships, dtype=np.int64) for ep, _, st in take])
                main.wait_event(b.event)
                move_rows(self.park, b.park, self.up_src.put(src, main), self.up_dst.put(dst, main), self.status,
                          main.cuda_stream)
                for ep, _, start in take:
                    last = self.step_no + ep.ticks - 1
                    self.live[ep.eid] = Live(ep, start, last)
                    self.ends.setdefault(last, []).append(ep.eid)
                    self.table.add(ep.eid, start, ep.ships)
                    self.live_rows += ep.ships
                self.stats.admitted += len(take)
                self._dirty = True
                with self._cv:
                    self.pending -= len(take)
            if b.next < len(b.episodes):
                return                                                # no room for the next one yet
            for name, _, _ in _STORAGE:                               # the staging park is read on the main stream
                getattr(b.park, "_" + name).record_stream(main)
            with self._cv:
                self.ready.popleft()
                self.staged_rows -= b.rows
                self._cv.notify_all()

    def _upload_plan(self) -> None:
        if not self._dirty:
            return
        c = self.table.count
        main = torch.cuda.current_stream(self.dev)
        wb, tb = self.up_worlds.buffer(2 * c), self.up_tiles.buffer(c + 1)
        worlds, tile_worlds = plan_worlds(self.table.start[:c], self.table.len[:c], self.tile_cap, wb, tb)
        self._plan = (self.up_worlds.send(len(worlds), main), self.up_tiles.send(len(tile_worlds), main),
                      len(tile_worlds) - 1)
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
            src_rows = self.up_src.put(src, main)
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
    def step(self) -> int:
        """One step (module docstring): admit, tick every live episode, retire; returns the ship-ticks it ran (0, with
        nothing recorded, when nothing is live). At most `depth` steps are in flight on the device: with depth 1 each
        step waits for its own tick, with 2 the host prepares a step while the device runs the one before."""
        if self._error is not None:
            raise RuntimeError("staging failed") from self._error
        t0 = time.perf_counter()
        with torch.cuda.device(self.dev):
            self._admit()
            if not self.live:
                self.flush()
                return 0
            self._upload_plan()
            main = torch.cuda.current_stream(self.dev)
            ev = self._events.pop() if self._events else tuple(torch.cuda.Event(enable_timing=k < 2) for k in range(3))
            ev[0].record(main)
            ran = self._tick()
            ev[1].record(main)
            self._retire()
            ev[2].record(main)
            self.inflight.append((t0, ev, ran))
            while len(self.inflight) >= self.depth:
                self._finish()
        self.step_no += 1
        return ran

    def _finish(self) -> None:
        """Wait for the oldest step in flight and record its latency, tick time and ship-ticks."""
        t0, ev, ran = self.inflight.popleft()
        ev[2].synchronize()
        self.stats.latency_ms.append((time.perf_counter() - t0) * 1e3)
        self.stats.tick_ms.append(ev[0].elapsed_time(ev[1]))
        self.stats.rows.append(ran)
        self._events.append(ev)

    def flush(self) -> None:
        """Wait for every step in flight."""
        while self.inflight:
            self._finish()

    def idle(self) -> bool:
        with self._cv:
            return not self.live and self.pending == 0

    def reset_stats(self) -> None:
        """Start the step statistics afresh (after a warm-up)."""
        self.flush()
        self.stats = StepStats()

    def check(self) -> None:
        """The device's status bits (a follow pointer leaving its world, a malformed tile, a bad move) as an error."""
        if self._error is not None:
            raise RuntimeError("staging failed") from self._error
        st = int(self.status.item())
        if st:
            raise RuntimeError(f"serving status {st:#x}: 1 a target outside its world, 2 a malformed tile, "
                               "4 a row or pointer outside a park in a move")

    def close(self) -> None:
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        self._thread.join(timeout=60)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def serve(server: Server, episodes: list, realtime: bool = True, max_steps: int | None = None) -> dict:
    """Run `episodes` through `server` until every one has finished (or max_steps steps have ticked): with
    `realtime`, each arrives at its `arrival` second of wall time after the start (an open loop); otherwise all wait
    from the start (a saturated, closed loop). Returns the step statistics' summary."""
    pending = deque(sorted(episodes, key=lambda e: e.arrival)) if realtime else deque()
    if not realtime:
        for ep in episodes:
            server.submit(ep)
    switch = sys.getswitchinterval()
    sys.setswitchinterval(SWITCH_INTERVAL_S)         # the staging thread gives the interpreter back to the loop quickly
    t0 = time.perf_counter()
    steps = 0
    try:
        while pending or not server.idle():
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                server.submit(pending.popleft())
            if server.step():
                steps += 1
                if max_steps is not None and steps >= max_steps:
                    break
            else:
                time.sleep(0.0001)                                    # nothing live yet: staging or waiting
        server.flush()
    finally:
        sys.setswitchinterval(switch)
    server.stats.wall_s += time.perf_counter() - t0
    server.check()
    return server.stats.summary()
