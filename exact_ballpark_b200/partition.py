"""The partition layer over ragged worlds: bubbles, the spatial partition and proximity sensors (the space layer,
exact_ballpark_b200.space) over a flight park whose worlds have uneven ship counts, packed with no padding.

The reference's layer (exact_ballpark.vec_space.VecSpace, vec_space.py:777) keeps W worlds of N slots, every world
padded to N, one thread a world in world order. Here the same per-world program runs over two arrangements of the
same worlds, with the same results world by world:

- `ragged=True` (the ragged batch): each world goes to the smallest size class (4, 8, 16, 32, 64 or 128 slots) that
  holds it, one layer a class, so a world's loops run over its class's slots and not 128; a class's worlds are
  ordered by size, largest first (the longest programs start first); the classes of 4 to 16 slots run a thread a
  world (a warp's 32 worlds of about the same size, so about the same program length), the classes of 32 to 128 slots
  a warp a world, its lanes splitting GetNearbyBalls' scan and sort (the sensors' O(N^2) part) and running the rest
  together;
- `ragged=False` (the plain per-configuration layout): one layer of 128 slots a world, the worlds in their order.

A tick (`tick`) is Destiny's Evolve with the layer on the master: every layer's dead-bubble rows (TIME-714), the
park's tick with those rows left out, then every layer's re-filings and HandleProximities (the events of the tick in
each layer's `ev`, cleared first). Nothing synchronises the host, so a tick can be captured as one CUDA graph
(`PartitionGraph`), with the server layer's pre-tick and send flags around it when a server rides on the park.
"""

from __future__ import annotations

import numpy as np
import torch

from .modes import WARP, VecModesPark
from .space import OP, VecSpace

CLASSES = (4, 8, 16, 32, 64, 128)
WARP_CLASS = 32                  # the ragged batch's classes from this size up run a warp a world
BOOL, I64 = torch.bool, torch.int64


class PartitionLayer:
    """The space layer over a flight park of ragged worlds whose rows are contiguous a world (`sizes` [W], world w's
    rows from sum(sizes[:w])). `events`: each world's event capacity a tick, by default N (N + 2) for a class of N
    slots (every pair entering and each ball's range and tracking events); `boxes`: box-table entries a world as a
    multiple of the class's slots (plus 64). `plan` {class: (lanes, block)}: how each size class runs (1 a thread a
    world, 32 a warp a world; threads a block), by default a warp a world from `warp_class` slots up, 128-thread
    blocks (`tune_partition` measures the best)."""

    def __init__(self, park: VecModesPark, sizes, ragged: bool = True, events: int | None = None,
                 boxes_per_slot: int = 16, seed: int = 1, warp_class: int = WARP_CLASS, plan: dict | None = None):
        self.park = park
        sizes = np.asarray(sizes, dtype=np.int64)
        if sizes.ndim != 1 or (sizes < 1).any() or sizes.max(initial=0) > CLASSES[-1]:
            raise ValueError(f"sizes: one ship count a world, from 1 to {CLASSES[-1]}")
        if int(sizes.sum()) != park.n:
            raise ValueError("the worlds' ships are not the park's rows")
        self.sizes, self.ragged = sizes, bool(ragged)
        starts = np.concatenate(([0], np.cumsum(sizes)[:-1])).astype(np.int64)
        if ragged:
            cls = np.searchsorted(np.asarray(CLASSES), sizes)          # the smallest class that holds the world
            groups = []
            for c, cap in enumerate(CLASSES):
                idx = np.nonzero(cls == c)[0]
                if len(idx):
                    idx = idx[np.argsort(-sizes[idx], kind="stable")]   # largest first
                    groups.append((cap, idx))
        else:
            groups = [(CLASSES[-1], np.arange(len(sizes)))]
        self.layers = []
        for cap, idx in groups:
            slots = np.full((len(idx), cap), -1, dtype=np.int64)
            k = sizes[idx]
            col = np.arange(cap)[None, :]
            slots[:] = np.where(col < k[:, None], starts[idx][:, None] + col, -1)
            lanes, block = (32 if ragged and cap >= warp_class else 1), 128
            if ragged and plan is not None and cap in plan:
                lanes, block = plan[cap]
            layer = VecSpace(park, slots, boxes=boxes_per_slot * cap + 64,
                             events=cap * (cap + 2) if events is None else int(events), umap_cap=cap,
                             seed=(idx + seed).tolist(), lanes=lanes, block=block)
            self.layers.append((layer, idx))
        self.last_dead = None

    # ---- set-up ----
    def load(self) -> None:
        """AddBall's filing of every ball (each world's ships in order)."""
        for layer, _ in self.layers:
            layer.load()

    def add_sensors(self, ranges, period: float = 1.0) -> None:
        """AddProximitySensor on every ship: `ranges` [n] each ship's sensor radius (by park row), the period."""
        rng = torch.as_tensor(np.asarray(ranges, dtype=np.float64))
        for layer, _ in self.layers:
            rows = layer.rows.t().cpu()                                   # [W, N]
            on = rows >= 0
            code = torch.where(on, OP["ADD_SENSOR"], OP["NONE"]).to(I64)
            slots = torch.arange(layer.N, dtype=I64).expand(layer.W, layer.N)
            f = torch.zeros(layer.W, layer.N, 4, dtype=torch.float64)
            f[..., 0] = torch.where(on, rng[rows.clamp(min=0)], 0.0)
            f[..., 1] = period
            layer.tape(code, slots, torch.zeros_like(code), f)

    # ---- the tick ----
    def dead_rows(self) -> torch.Tensor:
        """Every layer's dead-bubble rows [n] (phase 1's flags)."""
        dead = None
        for layer, _ in self.layers:
            d = layer.dead_rows()
            dead = d if dead is None else dead | d
        return dead

    def tick(self, park_tick=None) -> None:
        """One tick of the park with the layer: the dead bubbles' balls left out of the park's tick (flagged
        moribund for it), then each layer's events cleared, its re-filings and HandleProximities. `park_tick()` ticks
        the park (its `evolve` by default)."""
        park = self.park
        dead = self.dead_rows()
        self.last_dead = dead
        warp_proper = (park._mode == WARP) & (park._effect_stamp >= 0) & park._free & ~park._moribund & ~dead
        saved = park._moribund.clone()
        park._moribund.logical_or_(dead)
        if park_tick is None:
            park.evolve()
        else:
            park_tick()
        park._moribund.copy_(saved)
        dropped = warp_proper & (park._mode != WARP)
        for layer, _ in self.layers:
            layer.clear_events()
            layer.after_evolve(dropped)

    # ---- readers ----
    def event_counts(self) -> torch.Tensor:
        """Each world's events of the last tick [W] (by world index)."""
        out = torch.zeros(len(self.sizes), dtype=I64, device=self.park.dev)
        for layer, idx in self.layers:
            out[torch.as_tensor(idx, device=self.park.dev)] = layer.st["evn"]
        return out

    def flags(self) -> torch.Tensor:
        """Each world's domain flags [W] (by world index)."""
        out = torch.zeros(len(self.sizes), dtype=I64, device=self.park.dev)
        for layer, idx in self.layers:
            out[torch.as_tensor(idx, device=self.park.dev)] = layer.st["flags"]
        return out

    def world(self, w: int) -> tuple:
        """World w's layer and its column in it: (VecSpace, column)."""
        for layer, idx in self.layers:
            pos = np.nonzero(idx == w)[0]
            if len(pos):
                return layer, int(pos[0])
        raise IndexError(w)

    def check(self) -> None:
        for layer, _ in self.layers:
            layer.check()


class PartitionGraph:
    """One tick of a PartitionLayer captured as a CUDA graph: the server's pre-tick (when `server` rides on the park:
    the kernel path's queue, bubble update and history, one launch), the layer's tick around the park's tick, the
    server's send flags. `park_tick` ticks the park (the tiled schedule's launch, or the plain one). The state is
    written in place by every launch, so each `tick()` is one replay."""

    def __init__(self, part: PartitionLayer, park_tick, server=None, queue=None):
        self.part, self.park_tick, self.server, self.q = part, park_tick, server, queue
        park = part.park
        d = park.dev
        names = park.row_tensors()
        keep = [(getattr(park, k), getattr(park, k).clone()) for k in names]
        for layer, _ in part.layers:
            keep += [(t, t.clone()) for t in layer.st.values()]
        if server is not None:
            keep += [(t, t.clone()) for t in [park.cloaked, park.bubble, server.stamp_for_system, server._bubble_time,
                                              server.dead, server.settled, server._fresh, server._listed]
                     + [queue[k] for k in ("ok", "row", "trow", "loc", "route", "notice", "stamp", "clock",
                                           "has_character", "gets_bubble")]]
        side = torch.cuda.Stream(device=d)                 # a warm-up of every launch, undone
        side.wait_stream(torch.cuda.current_stream(d))
        with torch.cuda.stream(side):
            self._body()
        torch.cuda.current_stream(d).wait_stream(side)
        torch.cuda.synchronize(d)
        for t, v in keep:
            t.copy_(v)
        del keep
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._body()

    def _body(self) -> None:
        if self.server is not None:
            self.server._launch(self.q, 5)
        self.part.tick(self.park_tick)
        if self.server is not None:
            self.server._launch(self.q, 3)

    def tick(self) -> None:
        self.graph.replay()
        self.part.park.current_time += 1


def partition_setup(pw, dev, ragged: bool, server_on: bool = True, warp_class: int = WARP_CLASS,
                    plan: dict | None = None) -> dict:
    """A flight park of the partition worlds with the partition layer (ragged size classes, or the plain 128-slot
    layout), every ship's sensor added, and the server layer on top (a pilot a ship, GotoDirection and
    SetSpeedFraction queued for every ship every tick: a fixed schedule of 2 pushes a slot of the largest world, a
    world's pushes masked to its ships). The first tick runs eagerly; returns the parts and the captured tick."""
    from . import server
    from .modes import tick_plain, tick_tiled
    park = VecModesPark(pw.n, device=dev)
    park.load_columns(pw.cols)
    part = PartitionLayer(park, pw.sizes, ragged=ragged, warp_class=warp_class, plan=plan)
    part.load()
    part.add_sensors(pw.sensor_range, 1.0)
    park_tick = (lambda: tick_tiled(park)) if ragged else (lambda: tick_plain(park, park.block))
    if not ragged:
        park.scratch()
    srv = q = None
    W = len(pw.sizes)
    if server_on:
        srv = server.VecServer(server.ModesAdapter(park), (pw.cols["id"] - 1).tolist(), kernel="cuda")
        srv.pre_tick()                                      # the first tick (its additions) eagerly
        part.tick(park_tick)
        park.current_time += 1
        srv.post_tick()
        K = int(np.max(pw.sizes))                         # a world's most ships: the schedule's pilots
        sched = [k for _ in range(K) for k in ("GotoDirection", "SetSpeedFraction")]
        q = srv._queue([server.CODE[k] for k in sched])
        sizes = torch.as_tensor(pw.sizes, device=dev)
        starts = torch.as_tensor(pw.starts, device=dev)
        direction = torch.as_tensor(pw.direction, device=dev)
        speed = torch.as_tensor(pw.speed, device=dev)
        for k in range(K):
            on = sizes > k
            row = torch.where(on, starts + k, 0)
            for j, f in ((2 * k, direction[row]), (2 * k + 1, speed[row][:, None])):
                q["mask"][j].copy_(on.to(q["mask"].dtype))
                q["ball"][j].fill_(k + 1)
                q["f"][j][:, :f.shape[1]].copy_(f)
    else:
        part.tick(park_tick)
        park.current_time += 1
    g = PartitionGraph(part, park_tick, srv, q)
    return {"park": park, "part": part, "server": srv, "q": q, "graph": g, "park_tick": park_tick}


ARRANGEMENTS = ((1, 64), (1, 128), (32, 128))      # (lanes, block): a thread a world in 64- or 128-thread blocks; a warp


def tune_partition(pw, dev, warm: int = 1, ticks: int = 2, arrangements=ARRANGEMENTS) -> tuple:
    """The ragged batch's autotuner: each size class's arrangement (a thread a world, 2 or 4 warps of worlds a
    block; or a warp a world, 4 worlds a block), measured on the workload itself. For each arrangement every class
    runs it: the worlds are loaded, their sensors added, the server layer on top (the pilots' commands every tick, so
    the ships move as in the benchmark), `warm` ticks run, then `ticks` ticks each with every class's re-filings and
    HandleProximities timed alone (CUDA events); every arrangement starts from the same state and does the same work
    (its results are bit-identical). The classes run one after another in a tick, so each takes its fastest
    arrangement. Returns (plan {class: (lanes, block)}, {arrangement: {class: ms a tick}})."""
    times = {}
    for lanes, block in arrangements:
        plan = {cap: (lanes, block) for cap in CLASSES}
        r = partition_setup(pw, dev, ragged=True, server_on=True, plan=plan)
        part, park_tick, srv, q = r["part"], r["park_tick"], r["server"], r["q"]
        for _ in range(warm):
            r["graph"].tick()
        stream = torch.cuda.current_stream(dev)
        ms = {layer.N: 0.0 for layer, _ in part.layers}
        park = part.park
        for _ in range(ticks):
            srv._launch(q, 5)
            dead = part.dead_rows()
            saved = park._moribund.clone()
            park._moribund.logical_or_(dead)
            park_tick()
            park._moribund.copy_(saved)
            for layer, _ in part.layers:
                layer.clear_events()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                layer.after_evolve(None)
                b.record(stream)
                b.synchronize()
                ms[layer.N] += a.elapsed_time(b) / ticks
            srv._launch(q, 3)
            park.current_time += 1
        times[(lanes, block)] = ms
        del r, part, srv, q
        torch.cuda.empty_cache()
    best = {}
    for cap in CLASSES:
        have = [(t[cap], arr) for arr, t in times.items() if cap in t]
        if have:
            best[cap] = min(have)[1]
    return best, times
