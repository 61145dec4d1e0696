"""Packing worlds into tiles for the tiled (ragged, persistent) tick, and the plan's autotuned shape.

A tile is a run of whole worlds, at most `cap` rows, handled by one thread block of `block` threads (the records of
the tile in shared memory, the block's threads taking the tile's ships in the order of their last search cost).
Worlds of any size pack with no padding between them: the tile table is the row offsets of the tiles (tile_rows[t] ..
tile_rows[t + 1]). The grid is persistent: `grid` blocks take the tiles in turn (grid = tiles is one block a tile).

`plan_tiles` needs each world's rows contiguous (a world's rows one run, every world one run); otherwise it returns
None and the park ticks with the plain schedule. The shape (cap, block, grid) is chosen by `autotune`, which times
the candidates on the park itself and keeps the fastest (exact_ballpark_b200.autotune).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import torch

DEFAULT_CAP = 256
DEFAULT_BLOCK = 256
MAX_CAP = 4096


@dataclass
class TilePlan:
    tile_rows: list            # tiles + 1 row offsets
    cap: int                   # rows a tile holds at most
    block: int                 # threads a block (>= cap, a multiple of 32)
    grid: int                  # blocks of the persistent grid
    max_world: int             # the largest world's rows
    world_rows: list = field(default_factory=list)   # the worlds' row offsets ([0, ..., n]), when known
    _dev: dict = field(default_factory=dict, repr=False)

    @property
    def tiles(self) -> int:
        return len(self.tile_rows) - 1

    def worlds_on(self, dev) -> tuple:
        """The same plan as a list of worlds (the listed-worlds tick's form): world w is rows [worlds[2w],
        worlds[2w + 1]), tile t the worlds [tile_worlds[t], tile_worlds[t + 1]); device tensors, made once."""
        key = "worlds:" + str(dev)
        if key not in self._dev:
            runs = self.world_rows
            if len(runs) < 2:
                raise ValueError("the plan was made without its world offsets")
            pairs = [x for a, b in zip(runs[:-1], runs[1:]) for x in (a, b)]
            index = {r: k for k, r in enumerate(runs)}
            tile_worlds = [index[r] for r in self.tile_rows]
            self._dev[key] = (torch.tensor(pairs, dtype=torch.int64, device=dev),
                              torch.tensor(tile_worlds, dtype=torch.int64, device=dev))
        return self._dev[key]

    def tile_rows_on(self, dev) -> torch.Tensor:
        key = str(dev)
        if key not in self._dev:
            self._dev[key] = torch.tensor(self.tile_rows, dtype=torch.int64, device=dev)
        return self._dev[key]


def world_runs(world: torch.Tensor) -> list | None:
    """The row offsets of the worlds' runs ([0, ..., n]) when every world is one contiguous run, else None."""
    w = world.detach().to("cpu", torch.int64)
    n = int(w.numel())
    if n == 0:
        return [0]
    change = torch.nonzero(w[1:] != w[:-1]).reshape(-1) + 1
    starts = [0] + change.tolist()
    if len(starts) != int(torch.unique(w).numel()):
        return None
    return starts + [n]


def pack(runs: list, cap: int) -> list:
    """Greedy packing of consecutive world runs into tiles of at most cap rows (a world never split; every world at
    most cap rows)."""
    out = [runs[0]]
    for k in range(1, len(runs)):
        if runs[k] - out[-1] > cap:                  # world k-1 does not fit: the tile closes before it
            out.append(runs[k - 1])
    if out[-1] != runs[-1]:
        out.append(runs[-1])
    return out


def plan_tiles(world: torch.Tensor, cap: int = DEFAULT_CAP, block: int | None = None, grid: int | None = None):
    """The tile plan for a park's world column, or None when its worlds are not contiguous runs or a world is larger
    than MAX_CAP rows."""
    runs = world_runs(world)
    if runs is None or len(runs) < 2:
        return None
    max_world = max(b - a for a, b in zip(runs[:-1], runs[1:]))
    if max_world > MAX_CAP:
        return None
    cap = min(max(cap, max_world), MAX_CAP)
    tile_rows = pack(runs, cap)
    blk = block or DEFAULT_BLOCK
    if blk % 32 or not 32 <= blk <= 256:
        raise ValueError(f"block {blk}: a multiple of 32 up to 256")
    return TilePlan(tile_rows, cap, blk, grid or (len(tile_rows) - 1), max_world, runs)


@dataclass
class WorldsPlan:
    """A plan for the listed-worlds tick over a park's own worlds, packed best fit (include/ebb.h: ebb_plan_worlds):
    tiles of at most `cap` rows made of any whole worlds, not only neighbours, so small worlds fill the tiles that
    large ones leave room in. `worlds` [2W] row runs and `tile_worlds` [T + 1] as the kernel takes them."""
    worlds: list
    tile_worlds: list
    cap: int
    block: int
    grid: int
    _dev: dict = field(default_factory=dict, repr=False)

    @property
    def tiles(self) -> int:
        return len(self.tile_worlds) - 1

    def worlds_on(self, dev) -> tuple:
        key = str(dev)
        if key not in self._dev:
            self._dev[key] = (torch.tensor(self.worlds, dtype=torch.int64, device=dev),
                              torch.tensor(self.tile_worlds, dtype=torch.int64, device=dev))
        return self._dev[key]


def plan_best_fit(world: torch.Tensor, cap: int = DEFAULT_CAP, block: int | None = None) -> WorldsPlan | None:
    """The best-fit plan of a park's world column (each world one contiguous run of at most cap rows), one tile a
    block; None when the worlds are not contiguous runs or one is larger than cap."""
    import numpy as np

    from . import _native
    runs = world_runs(world)
    if runs is None or len(runs) < 2:
        return None
    r = np.asarray(runs, dtype=np.int64)
    starts, lens = np.ascontiguousarray(r[:-1]), np.ascontiguousarray(np.diff(r))
    if int(lens.max()) > cap:
        return None
    worlds = np.empty(2 * len(starts), dtype=np.int64)
    tile_worlds = np.empty(len(starts) + 1, dtype=np.int64)
    tiles = _native.lib().ebb_plan_worlds(starts.ctypes.data, lens.ctypes.data, len(starts), int(cap),
                                          worlds.ctypes.data, tile_worlds.ctypes.data)
    _native.check(int(tiles) if tiles < 0 else 0, "ebb_plan_worlds")
    blk = block or DEFAULT_BLOCK
    return WorldsPlan(worlds.tolist(), tile_worlds[:tiles + 1].tolist(), int(cap), blk, int(tiles))
