"""The serving loop's host logic without a GPU: the row allocator, the live table, the tile plan of listed worlds, the
episode stream, and the concatenation of worlds that staging relies on."""

import random

import numpy as np

from exact_ballpark_b200.serving import LiveTable, RowSpace, episode_stream, plan_worlds
from exact_ballpark_b200.workloads import FlightWorlds, flight_worlds


def test_the_row_space_allocates_first_fit_and_merges_free_runs():
    r = random.Random(3)
    cap = 500
    sp = RowSpace(cap)
    used = np.zeros(cap, dtype=bool)
    held = []
    for _ in range(3000):
        if held and (r.random() < 0.45 or sp.used > cap - 40):
            start, n = held.pop(r.randrange(len(held)))
            assert used[start:start + n].all()
            used[start:start + n] = False
            sp.free(start, n)
        else:
            n = r.randint(1, 40)
            start = sp.alloc(n)
            free_runs = [(s, ln) for s, ln in zip(sp.starts, sp.lens)]
            if start is None:                      # no free run of n rows
                assert all(ln < n for _, ln in free_runs)
                continue
            assert not used[start:start + n].any()
            used[start:start + n] = True
            held.append((start, n))
        assert sp.used == int(used.sum())
        # the free runs are exactly the free rows, sorted, maximal (merged)
        free = np.zeros(cap, dtype=bool)
        for s, ln in zip(sp.starts, sp.lens):
            free[s:s + ln] = True
        assert (free == ~used).all()
        assert sp.starts == sorted(sp.starts)
        assert all(a + la < b for a, la, b in zip(sp.starts, sp.lens, sp.starts[1:]))


def test_the_row_space_refuses_a_double_free():
    sp = RowSpace(10)
    a = sp.alloc(4)
    sp.free(a, 4)
    try:
        sp.free(a, 4)
    except ValueError:
        return
    raise AssertionError("a double free was accepted")


def test_the_live_table_swap_removes():
    t = LiveTable()
    ref = {}
    r = random.Random(9)
    for eid in range(500):
        t.add(eid, eid * 10, r.randint(1, 9))
        ref[eid] = (eid * 10, int(t.len[t.where[eid]]))
        if r.random() < 0.4:
            gone = r.choice(list(ref))
            t.remove(gone)
            del ref[gone]
    assert t.count == len(ref)
    got = {int(t.eid[k]): (int(t.start[k]), int(t.len[k])) for k in range(t.count)}
    assert got == ref


def test_the_tile_plan_lists_every_world_once_within_the_tile_size():
    r = random.Random(1)
    for cap in (64, 256, 384, 1024):
        for _ in range(50):
            e = r.randint(0, 400)
            lens = np.array([r.randint(1, min(cap, 256)) for _ in range(e)], dtype=np.int64)
            starts = np.cumsum(np.concatenate(([0], lens[:-1] + np.array([r.randint(0, 5) for _ in range(max(e - 1, 0))],
                                                                          dtype=np.int64)))).astype(np.int64)[:e]
            perm = np.array(r.sample(range(e), e), dtype=np.int64)
            worlds, tile_worlds = plan_worlds(starts[perm], lens[perm], cap)
            assert tile_worlds[0] == 0 and tile_worlds[-1] == e
            assert (np.diff(tile_worlds) > 0).all() or e == 0
            pairs = worlds.reshape(-1, 2)
            assert sorted(map(tuple, pairs.tolist())) == sorted(zip(starts.tolist(), (starts + lens).tolist()))
            total = int(lens.sum())
            for a, b in zip(tile_worlds[:-1], tile_worlds[1:]):
                rows = int((pairs[a:b, 1] - pairs[a:b, 0]).sum())
                assert rows <= cap and b - a <= cap
                assert (np.diff(pairs[a:b, 0]) > 0).all()                    # each tile's worlds in row order
            tiles = len(tile_worlds) - 1
            assert tiles <= max(1, 2 * -(-total // cap))                      # best fit: at most twice the least


def test_a_world_bigger_than_a_tile_is_refused():
    try:
        plan_worlds(np.array([0]), np.array([300]), 256)
    except ValueError:
        return
    raise AssertionError("a 300-row world was planned into 256-row tiles")


def test_the_episode_stream_is_seeded_and_shaped():
    a = episode_stream(7, 400, rate=2000.0)
    b = episode_stream(7, 400, rate=2000.0)
    assert [(e.ships, e.ticks, e.arrival) for e in a] == [(e.ships, e.ticks, e.arrival) for e in b]
    ships = np.array([e.ships for e in a])
    ticks = np.array([e.ticks for e in a])
    gaps = np.diff([0.0] + [e.arrival for e in a])
    assert ships.min() >= 1 and ships.max() <= 256 and ticks.min() >= 10 and ticks.max() <= 10000
    assert 0.0003 < gaps.mean() < 0.0007                    # Poisson at 2000 a second
    assert 20 < ships.mean() < 80                           # log-uniform in [1, 256]: about 46
    for e in a[:20]:
        assert len(e.world.rows) == e.ships and {r["world"] for r in e.world.rows} == {0}


def test_concatenated_worlds_keep_each_worlds_rows_and_targets():
    parts = [flight_worlds(s, 1, n) for s, n in ((1, 3), (2, 1), (3, 7), (4, 2))]
    c = FlightWorlds.concat(parts)
    assert c.worlds == 4 and c.sizes == [3, 1, 7, 2]
    base = 0
    for k, p in enumerate(parts):
        for j, row in enumerate(p.rows):
            q = c.rows[base + j]
            assert q["world"] == k and q["pos"] == row["pos"] and q["id"] == row["id"]
            t = p.target[j]
            assert c.target[base + j] == (t + base if t >= 0 else -1)
        base += len(p.rows)
