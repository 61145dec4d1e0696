"""The flight-mode tick on the GPU, through the C ABI (the package's VecModesPark and its schedules):

- against the golden traces recorded on the reference (every tick's state digest of every scenario: the reference's
  mode_cases and flight_cases families and the flight-mode benchmark's worlds), with the tiled and the plain schedule;
- against the CPU oracle on worlds beyond the fixtures (other seeds, 1024 worlds, dynamical orientation on and off,
  both orbit laws): every field of every ship after every tick, bit for bit;
- the schedules against each other, a CUDA graph's replays against eager ticks, and batch independence (a world
  alone, or with the worlds reordered, ticks to the same bits).
"""

import numpy as np
import pytest
import torch

import trace as tr
from golden_util import GOLDEN, available_traces, bit_equal

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]

COMPARE = ("pos", "vel", "old_pos", "old_vel", "goto", "last_g", "ang_vel", "old_ang_vel", "torque", "rot", "old_rot",
           "speed_fraction", "follow_range", "last_collision", "rot_roll", "mode", "effect_stamp", "follow_id",
           "owner_id", "follow_ptr", "clock", "free", "massive", "interactive", "sensor")


def _park(ctor: dict, schedule: str):
    from exact_ballpark_b200 import VecModesPark
    ctor = dict(ctor)
    p = VecModesPark(ctor.pop("n"), device="cuda", **ctor)
    return p


def _ticker(p, schedule: str):
    from exact_ballpark_b200 import tick_plain, tick_tiled

    def run():
        if schedule == "plain":
            tick_plain(p)
        elif schedule == "tiled":
            tick_tiled(p)
        else:
            p.evolve()
            return
        p.current_time += 1
    return run


@pytest.mark.parametrize("schedule", ["tiled", "plain"])
@pytest.mark.parametrize("name", available_traces())
def test_the_gpu_park_replays_the_golden_trace(name, schedule):
    groups = tr.load(GOLDEN / name)
    failures = []
    for gi, t in enumerate(groups):
        p = _park(t["ctor"], schedule)
        bad = []

        def on_tick(k, park):
            mm = tr.first_mismatch(t, k, tr.field_digests(park))
            if mm and not bad:
                bad.append((k, mm))
        run = None

        def tick():
            nonlocal run
            if run is None:
                if schedule == "tiled" and p.plan is None:
                    pytest.fail(f"{name} group {gi}: worlds not contiguous")
                run = _ticker(p, schedule)
            run()
        tr.replay(t, p, tick=tick, on_tick=on_tick)
        if bad:
            failures.append((gi, t["ctor"], bad[0]))
    assert not failures, f"{len(failures)} of {len(groups)} parks differ; first: {failures[:3]}"


def _compare(oracle, park, where: str) -> None:
    for f in COMPARE:
        a = np.asarray(getattr(oracle, f))
        b = getattr(park, f).detach().cpu().numpy()
        eq = bit_equal(a, b)
        if not eq.all():
            rows = np.unique(np.nonzero(eq.reshape(eq.shape[0], -1).all(axis=1) == 0)[0])
            raise AssertionError(f"{where}: {f} differs in {len(rows)} rows, first {rows[:5]}")


@pytest.mark.parametrize("do,new_orbit,seed", [(True, True, 101), (True, False, 102), (False, True, 103),
                                               (False, False, 104)])
@pytest.mark.parametrize("schedule", ["tiled", "plain"])
def test_the_gpu_tick_matches_the_oracle_beyond_the_fixtures(do, new_orbit, seed, schedule):
    from exact_ballpark_b200.workloads import flight_worlds
    from oracle.park import OraclePark
    w = flight_worlds(seed, 1024, 4)
    o = OraclePark(len(w.rows), dynamical_orientation=do, use_new_orbit=new_orbit)
    p = _park({"n": len(w.rows), "dynamical_orientation": do, "use_new_orbit": new_orbit}, schedule)
    for park in (o, p):
        park.load(w.rows)
        w.apply(park)
    run = _ticker(p, schedule)
    for k in range(60):
        o.evolve()
        run()
        if k % 10 == 9 or k < 3:
            _compare(o, p, f"tick {k}")


def test_ragged_worlds_match_the_oracle():
    """Worlds of 1 to 40 ships (log-uniform), packed with no padding, through the tiled schedule."""
    import random
    from exact_ballpark_b200.workloads import flight_worlds
    from oracle.park import OraclePark
    r = random.Random(5)
    rows, tgt, rng, pt, wf, fm, om, wm = [], [], [], [], [], [], [], []
    wid = 0
    while len(rows) < 3000:
        size = max(1, int(10 ** r.uniform(0, np.log10(40))))
        w = flight_worlds(1000 + wid, 1, size)
        base = len(rows)
        for i, row in enumerate(w.rows):
            row = dict(row, world=wid, id=base + i + 1)
            rows.append(row)
        tgt += [t + base if t >= 0 else -1 for t in w.target]
        rng += w.range_
        pt += w.point
        wf += w.warp_factor
        fm += w.follow_mask
        om += w.orbit_mask
        wm += w.warp_mask
        wid += 1
    from exact_ballpark_b200.workloads import FlightWorlds
    w = FlightWorlds(rows, fm, om, wm, tgt, rng, pt, wf, wid, 0)
    o = OraclePark(len(rows), dynamical_orientation=True, use_new_orbit=True)
    p = _park({"n": len(rows), "dynamical_orientation": True, "use_new_orbit": True}, "tiled")
    for park in (o, p):
        park.load(rows)
        w.apply(park)
    assert p.plan is not None and p.plan.max_world <= 40
    run = _ticker(p, "tiled")
    for k in range(40):
        o.evolve()
        run()
    _compare(o, p, "after 40 ticks")


@pytest.mark.parametrize("schedule", ["tiled", "tiled_rounds", "worlds", "plain"])
def test_worlds_of_65_to_128_ships_match_the_oracle(schedule):
    """The metric's largest worlds, 65 to 128 ships each, against the oracle under every schedule: tiles of whole
    worlds one a block (a tile up to 256 rows) and the persistent form with several rounds of ships a thread (tiles
    of up to 512 rows over 128-thread blocks), the listed-worlds kernel, and the plain two launches."""
    import random
    from exact_ballpark_b200 import tick_plain, tick_tiled, tick_worlds
    from exact_ballpark_b200.tiles import plan_tiles
    from exact_ballpark_b200.workloads import FlightWorlds, flight_worlds
    from oracle.park import OraclePark
    r = random.Random(65)
    w = FlightWorlds.concat([flight_worlds(7000 + k, 1, r.randint(65, 128)) for k in range(36)])
    assert min(w.sizes) >= 65 and max(w.sizes) > 120
    o = OraclePark(len(w.rows), dynamical_orientation=True, use_new_orbit=True)
    p = _park({"n": len(w.rows), "dynamical_orientation": True, "use_new_orbit": True}, "plain")
    for park in (o, p):
        park.load(w.rows)
        w.apply(park)
    if schedule == "tiled":
        plan = plan_tiles(p.world, cap=256, block=256)
        run = lambda: tick_tiled(p, plan)                                      # noqa: E731
    elif schedule == "tiled_rounds":
        plan = plan_tiles(p.world, cap=512, block=128, grid=5)
        run = lambda: tick_tiled(p, plan)                                      # noqa: E731
    elif schedule == "worlds":
        plan = plan_tiles(p.world, cap=512, block=128)
        run = lambda: tick_worlds(p, None, plan)                               # noqa: E731
    else:
        run = lambda: tick_plain(p)                                            # noqa: E731
    for k in range(25):
        o.evolve()
        run()
        if k in (0, 9, 24):
            _compare(o, p, f"{schedule}, tick {k}")
    assert int(p._status.item()) == 0


def _state(p) -> dict:
    return {f: getattr(p, f).detach().cpu().numpy().copy() for f in COMPARE}


def test_graph_replay_equals_eager_ticks():
    from exact_ballpark_b200 import ModesGraph
    from exact_ballpark_b200.workloads import flight_worlds
    w = flight_worlds(21, 512, 4)
    a = _park({"n": len(w.rows), "dynamical_orientation": True, "use_new_orbit": True}, "tiled")
    b = _park({"n": len(w.rows), "dynamical_orientation": True, "use_new_orbit": True}, "tiled")
    for park in (a, b):
        park.load(w.rows)
        w.apply(park)
    g = ModesGraph(b)
    for _ in range(25):
        a.evolve()
        g.tick()
    torch.cuda.synchronize()
    sa, sb = _state(a), _state(b)
    for f in COMPARE:
        assert bit_equal(sa[f], sb[f]).all(), f
    assert a.current_time == b.current_time == 25


def test_a_world_alone_and_reordered_ticks_the_same():
    """Batch independence: world 7 ticked alone, and the worlds in reverse order, equal world 7 in the batch."""
    from exact_ballpark_b200.workloads import FlightWorlds, flight_worlds
    w = flight_worlds(33, 64, 4)
    full = _park({"n": len(w.rows), "dynamical_orientation": True, "use_new_orbit": True}, "tiled")
    full.load(w.rows)
    w.apply(full)
    sel = list(range(28, 32))
    alone = FlightWorlds([dict(w.rows[i]) for i in sel], [w.follow_mask[i] for i in sel],
                         [w.orbit_mask[i] for i in sel], [w.warp_mask[i] for i in sel],
                         [w.target[i] - 28 if w.target[i] >= 0 else -1 for i in sel], [w.range_[i] for i in sel],
                         [w.point[i] for i in sel], [w.warp_factor[i] for i in sel], 1, 4)
    one = _park({"n": 4, "dynamical_orientation": True, "use_new_orbit": True}, "tiled")
    one.load(alone.rows)
    alone.apply(one)
    order = [wd * 4 + j for wd in reversed(range(64)) for j in range(4)]
    inv = {old: new for new, old in enumerate(order)}
    rev = FlightWorlds([dict(w.rows[i]) for i in order], [w.follow_mask[i] for i in order],
                       [w.orbit_mask[i] for i in order], [w.warp_mask[i] for i in order],
                       [inv[w.target[i]] if w.target[i] >= 0 else -1 for i in order], [w.range_[i] for i in order],
                       [w.point[i] for i in order], [w.warp_factor[i] for i in order], 64, 4)
    rp = _park({"n": len(w.rows), "dynamical_orientation": True, "use_new_orbit": True}, "plain")
    rp.load(rev.rows)
    rev.apply(rp)
    for _ in range(30):
        full.evolve()
        one.evolve()
        _ticker(rp, "plain")()
    sf, so, sr = _state(full), _state(one), _state(rp)
    rows_rev = [inv[i] for i in sel]
    for f in COMPARE:
        if f == "follow_ptr":                     # a row index: the same target row, in each park's own rows
            fp = sf[f][28:32]
            assert (np.where(fp >= 0, fp - 28, -1) == so[f]).all()
            back = {new: old for old, new in inv.items()}
            assert ([back[r] if r >= 0 else -1 for r in sr[f][rows_rev]] == fp).all()
            continue
        assert bit_equal(sf[f][28:32], so[f]).all(), f
        assert bit_equal(sf[f][28:32], sr[f][rows_rev]).all(), f


def test_the_masked_tick_keeps_the_other_worlds():
    from exact_ballpark_b200.workloads import flight_worlds
    w = flight_worlds(44, 32, 4)
    a = _park({"n": len(w.rows), "dynamical_orientation": True, "use_new_orbit": True}, "tiled")
    a.load(w.rows)
    w.apply(a)
    before = _state(a)
    active = torch.zeros(len(w.rows), dtype=torch.bool, device="cuda")
    active[:64] = True
    a.evolve(active=active)
    after = _state(a)
    for f in COMPARE:
        assert bit_equal(after[f][64:], before[f][64:]).all(), f
    assert (after["clock"][:64] == before["clock"][:64] + 1).all()
