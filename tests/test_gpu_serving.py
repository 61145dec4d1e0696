"""The listed-worlds tick, the row move and the serving loop on the GPU, through the C ABI:

- the listed-worlds tick over a park's own worlds equals the tiled tick, bit for bit; with OnTick's row mask inside
  the kernel it equals the reference's masked tick (every row ticked, the rows outside the mask put back);
- moving rows between parks keeps every field and moves follow pointers with their world;
- each episode served in a mix (continuous batching, admission as rows free up, holes left by finished episodes
  reused) ends bit for bit as the same episode run alone in its own park, and as the CPU oracle runs it alone.
"""

import numpy as np
import pytest
import torch

from golden_util import bit_equal

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]

COMPARE = ("pos", "vel", "old_pos", "old_vel", "goto", "last_g", "ang_vel", "old_ang_vel", "torque", "rot", "old_rot",
           "speed_fraction", "follow_range", "last_collision", "rot_roll", "mode", "effect_stamp", "follow_id",
           "owner_id", "follow_ptr", "clock", "free", "massive", "interactive", "sensor")


def _ragged(seed: int, worlds: int, max_ships: int):
    import random
    from exact_ballpark_b200.workloads import FlightWorlds, flight_worlds, ragged_ships
    r = random.Random(seed)
    return FlightWorlds.concat([flight_worlds(seed * 100 + k, 1, ragged_ships(r, max_ships)) for k in range(worlds)])


def _loaded(w, do=True, new_orbit=True):
    from exact_ballpark_b200 import VecModesPark
    p = VecModesPark(len(w.rows), device="cuda", dynamical_orientation=do, use_new_orbit=new_orbit)
    p.load(w.rows)
    w.apply(p)
    return p


def _state(p) -> dict:
    return {f: getattr(p, f).detach().cpu().numpy().copy() for f in COMPARE}


def _same_states(a: dict, b: dict, where: str) -> None:
    for f in COMPARE:
        eq = bit_equal(a[f], b[f])
        if not eq.all():
            rows = np.unique(np.nonzero(eq.reshape(eq.shape[0], -1).all(axis=1) == 0)[0])
            raise AssertionError(f"{where}: {f} differs in {len(rows)} rows, first {rows[:5]}")


@pytest.mark.parametrize("cap,block,grid", [(256, 256, None), (128, 256, None), (512, 128, None), (256, 128, 7),
                                            (128, 128, 5)])
def test_the_listed_worlds_tick_equals_the_tiled_and_plain_ticks(cap, block, grid):
    """Both forms of each tiled kernel: one tile a block of at most `block` rows, and the persistent grid with
    several rounds of ships a tile."""
    from exact_ballpark_b200 import tick_plain, tick_tiled, tick_worlds
    from exact_ballpark_b200.tiles import plan_tiles
    w = _ragged(3, 600, 64)
    a, b, c = _loaded(w), _loaded(w), _loaded(w)
    plan = plan_tiles(a.world, cap=cap, block=block, grid=grid)
    assert plan is not None
    for _ in range(30):
        tick_tiled(a, plan)
        tick_worlds(b, None, plan)
        tick_plain(c)
    torch.cuda.synchronize()
    sc = _state(c)
    _same_states(_state(a), sc, "tiled after 30 ticks")
    _same_states(_state(b), sc, "listed worlds after 30 ticks")
    assert int(a._status.item()) == 0 and int(b._status.item()) == 0


@pytest.mark.parametrize("per_world", [True, False])
def test_the_in_kernel_mask_equals_the_put_back(per_world):
    """OnTick's mask inside the listed-worlds kernel against the reference's form (tick every row, give the rows
    outside the mask their state back): per-world masks, and row masks that split worlds."""
    from exact_ballpark_b200 import tick_plain
    from exact_ballpark_b200.modes import masked_tick
    w = _ragged(4, 300, 24)
    a, b = _loaded(w), _loaded(w)
    g = torch.Generator().manual_seed(11)
    world = torch.tensor([r["world"] for r in w.rows])
    for k in range(25):
        if per_world:
            on = torch.rand(w.worlds, generator=g) < 0.6
            act = on[world].cuda()
        else:
            act = (torch.rand(len(w.rows), generator=g) < 0.6).cuda()
        a.evolve(active=act)                                   # in the kernel
        masked_tick(b, act, lambda: tick_plain(b))             # tick everything, put the others back
        b.current_time += 1
    torch.cuda.synchronize()
    _same_states(_state(a), _state(b), "after 25 masked ticks")


def test_a_masked_graph_uses_the_kernel_mask_and_equals_eager():
    from exact_ballpark_b200 import ModesGraph
    w = _ragged(5, 200, 16)
    a, b = _loaded(w), _loaded(w)
    g = ModesGraph(b, masked=True)
    assert g.in_kernel
    gen = torch.Generator().manual_seed(2)
    world = torch.tensor([r["world"] for r in w.rows])
    for _ in range(20):
        act = (torch.rand(w.worlds, generator=gen) < 0.5)[world].cuda()
        a.evolve(active=act)
        g.tick(act)
    torch.cuda.synchronize()
    _same_states(_state(a), _state(b), "graph vs eager")


def test_moving_rows_keeps_every_field_and_moves_targets():
    from exact_ballpark_b200.serving import Rows, move_rows
    w = _ragged(6, 40, 12)
    p = _loaded(w)
    for _ in range(5):
        p.evolve()
    out = Rows(p.n + 100, p)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    src = torch.arange(p.n, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    move_rows(out, p, src, src + 77, status, stream)
    back = _loaded(w)
    move_rows(back, out, src + 77, src, status, stream)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    fp = out.field("follow_ptr", 77, p.n).cpu().numpy()
    pf = p.follow_ptr.cpu().numpy()
    assert (np.where(pf >= 0, pf + 77, -1) == fp).all()
    _same_states(_state(p), _state(back), "moved out and back")


def _served(episodes, rows: int, **kw):
    from exact_ballpark_b200.serving import Server, serve
    srv = Server(rows=rows, max_ships=max(e.ships for e in episodes), **kw)
    try:
        summary = serve(srv, episodes, realtime=False)
    finally:
        srv.close()
    return srv, summary


def _alone(ep) -> dict:
    from exact_ballpark_b200 import tick_plain
    p = _loaded(ep.world)
    for _ in range(ep.ticks):
        tick_plain(p)
    torch.cuda.synchronize()
    return _state(p)


def _result_state(res) -> dict:
    return {f: res.field(f).detach().cpu().numpy().copy() for f in COMPARE}


def test_each_served_episode_equals_the_episode_alone():
    """30 episodes of 1-48 ships and 2-60 ticks through a 200-row server: most wait for rows, finished episodes leave
    holes that later ones fill, and every tick runs a different mix."""
    from exact_ballpark_b200.serving import episode_stream
    eps = episode_stream(17, 30, rate=0.0, max_ships=48, min_ticks=2, max_ticks=60)
    srv, summary = _served(eps, rows=200, tile_cap=128, stage_rows=64)
    assert summary["admitted"] == summary["retired"] == len(eps)
    assert summary["steps"] > max(e.ticks for e in eps)
    assert len(srv.results) == len(eps)
    for ep in eps:
        res = _result_state(srv.results[ep.eid])
        alone = _alone(ep)
        start = srv.results[ep.eid].start
        res["follow_ptr"] = np.where(res["follow_ptr"] >= 0, res["follow_ptr"] - start, -1)
        _same_states(res, alone, f"episode {ep.eid} ({ep.ships} ships, {ep.ticks} ticks)")


def test_served_episodes_match_the_oracle_alone():
    from exact_ballpark_b200.serving import episode_stream
    from oracle.park import OraclePark
    eps = episode_stream(23, 12, rate=0.0, max_ships=32, min_ticks=5, max_ticks=40)
    srv, _ = _served(eps, rows=120, tile_cap=64)
    for ep in eps:
        o = OraclePark(ep.ships, dynamical_orientation=True, use_new_orbit=True)
        o.load(ep.world.rows)
        ep.world.apply(o)
        for _ in range(ep.ticks):
            o.evolve()
        res = _result_state(srv.results[ep.eid])
        start = srv.results[ep.eid].start
        res["follow_ptr"] = np.where(res["follow_ptr"] >= 0, res["follow_ptr"] - start, -1)
        want = {f: np.asarray(getattr(o, f)) for f in COMPARE}
        _same_states(res, want, f"episode {ep.eid} against the oracle")


def test_served_episodes_of_129_to_256_ships_match_the_oracle_alone():
    """Config 4's largest episodes: 129 to 256 ships a world (tiles of up to 1024 rows, several rounds of ships a
    thread block), each against the oracle run alone."""
    from exact_ballpark_b200.serving import episode_stream
    from oracle.park import OraclePark
    eps = episode_stream(41, 8, rate=0.0, max_ships=256, min_ships=129, min_ticks=5, max_ticks=25)
    assert min(e.ships for e in eps) >= 129 and max(e.ships for e in eps) > 200
    srv, summary = _served(eps, rows=1200, tile_cap=1024)
    assert summary["admitted"] == summary["retired"] == len(eps)
    for ep in eps:
        o = OraclePark(ep.ships, dynamical_orientation=True, use_new_orbit=True)
        o.load(ep.world.rows)
        ep.world.apply(o)
        for _ in range(ep.ticks):
            o.evolve()
        res = _result_state(srv.results[ep.eid])
        start = srv.results[ep.eid].start
        res["follow_ptr"] = np.where(res["follow_ptr"] >= 0, res["follow_ptr"] - start, -1)
        want = {f: np.asarray(getattr(o, f)) for f in COMPARE}
        _same_states(res, want, f"episode {ep.eid} ({ep.ships} ships) against the oracle")


def test_open_loop_arrivals_are_served_and_timed():
    """Arrivals in wall time (an open loop): every episode is served and each step's latency is recorded."""
    from exact_ballpark_b200.serving import episode_stream
    from exact_ballpark_b200.serving import Server, serve
    eps = episode_stream(29, 60, rate=5000.0, max_ships=64, min_ticks=5, max_ticks=50)
    srv = Server(rows=4096, max_ships=64, tile_cap=256)
    try:
        summary = serve(srv, eps, realtime=True)
    finally:
        srv.close()
    assert summary["admitted"] == summary["retired"] == 60
    assert summary["p99_ms"] >= summary["p50_ms"] > 0
    for ep in eps[:10]:
        res = _result_state(srv.results[ep.eid])
        start = srv.results[ep.eid].start
        res["follow_ptr"] = np.where(res["follow_ptr"] >= 0, res["follow_ptr"] - start, -1)
        _same_states(res, _alone(ep), f"episode {ep.eid}")


def test_a_best_fit_plan_ticks_as_the_plain_schedule():
    """Tiles of any whole worlds (not only neighbours), packed best fit by ebb_plan_worlds."""
    from exact_ballpark_b200 import tick_plain, tick_worlds
    from exact_ballpark_b200.tiles import plan_best_fit
    w = _ragged(8, 700, 128)
    a, c = _loaded(w), _loaded(w)
    plan = plan_best_fit(a.world, cap=256, block=256)
    assert plan is not None and plan.tiles < len(w.rows) // 128
    for _ in range(25):
        tick_worlds(a, None, plan)
        tick_plain(c)
    torch.cuda.synchronize()
    _same_states(_state(a), _state(c), "best fit after 25 ticks")
    assert int(a._status.item()) == 0
