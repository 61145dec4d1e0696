"""The combat park on the GPU, through the C ABI (ebb_combat_tick) and the park's commands, against the golden
traces recorded on the reference's combat park (tests/golden/combat_trace.py): the reference's combat scenarios with
dynamical orientation (seed 1 development, seed 2 held out; missiles launched aimed and unaimed, at cloaked, removed
and warping targets, MissileFollow's refusals, formations reserved, followed, resized, left and freed, cloaks and
uncloaks, removals, velocity and massive setters, master and client, the missile exclusion of dynamical orientation
on and off): every field's digest after every step over the rows holding a ball, the DoCollision events and the
ReserveFormationSlot answers, bit for bit."""

import pytest
import torch

import combat_trace as ct

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


@pytest.mark.parametrize("seed", [1, 2], ids=["development", "held_out"])
def test_the_gpu_combat_park_replays_the_golden_batches(seed):
    from exact_ballpark_b200 import VecCombatPark
    formations, batches = ct.load(ct.GOLDEN / f"combat_{seed}")
    failures = []
    for bi, b in enumerate(batches):
        p, where = ct.make_park(VecCombatPark, b["cfg"], formations, "cuda")
        bad = ct.replay(p, b, where)
        p.check()
        if bad:
            failures.append((bi, bad[:2]))
    assert not failures, f"{len(failures)} of {len(batches)} batches differ, first {failures[:2]}"


@pytest.mark.parametrize("block", [128, 256])
def test_the_gpu_combat_park_matches_the_oracle_on_the_benchmark_worlds(block):
    """The combat benchmark's worlds (workloads.combat_worlds: 4 ships and 4 missiles launched aimed and massive, ships
    following, orbiting, flying to points, in formation) at 512 worlds, 60 ticks: every field of every row holding a
    ball after every 10th tick and every tick's events, GPU against the CPU oracle; then a CUDA graph's replays
    against eager ticks, bit for bit."""
    from exact_ballpark_b200 import CombatGraph, VecCombatPark
    from exact_ballpark_b200.workloads import combat_worlds
    from oracle.combat_park import OracleCombatPark
    w = combat_worlds(7, 512)
    n = len(w.rows)
    g = VecCombatPark(n, device="cuda", dynamical_orientation=True, use_new_orbit=True, block=block)
    o = OracleCombatPark(n, dynamical_orientation=True, use_new_orbit=True)
    for p in (g, o):
        p.load(w.rows)
        w.apply(p)
    events = 0
    for k in range(1, 61):
        g.evolve()
        o.evolve()
        ge, oe = g.events(), o.events()
        assert ge == oe, f"tick {k}: events differ"
        events += len(ge)
        if k % 10 == 0:
            want, got = ct.field_digests(o), ct.field_digests(g)
            assert not ct.first_mismatch(want, got), f"tick {k}: {ct.first_mismatch(want, got)}"
    g.check()
    assert events > 1000
    h = VecCombatPark(n, device="cuda", dynamical_orientation=True, use_new_orbit=True, block=block)
    h.load(w.rows)
    w.apply(h)
    e = VecCombatPark(n, device="cuda", dynamical_orientation=True, use_new_orbit=True, block=block)
    e.load(w.rows)
    w.apply(e)
    graph = CombatGraph(h)
    for k in range(20):
        graph.tick()
        e.evolve()
        assert h.events() == e.events()
    assert not ct.first_mismatch(ct.field_digests(e), ct.field_digests(h))


def _masked_against_put_back(park_cls, worlds_fn, fields):
    """OnTick's per-world mask inside the kernel against the reference's semantics (tick every world, then give the
    rows outside the mask back their state): 30 ticks, a different half of the worlds each tick, every field and the
    ticked worlds' events."""
    import torch
    from exact_ballpark_b200.modes import masked_tick
    w = worlds_fn()
    n = len(w.rows)
    a = park_cls(n, device="cuda", dynamical_orientation=True, use_new_orbit=True)
    b = park_cls(n, device="cuda", dynamical_orientation=True, use_new_orbit=True)
    for p in (a, b):
        p.load(w.rows)
        w.apply(p)
    world = a.world
    g = torch.Generator(device="cpu").manual_seed(5)
    for k in range(30):
        on = torch.rand(int(world.max()) + 1, generator=g) < 0.5
        act = on.to(world.device)[world]
        a.evolve(active=act)
        got = a.events()
        want = []
        masked_tick(b, act, lambda: (b.evolve(), want.extend(e for e in b.events() if bool(on[e[0]]))))
        assert got == want, f"tick {k}: events differ"
        assert not ct.first_mismatch(ct.field_digests(b, fields), ct.field_digests(a, fields), fields), \
            f"tick {k}: {ct.first_mismatch(ct.field_digests(b, fields), ct.field_digests(a, fields), fields)}"


def test_the_combat_parks_masked_tick_is_the_put_back():
    from exact_ballpark_b200 import VecCombatPark
    from exact_ballpark_b200.workloads import combat_worlds
    _masked_against_put_back(VecCombatPark, lambda: combat_worlds(13, 256), ct.FIELDS)
