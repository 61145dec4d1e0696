"""The composed park on the GPU, through the C ABI (ebb_composed_tick, ebb_composed_file) and the park's commands,
against the golden batches recorded on the reference's composed park (tests/golden/combat_trace.py with the
composed fields): the reference's composed scenarios with dynamical orientation (tests/park_cases.py; seed 1
development, seed 2 held out: ship clusters with fixed spheres meeting by the gradient method, FOLLOW and ORBIT at short
range, warps into the cluster dropping out among the others, the setters that re-file, cloaks, formations, missiles
launched at the ships): every field's digest after every step over the rows holding a ball (the collision
acceleration, the partition's filing and the collision list included), the DoCollision events and the
ReserveFormationSlot answers, bit for bit."""

import pytest
import torch

import combat_trace as ct

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


@pytest.mark.parametrize("seed", [1, 2], ids=["development", "held_out"])
def test_the_gpu_composed_park_replays_the_golden_batches(seed):
    from exact_ballpark_b200 import VecComposedPark
    formations, batches = ct.load(ct.GOLDEN / f"composed_{seed}")
    failures = []
    for bi, b in enumerate(batches):
        p, where = ct.make_park(VecComposedPark, b["cfg"], formations, "cuda")
        bad = ct.replay(p, b, where, fields=ct.COMPOSED_FIELDS)
        p.check()
        if bad:
            failures.append((bi, bad[:2]))
    assert not failures, f"{len(failures)} of {len(batches)} batches differ, first {failures[:2]}"


@pytest.mark.parametrize("block", [128, 256])
def test_the_gpu_composed_park_matches_the_oracle_on_the_benchmark_worlds(block):
    """The composed benchmark's worlds (workloads.composed_worlds: 6 massive ships, 1 fixed sphere and 2 missiles
    launched aimed and massive a world, within 5 km) at 512 worlds, 60 ticks: every composed field of every row
    holding a ball after every 10th tick and every tick's events, GPU against the sequential CPU oracle; then a CUDA
    graph's replays against eager ticks, bit for bit."""
    from exact_ballpark_b200 import CombatGraph, VecComposedPark
    from exact_ballpark_b200.workloads import composed_worlds
    from oracle.composed_park import OracleComposedPark
    w = composed_worlds(9, 512)
    n = len(w.rows)
    g = VecComposedPark(n, device="cuda", dynamical_orientation=True, use_new_orbit=True, block=block)
    o = OracleComposedPark(n, dynamical_orientation=True, use_new_orbit=True)
    for p in (g, o):
        p.load(w.rows)
        w.apply(p)
    events = contacts = 0
    for k in range(1, 61):
        g.evolve()
        o.evolve()
        ge, oe = g.events(), o.events()
        assert ge == oe, f"tick {k}: events differ"
        events += len(ge)
        contacts += int(o.hits_n.sum())
        if k % 10 == 0:
            want, got = ct.field_digests(o, ct.COMPOSED_FIELDS), ct.field_digests(g, ct.COMPOSED_FIELDS)
            assert not ct.first_mismatch(want, got, ct.COMPOSED_FIELDS), \
                f"tick {k}: {ct.first_mismatch(want, got, ct.COMPOSED_FIELDS)}"
    g.check()
    assert events > 100 and contacts > 1000
    h = VecComposedPark(n, device="cuda", dynamical_orientation=True, use_new_orbit=True, block=block)
    e = VecComposedPark(n, device="cuda", dynamical_orientation=True, use_new_orbit=True, block=block)
    for p in (h, e):
        p.load(w.rows)
        w.apply(p)
    graph = CombatGraph(h)
    for _ in range(20):
        graph.tick()
        e.evolve()
        assert h.events() == e.events()
    assert not ct.first_mismatch(ct.field_digests(e, ct.COMPOSED_FIELDS), ct.field_digests(h, ct.COMPOSED_FIELDS),
                                 ct.COMPOSED_FIELDS)


def test_the_composed_parks_masked_tick_is_the_put_back():
    from exact_ballpark_b200 import VecComposedPark
    from exact_ballpark_b200.workloads import composed_worlds
    from test_gpu_combat import _masked_against_put_back
    _masked_against_put_back(VecComposedPark, lambda: composed_worlds(13, 256), ct.COMPOSED_FIELDS)
