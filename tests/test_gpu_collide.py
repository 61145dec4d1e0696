"""The collision park on the GPU, through the C ABI (ebb_collide_load, ebb_collide_tick):

- against the golden traces recorded on the reference's collision park (its collide_cases scenarios, seeds 1 and 2, its
  static_cases scenarios with capsules and oriented boxes, seeds 1 and 2, and the collision benchmark's worlds): every
  field's digest after every tick, bit for bit;
- against the CPU oracle beyond the fixtures (the benchmark's worlds at other seeds, 1024 worlds, 150 ticks with the
  ships re-aimed): every field after every 25th tick; and on crowded worlds of 48 and 64 slots;
- a CUDA graph's replays against eager ticks, and inactive worlds (evolve(active)) keeping their state.
"""

import numpy as np
import pytest
import torch

import collide_trace as ct
from golden_util import bit_equal

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


@pytest.mark.parametrize("name", ["collide_cc1", "collide_cc2", "collide_w0", "collide_st1", "collide_st2",
                                  "collide_s0"])
def test_the_gpu_collision_park_replays_the_golden_trace(name):
    from exact_ballpark_b200 import VecCollidePark
    groups = ct.load(ct.GOLDEN / name)
    failures = []
    for gi, g in enumerate(groups):
        p = VecCollidePark(g["W"], g["N"], friction=g["friction"], tick_interval_ms=g["tick_interval_ms"],
                           statics=g.get("S", 0))
        bad = []

        def on_tick(k, park):
            mm = ct.first_mismatch(g, k, ct.field_digests(park))
            if mm and not bad:
                bad.append((k, mm))
        ct.replay(g, p, on_tick)
        p.check()
        if bad:
            failures.append((gi, bad[0]))
    assert not failures, f"{len(failures)} of {len(groups)} parks differ, first {failures[:3]}"


def _compare(o, p, where: str) -> None:
    for f in ct.FIELDS:
        a = np.asarray(getattr(o, f))
        b = getattr(p, f).detach().cpu().numpy()
        eq = bit_equal(a, b)
        if not eq.all():
            worlds = np.unique(np.nonzero(eq.reshape(eq.shape[0], -1).all(axis=1) == 0)[0])
            raise AssertionError(f"{where}: {f} differs in {len(worlds)} worlds, first {worlds[:5]}")


@pytest.mark.parametrize("seed", [7, 8])
def test_the_gpu_collision_tick_matches_the_oracle(seed):
    from exact_ballpark_b200 import VecCollidePark
    from exact_ballpark_b200.workloads import collide_worlds
    from oracle.collide_park import OracleCollidePark
    w = collide_worlds(seed, 1024, ticks=150)
    o = OracleCollidePark(1024, 16)
    p = VecCollidePark(1024, 16)
    o.load(w.worlds)
    p.load(w.worlds)
    for step in range(1, 151):
        w.apply(o, step)
        w.apply(p, step)
        o.evolve(threads=8)
        p.evolve()
        if step % 25 == 0 or step < 3:
            _compare(o, p, f"tick {step}")
    assert int(np.asarray(o.hits_n).sum()) > 0


@pytest.mark.parametrize("ships,spheres,fixed", [(8, 16, 24), (8, 24, 32)])
def test_the_gpu_collision_tick_matches_the_oracle_on_crowded_worlds(ships, spheres, fixed):
    """Worlds of 48 and 64 slots (the largest the park takes): blocks of 96 and 128 threads whose staged
    neighbourhoods and candidate tables take more than 48 KB of shared memory."""
    from exact_ballpark_b200 import VecCollidePark
    from exact_ballpark_b200.workloads import collide_worlds
    from oracle.collide_park import OracleCollidePark
    n = ships + spheres + fixed
    w = collide_worlds(11 + n, 256, ships=ships, spheres=spheres, statics=fixed, ticks=60, reaim=20)
    o = OracleCollidePark(256, n)
    p = VecCollidePark(256, n)
    o.load(w.worlds)
    p.load(w.worlds)
    for step in range(1, 61):
        w.apply(o, step)
        w.apply(p, step)
        o.evolve(threads=8)
        p.evolve()
        if step % 20 == 0 or step < 3:
            _compare(o, p, f"{n} slots, tick {step}")
    assert int(np.asarray(o.hits_n).sum()) > 0


def test_a_collision_graph_replays_the_eager_tick_and_inactive_worlds_keep_their_state():
    from exact_ballpark_b200 import CollideGraph, VecCollidePark
    from exact_ballpark_b200.workloads import collide_worlds
    w = collide_worlds(9, 256, ticks=40)
    a, b = VecCollidePark(256, 16), VecCollidePark(256, 16)
    a.load(w.worlds)
    b.load(w.worlds)
    g = CollideGraph(b)
    for step in range(1, 41):
        w.apply(a, step)
        w.apply(b, step)
        a.evolve()
        g.tick()
    torch.cuda.synchronize()
    for f in ct.FIELDS:
        assert bit_equal(getattr(a, f).cpu().numpy(), getattr(b, f).cpu().numpy()).all(), f
    before = {f: getattr(a, f).cpu().numpy().copy() for f in ct.FIELDS}
    active = torch.zeros(256, dtype=torch.bool)
    active[::3] = True
    a.evolve(active=active.cuda())
    after = {f: getattr(a, f).cpu().numpy() for f in ct.FIELDS}
    idle = ~active.numpy()
    for f in ct.FIELDS:
        assert bit_equal(after[f][idle], before[f][idle]).all(), f
    assert not np.array_equal(after["pos"][active.numpy()], before["pos"][active.numpy()])
