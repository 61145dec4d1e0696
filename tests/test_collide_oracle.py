"""The CPU oracle of the collision park (oracle/collide.cpp, oracle/collide_park.py) against the golden traces recorded
on the reference's batched collision park (tests/golden/collide_trace.py): the reference's collide_cases scenarios
(seed 1 development, seed 2 held out: approaching, glancing, overlapping and coincident balls, light balls, fixed
spheres as walls and fields, several contacts in a tick, near misses, chains, fast balls, balls on partition box faces,
space junk, cloaked and non-massive neighbours, racers with throttle and stop commands; ticks of 0.25 to 2 s, several
frictions), its static_cases scenarios (capsules and oriented boxes: ships through, at and along them, grazing, inside,
at rest beside, backing into them; faces, edges and corners of aligned, rotated, skewed and flat boxes; a box wider than
a top box; fields and clusters with racers; several static collidables touched in one tick) and the collision
benchmark's worlds (64 worlds of 4 ships, 4 free and 8 fixed spheres; and 64 worlds of 4 ships, 4 fixed spheres and 8
capsules and boxes; 100 ticks each; and crowded worlds of 48 and 64 slots, 60 ticks). Every field's digest after every
tick, bit for bit; a planted fault is caught. The static collidables' records (exact_ballpark_b200.statics) against the
reference park's own records, double for double."""

import numpy as np
import pytest

import collide_trace as ct

TRACES = ("collide_cc1", "collide_cc2", "collide_w0", "collide_st1", "collide_st2", "collide_s0", "collide_crowd")


def _replay(g, park, plant=None) -> list:
    bad = []

    def on_tick(k, p):
        if plant is not None:
            plant(k, p)
        mm = ct.first_mismatch(g, k, ct.field_digests(p))
        if mm and not bad:
            bad.append((k, mm))
    ct.replay(g, park, on_tick)
    return bad


@pytest.mark.parametrize("name", TRACES)
def test_the_oracle_replays_the_golden_collision_trace(name):
    from oracle.collide_park import OracleCollidePark
    groups = ct.load(ct.GOLDEN / name)
    failures = []
    for gi, g in enumerate(groups):
        p = OracleCollidePark(g["W"], g["N"], friction=g["friction"], tick_interval_ms=g["tick_interval_ms"],
                              statics=g.get("S", 0))
        bad = _replay(g, p)
        if bad:
            failures.append((gi, bad[0]))
    assert not failures, f"{len(failures)} of {len(groups)} parks differ, first {failures[:3]}"


def test_the_benchmark_worlds_collide_and_a_planted_fault_is_caught():
    from oracle.collide_park import OracleCollidePark
    g = ct.load(ct.GOLDEN / "collide_w0")[0]
    p = OracleCollidePark(g["W"], g["N"], friction=g["friction"], tick_interval_ms=g["tick_interval_ms"])
    hits = []
    assert not _replay(g, p, plant=lambda k, q: hits.append(int(q.hits_n.sum())))
    assert sum(hits) > 100 and sum(1 for h in hits if h) > 50           # contacts in most ticks

    def plant(k, q):                                                     # one ulp on a ship's velocity after tick 10
        if k == 10:
            q.vel[5, 0, 0] = np.nextafter(q.vel[5, 0, 0], np.inf)
    p = OracleCollidePark(g["W"], g["N"], friction=g["friction"], tick_interval_ms=g["tick_interval_ms"])
    bad = _replay(g, p, plant=plant)
    assert bad and bad[0][0] == 10 and "vel" in bad[0][1]


@pytest.mark.parametrize("name", ["collide_st1", "collide_st2"])
def test_the_static_records_are_the_references(name):
    from exact_ballpark_b200.statics import static_record
    n = 0
    for g in ct.load(ct.GOLDEN / name):
        f = g["filing"]
        for w, items in enumerate(g["statics"]):
            for j, item in enumerate(items):
                geo, ints, keys = static_record(item)
                assert (np.asarray(geo).view(np.uint64) == f["s_geo"][w, j].view(np.uint64)).all()
                assert list(ints) == f["s_int"][w, j].tolist()
                assert [list(k) for k in keys] == f["s_keys"][w, j][:ints[4]].tolist()
                n += 1
    assert n > 250
