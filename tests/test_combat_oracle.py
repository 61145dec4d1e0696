"""The CPU oracle of the combat park (oracle/combat_park.py's commands, oracle/flight.cpp's sequential tick with its
combat state) against the golden batches recorded on the reference's combat park (tests/golden/combat_trace.py: its
combat scenarios with dynamical orientation, seed 1 development, seed 2 held out): every field's digest after every
step over the rows holding a ball, the DoCollision events and the ReserveFormationSlot answers, bit for bit. A planted
fault is caught."""

import numpy as np
import pytest

import combat_trace as ct


@pytest.mark.parametrize("seed", [1, 2], ids=["development", "held_out"])
def test_the_oracle_replays_the_golden_combat_batches(seed):
    from oracle.combat_park import OracleCombatPark
    formations, batches = ct.load(ct.GOLDEN / f"combat_{seed}")
    failures = []
    for bi, b in enumerate(batches):
        p, where = ct.make_park(OracleCombatPark, b["cfg"], formations, "cpu")
        bad = ct.replay(p, b, where)
        if bad:
            failures.append((bi, bad[:2]))
    assert not failures, f"{len(failures)} of {len(batches)} batches differ, first {failures[:2]}"
    assert sum(len(b["events"]) for b in batches) > 100


def test_a_planted_fault_in_the_oracle_is_caught():
    from oracle.combat_park import OracleCombatPark
    formations, batches = ct.load(ct.GOLDEN / "combat_1")
    b = batches[1]
    p, where = ct.make_park(OracleCombatPark, b["cfg"], formations, "cpu")

    def tick(q):                                    # one ulp on a missile's position after its fourth tick
        q.evolve()
        if q.current_time == 4:
            rows = np.nonzero(q.exists & (q.mode == 5))[0]
            r = int(rows[0]) if len(rows) else int(np.nonzero(q.exists)[0][0])
            q.pos[r, 0] = np.nextafter(q.pos[r, 0], np.inf)
    bad = ct.replay(p, b, where, tick=tick)
    assert bad and bad[0][0] == 4 and "pos" in bad[0][1]


@pytest.mark.parametrize("seed", [1, 2], ids=["development", "held_out"])
def test_the_oracle_replays_the_golden_composed_batches(seed):
    """The composed park's oracle (the sequential tick: each massive ball's Gradient at its own turn) against the
    golden batches recorded on the reference's composed park: every field with the collision acceleration, the
    filing and the collision list, every step; the events and the slot answers."""
    from oracle.composed_park import OracleComposedPark
    formations, batches = ct.load(ct.GOLDEN / f"composed_{seed}")
    failures = []
    for bi, b in enumerate(batches):
        p, where = ct.make_park(OracleComposedPark, b["cfg"], formations, "cpu")
        bad = ct.replay(p, b, where, fields=ct.COMPOSED_FIELDS)
        if bad:
            failures.append((bi, bad[:2]))
    assert not failures, f"{len(failures)} of {len(batches)} batches differ, first {failures[:2]}"
    assert sum(len(b["events"]) for b in batches) > 400
