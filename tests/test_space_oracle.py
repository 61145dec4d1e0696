"""The CPU oracle of the master's partition and bubble partition of one world (oracle/space.cpp) against the golden
digests recorded on the reference's own SpaceBallpark (tests/golden/space_trace.py): 192 worlds (balls added near
top-box faces and corners, moved across top boxes, resized up to huge, removed and re-added, made interactive, kept
alive, cloaked; InitializeBubbles and CopyBubbles; sweeps past BoxAllocator's 256 kept boxes; the queries
GetNearbyBalls, CheckVisibility, GetBallIdsInRange from a ball or a point, GetBubbleAtCoordinates; proximity sensors
added (shuffled ones too, from the world's glibc rand) and removed, notification ranges in GOTO, tracked targets,
HandleProximities with its DoProximity, DoRange and DoTargetTracking events in the unordered maps' order; ticking
worlds whose ships fly GOTO legs across top boxes and bubbles: the flight tick of the free balls outside dead bubbles,
the re-filings of the balls that moved, HandleProximities; worlds of the follow, orbit and warp modes: FollowBall and
Orbit with the targets' follower sets in libstdc++'s order, WarpTo through alignment, warp proper and the drop-out
(re-filed at its drop-out point when nearly at rest there, massive again), StopAllFollowers when a target warps or is
removed, a re-added follower's kept target pointer); worlds of collisions inside the tick (Gradient at each massive
ball's turn in phase 3 over GetNearbyBalls' candidates, Potential's contacts with free and fixed balls, overlaps pushed
apart and recursed on, light balls, coincident centres, the latest contact kept), every state (each ball's mode, flight state and followers too)
and every answer after every operation. The first slice of the space layer: its kernel is built on this oracle."""

import numpy as np

import space_trace as sp
from oracle import space_world


def _scenarios():
    return sp.load(sp.GOLDEN / "space_bubbles")


def test_the_oracle_matches_the_references_partition_and_bubbles_after_every_operation():
    bad = []
    for sc in _scenarios():
        got = np.array([sp.digest(t) for t in space_world.run(sc["ops"], seed=sc["rand_seed"])], dtype=np.uint64)
        if got.shape != sc["digests"].shape or not (got == sc["digests"]).all():
            first = int(np.nonzero(got != sc["digests"])[0][0]) if got.shape == sc["digests"].shape else -1
            bad.append((sc["seed"], first))
    assert not bad, f"{len(bad)} worlds differ, first {bad[:3]}"


def test_the_streams_reach_the_partitions_paths():
    texts = [t for sc in _scenarios() for t in space_world.run(sc["ops"], seed=sc["rand_seed"])]
    kept = max(int(line.split()[1]) for t in texts for line in t.splitlines() if line.startswith("F "))
    assert kept == 256                                     # BoxAllocator full: later releases delete
    huge = sum(1 for t in texts for line in t.splitlines()
               if line.startswith("B ") and " - " not in line and bin(int(line.split()[11])).count("1") == 27)
    assert huge > 100                                      # huge balls in their 27 top boxes
    bubbles = max(int(line.split()[2]) for t in texts for line in t.splitlines() if line.startswith("F "))
    assert bubbles >= 5
    assert any(" -1:" in t or ":-1" in t for t in texts)   # a ball leaving a bubble before CopyBubbles
    answers = [t.splitlines()[-1] for t in texts if t.splitlines()[-1].startswith("Q")]
    assert len(answers) > 300
    assert sum(1 for a in answers if len(a.split()) > 2) > 50         # answers listing several balls
    assert any(":" in a for a in answers) and any(a == "Q None" for a in answers)
    assert any(a.split()[1:] and a.split()[1].isdigit() and int(a.split()[1]) > 0 for a in answers if len(a.split()) == 2)
    events = [e for a in answers for e in a.split()[1:] if e.count(":") == 2]
    assert sum(e.endswith(":1") for e in events) > 100 and sum(e.endswith(":0") for e in events) > 10
    assert any(line.startswith("S ") and len(line.split()) > 9 for t in texts for line in t.splitlines())
    assert any(e.startswith("R") for a in answers for e in a.split()[1:])
    assert any(e.startswith("T") for a in answers for e in a.split()[1:])
    ticking = [sc for sc in _scenarios() if sc["seed"].startswith("tick")]
    assert len(ticking) == 40 and sum(int((sc["ops"][:, 0] == sp.TICK).sum()) for sc in ticking) > 1000


def test_a_planted_fault_in_the_operations_is_seen():
    sc = _scenarios()[0]
    ops = sc["ops"].copy()
    k = next(i for i in range(len(ops)) if int(ops[i, 0]) == sp.ADD)
    ops[k, 7] += sp.TOP                                    # one ball added a top box further along x
    got = np.array([sp.digest(t) for t in space_world.run(ops, seed=sc["rand_seed"])], dtype=np.uint64)
    assert not (got == sc["digests"]).all()


def test_the_mode_worlds_reach_the_modes_paths():
    scs = [sc for sc in _scenarios() if sc["seed"].startswith("modes")]
    assert len(scs) == 40
    modes = [line.split() for sc in scs for t in space_world.run(sc["ops"], seed=sc["rand_seed"])
             for line in t.splitlines() if line.startswith("M ")]
    seen = {int(m[2]) for m in modes}
    assert {0, 1, 2, 3, 4} <= seen                         # GOTO, FOLLOW, STOP, WARP, ORBIT
    assert sum(1 for m in modes if m[-1] != ":") > 200     # balls with followers
    assert any(len(m) > 13 for m in modes)                 # a set of several followers, in its order
    assert any(m[2] == "2" and m[4] != "0" for m in modes)  # a stopped ball still pointing at its old target
    assert any(m[2] == "2" and m[3] == "1" for m in modes)  # massive again after a warp's drop-out


def test_a_planted_fault_in_a_warp_is_seen():
    sc = next(sc for sc in _scenarios() if sc["seed"].startswith("modes"))
    ops = sc["ops"].copy()
    k = next(i for i in range(len(ops)) if int(ops[i, 0]) == sp.WARP)
    ops[k, 2] += 1.0e6                                     # the warp's destination 1,000 km further along x
    got = np.array([sp.digest(t) for t in space_world.run(ops, seed=sc["rand_seed"])], dtype=np.uint64)
    assert not (got == sc["digests"]).all()


def test_collisions_inside_the_tick_change_the_worlds():
    scs = [sc for sc in _scenarios() if sc["seed"].startswith("collide")]
    assert len(scs) == 40
    changed = 0
    for sc in scs[:10]:
        ops = sc["ops"].copy()
        ops[ops[:, 0] == sp.ADD, 15] = 0.0                 # every ball added non-massive: no Gradient at all
        got = np.array([sp.digest(t) for t in space_world.run(ops, seed=sc["rand_seed"])], dtype=np.uint64)
        changed += not (got == sc["digests"]).all()
    assert changed >= 8


def test_the_oracle_matches_the_reference_in_crowded_sensing_worlds():
    """Worlds of 16 to 128 sensing ships (config 3's shape at a golden's size): each sensor's list and the proximity
    map grow past 13, 29, 59 and 127 keys, so the unordered maps' order follows the rehash policy's growths (13, 29,
    59, 127 and 257 buckets), every state and every tick's events digested against the reference's."""
    scs = sp.load(sp.GOLDEN / "space_crowd")
    assert len(scs) == 8
    longest = 0
    for sc in scs:
        texts = space_world.run(sc["ops"], seed=sc["rand_seed"])
        got = np.array([sp.digest(t) for t in texts], dtype=np.uint64)
        assert (got == sc["digests"]).all(), (sc["seed"], int(np.nonzero(got != sc["digests"])[0][0]))
        longest = max([longest] + [len(line.split()) - 8 for t in texts for line in t.splitlines()
                                   if line.startswith("S ")])
    assert longest == 127                                  # a list past 59 keys: 127 buckets, then 257
