"""The space layer (exact_ballpark_b200.space over csrc/ebb_space.cuh) against the oracle (oracle/space.cpp, held to
the reference's own SpaceBallpark by tests/test_space_oracle.py): the golden streams of tests/golden/space_bubbles.npz
(mixed operations, long streams, the sweeps past BoxAllocator's 256 kept boxes) driven through the layer, one world a
stream, and after every operation each ball's filing, bubble and old bubble, the dead-bubble flag, the live boxes per
level, BoxAllocator's kept count, the next bubble id, the bubble dictionaries in their order and the interactive and
keep-alive sets compared with the oracle's state text of the same operations; and the ticking and mode streams through
the layer's tick (the dead rows skipped by the park's tick, the drop-outs' and the commits' re-filings after it). The streams' sensor operations are left
out on both sides (the sensors are not in the layer's slice). On the CPU the layer's per-world program runs as its
host build (tests/native/space_host.cpp, the same source); on a GPU the product's VecSpace runs it, one CUDA thread a
world, and must give the same texts and the same state, word for word."""

import numpy as np
import pytest

import space_layer as sl
import space_trace as sp
from oracle import space_world

FAMILIES = ("mixed", "long", "sweep")
HUGE = 256                                                 # EBB_SPACE_FLAG_HUGE: a sensor meeting a huge ball


def _streams(families=FAMILIES):
    return [sc for sc in sp.load(sp.GOLDEN / "space_bubbles") if sc["seed"].split("-")[0] in families]


def _oracle_texts(sc):
    return [sl.oracle_lines(t, int(op[0])) for t, op in zip(space_world.run(sc["ops"], seed=sc["rand_seed"]),
                                                            sc["ops"])]


def _inputs(scs):
    return [(sc["ops"], sc["rand_seed"]) for sc in scs]


@pytest.mark.parametrize("world_major", [False, True])
def test_the_layers_program_matches_the_oracle_after_every_operation(world_major):
    """The host build over the interleaved state and over the world-major arena."""
    scs = _streams()
    assert len(scs) == 72
    texts, flags = sl.drive(_inputs(scs), "host", world_major=world_major)
    assert not (flags & ~HUGE).any()
    bad = []
    for sc, got in zip(scs, texts):
        want = _oracle_texts(sc)
        if got != want:
            bad.append((sc["seed"], next(i for i, (x, y) in enumerate(zip(want, got)) if x != y)))
    assert not bad, f"{len(bad)} worlds differ, first {bad[:3]}"


def test_the_streams_reach_the_layers_paths():
    scs = _streams()
    texts, _ = sl.drive(_inputs(scs), "host")
    lines = [line for t in texts for text in t for line in text.splitlines()]
    assert max(int(x.split()[1]) for x in lines if x.startswith("F ")) == 256   # BoxAllocator full, later deletions
    assert sum(1 for x in lines if x.startswith("B ") and " - " not in x and int(x.split()[11]) == (1 << 27) - 1) > 100
    assert max(int(x.split()[2]) for x in lines if x.startswith("F ")) >= 5      # bubbles made and joined
    assert any(":-1" in x for x in lines if x.startswith("U "))                 # a ball that left, before CopyBubbles
    assert any(x.startswith("K ") for x in lines) and any(x.startswith("I ") for x in lines)


def test_a_planted_fault_in_the_oracle_is_seen():
    sc = _streams(("mixed",))[0]
    texts, _ = sl.drive(_inputs([sc]), "host")
    ops = sc["ops"].copy()
    k = next(i for i in range(len(ops)) if int(ops[i, 0]) == sp.ADD)
    ops[k, 7] += sp.TOP                                    # the oracle's ball added a top box further along x
    want = [sl.oracle_lines(t, int(op[0])) for t, op in zip(space_world.run(ops, seed=sc["rand_seed"]), ops)]
    assert texts[0] != want


def test_a_full_box_table_flags_the_world_and_leaves_it_alone():
    sc = _streams(("sweep",))[0]
    park = sl.HostPark(40)
    park.ids[:] = np.arange(1, 41)
    layer = sl.HostLayer(1, 40, boxes=8)
    flagged_at = None
    for k, op in enumerate(sc["ops"][:200]):
        code, a, b, f = sl.translate(park, 0, op, 40)
        layer.tape(park, [code], [a], [b], np.asarray(f).reshape(1, 4, 1))
        if layer.st["flags"][0] and flagged_at is None:
            flagged_at = k
            frozen = {n: v.copy() for n, v in layer.st.items()}
    assert flagged_at is not None and layer.st["flags"][0] & 8                  # EBB_SPACE_FLAG_BOXES
    assert all((layer.st[n] == frozen[n]).all() for n in frozen)                # nothing ran after the flag


def _crowd():
    return sp.load(sp.GOLDEN / "space_crowd")


def test_the_layers_tick_matches_the_oracle_in_crowded_sensing_worlds_on_the_cpu():
    """16 to 128 sensing ships a world: the sensors' lists and the proximity map past every growth of the rehash
    policy, thousands of DoProximity events a world; the layer's host build around the flight oracle's tick."""
    bad = []
    for sc in _crowd():
        got = sl.drive_ticks_host(sc["ops"], sc["rand_seed"])
        want = _oracle_texts(sc)
        if got != want:
            bad.append((sc["seed"], next(i for i, (x, y) in enumerate(zip(want, got)) if x != y)))
    assert not bad, f"{len(bad)} worlds differ, first {bad[:3]}"


def test_the_layers_tick_matches_the_oracle_on_partition_worlds_on_the_cpu():
    """Worlds of the partition benchmark (the largest, one of about 45 ships, one small; sensors of 1-250 km on every
    ship, each flying its pilot's direction): the layer's host build, whose sensor checks there mostly skip their two
    re-filings (the inflated box's chain emptied and made again among them), against the oracle's tick."""
    from exact_ballpark_b200.workloads import partition_worlds
    pw = partition_worlds(11, 1200)
    order = np.argsort(-pw.sizes, kind="stable")
    goto = pw.cols["pos"] + pw.direction * 1e9
    bad = []
    for w in (int(order[0]), int(order[1]), int(order[150]), int(order[600])):
        ops = sl.partition_world_ops(pw, w, goto, 5)
        got = sl.drive_ticks_host(ops, seed=w + 1)
        want = [sl.oracle_lines(t, int(op[0])) for t, op in zip(space_world.run(ops, seed=w + 1), ops)]
        if got != want:
            bad.append((w, int(pw.sizes[w]), next(i for i, (x, y) in enumerate(zip(want, got)) if x != y)))
    assert not bad, f"{len(bad)} worlds differ, first {bad[:3]}"


@pytest.mark.parametrize("family,world_major", [("tick", False), ("modes", False), ("tick", True)])
def test_the_layers_tick_matches_the_oracle_on_the_cpu(family, world_major):
    """The ticking and the mode streams (GOTO and STOP ships; FollowBall, Orbit and WarpTo with drop-outs, releases
    and re-added followers): the layer's host build around the flight oracle's tick (dead rows skipped), every state
    after every operation against the space oracle's; the ticking ones over the world-major arena too."""
    scs = _streams((family,))
    assert len(scs) == 40
    bad = []
    for sc in scs:
        got = sl.drive_ticks_host(sc["ops"], sc["rand_seed"], world_major=world_major)
        want = _oracle_texts(sc)
        if got != want:
            bad.append((sc["seed"], next(i for i, (x, y) in enumerate(zip(want, got)) if x != y)))
    assert not bad, f"{len(bad)} worlds differ, first {bad[:3]}"


ARRANGEMENTS = [(1, False), (32, True), (1, True), (32, False)]   # (lanes, world-major): the defaults first


@pytest.mark.gpu
@pytest.mark.parametrize("lanes,world_major", ARRANGEMENTS)
def test_the_device_layer_matches_its_host_program_word_for_word(lanes, world_major):
    """A thread a world and a warp a world (its lanes splitting GetNearbyBalls' scan and sort), over the interleaved
    state and the world-major arena."""
    import torch
    assert torch.cuda.is_available()
    scs = _streams()
    streams = _inputs(scs)
    got, flags = sl.drive(streams, "cuda", lanes=lanes, world_major=world_major)
    want, _ = sl.drive(streams, "host")
    assert not (flags & ~HUGE).any()
    bad = [sc["seed"] for sc, g, w in zip(scs, got, want) if g != w]
    assert not bad, f"{len(bad)} worlds differ from the host program, first {bad[:3]}"
    bad = [sc["seed"] for sc, g in zip(scs, got) if g != _oracle_texts(sc)]
    assert not bad, f"{len(bad)} worlds differ from the oracle, first {bad[:3]}"


@pytest.mark.gpu
@pytest.mark.parametrize("lanes,world_major", ARRANGEMENTS[:3])
@pytest.mark.parametrize("family", ["tick", "modes"])
def test_the_layers_tick_over_the_flight_park_matches_the_oracle(family, lanes, world_major):
    """The ticking streams (GOTO and STOP ships across top boxes and bubbles, with sensors, tracked targets and
    notification ranges) and the mode streams (FollowBall, Orbit, WarpTo with drop-outs, releases, re-added
    followers, sensors): VecSpace.tick over a VecModesPark (the dead bubbles' rows skipped by the park's tick, then
    the re-filings of the balls that moved, in ascending id, then HandleProximities) against the oracle's tick, every
    state and every tick's events after every operation."""
    import torch
    assert torch.cuda.is_available()
    scs = _streams((family,))
    assert len(scs) == 40
    bad = []
    for sc in scs:
        got = sl.drive_ticks(sc["ops"], seed=sc["rand_seed"], lanes=lanes, world_major=world_major)
        want = _oracle_texts(sc)
        if got != want:
            bad.append((sc["seed"], next(i for i, (x, y) in enumerate(zip(want, got)) if x != y)))
    assert not bad, f"{len(bad)} worlds differ, first {bad[:3]}"


@pytest.mark.gpu
@pytest.mark.parametrize("lanes,world_major", ARRANGEMENTS[:2])
def test_the_layers_tick_matches_the_oracle_in_crowded_sensing_worlds(lanes, world_major):
    """The crowded worlds (16 to 128 sensing ships) through VecSpace.tick over a VecModesPark on the device, a thread
    a world over the interleaved state or a warp a world over the world-major arena."""
    import torch
    assert torch.cuda.is_available()
    bad = []
    for sc in _crowd():
        got = sl.drive_ticks(sc["ops"], seed=sc["rand_seed"], lanes=lanes, world_major=world_major)
        want = _oracle_texts(sc)
        if got != want:
            bad.append((sc["seed"], next(i for i, (x, y) in enumerate(zip(want, got)) if x != y)))
    assert not bad, f"{len(bad)} worlds differ, first {bad[:3]}"
