"""The partition layer over ragged worlds (exact_ballpark_b200.partition): the metric's workload at a test's size.

Ragged worlds of 1 to 128 ships in Gaussian blobs with a sensor on every ship (workloads.partition_worlds), the space
layer in its two arrangements (size classes with the worlds ordered by size, and the plain 128-slot layout in world
order) over the flight park: both must give the same park and the same layer state world by world, bit for bit, and
sampled worlds must match the space oracle (oracle/space.cpp, held to the reference's SpaceBallpark) run on the same
world alone: every state and every tick's events."""

import numpy as np
import pytest

import space_layer as sl
import space_trace as sp
from oracle import space_world

pytestmark = pytest.mark.gpu


def _world_text(part, park, pw, w: int, events: bool) -> str:
    """World w's layer state as the oracle's state text (and the last tick's events)."""
    layer, col = part.world(w)
    st = {k: v[..., col:col + 1].cpu().numpy() for k, v in layer.st.items()}
    N, s0, k = layer.N, int(pw.starts[w]), int(pw.sizes[w])
    ids = np.zeros(N, np.int64)
    mode = np.zeros(N, np.int64)
    sensor = np.zeros(N, np.uint8)
    rows = np.arange(s0, s0 + k)
    ids[:k] = park._ids[rows].cpu().numpy()
    mode[:k] = park._mode[rows].cpu().numpy()
    sensor[:k] = park._sensor[rows].cpu().numpy()
    t = sl.text(st, ids, mode, 0, sensor)
    return t + (sl.events_text(st, ids, 0, N) if events else "")


def _run(pw, ragged: bool, goto, ticks: int, dev, plan=None):
    import torch

    from exact_ballpark_b200 import VecModesPark
    from exact_ballpark_b200.modes import tick_plain, tick_tiled
    from exact_ballpark_b200.partition import PartitionLayer
    park = VecModesPark(pw.n, device=dev)
    park.load_columns(pw.cols)
    part = PartitionLayer(park, pw.sizes, ragged=ragged, plan=plan)
    part.load()
    part.add_sensors(pw.sensor_range, 1.0)
    park.goto_point(torch.ones(pw.n, dtype=torch.bool, device=dev), torch.as_tensor(goto, device=dev))
    step = (lambda: tick_tiled(park)) if ragged else (lambda: tick_plain(park, park.block))
    for _ in range(ticks):
        part.tick(step)
        park.current_time += 1
    return park, part


def test_the_ragged_batch_matches_the_plain_layout_and_the_oracle():
    import torch
    from exact_ballpark_b200.workloads import partition_worlds
    dev = torch.device("cuda")
    pw = partition_worlds(5, 300)
    assert pw.sizes.max() >= 100 and pw.sizes.min() == 1        # the classes from 4 to 128 slots all in use
    g = np.random.default_rng(3)
    goto = pw.cols["pos"] + g.normal(0.0, 3e4, (pw.n, 3))
    ticks = 6
    pr, ragged = _run(pw, True, goto, ticks, dev)
    pp, plain = _run(pw, False, goto, ticks, dev)
    torch.cuda.synchronize()
    assert len(ragged.layers) >= 5 and len(plain.layers) == 1
    for k in ("pos", "vel", "old_pos", "mode", "clock", "sensor", "radius"):
        assert torch.equal(getattr(pr, "_" + k), getattr(pp, "_" + k)), k
    assert not (ragged.flags() != 0).any() and not (plain.flags() != 0).any()
    assert torch.equal(ragged.event_counts(), plain.event_counts())
    for w in range(len(pw.sizes)):
        assert _world_text(ragged, pr, pw, w, True) == _world_text(plain, pp, pw, w, True), w
    # sampled worlds against the oracle run alone: the largest, the smallest and a few between
    order = np.argsort(pw.sizes)
    sample = sorted(set([int(order[-1]), int(order[-2]), int(order[0])] + [int(x) for x in order[::60]]))
    for w in sample:
        want = space_world.run(sl.partition_world_ops(pw, w, goto, ticks), seed=w + 1)[-1]
        assert _world_text(ragged, pr, pw, w, True) == sl.oracle_lines(want, sp.TICK), (w, int(pw.sizes[w]))


def test_every_arrangement_of_the_classes_gives_the_same_worlds():
    """The autotuner's choices change no result: the classes crossed (the small ones a warp a world, the large ones a
    thread a world in 64-thread blocks) against the default, and the tuner's own plan, every world bit for bit."""
    import torch
    from exact_ballpark_b200.partition import CLASSES, tune_partition
    from exact_ballpark_b200.workloads import partition_worlds
    dev = torch.device("cuda")
    pw = partition_worlds(7, 200)
    goto = pw.cols["pos"] + np.random.default_rng(4).normal(0.0, 3e4, (pw.n, 3))
    ticks = 4
    base_park, base = _run(pw, True, goto, ticks, dev)
    crossed = {c: ((32, 128) if c <= 16 else (1, 64)) for c in CLASSES}
    plan, times = tune_partition(pw, dev, warm=1, ticks=1)
    assert set(plan) == {layer.N for layer, _ in base.layers}
    assert all(set(t) == set(plan) for t in times.values())
    for p in (crossed, plan):
        park, part = _run(pw, True, goto, ticks, dev, plan=p)
        assert [(layer.lanes, layer.block) for layer, _ in part.layers] == [p[layer.N] for layer, _ in part.layers]
        for k in ("pos", "vel", "mode", "clock"):
            assert torch.equal(getattr(park, "_" + k), getattr(base_park, "_" + k)), k
        assert torch.equal(part.event_counts(), base.event_counts())
        for w in range(len(pw.sizes)):
            assert _world_text(part, park, pw, w, True) == _world_text(base, base_park, pw, w, True), w
