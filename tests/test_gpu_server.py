"""The server layer (exact_ballpark_b200.server: the server kernel, its only path) over the GPU flight park against the
golden traces recorded on the reference's own server layer (tests/golden/server_trace.py): the reference's server
scenarios over the flight-mode park, without and with dynamical orientation (seed 1 development, seed 2 held out; 40
worlds of one bubble each, 14 ticks of Actions calls: conflicting commands, duplicates dropped and kept, cloaks and
uncloaks in both orders, local and non-local SetBallPosition, follows and orbits of a cloaking ship, warps and
warp-ins, every setter, refused values), its pending-query scenarios and its OnTick scenarios. After every tick (or
call): every park field's digest, the update batch's digest (stamps, queued flags and rows, routes, the uncloaks'
recipients and the park's fields there, the bubble's additions, the narrowcast and character flags), the answers and
what every client is sent, bit for bit. Then the queue's duplicate rule and lookups on a small park, and a
ServerGraph's replays against eager ticks on random queues. On the CPU: OnTick's interval arithmetic."""

import random
from types import SimpleNamespace

import numpy as np
import pytest
import torch

import server_trace as st
import trace as tr


def _golden(name):
    return st.load(st.GOLDEN / name)


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")
@pytest.mark.parametrize("name", ["server_modes", "server_modes_do"], ids=["euler", "dynamical"])
@pytest.mark.parametrize("run", [0, 1], ids=["development", "held_out"])
def test_the_server_layer_replays_the_golden_ticks(name, run):
    from exact_ballpark_b200 import VecModesPark, server
    r = _golden(name)[run]
    bad = st.replay(server, VecModesPark, r, "cuda")
    assert not bad, f"{len(bad)} differences, first {bad[:3]}"


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")
@pytest.mark.parametrize("run", [0, 1], ids=["development", "held_out"])
def test_the_pending_queries_and_undos_replay_the_golden_ticks(run):
    """The reference's pending-query scenarios (queries of every kind among the calls, undos of a pending cloak, the
    prune's edge): every answer (from the kernel's test of the queue), the park and the update batch after every
    tick."""
    from exact_ballpark_b200 import VecModesPark, server
    r = _golden("server_pending")[run]
    bad = st.replay(server, VecModesPark, r, "cuda")
    assert not bad, f"{len(bad)} differences, first {bad[:3]}"


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")
@pytest.mark.parametrize("run", [0, 1, 2, 3], ids=["euler-development", "euler-held_out", "dynamical-development",
                                                   "dynamical-held_out"])
def test_on_tick_replays_the_golden_calls(run):
    """The reference's OnTick scenarios (each world's own clock: calls too early, first calls, remainders, the
    master's resynchronisation, masked rounds, kept queues): after every call the park, each world's clocks and every
    round's worlds and update batch."""
    from exact_ballpark_b200 import VecModesPark, server
    r = _golden("server_ontick")[run]
    bad = st.replay(server, VecModesPark, r, "cuda")
    assert not bad, f"{len(bad)} differences, first {bad[:3]}"


# ---- random queues ----

def _random_worlds(seed: int, W: int, do: bool) -> list:
    """W worlds of 1 to 6 balls (ids 1 to 40, distinct in a world), mostly interactive, about half piloted."""
    r = random.Random(seed)
    cs = []
    for w in range(W):
        ids = r.sample(range(1, 41), r.randint(1, 6))
        centre = [r.uniform(-1e5, 1e5) for _ in range(3)]
        balls = [{"id": i, "mass": 10 ** r.uniform(5, 8), "radius": r.uniform(10, 300), "max_vel": r.uniform(50, 500),
                  "pos": [c + r.uniform(-5e3, 5e3) for c in centre], "vel": [r.uniform(-50, 50) for _ in range(3)],
                  "agility": r.uniform(0.2, 2.0), "sf": r.choice([0.0, 0.5, 1.0]), "massive": r.random() < 0.5,
                  "interactive": r.random() < 0.8, "max_ang_vel": r.uniform(0.1, 1.0), "rot_agility": r.uniform(0.1, 1)}
                 for i in ids]
        pilots = {b["id"]: k for k, b in enumerate(balls) if r.random() < 0.5}
        cs.append({"id": 1000 + 7 * w, "balls": balls, "pilots": pilots, "ticks": []})
    return cs


def _value(r: random.Random, lo: float, hi: float) -> float:
    x = r.random()
    if x < 0.03:
        return float("nan")
    if x < 0.05:
        return float("inf")
    if x < 0.15:
        return -r.uniform(lo, hi)
    if x < 0.2:
        return 0.0
    return r.uniform(lo, hi)


def _random_pushes(r: random.Random, cs: list, kinds: list, dev) -> list:
    """One tick's pushes: 0 to 14 calls of random kinds, worlds masked at random, arguments with edge values; a push
    repeated as it was now and then (the duplicate rule)."""
    W = len(cs)
    out = []
    for _ in range(r.randint(0, 14)):
        if out and r.random() < 0.2:
            out.append(out[-1])
            continue
        kind = r.choice(kinds)
        mask = torch.tensor([r.random() < 0.7 for _ in range(W)])
        pick = lambda w: r.choice([b["id"] for b in cs[w]["balls"]]) if r.random() < 0.93 else r.choice([0, 99])  # noqa: E731
        ball = torch.tensor([pick(w) for w in range(W)], dtype=torch.int64)
        target = torch.tensor([pick(w) for w in range(W)], dtype=torch.int64)
        if kind in ("GotoPoint", "WarpTo", "EntityWarpIn", "SetBallPosition"):
            f = [[_value(r, 1e3, 1e7) for _ in range(3)] + [_value(r, 0, 1e5)] for _ in range(W)]
        elif kind in ("GotoDirection", "SetBallVelocity", "SetBallAngularVelocity", "SetBallRotation"):
            f = [[_value(r, 0, 2) for _ in range(4)] for _ in range(W)]
        else:
            f = [[_value(r, 0, 1.5) if kind in ("SetSpeedFraction", "SetBallAgility") else _value(r, 0, 1e6)]
                 + [0.0] * 3 for _ in range(W)]
        n = torch.tensor([r.choice([-3, 0, 1, 2, 3, 5, 257, 300]) for _ in range(W)], dtype=torch.int64)
        loc = torch.tensor([r.choice([0, 0, 1]) for _ in range(W)], dtype=torch.int64)
        out.append((kind, *(x.to(dev) for x in (mask, ball, target, torch.tensor(f, dtype=torch.float64), n, loc))))
    return out


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")
def test_a_server_graph_replays_eager_kernel_ticks():
    from exact_ballpark_b200 import VecModesPark, server
    cs = _random_worlds(9, 1024, True)
    sched = ["GotoDirection", "SetSpeedFraction", "FollowBall", "SetMaxSpeed", "Orbit", "GotoDirection",
             "CloakBall", "SetSpeedFraction"]
    g = torch.Generator().manual_seed(3)
    W = len(cs)
    ins = []
    for k in sched:
        ids = torch.tensor([w["balls"][int(torch.randint(len(w["balls"]), (1,), generator=g))]["id"] for w in cs])
        tgt = torch.tensor([w["balls"][0]["id"] for w in cs])
        f = torch.rand(W, 4, generator=g, dtype=torch.float64) * 2 - 1
        ins.append({"mask": torch.rand(W, generator=g) < 0.8, "ball": ids, "target": tgt, "f": f,
                    "n": torch.ones(W, dtype=torch.int64), "loc": torch.zeros(W, dtype=torch.int64)})
    eager, _ = st.build(server, VecModesPark, cs, True, "cuda")
    graphed, _ = st.build(server, VecModesPark, cs, True, "cuda")
    for s in (eager, graphed):                             # the first tick (its additions' fields) eagerly
        s.pre_tick()
        s.evolve()
        s.post_tick()
    gr = server.ServerGraph(graphed, sched)
    for j, inp in enumerate(ins):
        for key, v in inp.items():
            gr.inputs[j][key].copy_(v.to("cuda"))
    for t in range(12):
        for k, inp in zip(sched, ins):
            eager.push(k, *(inp[key].to("cuda") for key in ("mask", "ball", "target", "f", "n", "loc")))
        eager.pre_tick(snapshot=False)
        eager.evolve()
        eager.post_tick()
        out = gr.tick()
        fa, fb = tr.field_digests(eager.a.park), tr.field_digests(graphed.a.park)
        assert np.array_equal(fa, fb), f"tick {t}: park fields differ"
        assert graphed.a.park.current_time == eager.a.park.current_time
        for key in ("has_character", "gets_bubble"):
            assert torch.equal(getattr(out, key), getattr(eager.batch, key)), (t, key)
        assert torch.equal(out.route, eager.batch.route) and torch.equal(out.stamp, eager.batch.stamp)
        assert torch.equal(graphed.dead, eager.dead)
        for j in range(len(sched)):
            assert torch.equal(out.slots[j].ok, eager.batch.slots[j].ok), (t, j)


def test_every_server_golden_carries_the_clients_sends():
    for name in ("server_modes", "server_modes_do", "server_pending", "server_ontick"):
        for r in _golden(name):
            assert r["decoded"] and len(r["decode"]) == len(r["park"])


def test_the_on_tick_goldens_hold_masked_rounds_and_kept_queues():
    runs = _golden("server_ontick")
    assert len(runs) == 4 and all(r["ontick"] for r in runs)
    for r in runs:
        T = len(r["cases"][0]["clock"])
        assert r["park"].shape[0] == T and len(r["batch"]) == T
        rounds = [int(d[3]) for d in r["batch"]]
        assert sum(rounds) > 20 and 0 in rounds              # calls with no round, calls with several
        assert max(rounds) > 1


def test_the_pending_goldens_hold_queries_and_undos():
    runs = _golden("server_pending")
    assert len(runs) == 2
    for r in runs:
        names = [c[0] for w in r["cases"] for t in w["ticks"] for c in t]
        assert names.count(st.UNDO) >= 300
        for q in st.QUERIES:
            assert names.count(q) >= 50, q
        assert len(r["answers"]) == len(r["park"]) and sum(len(a) for a in r["answers"]) > 100


def test_the_server_goldens_hold_every_action_kind():
    from exact_ballpark_b200 import server
    for name in ("server_modes", "server_modes_do"):
        runs = _golden(name)
        assert len(runs) == 2
        kinds = {c[0] for r in runs for w in r["cases"] for t in w["ticks"] for c in t}
        assert {st.ACTION_KINDS[k] for k in kinds} <= set(server.CODE)
        assert len(kinds) >= 18
        for r in runs:
            T = len(r["cases"][0]["ticks"])
            assert r["park"].shape[0] == T and len(r["batch"]) == T


def _small_server():
    """Two worlds of three piloted balls (ids 10, 11, 12 and 20, 21, 22) on the GPU flight park."""
    from exact_ballpark_b200 import VecModesPark, server
    rows = [{"id": i, "world": w, "time": 0, "mass": 1e7, "radius": 50.0, "max_vel": 200.0,
             "pos": [1e3 * k, 0.0, 0.0], "vel": [0.0, 0.0, 0.0], "agility": 1.0, "speed_fraction": 1.0,
             "free": True, "massive": False, "interactive": True}
            for w, ids in enumerate(((10, 11, 12), (20, 21, 22))) for k, i in enumerate(ids)]
    p = VecModesPark(len(rows), device="cuda")
    p.load(rows)
    return server.VecServer(server.ModesAdapter(p), list(range(6)))


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")
def test_the_queue_drops_a_call_equal_to_the_worlds_last_and_keeps_the_rest():
    """TIME-710 in the kernel: a call equal to the world's last queued call is dropped (a NaN equals nothing), one
    equal to an earlier call is queued again, a call for a ball not in the world finds no row, a CloakBall of a ball
    not in the park is not queued and is queued in its ball's bubble otherwise; the pending queries see the same
    test."""
    s = _small_server()
    s.tick()                                               # the first tick: every ball settled in its bubble
    both = torch.tensor([True, True], device="cuda")
    ids = lambda a, b: torch.tensor([a, b], device="cuda")          # noqa: E731
    fl = lambda a, b: torch.tensor([[a], [b]], dtype=torch.float64, device="cuda")   # noqa: E731
    a = s.push("SetMaxSpeed", both, ids(11, 22), f=fl(3.0, float("nan")))
    b = s.push("SetMaxSpeed", both, ids(11, 22), f=fl(3.0, float("nan")))
    c = s.push("SetMaxSpeed", both, ids(11, 23), f=fl(3.5, 1.0))
    d = s.push("SetMaxSpeed", torch.tensor([True, False], device="cuda"), ids(11, 23), f=fl(3.0, 1.0))
    e = s.push("CloakBall", both, ids(10, 24), n=ids(1, 1), f=fl(9.0, 9.0))
    assert s.has_pending_cloak(both, ids(10, 24)).tolist() == [True, False]
    s.pre_tick()
    assert a.ok.tolist() == [True, True] and a.row.tolist() == [1, 5]
    assert b.ok.tolist() == [False, True]
    assert c.ok.tolist() == [True, True] and c.row.tolist() == [1, -1]
    assert d.ok.tolist() == [True, False]
    assert e.ok.tolist() == [True, False] and e.loc.tolist()[0] == 0
    s.evolve()
    s.post_tick()


def test_on_tick_clocks_count_whole_intervals_and_carry_the_rest():
    """OnTick's arithmetic (Ballpark.cpp:219-330) on the CPU: too early, a first call, whole intervals with the
    remainder carried, and the master's backlog of more than five intervals cut to one without a remainder."""
    from exact_ballpark_b200.server import _Clocks
    iv = 10_000_000
    elapsed = torch.tensor([iv - 1, iv, 3 * iv + 7, 9 * iv + 5, 9 * iv + 5])
    first = torch.tensor([False, True, False, False, False])
    c = _Clocks.of(elapsed, iv, first, master=True)
    assert c.due.tolist() == [False, True, True, True, True]
    assert c.first.tolist() == [False, True, False, False, False]
    assert c.runs.tolist() == [0, 0, 3, 1, 1] and c.left.tolist() == [0, 0, 7, 0, 0]
    assert c.resync.tolist() == [False, False, False, True, True]
    c = _Clocks.of(elapsed, iv, first, master=False)
    assert c.runs.tolist() == [0, 0, 3, 9, 9] and c.left.tolist() == [0, 0, 7, 5, 5]
