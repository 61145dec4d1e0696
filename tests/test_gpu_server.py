"""The server layer (exact_ballpark_b200.server) over the GPU flight park against the golden traces recorded on the
reference's own server layer (tests/golden/server_trace.py): the reference's server scenarios over the flight-mode
park, without and with dynamical orientation (seed 1 development, seed 2 held out; 40 worlds of one bubble each, 14
ticks of Actions calls: conflicting commands, duplicates dropped and kept, cloaks and uncloaks in both orders, local and
non-local SetBallPosition, follows and orbits of a cloaking ship, warps and warp-ins, every setter, refused values).
After every tick: every park field's digest and the update batch's digest (stamps, queued flags and rows, routes, the
uncloaks' recipients and the park's fields there, the bubble's additions, the narrowcast and character flags), bit for
bit, on both paths (the park's commands over all worlds; the server kernel, one thread a world). Then the kernel
against the torch path on random queues over 1,536 worlds (every kind the flight park applies, refused and edge
values, duplicates, misses), and a ServerGraph's replays against eager kernel ticks. The CPU tests hold the queue's
duplicate rule and the world lookup on a stand-in park."""

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
@pytest.mark.parametrize("kernel", ["torch", "cuda"])
def test_the_server_layer_replays_the_golden_ticks(name, run, kernel):
    from exact_ballpark_b200 import VecModesPark, server
    r = _golden(name)[run]
    bad = st.replay(server, VecModesPark, r, "cuda", kernel=kernel)
    assert not bad, f"{len(bad)} differences, first {bad[:3]}"


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")
@pytest.mark.parametrize("run", [0, 1], ids=["development", "held_out"])
@pytest.mark.parametrize("kernel", ["torch", "cuda"])
def test_the_pending_queries_and_undos_replay_the_golden_ticks(run, kernel):
    """The reference's pending-query scenarios (queries of every kind among the calls, undos of a pending cloak, the
    prune's edge): every answer, the park and the update batch after every tick, on both paths."""
    from exact_ballpark_b200 import VecModesPark, server
    r = _golden("server_pending")[run]
    bad = st.replay(server, VecModesPark, r, "cuda", kernel=kernel)
    assert not bad, f"{len(bad)} differences, first {bad[:3]}"


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")
@pytest.mark.parametrize("run", [0, 1, 2, 3], ids=["euler-development", "euler-held_out", "dynamical-development",
                                                   "dynamical-held_out"])
@pytest.mark.parametrize("kernel", ["torch", "cuda"])
def test_on_tick_replays_the_golden_calls(run, kernel):
    """The reference's OnTick scenarios (each world's own clock: calls too early, first calls, remainders, the
    master's resynchronisation, masked rounds, kept queues): after every call the park, each world's clocks and every
    round's worlds and update batch, on both paths."""
    from exact_ballpark_b200 import VecModesPark, server
    r = _golden("server_ontick")[run]
    bad = st.replay(server, VecModesPark, r, "cuda", kernel=kernel)
    assert not bad, f"{len(bad)} differences, first {bad[:3]}"


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")
@pytest.mark.parametrize("name,run", [("server_collide", 0), ("server_collide", 1), ("server_collide_ontick", 0)],
                         ids=["development", "held_out", "on_tick"])
def test_the_server_layer_over_the_collision_park_replays_the_golden_ticks(name, run):
    """The reference's server scenarios over the collision park (massive balls within 3 km that meet, cloaks,
    SetBallMassive, SetBallInteractive) and its OnTick scenarios there: the park's every field, the batch and every
    client's sends, every tick or call."""
    from exact_ballpark_b200 import VecCollidePark, server
    r = _golden(name)[run]
    bad = st.replay(server, VecCollidePark, r, "cuda")
    assert not bad, f"{len(bad)} differences, first {bad[:3]}"


# ---- random queues: the kernel against the torch path ----

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
@pytest.mark.parametrize("do", [False, True], ids=["euler", "dynamical"])
def test_the_server_kernel_matches_the_torch_path_on_random_queues(do):
    from exact_ballpark_b200 import VecModesPark, server
    cs = _random_worlds(5 + int(do), 1536, do)
    a, _ = st.build(server, VecModesPark, cs, do, "cuda", kernel="torch")
    b, _ = st.build(server, VecModesPark, cs, do, "cuda", kernel="cuda")
    kinds = sorted(server.KINDS[k] for k in a.a.kinds)
    assert len(kinds) == (25 if do else 20)
    r = random.Random(11)
    routed = 0
    for t in range(24):
        pushes = _random_pushes(r, cs, kinds, "cuda")
        for p in pushes:
            a.push(*p)
            b.push(*p)
        for s in (a, b):
            s.pre_tick()
            s.evolve()
            s.post_tick()
        fa, fb = tr.field_digests(a.a.park), tr.field_digests(b.a.park)
        bad = [st.PARK_FIELDS[k] for k in range(len(fa)) if fa[k] != fb[k]]
        assert not bad, f"tick {t}: park fields {bad} differ"
        da, db = st.batch_digests(a), st.batch_digests(b)
        assert da.shape == db.shape and (da == db).all(), f"tick {t}: the update batches differ"
        routed += int((a.batch.route != 0).sum())
        assert torch.equal(a.dead, b.dead)
    assert routed > 10000


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
    eager, _ = st.build(server, VecModesPark, cs, True, "cuda", kernel="cuda")
    graphed, _ = st.build(server, VecModesPark, cs, True, "cuda", kernel="cuda")
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
    for name in ("server_modes", "server_modes_do", "server_pending", "server_ontick", "server_collide",
                 "server_collide_ontick"):
        for r in _golden(name):
            assert r["decoded"] and len(r["decode"]) == len(r["park"])
    kinds = {c[0] for r in _golden("server_collide") for w in r["cases"] for t in w["ticks"] for c in t}
    assert {"cloak_ball", "uncloak_ball", "set_ball_massive", "go_to_point", "stop"} <= kinds


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


class _StandIn:
    """A park the server layer reads on the CPU: two worlds of three balls (ids 10, 11, 12 and 20, 21, 22)."""

    def __init__(self):
        from exact_ballpark_b200 import server
        self.dev = torch.device("cpu")
        self.R, self.W = 6, 2
        self.world = torch.tensor([0, 0, 0, 1, 1, 1])
        self.rows_of_world = torch.tensor([[0, 1, 2], [3, 4, 5]])
        self.ids_of_world = torch.tensor([[10, 11, 12], [20, 21, 22]])
        self.arange = torch.arange(6)
        self.kinds = frozenset(k for k in range(1, len(server.KINDS)) if k not in server.NOT_APPLIED)
        self.lookup = server.ModesAdapter.lookup.__get__(self)
        self.any_in_world = server.ModesAdapter.any_in_world.__get__(self)

    def clock(self):
        return torch.tensor([5, 5])


def test_push_drops_a_call_equal_to_the_worlds_last_and_keeps_the_rest():
    from exact_ballpark_b200 import server
    A = _StandIn()
    s = server.VecServer.__new__(server.VecServer)
    s.a, s.W, s.R, s.dev, s.kernel = A, A.W, A.R, A.dev, "torch"
    s.settled = torch.tensor([True, False, False, True, True, True])
    s.slots = []
    s._reset_last()
    both = torch.tensor([True, True])
    a = s.push("SetMaxSpeed", both, torch.tensor([11, 22]), f=torch.tensor([[3.0], [float("nan")]]))
    assert a.ok.tolist() == [True, True] and a.row.tolist() == [1, 5]
    b = s.push("SetMaxSpeed", both, torch.tensor([11, 22]), f=torch.tensor([[3.0], [float("nan")]]))
    assert b.ok.tolist() == [False, True]          # the same call dropped; a NaN equals nothing
    c = s.push("SetMaxSpeed", both, torch.tensor([11, 23]), f=torch.tensor([[3.5], [1.0]]))
    assert c.ok.tolist() == [True, True] and c.row.tolist() == [1, -1]
    d = s.push("SetMaxSpeed", torch.tensor([True, False]), torch.tensor([11, 23]), f=torch.tensor([[3.0], [1.0]]))
    assert d.ok.tolist() == [True, False]          # not the last call any more: queued again
    e = s.push("CloakBall", both, torch.tensor([10, 24]), n=torch.tensor([1, 1]), f=torch.tensor([[9.0], [9.0]]))
    assert e.ok.tolist() == [True, False]          # not queued for a ball not in the park
    assert e.loc.tolist()[0] == 0                  # the bubble it was queued in
    f = s.push("CloakBall", both, torch.tensor([12, 21]), n=torch.tensor([1, 1]), f=torch.tensor([[9.0], [9.0]]))
    assert f.ok.tolist() == [True, True] and f.loc.tolist() == [-1, 0]
    g = s.push("FollowBall", both, torch.tensor([10, 20]), target=torch.tensor([12, 29]), f=torch.tensor([[5.0], [5.0]]))
    assert g.trow.tolist() == [2, -1]
    with pytest.raises(ValueError):
        s.push("LaunchMissile", both, torch.tensor([10, 20]))
    assert len(s.slots) == 7
    assert SimpleNamespace(**s.last).kind.tolist() == [server.CODE["FollowBall"]] * 2


def _standin_server(kernel: str):
    from exact_ballpark_b200 import server
    A = _StandIn()
    s = server.VecServer.__new__(server.VecServer)
    s.a, s.W, s.R, s.dev, s.kernel = A, A.W, A.R, A.dev, kernel
    s.settled = torch.tensor([True, True, True, True, True, True])
    A.cloaked = torch.tensor([0, 0, 0, 0, 0, 2])
    s.slots = []
    s._reset_last()
    return s


@pytest.mark.parametrize("kernel", ["torch", "cuda"])
def test_an_undo_prunes_the_pending_cloaks_and_the_calls_around_them_stand(kernel):
    """X, CloakBall, X, undo: both X stay queued (the second was tested against the cloak); a cloak pushed twice is
    queued once and the undo takes it out; the pending mode falls back to the ball's cloak byte. On the kernel path the
    calls are tested at the query, as the kernel tests them, and the undo marks them tested."""
    s = _standin_server(kernel)
    both = torch.tensor([True, True])
    x = ("SetSpeedFraction", both, torch.tensor([11, 21]), None, torch.tensor([[0.5], [0.5]]))
    cloak = ("CloakBall", both, torch.tensor([10, 22]), None, torch.tensor([[900.0], [900.0]]), torch.tensor([1, 3]))
    s.push(*x)
    s.push(*cloak)
    s.push(*cloak)                                   # the same cloak again: a duplicate
    s.push(*x)
    assert [q.tolist() for q in s._queued()] == [[True, True], [True, True], [False, False], [True, True]]
    assert s.has_pending_cloak(both, torch.tensor([10, 22])).tolist() == [True, True]
    mode, known = s.get_pending_cloak_mode(both, torch.tensor([10, 22]))
    assert mode.tolist() == [1, 3] and known.tolist() == [True, True]
    s.undo_pending_cloak(torch.tensor([True, False]), torch.tensor([10, 22]))
    assert s.has_pending_cloak(both, torch.tensor([10, 22])).tolist() == [False, True]
    mode, known = s.get_pending_cloak_mode(both, torch.tensor([10, 22]))
    assert mode.tolist() == [0, 3] and known.tolist() == [True, True]
    mode, known = s.get_pending_cloak_mode(both, torch.tensor([99, 23]))
    assert known.tolist() == [False, False]
    assert [q.tolist() for q in s._queued()] == [[True, True], [False, True], [False, False], [True, True]]
    s.push(*x)                                       # now equal to the world's last queued call: dropped
    assert s._queued()[-1].tolist() == [False, False]
    if kernel == "cuda":
        assert all(getattr(q, "resolved", False) for q in s.slots[:4]) and not getattr(s.slots[4], "resolved", False)


def test_a_masked_split_keeps_the_same_queue_on_both_paths():
    """OnTick's queue split: a world without a tick keeps its queued calls (a duplicate dropped), in order, and the
    ticking worlds' calls go to the pre-tick, alike on the torch path (tested at each push) and the kernel path (tested
    at the split, as the kernel tests them)."""
    both = torch.tensor([True, True])
    on = torch.tensor([True, False])
    kept = {}
    for kernel in ("torch", "cuda"):
        s = _standin_server(kernel)
        s.push("SetSpeedFraction", both, torch.tensor([11, 21]), f=torch.tensor([[0.5], [0.5]]))
        s.push("SetSpeedFraction", both, torch.tensor([11, 21]), f=torch.tensor([[0.5], [0.5]]))   # duplicates
        s.push("CloakBall", torch.tensor([False, True]), torch.tensor([10, 22]), n=torch.tensor([1, 1]),
               f=torch.tensor([[9.0], [9.0]]))
        if kernel == "cuda":
            s._test_pending(commit=True)
        flag = "ok" if kernel == "torch" else "mask"
        going = s._split_queue(on, flag)
        kept[kernel] = [(q.kind, getattr(q, flag).tolist(), q.loc.tolist()) for q in s.slots]
        assert [getattr(q, flag).tolist() for q in going] == [[True, False], [False, False], [False, False]]
    assert kept["torch"] == kept["cuda"]
    assert [k[1] for k in kept["torch"]] == [[False, True], [False, True]]


def _fields(mode: int, free: bool = True, dynamical: bool = False) -> dict:
    f = {"ids": torch.tensor([7]), "mode": torch.tensor([mode]), "radius": torch.tensor([12.5]),
         "pos": torch.tensor([[1.0, -2.0, 3.5]], dtype=torch.float64), "free": torch.tensor([free]),
         "massive": torch.tensor([True]), "interactive": torch.tensor([False]), "mass": torch.tensor([1e6]),
         "cloaked": torch.tensor([200]), "max_vel": torch.tensor([150.0]),
         "vel": torch.tensor([[4.0, 5.0, 6.0]], dtype=torch.float64), "agility": torch.tensor([0.75]),
         "speed_fraction": torch.tensor([0.5]), "goto": torch.tensor([[9.0, 8.0, 7.0]], dtype=torch.float64),
         "follow_id": torch.tensor([42]), "follow_range": torch.tensor([250.0]),
         "effect_stamp": torch.tensor([(1 << 32) + 5]), "last_collision": torch.tensor([3.25]),
         "owner_id": torch.tensor([3000]), "rot": torch.tensor([[0.0, 0.0, 0.0, 1.0]]),
         "max_ang_vel": torch.tensor([1.0]), "ang_vel": torch.tensor([[0.0, 0.5, 0.0]]),
         "rot_agility": torch.tensor([0.9]), "dynamical": dynamical}
    return f


def test_a_ball_stream_has_write_ball_to_streams_layout():
    import struct

    from exact_ballpark_b200 import server
    blob = server.ball_stream(_fields(3), [0], 12)                       # a free ball in WARP
    tag, time = struct.unpack_from("<Bi", blob, 0)
    head = struct.unpack_from("<qBf3dB", blob, 5)
    assert (tag, time) == (1, 12) and head == (7, 3, 12.5, 1.0, -2.0, 3.5, 0x01 | 0x04)
    o = 5 + struct.calcsize("<qBf3dB")
    assert struct.unpack_from("<dbqii", blob, o) == (1e6, 200 - 256, -1, -1, -1)     # the cloak as a signed char
    o += struct.calcsize("<dbqii")
    assert struct.unpack_from("<f3dff", blob, o) == (150.0, 4.0, 5.0, 6.0, 0.75, 0.5)
    o += struct.calcsize("<f3dff")
    assert struct.unpack_from("<b", blob, o) == (-1,)                               # no formation
    o += 1
    assert struct.unpack_from("<3didqq", blob, o) == (9.0, 8.0, 7.0, 5, 3.25, 42, 3000)
    assert len(blob) == o + struct.calcsize("<3didqq")
    held = server.ball_stream(_fields(2, free=False), [0], 12)            # STOP, not free: no motion block, no tail
    assert len(held) == 5 + struct.calcsize("<qBf3dB") + struct.calcsize("<dbqii") + 1
    rigid = server.ball_stream(_fields(11, free=False), [0], 12)          # RIGID: no mass block either
    assert len(rigid) == 5 + struct.calcsize("<qBf3dB") + 1
    turning = server.ball_stream(_fields(0, dynamical=True), [0], -1)     # GOTO with the orientation block
    assert struct.unpack_from("<Bi", turning, 0) == (1, -1)
    assert len(turning) == len(blob) - struct.calcsize("<3didqq") + struct.calcsize("<4ff3ff") + 24


class _ClockPark:
    """A stand-in park with what the torch path reads: per-row clocks that its tick moves, flags, no motion."""

    def __init__(self, worlds: int, per: int, interactive=True):
        from exact_ballpark_b200 import server
        self.n, self.dev, self.dt = worlds * per, torch.device("cpu"), 1.0
        self.ids = torch.tensor([k + 1 for _ in range(worlds) for k in range(per)])
        self.world = torch.arange(self.n) // per
        self.clock = torch.zeros(self.n, dtype=torch.int64)
        self.interactive = torch.full((self.n,), bool(interactive))
        self.cloaked = torch.zeros(self.n, dtype=torch.int64)
        self.massive = torch.zeros(self.n, dtype=torch.bool)
        self.ticks = []
        self.kinds = frozenset({server.CODE["SetSpeedFraction"], server.CODE["Stop"]})

    def evolve(self, active=None):
        act = torch.ones(self.n, dtype=torch.bool) if active is None else active
        self.clock += act.to(torch.int64)
        self.ticks.append(act.clone())


def _clock_server(worlds: int = 4, per: int = 2, pilots=None):
    from exact_ballpark_b200 import server
    park = _ClockPark(worlds, per)
    a = server.ModesAdapter.__new__(server.ModesAdapter)
    a.park, a.R, a.dev, a.master, a.ids = park, park.n, park.dev, True, park.ids
    a.exists = torch.ones(park.n, dtype=torch.bool)
    a._index_worlds(park.world.tolist())
    a.kinds = park.kinds
    a.apply = lambda kind, m, trow, f, n: None
    a.stream_fields = lambda: {"ids": park.ids.clone()}
    return server.VecServer(a, pilots if pilots is not None else list(range(park.n))), park


def test_on_tick_runs_each_worlds_whole_intervals_and_carries_the_rest():
    """OnTick's arithmetic (Ballpark.cpp:219-330): too early, a first call (one evolve, no pre-tick), whole
    intervals under a mask, the remainder carried, the master's backlog of more than five intervals cut to one."""
    s, park = _clock_server()
    I = 10_000_000                                          # a 1 s interval in 100 ns units
    assert s.on_tick(torch.tensor([0, I - 1, I, 3 * I + 7])) == []      # first calls evolve once: worlds 2 and 3
    assert s.tick_counts == {"worlds too early": 2, "first calls": 2, "resynchronisations": 0, "intervals run": 0,
                             "remainders carried": 0}
    assert park.ticks[-1].tolist() == [False, False, False, False, True, True, True, True]
    assert s.time.tolist() == [0, 0, I, 3 * I + 7] and s.first_time.tolist() == [True, True, False, False]
    batches = s.on_tick(torch.tensor([I, I - 1, 3 * I + 5, 5 * I + 6]))   # world 0's first call; 2 runs 2, 3 runs 1
    assert [b.ticked.tolist() for b in batches] == [[False, False, True, True], [False, False, True, False]]
    assert s.time.tolist() == [I, 0, 3 * I, 4 * I + 7]                   # world 3 carries 2 I - 1
    assert s.tick_counts["remainders carried"] == 2
    assert park.clock.tolist() == [1, 1, 0, 0, 3, 3, 2, 2]
    batches = s.on_tick(torch.tensor([2 * I, I, 3 * I, 14 * I + 8]))      # world 3: ten intervals behind: one
    assert s.tick_counts["resynchronisations"] == 1
    assert s.time.tolist() == [2 * I, I, 3 * I, 14 * I + 8]
    assert [b.ticked.tolist() for b in batches] == [[True, False, False, True]]


def test_a_masked_tick_keeps_the_queue_and_the_stamp_of_a_world_without_a_tick():
    s, park = _clock_server(worlds=2, per=2)
    both = torch.tensor([True, True])
    s.push("SetSpeedFraction", both, torch.tensor([1, 2]), f=torch.tensor([[0.5], [0.5]]))
    on = torch.tensor([True, False])
    s.pre_tick(mask=on)
    s.evolve(mask=on)
    s.post_tick(mask=on)
    assert s.batch.slots[0].ok.tolist() == [True, False] and s.batch.ticked.tolist() == [True, False]
    assert [q.ok.tolist() for q in s.slots] == [[False, True]]           # world 1's call kept
    assert s.stamp_for_system.tolist() == [1, 0]
    assert s.batch.has_character.tolist()[2:] == [False, False]          # a world without a tick sends nothing
    s.push("SetSpeedFraction", both, torch.tensor([1, 2]), f=torch.tensor([[0.5], [0.5]]))
    assert s.slots[-1].ok.tolist() == [True, False]                      # world 1: the same call is still its last
    s.pre_tick()
    assert [q.ok.tolist() for q in s.batch.slots] == [[False, True], [True, False]]


def test_decode_sends_each_pilot_its_updates_in_destinys_order():
    """One world, two piloted balls: a call routed to the bubble goes to both pilots' narrowcast; the first pre-tick's
    additions (none listed without a cloak change here: the fields stand in) are a PackagedAction in the singlecast."""
    from exact_ballpark_b200 import server
    s, park = _clock_server(worlds=1, per=2, pilots=[0, 1])
    s.push("SetSpeedFraction", torch.tensor([True]), torch.tensor([2]), f=torch.tensor([[0.25]]))
    s.pre_tick(snapshot=False)
    s.evolve()
    s.post_tick()
    b = s.batch
    assert b.route.tolist() == [[server.BUBBLE]]
    assert b.gets_bubble.tolist() == [True, True] and b.has_character.tolist() == [True, True]
    with pytest.raises(ValueError):                       # the additions' streams were not recorded
        server.decode(s)
    b.additions = (torch.zeros(2, dtype=torch.bool), b.additions[1], None)
    b.has_character = torch.zeros(2, dtype=torch.bool)
    sent = server.decode(s)
    event = (0, ("SetSpeedFraction", (2, 0.25)))
    assert sent == [{10000: [("narrow", "DoDestinyUpdate", [event], False, server.ClientUpdateCountThisTick.ONE)],
                     10001: [("narrow", "DoDestinyUpdate", [event], False, server.ClientUpdateCountThisTick.ONE)]}]


def test_a_client_view_lags_down_ticks_and_hides_the_other_pilots_cloaked_ships():
    from exact_ballpark_b200 import server
    s, park = _clock_server(worlds=2, per=2)
    park.pos = torch.zeros(4, 3, dtype=torch.float64)
    view = server.ClientView(s, down=2, fields=("pos", "clock"))
    with pytest.raises(ValueError):
        server.ClientView(s, down=-1)
    for t in range(1, 6):
        park.pos[:, 0] = float(t)
        park.cloaked.copy_(torch.tensor([0, 1, 0, 0]) if t >= 3 else torch.zeros(4, dtype=torch.int64))
        s.evolve()
        view.record(t)
        time, fields, present = view.view()
        if t <= 2:
            assert time == -1 and fields == {} and present is None
            continue
        assert time == t - 2
        assert fields["pos"][:, 0].tolist() == [float(t - 2)] * 4
        assert fields["clock"].tolist() == [t - 2] * 4
        hidden = t - 2 >= 3                                   # row 1 cloaked in the state the clients hold
        assert present[1].tolist() == [not hidden, True, False, False]      # its own pilot still holds it
        assert present[0].tolist() == [True, True, False, False]
        assert present[2].tolist() == [False, False, True, True]


def test_the_kernel_path_wants_a_cuda_device_and_a_known_path():
    from exact_ballpark_b200 import server
    with pytest.raises(ValueError):
        server.VecServer(_StandIn(), kernel="triton")
    with pytest.raises(ValueError):
        server.VecServer(_StandIn(), kernel="cuda")
