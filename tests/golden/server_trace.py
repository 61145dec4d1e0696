"""Golden traces of the server layer over the flight-mode park: the reference's server scenarios (worlds of one bubble
with their pilots and each tick's Actions calls, as its server scenario generator states them), the driver that runs
them through any server layer with the reference's API (push, pre_tick, evolve, post_tick, batch), and each tick's
digests: the park's state and the update batch (the stamps, each queued call's flags and rows, the routes, the
uncloaks' recipients and the bubble's additions with the park's fields at each of them, and who gets the bubble's
narrowcast and a character update).

`make_golden.py` records traces by driving the reference's own batched server layer (exact_ballpark.vec_server's
VecServer, its torch path, over its VecModesPark on the CPU), which the reference holds bit for bit to its scalar
server layer (exact_ballpark.server over FullBallpark) on these very scenarios; the tests replay them on this
package's server layer.
"""

from __future__ import annotations

import gzip
import hashlib
import json
from collections import defaultdict
from pathlib import Path

import numpy as np
import torch

import collide_trace as ct
import trace as tr

GOLDEN = Path(__file__).resolve().parent
PARK_FIELDS = tr.FIELDS
STREAM_FIELDS = ("ids", "mode", "radius", "pos", "free", "massive", "interactive", "mass", "cloaked", "max_vel", "vel",
                 "agility", "speed_fraction", "goto", "follow_id", "follow_range", "effect_stamp", "last_collision",
                 "owner_id", "rot", "max_ang_vel", "ang_vel", "rot_agility")
ACTION_KINDS = {"go_to_point": "GotoPoint", "go_to_direction": "GotoDirection", "stop": "Stop",
                "follow_ball": "FollowBall", "orbit": "Orbit", "warp_to": "WarpTo", "entity_warp_in": "EntityWarpIn",
                "set_speed_fraction": "SetSpeedFraction", "set_max_speed": "SetMaxSpeed",
                "set_ball_mass": "SetBallMass", "set_ball_agility": "SetBallAgility",
                "set_ball_radius": "SetBallRadius", "set_ball_velocity": "SetBallVelocity",
                "set_ball_massive": "SetBallMassive", "set_ball_interactive": "SetBallInteractive",
                "set_ball_position": "SetBallPosition", "cloak_ball": "CloakBall", "uncloak_ball": "UncloakBall",
                "set_max_angular_speed": "SetMaxAngularSpeed", "set_ball_angular_velocity": "SetBallAngularVelocity",
                "set_ball_rotation": "SetBallRotation", "set_ball_angular_agility": "SetBallAngularAgility",
                "set_max_angular_velocity": "SetMaxAngularVelocity"}


def _h(name: str, a) -> np.uint64:
    x = tr.canonical(a)
    d = hashlib.sha256(name.encode() + str(x.shape).encode() + x.tobytes()).digest()
    return np.frombuffer(d[:8], dtype=np.uint64)[0]


def _fields_digest(fields) -> np.uint64:
    if fields is None:
        return np.uint64(0)
    parts = [_h(k, fields[k]) for k in STREAM_FIELDS if k in fields]      # (a collision park has no rotation)
    d = hashlib.sha256(np.array(parts, dtype=np.uint64).tobytes() + bytes([int(bool(fields["dynamical"]))])).digest()
    return np.frombuffer(d[:8], dtype=np.uint64)[0]


def batch_digests(server, b=None) -> np.ndarray:
    """The last tick's update batch (or the batch b) as digests (uint64): the stamps and clocks, the routes, each
    queued call's kind, queued flag, row, target row and local argument, each uncloak's recipients and the park's
    fields there, the bubble's additions (fresh, listed, fields), and the narrowcast and character flags."""
    b = server.batch if b is None else b
    out = [_h("stamp", b.stamp), _h("clock", b.clock), _h("route", b.route.to(torch.int64))]
    for j, s in enumerate(b.slots):
        out += [np.uint64(s.kind), _h(f"ok{j}", s.ok), _h(f"row{j}", s.row), _h(f"trow{j}", s.trow),
                _h(f"loc{j}", s.loc)]
    for j, rec, fields in b.notices:
        out += [np.uint64(j), _h("notice", rec), _fields_digest(fields)]
    fresh, listed, fields = b.additions
    out += [_h("fresh", fresh), _h("listed", listed), _fields_digest(fields), _h("gets_bubble", b.gets_bubble),
            _h("has_character", b.has_character)]
    return np.array(out, dtype=np.uint64)


# ---- the batch's park and server ----

def park_digests(park_kind: str, park) -> np.ndarray:
    return (ct.field_digests(park) if park_kind == "collide" else tr.field_digests(park))


def park_fields(park_kind: str) -> tuple:
    return ct.FIELDS if park_kind == "collide" else PARK_FIELDS


def build(server_mod, park_cls, cs: list, do: bool, device, friction: float = 1.0e6, tick_ms: int = 1000,
          kernel: str | None = None, park: str = "modes"):
    """The server layer (server_mod's VecServer over its ModesAdapter, or its CollideAdapter for park "collide";
    `kernel` its path, when given) over a park of the worlds cs: (server, {(world, ball id): row})."""
    if park == "collide":                                # W worlds of N slots, a world's balls in ascending id
        slots = max(len(w["balls"]) for w in cs)
        p = park_cls(len(cs), slots, friction=friction, tick_interval_ms=tick_ms, device=device)
        p.load([[{"id": b["id"], "mass": b["mass"], "radius": b["radius"], "max_vel": b["max_vel"],
                  "agility": b["agility"], "speed_fraction": b["sf"], "pos": b["pos"], "vel": b["vel"], "free": True,
                  "massive": b["massive"]} for b in w["balls"]] for w in cs])
        index, inter = {}, []
        for wi, w in enumerate(cs):
            by_id = {b["id"]: b for b in w["balls"]}
            flags = [False] * slots
            for k, bid in enumerate(sorted(by_id)):
                index[(w["id"], bid)] = wi * slots + k
                flags[k] = by_id[bid]["interactive"]
            inter += flags
        a = server_mod.CollideAdapter(p, interactive=inter)
        pilots = [-1] * a.R
        for w in cs:
            for bid, pp in w["pilots"].items():
                pilots[index[(w["id"], int(bid))]] = pp
        return server_mod.VecServer(a, pilots), index
    rows = [(w, b) for w in cs for b in w["balls"]]
    p = park_cls(len(rows), friction=friction, tick_interval_ms=tick_ms, device=device, dynamical_orientation=do)
    p.load([{"id": b["id"], "world": w["id"], "time": 0, "mass": b["mass"], "radius": b["radius"],
             "max_vel": b["max_vel"], "pos": b["pos"], "vel": b["vel"], "agility": b["agility"],
             "speed_fraction": b["sf"], "free": True, "massive": b["massive"], "interactive": b["interactive"],
             "cloaked": 0, "bubble": 0, "moribund": False, "max_ang_vel": b["max_ang_vel"],
             "rot_agility": b["rot_agility"]} for w, b in rows])
    a = server_mod.ModesAdapter(p)
    index = {(w["id"], b["id"]): i for i, (w, b) in enumerate(rows)}
    pilots = [-1] * a.R
    for w in cs:
        for bid, pp in w["pilots"].items():
            pilots[index[(w["id"], int(bid))]] = pp
    if kernel is None:
        return server_mod.VecServer(a, pilots), index
    return server_mod.VecServer(a, pilots, kernel=kernel), index


def _group(by_kind: dict, W: int, device) -> list:
    """One push a kind for the calls {kind: [(world index, args)]}: [(kind, mask, ball, target, f, n, loc)]."""
    out = []
    for kind, items in by_kind.items():
        mask = torch.zeros(W, dtype=torch.bool)
        ball, target, n, loc = (torch.zeros(W, dtype=torch.int64) for _ in range(4))
        f = torch.zeros(W, 4, dtype=torch.float64)
        for wi, args in items:
            mask[wi] = True
            ball[wi] = int(args[0])
            rest = list(args[1:])
            if kind in ("FollowBall", "Orbit"):
                target[wi], f[wi, 0] = int(rest[0]), float(rest[1])
            elif kind == "WarpTo":
                f[wi, :4] = torch.tensor([float(x) for x in rest[:4]], dtype=torch.float64)
                n[wi] = int(rest[4])
            elif kind == "EntityWarpIn":
                f[wi, :3] = torch.tensor([float(x) for x in rest[:3]], dtype=torch.float64)
                n[wi] = int(rest[3])
            elif kind in ("SetBallMassive", "SetBallInteractive"):
                n[wi] = int(rest[0])
            elif kind == "SetBallPosition":
                f[wi, :3] = torch.tensor([float(x) for x in rest[:3]], dtype=torch.float64)
                loc[wi] = 1 if rest[3] is True else 0
            elif kind == "CloakBall":
                n[wi], f[wi, 0] = int(rest[0]), float(rest[1])
            elif rest:
                f[wi, :len(rest)] = torch.tensor([float(x) for x in rest], dtype=torch.float64)
        out.append((kind, *(x.to(device) for x in (mask, ball, target, f, n, loc))))
    return out


def pushes(cs: list, t: int, device) -> list:
    """Tick t's calls of every world as pushes: the j-th calls of one kind of all worlds together, each world's calls
    in its own order: [(kind, mask, ball, target, f, n, loc)]."""
    out = []
    width = max((len(w["ticks"][t]) for w in cs), default=0)
    for j in range(width):
        by_kind = defaultdict(list)
        for wi, w in enumerate(cs):
            calls = w["ticks"][t]
            if j < len(calls):
                by_kind[ACTION_KINDS[calls[j][0]]].append((wi, calls[j][1]))
        out += _group(by_kind, len(cs), device)
    return out


# the game's queries of the Actions queue and the undo of a pending cloak, between the calls
QUERIES = ("has_pending_cloak", "has_pending_uncloak", "get_pending_cloak_mode", "get_pending_interactive_state",
           "get_pending_speed_fraction")
UNDO = "undo_pending_cloak"


def steps(cs: list, t: int, device) -> list:
    """Tick t of every world with queries and undos among its calls: for each position j, the calls at j as pushes
    (one a kind), then the queries and undos at j (one a name): ("push", ...), ("query", name, mask, ball),
    ("undo", mask, ball)."""
    W = len(cs)
    out = []
    width = max((len(w["ticks"][t]) for w in cs), default=0)
    for j in range(width):
        by_kind, asks = defaultdict(list), defaultdict(list)
        for wi, w in enumerate(cs):
            calls = w["ticks"][t]
            if j >= len(calls):
                continue
            name, args = calls[j]
            if name in QUERIES or name == UNDO:
                asks[name].append((wi, int(args[0])))
            else:
                by_kind[ACTION_KINDS[name]].append((wi, args))
        out += [("push", *p) for p in _group(by_kind, W, device)]
        for name, items in asks.items():
            mask = torch.zeros(W, dtype=torch.bool)
            ball = torch.zeros(W, dtype=torch.int64)
            for wi, b in items:
                mask[wi], ball[wi] = True, b
            mask, ball = mask.to(device), ball.to(device)
            out.append(("undo", mask, ball) if name == UNDO else ("query", name, mask, ball))
    return out


def answer_digest(name: str, res, mask: torch.Tensor) -> np.uint64:
    """A query's answer over every world as one digest: the flag (has_*), or the value where known and the known
    flags (get_*)."""
    if name.startswith("has_"):
        parts = [_h(name, res & mask)]
    else:
        value, known = res
        parts = [_h(name + ":v", torch.where(known, value, torch.zeros_like(value))), _h(name + ":k", known)]
    d = hashlib.sha256(np.array(parts, dtype=np.uint64).tobytes()).digest()
    return np.frombuffer(d[:8], dtype=np.uint64)[0]


def drive_pending(server, cs: list, device, on_tick) -> None:
    """Each tick: the steps in order (pushes, queries, undos), the pre-tick, the park's tick, the post-tick;
    on_tick(t, server, [the answers' digests])."""
    for t in range(len(cs[0]["ticks"])):
        answers = []
        for st in steps(cs, t, device):
            if st[0] == "push":
                server.push(*st[1:])
            elif st[0] == "undo":
                server.undo_pending_cloak(st[1], st[2])
            else:
                name, mask, ball = st[1:]
                answers.append(answer_digest(name, getattr(server, name)(mask, ball), mask))
        server.pre_tick()
        server.evolve()
        server.post_tick()
        on_tick(t, server, np.array(answers, dtype=np.uint64))


def drive(server, cs: list, evolve: bool, device, on_tick=None) -> None:
    """Each tick: the worlds' calls pushed, the pre-tick, the park's tick (unless `evolve` is false), the post-tick;
    on_tick(t, server) after each."""
    for t in range(len(cs[0]["ticks"])):
        for kind, mask, ball, target, f, n, loc in pushes(cs, t, device):
            server.push(kind, mask, ball, target, f, n, loc)
        server.pre_tick()
        if evolve:
            server.evolve()
        server.post_tick()
        if on_tick is not None:
            on_tick(t, server)


def ontick_digests(server, batches: list) -> np.ndarray:
    """One OnTick call as digests: each world's time, first-time flag and park time, the number of rounds run, and
    each round's worlds and update batch."""
    out = [_h("time", server.time), _h("first_time", server.first_time), _h("clock", server.a.clock()),
           np.uint64(len(batches))]
    for b in batches:
        out.append(_h("ticked", b.ticked))
        out += list(batch_digests(server, b))
    return np.array(out, dtype=np.uint64)


def drive_ontick(server, cs: list, device, on_tick) -> None:
    """Each call: the worlds' calls pushed, then OnTick at each world's own simulation time (w["clock"][t]);
    on_tick(t, server, batches)."""
    for t in range(len(cs[0]["clock"])):
        for kind, mask, ball, target, f, n, loc in pushes(cs, t, device):
            server.push(kind, mask, ball, target, f, n, loc)
        sim = torch.tensor([w["clock"][t] for w in cs], dtype=torch.int64)
        on_tick(t, server, server.on_tick(sim))


def canon(x):
    """A decoded value as compared: floats by their bits, ints and bools apart, bytes, a marshalled payload by its
    value (either layer's Marshalled), sequences by type and item."""
    if isinstance(x, bool):
        return ("b", x)
    if isinstance(x, int):
        return ("i", int(x))
    if isinstance(x, float):
        return ("f", "nan" if x != x else x.hex())
    if isinstance(x, (bytes, bytearray)):
        return ("B", bytes(x).hex())
    if type(x).__name__ == "Marshalled":
        return ("M", canon(x.value))
    if isinstance(x, (list, tuple)):
        return (type(x).__name__, tuple(canon(v) for v in x))
    if isinstance(x, dict):
        return ("d", tuple((canon(k), canon(v)) for k, v in x.items()))
    if isinstance(x, str):
        return ("s", x)
    raise TypeError(type(x))


def decode_digest(decoded) -> np.uint64:
    """What every client of every world is sent (a decode's result, or a list of them) as one digest."""
    d = hashlib.sha256(repr(canon(decoded)).encode()).digest()
    return np.frombuffer(d[:8], dtype=np.uint64)[0]


# ---- the golden bundle ----

def save(path: Path, runs: list) -> None:
    """runs: [{"cases", "do", "evolve", "park" [T, F] uint64, "batch": [T arrays], and for runs with queries
    "answers": [T arrays]}]."""
    body = [{"cases": r["cases"], "do": r["do"], "evolve": r["evolve"], "pending": "answers" in r,
             "ontick": bool(r.get("ontick")), "decoded": "decode" in r, "park_kind": r.get("park_kind", "modes")}
            for r in runs]
    with gzip.open(str(path) + ".json.gz", "wt") as f:
        json.dump(body, f)
    arrays = {}
    for i, r in enumerate(runs):
        arrays[f"r{i}_park"] = r["park"]
        for t, b in enumerate(r["batch"]):
            arrays[f"r{i}_batch{t}"] = b
        for t, a in enumerate(r.get("answers", [])):
            arrays[f"r{i}_answers{t}"] = a
        if "decode" in r:
            arrays[f"r{i}_decode"] = np.array(r["decode"], dtype=np.uint64)
    np.savez_compressed(str(path) + ".npz", **arrays)


def load(path: Path) -> list:
    with gzip.open(str(path) + ".json.gz", "rt") as f:
        body = json.load(f)
    z = np.load(str(path) + ".npz")
    for i, r in enumerate(body):
        r["park"] = z[f"r{i}_park"]
        r["batch"] = [z[f"r{i}_batch{t}"] for t in range(len(r["park"]))]
        if r.get("pending"):
            r["answers"] = [z[f"r{i}_answers{t}"] for t in range(len(r["park"]))]
        if r.get("decoded"):
            r["decode"] = z[f"r{i}_decode"]
        for w in r["cases"]:
            w["pilots"] = {int(k): v for k, v in w["pilots"].items()}
            w["ticks"] = [[(c[0], tuple(c[1])) for c in calls] for calls in w["ticks"]]
    return body


def replay(server_mod, park_cls, run: dict, device, kernel: str | None = None) -> list:
    """A recorded run on server_mod's layer over park_cls: the differences [(tick, 'park', fields), (tick, 'batch'),
    (tick, 'answers') or (tick, 'sends')]."""
    kind = run.get("park_kind", "modes")
    server, _ = build(server_mod, park_cls, run["cases"], run["do"], device, kernel=kernel, park=kind)
    names = park_fields(kind)
    bad = []

    def sends(t, decoded):
        if "decode" in run and decode_digest(decoded) != run["decode"][t]:
            bad.append((t, "sends"))

    def check(t, s):
        sends(t, server_mod.decode(s))
        got = park_digests(kind, s.a.park)
        mm = [names[k] for k in range(len(names)) if got[k] != run["park"][t][k]]
        if mm:
            bad.append((t, "park", mm))
        b = batch_digests(s)
        want = run["batch"][t]
        if b.shape != want.shape or not (b == want).all():
            bad.append((t, "batch"))

    if run.get("ontick"):
        def on_call(t, s, batches):
            sends(t, [server_mod.decode(s, b) for b in batches])
            got = park_digests(kind, s.a.park)
            mm = [names[k] for k in range(len(names)) if got[k] != run["park"][t][k]]
            if mm:
                bad.append((t, "park", mm))
            d = ontick_digests(s, batches)
            want = run["batch"][t]
            if d.shape != want.shape or not (d == want).all():
                bad.append((t, "batches"))
        drive_ontick(server, run["cases"], device, on_call)
    elif run.get("pending"):
        def on_tick(t, s, answers):
            check(t, s)
            want = run["answers"][t]
            if answers.shape != want.shape or not (answers == want).all():
                bad.append((t, "answers"))
        drive_pending(server, run["cases"], device, on_tick)
    else:
        drive(server, run["cases"], run["evolve"], device, check)
    return bad
