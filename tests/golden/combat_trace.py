"""Golden traces of the combat park (missiles, formations, cloaking, AddBall and RemoveBall mid-run): a scenario as
the reference's combat scenario generator states it (worlds of ships, a pool of missile rows, records applied at
given steps), the driver that applies it to any park with the reference's combat API, and the park's state after
every step as per-field digests.

A scenario batch is a configuration (friction, tick, the orbit law, master or client, dynamical orientation's missile
exclusion) and its worlds; each world is its ships, its pool's empty rows and its records [(step, op, *args)]. Step 0
is the set-up; after the records of each later step every park evolves one tick. The driver applies a step's j-th
record of every world together, one masked command per kind of record (the worlds are independent), as the
reference's batch harness does; the ReserveFormationSlot answers are collected per world, and the DoCollision events
after every tick.

`make_golden.py` records batches by driving the reference's own combat park (exact_ballpark.vec_combat.VecCombatPark,
its tick on tensors on the CPU, held bit for bit by the reference to its scalar FullBallpark) with this driver; the
tests replay the same batches on this package's park and on the oracle and compare the digests step by step.

A step's digest covers every field a command or a tick may change (FIELDS), over the rows holding a ball at that step
(`exists`, itself a field over every row), each canonicalised: floats as float64 bit patterns with every NaN made one
quiet NaN, integers and flags as int64.
"""

from __future__ import annotations

import gzip
import hashlib
import json
from collections import defaultdict
from pathlib import Path

import numpy as np
import torch

GOLDEN = Path(__file__).resolve().parent

FIELDS = ("pos", "vel", "old_pos", "old_vel", "goto", "last_g", "mode", "effect_stamp", "follow_id", "owner_id",
          "massive", "cloaked", "speed_fraction", "follow_range", "last_collision", "formation_id", "formation_slots",
          "mass", "radius", "max_vel", "agility", "time_factor", "rot", "old_rot", "ang_vel", "old_ang_vel", "torque",
          "rot_roll", "ids", "free", "moribund", "interactive", "sensor", "follow_ptr", "owner_ptr", "clock")
_QNAN = np.uint64(0x7FF8000000000000)


def canonical(t) -> np.ndarray:
    a = t.detach().cpu() if isinstance(t, torch.Tensor) else torch.as_tensor(np.asarray(t))
    if a.dtype in (torch.float64, torch.float32, torch.float16):
        x = np.ascontiguousarray(a.to(torch.float64).numpy())
        bits = x.view(np.uint64).copy()
        bits[np.isnan(x)] = _QNAN
        return bits.view(np.float64)
    return np.ascontiguousarray(a.to(torch.int64).numpy())


COMPOSED_FIELDS = FIELDS + ("last_c", "level", "key", "mod", "hits_n", "collisions")
LIST_WIDTH = 192                    # a collision list as a digest holds it: its entries, then -1 up to this width


def _field(park, f: str) -> np.ndarray:
    if f != "collisions":
        return canonical(getattr(park, f))
    hits, n = canonical(park.hits), canonical(park.hits_n)
    out = np.full((hits.shape[0], LIST_WIDTH), -1, dtype=np.int64)
    for r in np.nonzero(n)[0].tolist():
        out[r, :n[r]] = hits[r, :n[r]]
    return out


def field_digests(park, fields: tuple = FIELDS) -> np.ndarray:
    """[len(fields) + 1] uint64: each field's digest over the rows holding a ball, then `exists` over every row (the
    collision list as its entries, padded with -1 to LIST_WIDTH)."""
    exists = canonical(park.exists).astype(bool)
    out = np.zeros(len(fields) + 1, dtype=np.uint64)
    for i, f in enumerate(fields):
        a = _field(park, f)[exists]
        h = hashlib.sha256(f.encode() + str(a.shape).encode() + a.tobytes()).digest()
        out[i] = np.frombuffer(h[:8], dtype=np.uint64)[0]
    e = exists.astype(np.int64)
    out[-1] = np.frombuffer(hashlib.sha256(b"exists" + e.tobytes()).digest()[:8], dtype=np.uint64)[0]
    return out


def first_mismatch(want: np.ndarray, got: np.ndarray, fields: tuple = FIELDS) -> list:
    names = fields + ("exists",)
    return [names[i] for i in range(len(names)) if want[i] != got[i]]


# ---- the batch's rows ----

def rows_for(cfg: dict) -> tuple:
    """Each world's ships then its pool's empty rows, in world order: (rows, {(world, id): row})."""
    rows, where = [], {}
    bubble = 0 if cfg["master"] else -1
    for wi, w in enumerate(cfg["worlds"]):
        for s in w["ships"]:
            where[(wi, s["id"])] = len(rows)
            rows.append({**s, "world": wi, "time": w["start"], "bubble": bubble})
        for mid in w["pool"]:
            where[(wi, mid)] = len(rows)
            rows.append({"id": mid, "world": wi, "time": w["start"], "exists": False, "mass": 1.0, "radius": 1.0,
                         "max_vel": 1.0, "pos": [0.0, 0.0, 0.0], "vel": [0.0, 0.0, 0.0], "agility": 1.0,
                         "speed_fraction": 1.0, "bubble": bubble})
    return rows, where


def make_park(park_cls, cfg: dict, formations: list, device, **extra):
    rows, where = rows_for(cfg)
    p = park_cls(len(rows), cfg["friction"], cfg["tick"], device, True, cfg["new_orbit"], master=cfg["master"],
                 disable_do_for_missiles=cfg["do_off"], **extra)
    p.load(rows)
    p.load_formations(formations)
    return p, where


# ---- the driver ----

def _t(x, dev) -> torch.Tensor:
    """A park's per-row array as a tensor (the oracle's parks hold numpy arrays)."""
    return x if isinstance(x, torch.Tensor) else torch.as_tensor(np.asarray(x), device=dev)


def _one_kind(p, op: str, group: dict, where: dict, n: int, answers: list, dev) -> None:
    """The records `group` {world: record} of one kind, as one masked command (or, for the slot calls, one call a
    world in world order)."""
    I64, F64, BOOL = torch.int64, torch.float64, torch.bool
    if op == "add":
        placed = sorted((where[(wi, rec[2]["id"])], rec[2]) for wi, rec in group.items())
        m = torch.zeros(n, dtype=BOOL, device=dev)
        m[[r for r, _ in placed]] = True
        p.add_balls(m, [b for _, b in placed])
        return
    if op in ("reserve_follow", "reserve", "free"):
        for wi in sorted(group):
            args = group[wi][2:]
            r = where.get((wi, args[0]))
            if r is None:
                continue
            if op == "reserve_follow":
                lr = where.get((wi, args[1]))
                slot = p.reserve_formation_slot(lr) if lr is not None and bool(p.exists[lr]) else -1
                answers[wi].append(slot)
                if slot >= 0:
                    one = torch.zeros(n, dtype=BOOL, device=dev)
                    one[r] = True
                    p.formation_follow(one, torch.full((n,), args[1], dtype=I64, device=dev),
                                       torch.full((n,), slot, dtype=I64, device=dev))
            elif op == "reserve":
                answers[wi].append(p.reserve_formation_slot(r) if bool(p.exists[r]) else -1)
            elif bool(p.exists[r]):
                p.free_formation_slot(r, args[1])
        return
    mask = np.zeros(n, dtype=bool)
    ints = np.zeros((4, n), dtype=np.int64)
    vec = np.zeros((n, 3), dtype=np.float64)
    one = np.zeros(n, dtype=np.float64)
    for wi, rec in group.items():
        args = rec[2:]
        r = where.get((wi, args[0]))
        if r is None:
            continue
        mask[r] = True
        if op in ("goto", "dir", "vel"):
            vec[r] = args[1:4]
        elif op == "warp":
            vec[r], one[r], ints[0, r] = args[1:4], args[4], args[5]
        elif op in ("massive", "cloak", "setform"):
            ints[0, r] = args[1]
        elif op == "launch":
            ints[:, r] = args[1:5]
        elif op in ("mfollow", "formfollow"):
            ints[0, r], ints[1, r] = args[1], args[2]
        elif op in ("follow", "orbit"):
            ints[0, r], one[r] = where.get((wi, args[1]), -1), args[2]
        elif op == "warpin":
            vec[r], ints[0, r] = args[1:4], args[4]
        elif op in ("radius", "maxvel", "sf", "mass"):
            one[r] = args[1]
    m = torch.tensor(mask, dtype=BOOL, device=dev)
    A, B, C, D = (torch.tensor(ints[k], dtype=I64, device=dev) for k in range(4))
    V = torch.tensor(vec, dtype=F64, device=dev)
    live = m & _t(p.exists, dev)
    if op == "goto":
        p.goto_point(live, V)
    elif op == "dir":
        p.goto_direction(live, V)
    elif op == "stop":
        p.stop(live)
    elif op == "warp":
        p.warp_to(live, V, torch.tensor(one, dtype=F64, device=dev), A)
    elif op == "vel":
        p.set_velocity(live, V)
    elif op == "massive":
        p.massive = torch.where(live, A != 0, _t(p.massive, dev))
    elif op == "launch":
        p.launch_missile(m, A, B, C, D)
    elif op == "mfollow":
        p.missile_follow(m, A, B)
    elif op == "cloak":
        p.cloak(m, A)
    elif op == "uncloak":
        p.uncloak(m)
    elif op == "remove":
        p.remove(m)
    elif op == "setform":
        p.set_ball_formation(m, A)
    elif op == "formfollow":
        p.formation_follow(m, A, B)
    elif op in ("follow", "orbit", "warpin", "radius", "maxvel", "sf", "mass"):
        X1 = torch.tensor(one, dtype=F64, device=dev)
        if op == "follow":
            p.follow(live, A, X1)
        elif op == "orbit":
            p.orbit(live, A, X1)
        elif op == "warpin":
            p.entity_warp_in(live, V, A)
        elif op == "radius":
            p.set_radius(live, X1)
        elif op == "maxvel":
            p.set_max_velocity(live, X1)
        elif op == "sf":
            p.set_speed_fraction(live, X1)
        else:
            p.set_mass(live, X1)
    else:
        raise ValueError(f"unknown record {op!r}")


def drive(p, cfg: dict, where: dict, on_step=None, tick=None) -> dict:
    """Run a batch on park p (made by make_park): {"A": answers per world, "E": events [(world, time, missile,
    collider)]}. on_step(step, park) after each step's records and tick; tick(park) replaces p.evolve()."""
    W = len(cfg["worlds"])
    n = p.n
    dev = p.dev
    answers = [[] for _ in range(W)]
    events = []
    by_step = [defaultdict(list) for _ in range(W)]
    for wi, w in enumerate(cfg["worlds"]):
        for rec in w["records"]:
            by_step[wi][rec[0]].append(rec)
    for s in range(cfg["steps"] + 1):
        depth = max(len(by_step[wi].get(s, ())) for wi in range(W))
        for j in range(depth):
            kinds: dict = {}
            for wi in range(W):
                recs = by_step[wi].get(s, ())
                if j < len(recs):
                    kinds.setdefault(recs[j][1], {})[wi] = recs[j]
            for op, group in kinds.items():
                _one_kind(p, op, group, where, n, answers, dev)
        if s > 0:
            (tick or (lambda q: q.evolve()))(p)
            events.extend(tuple(int(x) for x in e) for e in p.events())
        if on_step is not None:
            on_step(s, p)
    return {"A": answers, "E": events}


# ---- the golden bundle ----

def _tuples(x):
    if isinstance(x, list):
        return tuple(_tuples(v) for v in x)
    return x


def save(path: Path, formations: list, batches: list) -> None:
    """batches: [{"cfg", "digests" [steps + 1, F + 1] uint64, "events", "answers"}]."""
    body = {"formations": formations,
            "batches": [{"cfg": b["cfg"], "events": b["events"], "answers": b["answers"]} for b in batches]}
    with gzip.open(str(path) + ".json.gz", "wt") as f:
        json.dump(body, f)
    np.savez_compressed(str(path) + ".npz", **{f"b{i}": b["digests"] for i, b in enumerate(batches)})


def load(path: Path) -> tuple:
    """(formations, batches) with each batch's cfg records as tuples, digests, events and answers."""
    with gzip.open(str(path) + ".json.gz", "rt") as f:
        body = json.load(f)
    z = np.load(str(path) + ".npz")
    out = []
    for i, b in enumerate(body["batches"]):
        cfg = b["cfg"]
        for w in cfg["worlds"]:
            w["records"] = [tuple(r) for r in w["records"]]
        out.append({"cfg": cfg, "digests": z[f"b{i}"], "events": [tuple(e) for e in b["events"]],
                    "answers": b["answers"]})
    return body["formations"], out


def replay(p, batch: dict, where: dict, tick=None, fields: tuple = FIELDS) -> list:
    """Drive a recorded batch on park p; the differences: [(step, fields)] for digests, then events and answers."""
    bad = []

    def on_step(s, q):
        mm = first_mismatch(batch["digests"][s], field_digests(q, fields), fields)
        if mm:
            bad.append((s, mm))
    got = drive(p, batch["cfg"], where, on_step, tick)
    if [tuple(e) for e in got["E"]] != [tuple(e) for e in batch["events"]]:
        bad.append(("events", got["E"][:6], batch["events"][:6]))
    if got["A"] != batch["answers"]:
        bad.append(("answers", got["A"], batch["answers"]))
    return bad
