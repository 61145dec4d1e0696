"""The collision park on a B200: a drop-in for exact_ballpark.vec_collide.VecCollidePark's gradient method (spheres free
and fixed, and static collidables: capsules and oriented boxes).

The public API is the reference park's (exact_ballpark/vec_collide.py:432-700, 990): the constructor (W worlds of N
ball slots, friction, tick), `load(worlds)` (each world a list of AddBall's arguments), the commands goto_point,
goto_direction, stop and set_speed_fraction on [W, N] masks, `evolve(active=None)`, `check()`, and the [W, N] state
tensors (pos, vel, old_pos, old_vel, goto, last_g, last_c, last_collision, mode, level, key, mod, hits, hits_n, the
impact record imp_slot, imp_s, imp_closing, imp_n, and the balls' properties), in the reference's layout and dtypes.

The tick is the native library's (include/ebb.h: ebb_collide_tick): one launch, a thread block a group of whole worlds,
every free ball's behaviour, Gradient for every free massive ball with its candidates in Partition::GetNearbyBalls'
order, the commit and the re-filing. Nothing waits for the host and nothing is pruned on the host, so the tick can be
captured in a CUDA graph; every contact a ball has is handled (no contact_slots overflow). There is no CPU tick.

Not here (the constructor or the load refuses them): the iterative collision method, minis and force fields, global
balls, the master's bubbles, the `rows` lever (every slot is a row), turning collisions off; balls filed at the
partition grid's edge or wider than a top box and static collidables at its edge (the reference refuses them).
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _native
from .statics import G_SIZE, I_SIZE, static_record

F64, I64, BOOL = torch.float64, torch.int64, torch.bool
GOTO, STOP = 0, 2


class CollideState(ctypes.Structure):
    """include/ebb.h's EbbCollideState, field for field."""
    _fields_ = ([("worlds", ctypes.c_int64), ("slots", ctypes.c_int64), ("hit_cap", ctypes.c_int64),
                 ("impact_cap", ctypes.c_int64), ("friction", ctypes.c_double), ("dt", ctypes.c_double)]
                + [(k, ctypes.c_void_p) for k in (
                    "pos", "vel", "old_pos", "old_vel", "goto_pt", "last_g", "last_c", "mass", "radius", "max_vel",
                    "agility", "speed_fraction", "time_factor", "last_collision", "id", "mode", "level", "key", "mod",
                    "exists", "free_", "massive", "junk", "cloaked", "hits", "hits_n", "imp_slot", "imp_n", "imp_s",
                    "imp_closing")]
                + [("statics", ctypes.c_int64), ("boxes", ctypes.c_int64)]
                + [(k, ctypes.c_void_p) for k in ("s_exists", "s_geo", "s_int", "s_keys")])


_STATE_NAME = {"goto_pt": "goto", "free_": "free"}
_VEC = ("pos", "vel", "old_pos", "old_vel", "goto", "last_g", "last_c")
_SCALAR = ("mass", "radius", "max_vel", "agility", "speed_fraction", "time_factor", "last_collision")
_FLAGS = ("exists", "free", "massive", "junk", "cloaked")


def _f32(x: float) -> float:
    """A double rounded to a float and back; an overflow is an infinity (vec_collide.py:160)."""
    with np.errstate(over="ignore"):
        return float(np.float32(x))


def _normalized(v: torch.Tensor) -> torch.Tensor:
    """Vector3d's Normalize (vec_collide.py:172): times the reciprocal of the length; a zero vector stays zero."""
    n = torch.sqrt(v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1] + v[..., 2] * v[..., 2])
    zero = n == 0.0
    inv = 1.0 / torch.where(zero, torch.ones_like(n), n)
    return torch.where(zero[..., None], v, v * inv[..., None])


class VecCollidePark:
    """W worlds of N ball slots (module docstring); each world's balls fill its first slots in ascending id."""

    def __init__(self, worlds: int, slots: int, friction: float = 1.0e6, tick_interval_ms: int = 1000,
                 iterative: bool = False, collisions: bool = True, contact_slots: int | None = None,
                 locations: int = 48, device="cuda", rows: int | None = None, impact_slots: int | None = None,
                 kernel: str = "cuda", statics: int = 0, minis: bool = False, fields: bool = False,
                 global_balls: bool = False):
        dev = torch.device(device)
        if dev.type != "cuda":
            raise ValueError("the B200 collision park ticks on a CUDA device only (there is no CPU tick)")
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        if iterative or not collisions or minis or fields or global_balls:
            raise ValueError("this park runs the gradient method: no iterative method, minis, force fields or global "
                             "balls, and collisions on")
        if not 0 <= int(statics) <= _native.COLLIDE_MAX_STATICS:
            raise ValueError(f"statics: 0 to {_native.COLLIDE_MAX_STATICS} slots a world")
        if rows is not None and int(rows) != int(slots):
            raise ValueError("every slot is a row here (the rows lever is not taken)")
        if not 1 <= int(slots) <= _native.COLLIDE_MAX_SLOTS:
            raise ValueError(f"slots: 1 to {_native.COLLIDE_MAX_SLOTS}")
        self.W, self.N, self.R, self.S, self.dev = int(worlds), int(slots), int(slots), int(statics), dev
        self.friction, self.dt = float(friction), tick_interval_ms * 0.001
        self.contact_slots, self.impact_slots = contact_slots, impact_slots     # accepted: nothing overflows here
        self.current_time = 0
        W, N = self.W, self.N
        self.C, self.I = max(1, 3 * (N - 1)) + self.S, max(1, N - 1)
        z = lambda *s: torch.zeros((W, N) + s, dtype=F64, device=dev)
        for k in _VEC:
            setattr(self, k, z(3))
        for k in _SCALAR:
            setattr(self, k, z())
        self.last_collision.fill_(-1.0)
        self.id = torch.zeros(W, N, dtype=I64, device=dev)
        self.mode = torch.full((W, N), STOP, dtype=I64, device=dev)
        self.level = torch.zeros(W, N, dtype=I64, device=dev)
        self.key = torch.zeros(W, N, 3, dtype=I64, device=dev)
        self.mod = torch.zeros(W, N, 3, dtype=I64, device=dev)
        for k in _FLAGS:
            setattr(self, k, torch.zeros(W, N, dtype=BOOL, device=dev))
        self.hits = torch.full((W, N, self.C), -1, dtype=I64, device=dev)
        self.hits_n = torch.zeros(W, N, dtype=I64, device=dev)
        self.imp_slot = torch.full((W, N, self.I), -1, dtype=I64, device=dev)
        self.imp_s = torch.zeros(W, N, self.I, dtype=F64, device=dev)
        self.imp_closing = torch.zeros(W, N, self.I, dtype=F64, device=dev)
        self.imp_n = torch.zeros(W, N, dtype=I64, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self._empty_statics(1)
        self._state = None

    def _empty_statics(self, boxes: int) -> None:
        """The static collidable slots, none filled: records [W, S] (exact_ballpark_b200.statics) and box keys."""
        W, S = (self.W, self.S) if self.S else (1, 1)       # a park without static slots holds one empty record
        self.B = max(1, int(boxes))
        self.s_exists = torch.zeros(W, S, dtype=BOOL, device=self.dev)
        self.s_geo = torch.zeros(W, S, G_SIZE, dtype=F64, device=self.dev)
        self.s_int = torch.zeros(W, S, I_SIZE, dtype=I64, device=self.dev)
        self.s_keys = torch.zeros(W, S, self.B, 3, dtype=I64, device=self.dev)
        self._state = None

    def state(self) -> CollideState:
        """include/ebb.h's EbbCollideState over the park's tensors (the same buffers every tick)."""
        if self._state is None:
            s = CollideState()
            s.worlds, s.slots, s.hit_cap, s.impact_cap = self.W, self.N, self.C, self.I
            s.friction, s.dt = self.friction, self.dt
            s.statics, s.boxes = self.S, self.B
            for name, _ in CollideState._fields_[6:]:
                if name in ("statics", "boxes"):
                    continue
                t = getattr(self, _STATE_NAME.get(name, name))
                if not t.is_contiguous():
                    raise RuntimeError(f"{name} is not contiguous")
                setattr(s, name, t.data_ptr())
            self._state = s
        return self._state

    def _stream(self) -> int:
        return torch.cuda.current_stream(self.dev).cuda_stream

    # ---- loading (vec_collide.py:550) ----
    def load(self, worlds: list, statics: list | None = None) -> None:
        """Each world a list of balls (AddBall's arguments: id, mass, radius, max_vel, agility, speed_fraction, pos,
        vel, free, massive, and optionally junk and cloaked): the balls in ascending id in the world's first slots,
        AddBall's float members and clamps, every ball in STOP with its goto point at the origin; on the device the
        decay factors and the first filing. `statics` (a park made with static slots): each world's capsules and
        oriented boxes as AddCapsule and AddOrientedBox take them ({"kind": "capsule", "id", "parent", "a", "b",
        "radius"} or {"kind": "box", "id", "parent", "corner", "lx", "ly", "lz"}), their records made on the host."""
        if len(worlds) != self.W:
            raise ValueError(f"{len(worlds)} worlds for a park of {self.W}")
        W, N = self.W, self.N
        sc = {k: np.zeros((W, N)) for k in ("mass", "radius", "max_vel", "agility", "speed_fraction")}
        vec = {k: np.zeros((W, N, 3)) for k in ("pos", "vel", "old_pos")}
        fl = {k: np.zeros((W, N), dtype=bool) for k in _FLAGS}
        ids = np.zeros((W, N), dtype=np.int64)
        for w, balls in enumerate(worlds):
            if len(balls) > N:
                raise ValueError(f"world {w} has {len(balls)} balls for {N} slots")
            seen = [int(b["id"]) for b in balls]
            if len(set(seen)) != len(seen) or min(seen, default=1) <= 0:
                raise ValueError(f"world {w}: ball ids must be positive and distinct")
            if any("owner" in b or "miniball" in b or b.get("global", False) for b in balls):
                raise ValueError(f"world {w}: owners, miniballs and global balls are not in this park")
            for j, b in enumerate(sorted(balls, key=lambda b: int(b["id"]))):
                radius, max_vel = _f32(b["radius"]), _f32(b["max_vel"])
                agility, sf = _f32(b.get("agility", 0.0)), _f32(b.get("speed_fraction", 0.0))
                mass = float(b["mass"])
                mass = 0.0 if mass < 0.0 else mass
                agility = 1.0 if agility <= 0.0 else agility
                free = bool(b["free"])
                if free and not mass * agility > 0.0:
                    raise ValueError(f"world {w}, ball {b['id']}: a free ball needs a positive mass x agility")
                sc["mass"][w, j], sc["radius"][w, j] = mass, 0.0 if radius < 0.0 else radius
                sc["max_vel"][w, j], sc["agility"][w, j] = 0.0 if max_vel < 0.0 else max_vel, agility
                sc["speed_fraction"][w, j] = 0.0 if sf < 0.0 else sf
                p = [float(c) for c in b["pos"]]
                v = [float(c) for c in b.get("vel", (0.0, 0.0, 0.0))]
                vec["pos"][w, j], vec["vel"][w, j] = p, v
                vec["old_pos"][w, j] = [p[i] - v[i] * self.dt for i in range(3)]
                fl["exists"][w, j], fl["free"][w, j] = True, free
                fl["massive"][w, j], fl["junk"][w, j] = bool(b["massive"]), bool(b.get("junk", False))
                fl["cloaked"][w, j] = bool(int(b.get("cloaked", 0)) & 0xFF)
                ids[w, j] = int(b["id"])
        put = lambda t, a: t.copy_(torch.from_numpy(a))
        for k, a in sc.items():
            put(getattr(self, k), a)
        for k, a in vec.items():
            put(getattr(self, k), a)
        self.old_vel.copy_(self.vel)
        for k, a in fl.items():
            put(getattr(self, k), a)
        put(self.id, ids)
        self.mode.fill_(STOP)
        for t in (self.goto, self.last_g, self.last_c, self.time_factor):
            t.zero_()
        self.last_collision.fill_(-1.0)
        self.level.zero_()
        self.key.zero_()
        self.mod.zero_()
        self.hits.fill_(-1)
        self.hits_n.zero_()
        self.imp_slot.fill_(-1)
        self.imp_s.zero_()
        self.imp_closing.zero_()
        self.imp_n.zero_()
        self.status.zero_()
        self._load_statics(statics)
        with torch.cuda.device(self.dev):
            rc = _native.lib().ebb_collide_load(ctypes.byref(self.state()), self.status.data_ptr(), self._stream())
        _native.check(rc, "ebb_collide_load")
        if int(self.status.item()) & 1:
            raise ValueError("a ball at the partition's edge or wider than a top box: not in this module")
        self.current_time = 0

    def _load_statics(self, statics: list | None) -> None:
        """The worlds' static collidables into the static slots (vec_collide.py:1329): records and filings made once
        on the host (exact_ballpark_b200.statics.static_record); refused beyond the park's slots."""
        if statics is None:
            self._empty_statics(1)
            return
        if len(statics) != self.W:
            raise ValueError(f"{len(statics)} worlds of static collidables for a park of {self.W}")
        recs = []
        for w, items in enumerate(statics):
            if len(items) > self.S:
                raise ValueError(f"world {w} has {len(items)} static collidables for the park's {self.S} slots")
            ids = [int(x["id"]) for x in items]
            if len(set(ids)) != len(ids):
                raise ValueError(f"world {w}: static collidable ids must be distinct")
            recs.append([static_record(x) for x in items])
        self._empty_statics(max([len(r[2]) for rs in recs for r in rs], default=1))
        W, S = self.s_exists.shape
        geo = np.zeros((W, S, G_SIZE))
        ints = np.zeros((W, S, I_SIZE), dtype=np.int64)
        keys = np.zeros((W, S, self.B, 3), dtype=np.int64)
        exists = np.zeros((W, S), dtype=bool)
        for w, rs in enumerate(recs):
            for j, (g, i, k) in enumerate(rs):
                geo[w, j], ints[w, j], exists[w, j] = g, i, True
                if k:
                    keys[w, j, :len(k)] = k
        self.s_geo.copy_(torch.from_numpy(geo))
        self.s_int.copy_(torch.from_numpy(ints))
        self.s_keys.copy_(torch.from_numpy(keys))
        self.s_exists.copy_(torch.from_numpy(exists))

    # ---- commands (vec_collide.py:669-697) ----
    def goto_point(self, mask: torch.Tensor, point: torch.Tensor) -> None:
        """GotoPoint (Ballpark.cpp:4529): ignored for a non-finite point; the point, a speed fraction of 1 if it was
        0, GOTO."""
        point = point.to(device=self.dev, dtype=F64)
        ok = mask.to(self.dev) & self.exists & torch.isfinite(point).all(-1)
        self.goto.copy_(torch.where(ok[..., None], point, self.goto))
        sf0 = ok & (self.speed_fraction == 0.0)
        self.speed_fraction.copy_(torch.where(sf0, torch.ones_like(self.speed_fraction), self.speed_fraction))
        self.mode.copy_(torch.where(ok, torch.full_like(self.mode, GOTO), self.mode))

    def goto_direction(self, mask: torch.Tensor, direction: torch.Tensor) -> None:
        """GotoDirection (Ballpark.cpp:4483): a point 1e17 m along the unit direction."""
        direction = direction.to(device=self.dev, dtype=F64)
        ok = mask.to(self.dev) & torch.isfinite(direction).all(-1)
        self.goto_point(ok, self.pos + _normalized(direction) * 1.0e17)

    def stop(self, mask: torch.Tensor) -> None:
        """Stop (Ballpark.cpp:4556)."""
        self.mode.copy_(torch.where(mask.to(self.dev) & self.exists, torch.full_like(self.mode, STOP), self.mode))

    def set_speed_fraction(self, mask: torch.Tensor, s: torch.Tensor) -> None:
        """SetSpeedFraction: a float, finite only, clamped to [0, 1]."""
        s = s.to(device=self.dev, dtype=F64).to(torch.float32).to(F64)
        ok = mask.to(self.dev) & self.exists & torch.isfinite(s)
        s = torch.where(s < 0.0, torch.zeros_like(s), torch.where(s > 1.0, torch.ones_like(s), s))
        self.speed_fraction.copy_(torch.where(ok, s, self.speed_fraction))

    # ---- the tick ----
    def evolve(self, active: torch.Tensor | None = None, skip: torch.Tensor | None = None) -> None:
        """One tick in every world, or in the worlds where `active` [W] (the others keep their state bit for bit); in
        place, on the device, no host synchronisation."""
        if skip is not None:
            raise ValueError("the master's dead bubbles (skip) are not in this park")
        act = None
        if active is not None:
            act = active.to(device=self.dev, dtype=BOOL).reshape(self.W).contiguous()
        with torch.cuda.device(self.dev):
            rc = _native.lib().ebb_collide_tick(ctypes.byref(self.state()), 0 if act is None else act.data_ptr(),
                                                self.status.data_ptr(), self._stream())
        _native.check(rc, "ebb_collide_tick")
        self.current_time += 1

    def check(self) -> None:
        """The device's status (a re-filing at the partition grid's edge) as an error."""
        st = int(self.status.item())
        if st:
            raise RuntimeError(f"collision park status {st:#x}: a filing at the partition grid's edge")


class CollideGraph:
    """The collision park's tick captured once as a CUDA graph on the park's own buffers: each `tick()` is one replay
    (the commands write the buffers in place)."""

    def __init__(self, park: VecCollidePark):
        self.park = park
        names = [n for n in vars(park) if isinstance(getattr(park, n), torch.Tensor)]
        keep = {n: getattr(park, n).clone() for n in names}
        side = torch.cuda.Stream(device=park.dev)
        side.wait_stream(torch.cuda.current_stream(park.dev))
        with torch.cuda.stream(side):                             # a warm-up launch, undone
            park.evolve()
            for n, v in keep.items():
                getattr(park, n).copy_(v)
        torch.cuda.current_stream(park.dev).wait_stream(side)
        torch.cuda.synchronize(park.dev)
        park.current_time -= 1
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            park.evolve()
        park.current_time -= 1

    def tick(self) -> None:
        self.graph.replay()
        self.park.current_time += 1
