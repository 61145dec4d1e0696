"""TEST INFRASTRUCTURE, NOT THE PRODUCT. The CPU oracle's collision park: the reference's batched collision park's API
(exact_ballpark/vec_collide.py, VecCollidePark: the constructor's worlds x slots, load :550, goto_point :669,
goto_direction :678, stop :683, set_speed_fraction :687, evolve :990) on numpy arrays in its [W, N] layout, the tick in
the C oracle (oracle/collide.cpp, built into oracle/liboracle.so). Only tests/, __graft_entry__.smoke() and bench.py's
CPU baseline use it, as the checker.

The load and the commands restate the reference's on numpy: the same clamps, float32 roundings and guards, in their
order; the decay factor is glibc's exp (the oracle's libm).
"""

from __future__ import annotations

import ctypes
import math

import numpy as np

from .park import f32, lib, libm

GOTO, STOP = 0, 2


class _Collide(ctypes.Structure):
    _fields_ = ([("W", ctypes.c_int64), ("N", ctypes.c_int64), ("C", ctypes.c_int64), ("I", ctypes.c_int64),
                 ("k", ctypes.c_double), ("dt", ctypes.c_double)]
                + [(k, ctypes.c_void_p) for k in (
                    "pos", "vel", "old_pos", "old_vel", "goto", "last_g", "last_c", "mass", "radius", "max_vel",
                    "agility", "speed_fraction", "time_factor", "last_collision", "id", "mode", "level", "key", "mod",
                    "exists", "free", "massive", "junk", "cloaked", "hits", "hits_n", "imp_slot", "imp_n", "imp_s",
                    "imp_closing")]
                + [("S", ctypes.c_int64), ("B", ctypes.c_int64)]
                + [(k, ctypes.c_void_p) for k in ("s_exists", "s_geo", "s_int", "s_keys")])


def _normalized(v: np.ndarray) -> np.ndarray:
    n = np.sqrt(v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1] + v[..., 2] * v[..., 2])
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / np.where(n == 0.0, 1.0, n)
    return np.where((n == 0.0)[..., None], v, v * inv[..., None])


class OracleCollidePark:
    """W worlds of N ball slots on the CPU (module docstring): each world's balls in the first slots, ascending id."""

    def __init__(self, worlds: int, slots: int, friction: float = 1.0e6, tick_interval_ms: int = 1000, device="cpu",
                 statics: int = 0, **_):
        self.W, self.N, self.S = int(worlds), int(slots), int(statics)
        self.dev = "cpu"
        self.friction, self.dt = float(friction), tick_interval_ms * 0.001
        self.current_time = 0
        W, N = self.W, self.N
        self.C, self.I = max(1, 3 * (N - 1)) + self.S, max(1, N - 1)
        self._statics(1)
        z = lambda *s: np.zeros((W, N) + s)
        self.pos, self.vel, self.old_pos, self.old_vel = z(3), z(3), z(3), z(3)
        self.goto, self.last_g, self.last_c = z(3), z(3), z(3)
        self.mass, self.radius, self.max_vel, self.agility, self.speed_fraction, self.time_factor = (
            z(), z(), z(), z(), z(), z())
        self.last_collision = np.full((W, N), -1.0)
        self.id = np.zeros((W, N), dtype=np.int64)
        self.mode = np.full((W, N), STOP, dtype=np.int64)
        self.level = np.zeros((W, N), dtype=np.int64)
        self.key = np.zeros((W, N, 3), dtype=np.int64)
        self.mod = np.zeros((W, N, 3), dtype=np.int64)
        for k in ("exists", "free", "massive", "junk", "cloaked"):
            setattr(self, k, np.zeros((W, N), dtype=bool))
        self.hits = np.full((W, N, self.C), -1, dtype=np.int64)
        self.hits_n = np.zeros((W, N), dtype=np.int64)
        self.imp_slot = np.full((W, N, self.I), -1, dtype=np.int64)
        self.imp_s = np.zeros((W, N, self.I))
        self.imp_closing = np.zeros((W, N, self.I))
        self.imp_n = np.zeros((W, N), dtype=np.int64)
        lib().oracle_collide_tick.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        lib().oracle_collide_filing.argtypes = [ctypes.c_void_p, ctypes.c_void_p]

    def _statics(self, boxes: int) -> None:
        W, S = self.W, max(self.S, 1)
        self.B = max(1, int(boxes))
        self.s_exists = np.zeros((W, S), dtype=bool)
        self.s_geo = np.zeros((W, S, 175))
        self.s_int = np.zeros((W, S, 5), dtype=np.int64)
        self.s_keys = np.zeros((W, S, self.B, 3), dtype=np.int64)

    def _state(self) -> _Collide:
        s = _Collide()
        s.W, s.N, s.C, s.I, s.k, s.dt = self.W, self.N, self.C, self.I, self.friction, self.dt
        s.S, s.B = self.S, self.B
        for name, _ in _Collide._fields_[6:]:
            if name in ("S", "B"):
                continue
            a = getattr(self, name)
            if not a.flags["C_CONTIGUOUS"]:
                a = np.ascontiguousarray(a)
                setattr(self, name, a)
            setattr(s, name, a.ctypes.data)
        return s

    def load(self, worlds: list, statics: list | None = None) -> None:
        """AddBall for each world's balls (vec_collide.py:550): ascending id in the slots, the float members rounded
        to floats, AddBall's clamps, the decay factor, STOP, the first filing; then each world's static collidables
        (vec_collide.py:1329; their records from exact_ballpark_b200.statics, which the tests pin to the reference's
        own records)."""
        if len(worlds) != self.W:
            raise ValueError(f"{len(worlds)} worlds for a park of {self.W}")
        self.__init__(self.W, self.N, self.friction, int(round(self.dt * 1000)), statics=self.S)
        if statics is not None:
            from exact_ballpark_b200.statics import static_record
            recs = [[static_record(x) for x in items] for items in statics]
            self._statics(max([len(r[2]) for rs in recs for r in rs], default=1))
            for w, rs in enumerate(recs):
                for j, (g, i, k) in enumerate(rs):
                    self.s_geo[w, j], self.s_int[w, j], self.s_exists[w, j] = g, i, True
                    for b, key in enumerate(k):
                        self.s_keys[w, j, b] = key
        m_all = np.zeros((self.W, self.N))
        for w, balls in enumerate(worlds):
            if len(balls) > self.N:
                raise ValueError(f"world {w} has {len(balls)} balls for {self.N} slots")
            for j, b in enumerate(sorted(balls, key=lambda b: int(b["id"]))):
                radius, max_vel = float(f32(b["radius"])), float(f32(b["max_vel"]))
                agility, sf = float(f32(b.get("agility", 0.0))), float(f32(b.get("speed_fraction", 0.0)))
                mass = float(b["mass"])
                mass = 0.0 if mass < 0.0 else mass
                agility = 1.0 if agility <= 0.0 else agility
                free = bool(b["free"])
                if free and not mass * agility > 0.0:
                    raise ValueError(f"world {w}, ball {b['id']}: a free ball needs a positive mass x agility")
                self.mass[w, j], self.radius[w, j] = mass, 0.0 if radius < 0.0 else radius
                self.max_vel[w, j], self.agility[w, j] = 0.0 if max_vel < 0.0 else max_vel, agility
                self.speed_fraction[w, j] = 0.0 if sf < 0.0 else sf
                m_all[w, j] = mass * agility
                p = [float(c) for c in b["pos"]]
                v = [float(c) for c in b.get("vel", (0.0, 0.0, 0.0))]
                self.pos[w, j], self.vel[w, j] = p, v
                self.old_pos[w, j] = [p[i] - v[i] * self.dt for i in range(3)]
                self.exists[w, j], self.free[w, j] = True, free
                self.massive[w, j], self.junk[w, j] = bool(b["massive"]), bool(b.get("junk", False))
                self.cloaked[w, j] = bool(int(b.get("cloaked", 0)) & 0xFF)
                self.id[w, j] = int(b["id"])
        self.old_vel = self.vel.copy()
        pos_m = m_all > 0
        x = np.where(pos_m, -self.friction * self.dt / np.where(pos_m, m_all, 1.0), 0.0)
        self.time_factor = np.where(pos_m, libm("exp", x.reshape(-1)).reshape(x.shape), 0.0)
        which = np.ascontiguousarray(self.exists.astype(np.uint8))
        lib().oracle_collide_filing(ctypes.byref(self._state()), which.ctypes.data)

    # ---- commands (vec_collide.py:669-697) ----
    def goto_point(self, mask, point) -> None:
        point = np.asarray(point, dtype=np.float64)
        ok = np.asarray(mask, dtype=bool) & self.exists & np.isfinite(point).all(-1)
        self.goto = np.where(ok[..., None], point, self.goto)
        sf0 = ok & (self.speed_fraction == 0.0)
        self.speed_fraction = np.where(sf0, 1.0, self.speed_fraction)
        self.mode = np.where(ok, GOTO, self.mode)

    def goto_direction(self, mask, direction) -> None:
        direction = np.asarray(direction, dtype=np.float64)
        ok = np.asarray(mask, dtype=bool) & np.isfinite(direction).all(-1)
        with np.errstate(invalid="ignore", over="ignore"):
            self.goto_point(ok, self.pos + _normalized(direction) * 1.0e17)

    def stop(self, mask) -> None:
        self.mode = np.where(np.asarray(mask, dtype=bool) & self.exists, STOP, self.mode)

    def set_speed_fraction(self, mask, s) -> None:
        s = f32(np.asarray(s, dtype=np.float64))
        ok = np.asarray(mask, dtype=bool) & self.exists & np.isfinite(s)
        s = np.where(s < 0.0, 0.0, np.where(s > 1.0, 1.0, s))
        self.speed_fraction = np.where(ok, s, self.speed_fraction)

    def evolve(self, active=None, threads: int = 1) -> None:
        act = None if active is None else np.ascontiguousarray(np.asarray(active, dtype=np.uint8))
        lib().oracle_collide_tick(ctypes.byref(self._state()), None if act is None else act.ctypes.data,
                                  int(threads))
        self.current_time += 1
