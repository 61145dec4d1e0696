"""TEST INFRASTRUCTURE, NOT THE PRODUCT. The CPU oracle's flight-mode park: the reference park's API (load, the
commands, the setters, evolve) on numpy arrays in the reference's layout, with the tick, SnapOrientation and the
libm in the C oracle (oracle/flight.cpp, oracle/oracle_libm.cpp, built into oracle/liboracle.so). Only tests/,
__graft_entry__.smoke() and bench.py's CPU baseline use it, as the checker.

The commands restate exact_ballpark/vec_modes.py (VecModesPark, :221-483) and exact_ballpark/vec_orient.py
(VecOrientPark's setters, :382-478) on numpy: the same guards, the same stores, in their order.
"""

from __future__ import annotations

import ctypes
import struct
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

GOTO, FOLLOW, STOP, WARP, ORBIT, MISSILE = 0, 1, 2, 3, 4, 5
BOID, TROLL, MINIBALL, FIELD, RIGID = 7, 8, 9, 10, 11
INERT = (BOID, MINIBALL, FIELD, RIGID)
AU = .1495978707e12
MIN_WARP_DISTANCE_SQ = 10000000000.0

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is not built (run __graft_entry__.build())")
        _lib = ctypes.CDLL(str(LIB_PATH))
        p, i64 = ctypes.c_void_p, ctypes.c_int64
        _lib.oracle_libm.argtypes = [ctypes.c_int, i64, p, p, p]
        _lib.oracle_flight_tick.argtypes = [p]
        _lib.oracle_flight_tick_mt.argtypes = [p, ctypes.c_int]
        _lib.oracle_combat_tick_mt.argtypes = [p, p, ctypes.c_int]
        _lib.oracle_composed_tick_mt.argtypes = [p, p, p, ctypes.c_int]
        _lib.oracle_composed_file.argtypes = [p, p, p, p, p, p, p]
        _lib.oracle_snap.argtypes = [i64, p, p, p, p, p, p]
        _lib.oracle_q_rot_mul.argtypes = [i64, p, p, p, p]
    return _lib


LIBM_FUNCS = {"sin": 0, "cos": 1, "log": 2, "exp": 3, "sincos_sin": 4, "sincos_cos": 5, "pow": 6, "expf": 10,
              "logf": 11, "sinf": 12, "cosf": 13, "acosf": 14, "atanf": 15, "atan2f": 16, "powf": 17}


def libm(name: str, x, y=None) -> np.ndarray:
    """The oracle's glibc function `name` elementwise (floats held in doubles for the float functions; atan2f(y, x),
    pow(x, y))."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(x if y is None else y, dtype=np.float64)
    out = np.empty_like(x)
    rc = lib().oracle_libm(LIBM_FUNCS[name], x.size, x.ctypes.data, y.ctypes.data, out.ctypes.data)
    if rc:
        raise ValueError(name)
    return out


def f32(x) -> np.ndarray:
    with np.errstate(over="ignore"):
        return np.asarray(x, dtype=np.float64).astype(np.float32).astype(np.float64)


class _State(ctypes.Structure):
    _fields_ = ([("n", ctypes.c_int64), ("friction", ctypes.c_double), ("dt", ctypes.c_double),
                 ("ffriction", ctypes.c_float), ("fdt", ctypes.c_float), ("new_orbit", ctypes.c_int32),
                 ("dynamical", ctypes.c_int32)]
                + [(k, ctypes.c_void_p) for k in (
                    "pos", "vel", "old_pos", "old_vel", "goto", "last_g", "mass", "time_factor", "last_collision",
                    "radius", "max_vel", "agility", "speed_fraction", "follow_range", "max_ang_vel", "rot_agility",
                    "rot_roll", "rot", "old_rot", "ang_vel", "old_ang_vel", "torque", "ids", "world", "mode",
                    "effect_stamp", "follow_id", "owner_id", "follow_ptr", "clock", "free", "moribund", "massive",
                    "interactive", "sensor")])


_F64 = ("pos", "vel", "old_pos", "old_vel", "goto", "last_g", "mass", "time_factor", "last_collision", "radius",
        "max_vel", "agility", "speed_fraction", "follow_range", "max_ang_vel", "rot_agility", "rot_roll", "rot",
        "old_rot", "ang_vel", "old_ang_vel", "torque")
_I64 = ("ids", "world", "mode", "effect_stamp", "follow_id", "owner_id", "follow_ptr", "clock", "cloaked", "bubble",
        "refiled")
_BOOL = ("free", "moribund", "massive", "interactive", "sensor")


def _unit(d: np.ndarray) -> np.ndarray:
    norm = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / np.where(norm == 0.0, 1.0, norm)
    return np.where((norm == 0.0)[:, None], d, d * inv[:, None])


class OraclePark:
    """The reference park's API on the CPU (module docstring)."""

    def __init__(self, n: int, friction: float = 1.0e6, tick_interval_ms: int = 1000, device="cpu",
                 dynamical_orientation: bool = False, use_new_orbit: bool = False, block: int = 128, ypr="host"):
        self.n = int(n)
        self.dev = "cpu"
        self.friction = float(friction)
        self.dt = tick_interval_ms * 0.001
        self.fdt = struct.unpack("f", struct.pack("f", self.dt))[0]
        self.ffriction = struct.unpack("f", struct.pack("f", self.friction))[0]
        self.dynamical_orientation = bool(dynamical_orientation)
        self.use_new_orbit = bool(use_new_orbit)
        self.current_time = 0
        z3 = lambda: np.zeros((n, 3))
        self.pos, self.vel, self.old_pos, self.old_vel, self.goto, self.last_g = z3(), z3(), z3(), z3(), z3(), z3()
        self.ang_vel, self.old_ang_vel, self.torque = z3(), z3(), z3()
        self.rot, self.old_rot = np.zeros((n, 4)), np.zeros((n, 4))
        self.rot[:, 3] = 1.0
        self.old_rot[:, 3] = 1.0
        for k in ("mass", "time_factor", "radius", "max_vel", "agility", "speed_fraction", "max_ang_vel",
                  "rot_agility", "rot_roll"):
            setattr(self, k, np.zeros(n))
        self.last_collision = np.full(n, -1.0)
        self.follow_range = np.full(n, 10.0)
        self.ids = np.arange(1, n + 1, dtype=np.int64)
        for k in ("world", "clock", "effect_stamp", "follow_id", "owner_id", "cloaked", "refiled", "mode"):
            setattr(self, k, np.zeros(n, dtype=np.int64))
        self.mode[:] = STOP
        self.follow_ptr = np.full(n, -1, dtype=np.int64)
        self.bubble = np.full(n, -1, dtype=np.int64)
        for k in _BOOL:
            setattr(self, k, np.zeros(n, dtype=bool))

    # ---- load (vec_modes.py:221) ----
    def _decay(self, m: np.ndarray) -> np.ndarray:
        with np.errstate(divide="ignore", invalid="ignore"):
            x = np.full_like(m, -self.friction * self.dt) / m
        return np.where(m <= 0.0, 0.0, libm("exp", x))

    def load(self, rows: list) -> None:
        n = len(rows)
        if n != self.n:
            raise ValueError(f"{n} rows for a park of {self.n}")
        g = lambda k, d=None: np.array([float(r[k] if d is None else r.get(k, d)) for r in rows])
        self.mass = g("mass")
        self.mass = np.where(self.mass < 0.0, 0.0, self.mass)
        self.radius = f32(g("radius"))
        self.radius = np.where(self.radius < 0.0, 0.0, self.radius)
        self.max_vel = f32(g("max_vel"))
        self.max_vel = np.where(self.max_vel < 0.0, 0.0, self.max_vel)
        self.agility = f32(g("agility"))
        self.agility = np.where(self.agility <= 0.0, 1.0, self.agility)
        self.speed_fraction = f32(g("speed_fraction"))
        self.speed_fraction = np.where(self.speed_fraction < 0.0, 0.0, self.speed_fraction)
        self.pos = np.array([[float(c) for c in r["pos"]] for r in rows]).reshape(n, 3)
        self.vel = np.array([[float(c) for c in r["vel"]] for r in rows]).reshape(n, 3)
        self.old_pos = self.pos - self.vel * self.dt
        self.old_vel = self.vel.copy()
        self.goto, self.last_g = np.zeros((n, 3)), np.zeros((n, 3))
        self.time_factor = self._decay(self.mass * self.agility)
        self.rot = np.tile([0.0, 0.0, 0.0, 1.0], (n, 1))
        self.old_rot = self.rot.copy()
        self.ang_vel, self.old_ang_vel, self.torque = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3))
        self.rot_roll = np.zeros(n)
        if self.dynamical_orientation:
            self.max_ang_vel = f32(g("max_ang_vel", 1.0))
            self.max_ang_vel = np.where(self.max_ang_vel < 0.0, 0.0, self.max_ang_vel)
            self.rot_agility = f32(g("rot_agility", 0.9))
            self.rot_agility = np.where(self.rot_agility <= 0.0, 1.0, self.rot_agility)
            angle = f32(-self.fdt * np.zeros(n))                     # -dt |angVel| of a new ball (at rest)
            out = np.zeros((n, 4))
            rot = np.ascontiguousarray(self.rot)
            axis = np.ascontiguousarray(self.ang_vel)
            lib().oracle_q_rot_mul(n, rot.ctypes.data, axis.ctypes.data, np.ascontiguousarray(angle).ctypes.data,
                                   out.ctypes.data)
            self.old_rot = out
            self._snap(np.ones(n, dtype=bool))
        else:
            self.max_ang_vel, self.rot_agility = np.ones(n), f32(np.full(n, 0.9))
        self.ids = np.array([int(r["id"]) for r in rows], dtype=np.int64)
        self.world = np.array([int(r.get("world", 0)) for r in rows], dtype=np.int64)
        self.clock = np.array([int(r.get("time", 0)) for r in rows], dtype=np.int64)
        self.mode = np.array([int(r.get("mode", STOP)) for r in rows], dtype=np.int64)
        b = lambda k, d: np.array([bool(r.get(k, d)) for r in rows], dtype=bool)
        self.free, self.massive = b("free", True), b("massive", False)
        self.interactive, self.moribund = b("interactive", False), b("moribund", False)
        self.cloaked = np.array([int(r.get("cloaked", 0)) for r in rows], dtype=np.int64)
        self.bubble = np.array([int(r.get("bubble", -1)) for r in rows], dtype=np.int64)
        self.sensor = np.zeros(n, dtype=bool)
        self.effect_stamp = np.zeros(n, dtype=np.int64)
        self.follow_id = np.zeros(n, dtype=np.int64)
        self.owner_id = np.zeros(n, dtype=np.int64)
        self.follow_ptr = np.full(n, -1, dtype=np.int64)
        self.follow_range = np.full(n, 10.0)
        self.last_collision = np.full(n, -1.0)

    def _snap(self, mask: np.ndarray) -> None:
        arrs = [np.ascontiguousarray(getattr(self, k)) for k in ("vel", "rot", "old_rot", "ang_vel", "old_ang_vel")]
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        lib().oracle_snap(self.n, m.ctypes.data, *[a.ctypes.data for a in arrs])
        for k, a in zip(("vel", "rot", "old_rot", "ang_vel", "old_ang_vel"), arrs):
            setattr(self, k, a)

    # ---- commands (vec_modes.py:286-483) ----
    def _m(self, mask) -> np.ndarray:
        return np.asarray(mask.cpu() if hasattr(mask, "cpu") else mask).astype(bool).reshape(self.n)

    @staticmethod
    def _a(x) -> np.ndarray:
        return np.asarray(x.cpu() if hasattr(x, "cpu") else x)

    def _following(self) -> np.ndarray:
        return (self.mode == FOLLOW) | (self.mode == ORBIT)

    def _stop_rows(self, mask: np.ndarray) -> None:
        follower = mask & self._following()
        self.effect_stamp = np.where(follower, 0, self.effect_stamp)
        self.follow_ptr = np.where(follower, -1, self.follow_ptr)
        self.follow_id = np.where(follower, 0, self.follow_id)
        self.owner_id = np.where(follower, 0, self.owner_id)
        self.follow_range = np.where(follower, 0.0, self.follow_range)
        self.mode = np.where(mask, STOP, self.mode)

    def stop(self, mask) -> None:
        m = self._m(mask)
        self._stop_rows(m & (self.mode != STOP))

    def goto_point(self, mask, point) -> None:
        m, point = self._m(mask), self._a(point).astype(np.float64).reshape(self.n, 3)
        ok = m & np.isfinite(point).all(axis=1)
        self._stop_rows(ok)
        self.goto = np.where(ok[:, None], point, self.goto)
        self.speed_fraction = np.where(ok & (self.speed_fraction == 0.0), 1.0, self.speed_fraction)
        self.mode = np.where(ok, GOTO, self.mode)

    def goto_direction(self, mask, direction) -> None:
        m, d = self._m(mask), self._a(direction).astype(np.float64).reshape(self.n, 3)
        ok = m & np.isfinite(d).all(axis=1)
        with np.errstate(over="ignore", invalid="ignore"):
            self.goto_point(ok, self.pos + _unit(d) * 1.0e17)

    def _follow(self, mask, target, range_, mode) -> None:
        m = self._m(mask)
        rng = f32(self._a(range_).astype(np.float64))
        target = self._a(target).astype(np.int64)
        inr = (target >= 0) & (target < self.n)
        safe = np.where(inr, target, 0)
        rows = np.arange(self.n)
        ok = (m & np.isfinite(rng) & inr & (safe != rows) & (self.world[safe] == self.world) & ~self.moribund[safe]
              & (self.bubble[safe] == self.bubble) & (self.cloaked[safe] == 0))
        self._stop_rows(ok)
        self.follow_id = np.where(ok, self.ids[safe], self.follow_id)
        self.follow_ptr = np.where(ok, safe, self.follow_ptr)
        self.follow_range = np.where(ok, rng, self.follow_range)
        self.mode = np.where(ok, mode, self.mode)

    def follow(self, mask, target, range_) -> None:
        self._follow(mask, target, range_, FOLLOW)

    def orbit(self, mask, target, range_) -> None:
        self._follow(mask, target, range_, ORBIT)

    def warp_to(self, mask, point, min_range, warp_factor) -> None:
        m = self._m(mask)
        point = self._a(point).astype(np.float64).reshape(self.n, 3)
        mr = self._a(min_range).astype(np.float64)
        wf = self._a(warp_factor).astype(np.int64)
        ok = m & np.isfinite(point).all(axis=1)
        mr = np.where(mr < 0.0, 0.0, mr)
        wf = np.where(wf <= 0, 1, wf)
        d = self.pos - point
        with np.errstate(over="ignore", invalid="ignore"):
            short = ok & ((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]) < MIN_WARP_DISTANCE_SQ)
        self.goto_point(short, point)
        ok = ok & ~short & ~((self.mode == WARP) & (self.goto == point).all(axis=1))
        self._stop_rows(ok)
        self.goto = np.where(ok[:, None], point, self.goto)
        self.effect_stamp = np.where(ok, -1, self.effect_stamp)
        self.follow_range = np.where(ok, 0.0, self.follow_range)
        self.follow_id = np.where(ok, np.ascontiguousarray(mr).view(np.int64), self.follow_id)
        self.owner_id = np.where(ok, wf, self.owner_id)
        self.mode = np.where(ok, WARP, self.mode)

    def _members(self, rows: np.ndarray) -> np.ndarray:
        safe = np.where(self.follow_ptr >= 0, self.follow_ptr, 0)
        return (self.follow_ptr >= 0) & (self.follow_id == self.ids[safe]) & rows[safe]

    def entity_warp_in(self, mask, point, warp_factor) -> None:
        m = self._m(mask)
        point = self._a(point).astype(np.float64).reshape(self.n, 3)
        self.warp_to(m, point, np.zeros(self.n), warp_factor)
        go = m & (self.mode != GOTO)
        f = self._members(go)                                          # StopAllFollowers
        orbiter = f & self.interactive & (self.mode == ORBIT)
        self._stop_rows(f & ~orbiter)
        self.goto_direction(orbiter, self.vel.copy())
        with np.errstate(over="ignore", invalid="ignore"):
            delta = _unit(self.pos - self.goto)
            mr = np.ascontiguousarray(self.follow_id).view(np.float64)
            dst = self.goto + delta * mr[:, None]
        self.goto = np.where(go[:, None], dst, self.goto)
        self.massive = np.where(go, False, self.massive)
        self.sensor = np.where(go, False, self.sensor)
        self.vel = np.where(go[:, None], _unit(point) * AU, self.vel)
        if self.dynamical_orientation:
            self._snap(go)
        self.effect_stamp = np.where(go, np.maximum(self.clock - 5, 0), self.effect_stamp)
        back = self.pos - self.goto
        with np.errstate(over="ignore", invalid="ignore"):
            length = np.sqrt(back[:, 0] * back[:, 0] + back[:, 1] * back[:, 1] + back[:, 2] * back[:, 2])
        self.last_collision = np.where(go, length, self.last_collision)

    def set_velocity(self, mask, v) -> None:
        m, v = self._m(mask), self._a(v).astype(np.float64).reshape(self.n, 3)
        self.vel = np.where(m[:, None], v, self.vel)
        self.old_vel = np.where(m[:, None], v, self.old_vel)
        if self.dynamical_orientation:
            self._snap(m)

    def set_free(self, mask, flag) -> None:
        m, flag = self._m(mask), self._a(flag) != 0
        change = m & (flag != self.free)
        fix = change & ~flag
        self.free = np.where(change, flag, self.free)
        self._stop_rows(fix)
        self.set_velocity(fix, np.zeros_like(self.vel))
        self.last_g = np.where(fix[:, None], 0.0, self.last_g)

    def set_ball_rigid(self, mask) -> None:
        m = self._m(mask)
        self._stop_rows(m)
        self.mode = np.where(m, RIGID, self.mode)

    def set_boid(self, mask, on) -> None:
        m, on = self._m(mask), self._a(on) != 0
        self.mode = np.where(m & on, BOID, self.mode)
        self._stop_rows(m & ~on)

    def set_interactive(self, mask, flag) -> None:
        m = self._m(mask)
        self.interactive = np.where(m, self._a(flag) != 0, self.interactive)

    def set_ball_troll(self, mask, delay) -> None:
        m = self._m(mask)
        d = self._a(delay).astype(np.int64)
        d = np.where(d < 1, 1, d)
        self._stop_rows(m)
        self.set_free(m, np.ones(self.n, dtype=bool))
        self.set_interactive(m, np.ones(self.n, dtype=bool))
        self.effect_stamp = np.where(m, self.clock + d, self.effect_stamp)
        self.mode = np.where(m, TROLL, self.mode)

    # ---- setters (vec_orient.py:403-465) ----
    def set_mass(self, mask, mass) -> None:
        m, v = self._m(mask), self._a(mass).astype(np.float64)
        ok = m & ~(v <= 0.0)
        self.mass = np.where(ok, v, self.mass)
        self.time_factor = np.where(ok, self._decay(self.mass * self.agility), self.time_factor)

    def set_agility(self, mask, a) -> None:
        m, v = self._m(mask), f32(self._a(a))
        ok = m & ~(v <= 0.0)
        self.agility = np.where(ok, v, self.agility)
        self.time_factor = np.where(ok, self._decay(self.mass * self.agility), self.time_factor)

    def set_max_velocity(self, mask, v) -> None:
        m, v = self._m(mask), f32(self._a(v))
        ok = m & ~(v < 0.0)
        self.max_vel = np.where(ok, v, self.max_vel)
        self.refiled = self.refiled + ok.astype(np.int64)

    def set_speed_fraction(self, mask, s) -> None:
        m, s = self._m(mask), f32(self._a(s))
        ok = m & np.isfinite(s)
        s = np.where(s < 0.0, 0.0, np.where(s > 1.0, 1.0, s))
        self.speed_fraction = np.where(ok, s, self.speed_fraction)

    def set_radius(self, mask, r) -> None:
        m, r = self._m(mask), f32(self._a(r))
        ok = m & ~(r < 0.0)
        self.radius = np.where(ok, r, self.radius)
        self.refiled = self.refiled + ok.astype(np.int64)

    def set_max_angular_speed(self, mask, w) -> None:
        m, w = self._m(mask), f32(self._a(w))
        ok = m & ~(w < 0.0)
        self.max_ang_vel = np.where(ok, w, self.max_ang_vel)

    def set_rot_agility(self, mask, a) -> None:
        m, a = self._m(mask), f32(self._a(a))
        ok = m & ~(a <= 0.0)
        self.rot_agility = np.where(ok, a, self.rot_agility)

    def set_angular_velocity(self, mask, w) -> None:
        m, w = self._m(mask), f32(self._a(w).reshape(self.n, 3))
        self.ang_vel = np.where(m[:, None], w, self.ang_vel)
        self.old_ang_vel = np.where(m[:, None], w, self.old_ang_vel)

    def set_rotation(self, mask, q) -> None:
        m = self._m(mask)
        q = f32(self._a(q).reshape(self.n, 4)).astype(np.float32)
        with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
            l2 = ((q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1]) + q[:, 2] * q[:, 2]) + q[:, 3] * q[:, 3]
            length = np.sqrt(l2).astype(np.float32)
            ok = m & (length.astype(np.float64) > 1e-20)
            d = (np.float32(1.0) / np.where(ok, length, np.float32(1.0))).astype(np.float32)
            rot = (q * d[:, None]).astype(np.float32).astype(np.float64)
        self.rot = np.where(ok[:, None], rot, self.rot)
        self.old_rot = np.where(ok[:, None], rot, self.old_rot)
        self.ang_vel = np.where(ok[:, None], 0.0, self.ang_vel)
        self.old_ang_vel = np.where(ok[:, None], 0.0, self.old_ang_vel)

    # ---- the tick ----
    def evolve(self, lib_=None, active=None, threads: int = 1) -> None:
        """One tick of every world (`threads` host threads over disjoint worlds)."""
        if active is not None:
            raise NotImplementedError("the oracle ticks every world")
        for k in _F64:
            setattr(self, k, np.ascontiguousarray(getattr(self, k), dtype=np.float64))
        for k in _I64:
            setattr(self, k, np.ascontiguousarray(getattr(self, k), dtype=np.int64))
        bools = {k: np.ascontiguousarray(getattr(self, k), dtype=np.uint8) for k in _BOOL}
        s = _State()
        s.n, s.friction, s.dt, s.ffriction, s.fdt = self.n, self.friction, self.dt, self.ffriction, self.fdt
        s.new_orbit, s.dynamical = int(self.use_new_orbit), int(self.dynamical_orientation)
        for k in _F64 + ("ids", "world", "mode", "effect_stamp", "follow_id", "owner_id", "follow_ptr", "clock"):
            setattr(s, k, getattr(self, k).ctypes.data)
        for k, a in bools.items():
            setattr(s, k, a.ctypes.data)
        lib().oracle_flight_tick_mt(ctypes.byref(s), int(threads))
        for k, a in bools.items():
            setattr(self, k, a.astype(bool))
        self.current_time += 1
