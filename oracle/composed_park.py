"""TEST INFRASTRUCTURE, NOT THE PRODUCT. The CPU oracle's composed park: the reference composed park's API (the combat
park's, with the collision acceleration, the partition's filing, the collision lists and the commands that re-file) on
numpy arrays, with the tick in the C oracle (oracle/flight.cpp's sequential tick with the composed state: each
massive ball's Gradient at its own turn in ascending id, the others as they stand then; oracle_composed_tick_mt) and
the filings there too (oracle_composed_file). Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it.

The commands restate exact_ballpark/vec_composed.py (VecComposedPark, :208-300) on numpy.
"""

from __future__ import annotations

import ctypes

import numpy as np

from .combat_park import FLAG_DEFENDER, OracleCombatPark, _Combat
from .park import _BOOL, _F64, _State, f32, lib

FLAG_SENSOR = 256


class _Composed(ctypes.Structure):
    _fields_ = ([(k, ctypes.c_void_p) for k in ("last_c", "level", "key", "mod", "hits")]
                + [("hit_cap", ctypes.c_int64)])


class OracleComposedPark(OracleCombatPark):
    """The reference composed park's API on the CPU (module docstring); collisions on."""

    def __init__(self, n: int, friction: float = 1.0e6, tick_interval_ms: int = 1000, device="cpu",
                 dynamical_orientation: bool = True, use_new_orbit: bool = False, block: int = 128,
                 master: bool = False, disable_do_for_missiles: bool = False, collisions: bool = True):
        if not collisions:
            raise ValueError("the oracle's composed park runs with collisions (without them it is the combat park)")
        super().__init__(n, friction, tick_interval_ms, device, dynamical_orientation, use_new_orbit, block, master,
                         disable_do_for_missiles)
        self.collisions = True
        self.last_c = np.zeros((n, 3))
        self.level = np.zeros(n, dtype=np.int64)
        self.key, self.mod = np.zeros((n, 3), dtype=np.int64), np.zeros((n, 3), dtype=np.int64)
        self.hits = np.full((n, 1), -1, dtype=np.int64)

    # ---- the native calls ----
    def _structs(self):
        for k in _F64:
            setattr(self, k, np.ascontiguousarray(getattr(self, k), dtype=np.float64))
        for k in ("ids", "world", "mode", "effect_stamp", "follow_id", "owner_id", "follow_ptr", "clock", "cloaked",
                  "bubble", "formation_id", "formation_slots", "owner_ptr", "hits_n", "ev_n", "flags", "level", "key",
                  "mod", "hits"):
            setattr(self, k, np.ascontiguousarray(getattr(self, k), dtype=np.int64))
        self.last_c = np.ascontiguousarray(self.last_c, dtype=np.float64)
        bools = {k: np.ascontiguousarray(getattr(self, k), dtype=np.uint8) for k in _BOOL + ("exists", "ev_self")}
        s = _State()
        s.n, s.friction, s.dt, s.ffriction, s.fdt = self.n, self.friction, self.dt, self.ffriction, self.fdt
        s.new_orbit, s.dynamical = int(self.use_new_orbit), 1
        for k in _F64 + ("ids", "world", "mode", "effect_stamp", "follow_id", "owner_id", "follow_ptr", "clock"):
            setattr(s, k, getattr(self, k).ctypes.data)
        for k in _BOOL:
            setattr(s, k, bools[k].ctypes.data)
        c = _Combat()
        for k in ("formation_id", "formation_slots", "owner_ptr", "hits_n", "ev_n", "bubble", "cloaked", "flags"):
            setattr(c, k, getattr(self, k).ctypes.data)
        c.exists, c.ev_self = bools["exists"].ctypes.data, bools["ev_self"].ctypes.data
        table = np.ascontiguousarray(self.formation_table, dtype=np.float64)
        lens = np.ascontiguousarray(self.formation_lengths, dtype=np.int64)
        c.formations, c.formation_len = table.ctypes.data, lens.ctypes.data
        c.n_formations, c.max_slots, c.tick_ms = self.n_formations, self.max_slots, self.tick_ms
        c.do_missiles_off, c.master = int(self.disable_do_for_missiles), int(self.master)
        x = _Composed()
        for k in ("last_c", "level", "key", "mod", "hits"):
            setattr(x, k, getattr(self, k).ctypes.data)
        x.hit_cap = self.hits.shape[1]
        return s, c, x, bools, (table, lens)

    def _done(self, bools) -> None:
        for k, a in bools.items():
            setattr(self, k, a.astype(bool))

    def _file(self, which, pos=None, vel=None, sf=None) -> None:
        which = np.asarray(which, dtype=bool)
        if not which.any():
            return
        s, c, x, bools, keep = self._structs()
        m = np.ascontiguousarray(which, dtype=np.uint8)
        arrs = [None if a is None else np.ascontiguousarray(np.asarray(a, dtype=np.float64)) for a in (pos, vel, sf)]
        ptr = [None if a is None else a.ctypes.data for a in arrs]
        lib().oracle_composed_file(ctypes.byref(s), ctypes.byref(c), ctypes.byref(x), m.ctypes.data, *ptr)
        self._done(bools)

    # ---- loading, adding, the setters that re-file ----
    def load(self, rows: list) -> None:
        super().load(rows)
        S = self.rows_of_world.shape[1] if self.rows_of_world.size else 1
        self.hits = np.full((self.n, max(1, 3 * (S - 1)) + 1), -1, dtype=np.int64)
        self.last_c = np.zeros((self.n, 3))
        self.level = np.zeros(self.n, dtype=np.int64)
        self.key, self.mod = np.zeros((self.n, 3), dtype=np.int64), np.zeros((self.n, 3), dtype=np.int64)
        self._file(self.exists & ~self.moribund)

    def add_balls(self, mask, rows: list) -> None:
        m = self._m(mask)
        super().add_balls(m, rows)
        new = m & self.exists
        self.last_c = np.where(new[:, None], 0.0, self.last_c)
        self.hits = np.where(new[:, None], -1, self.hits)
        self.hits_n = np.where(new, 0, self.hits_n)
        self._file(new)

    def set_radius(self, mask, r) -> None:
        m, v = self._m(mask), self._a(r).astype(np.float64)
        ok = m & ~(f32(v) < 0.0) & self.exists
        super().set_radius(m, v)
        self._file(ok)

    def set_max_velocity(self, mask, v) -> None:
        m, val = self._m(mask), self._a(v).astype(np.float64)
        ok = m & ~(f32(val) < 0.0) & self.exists
        super().set_max_velocity(m, val)
        self._file(ok)

    def launch_missile(self, mask, target, owner, aimed, massive) -> None:
        m = self._m(mask)
        dst, own = self._a(target).astype(np.int64), self._a(owner).astype(np.int64)
        go = m & (dst >= 0) & (self.lookup(np.arange(self.n), np.abs(own)) >= 0) & self.exists
        vel0, sf0 = self.vel.copy(), np.array(self.speed_fraction, dtype=np.float64)
        super().launch_missile(m, dst, own, aimed, massive)
        self._file(go, vel=vel0, sf=sf0)

    def missile_follow(self, mask, target, owner) -> None:
        before = self.flags.copy()
        super().missile_follow(mask, target, owner)
        self.flags = (self.flags & ~FLAG_DEFENDER) | (before & FLAG_DEFENDER)

    def set_free(self, mask, flag) -> None:
        m = self._m(mask)
        f = self._a(flag) != 0
        fix = m & (f != self.free) & ~f
        super().set_free(m, f)
        self._file(fix & self.exists)

    def cloak(self, mask, mode, range_=None) -> None:
        before = self.sensor.copy()
        super().cloak(mask, mode, range_)
        if self.master:
            self.flags = self.flags | np.where(self.sensor & ~before, FLAG_SENSOR, 0)

    # ---- the tick ----
    def watch(self) -> None:
        """With collisions two massive balls meet here: no refusal."""

    def evolve(self, lib_=None, active=None, threads: int = 1) -> None:
        if active is not None:
            raise NotImplementedError("the oracle ticks every world")
        s, c, x, bools, keep = self._structs()
        lib().oracle_composed_tick_mt(ctypes.byref(s), ctypes.byref(c), ctypes.byref(x), int(threads))
        self._done(bools)
        self.current_time += 1

    def events(self) -> list:
        sel = (self.ev_n > 0) | self.ev_self
        order = {w: k for k, w in enumerate(self.labels)}
        out = []
        for r in sorted(np.nonzero(sel)[0].tolist(), key=lambda r: (order[int(self.world[r])], int(self.ids[r]))):
            w, t, i = int(self.world[r]), int(self.clock[r]) - 1, int(self.ids[r])
            out.extend((w, t, i, int(self.hits[r, k])) for k in range(int(self.ev_n[r])))
            if self.ev_self[r]:
                out.append((w, t, i, i))
        return out

    def collision_lists(self) -> list:
        return [tuple(int(v) for v in h[:k]) for h, k in zip(self.hits, self.hits_n)]
