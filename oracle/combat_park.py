"""TEST INFRASTRUCTURE, NOT THE PRODUCT. The CPU oracle's combat park: the reference combat park's API (load with
empty rows, add_balls, missile_follow, launch_missile, load_formations, set_ball_formation, formation_follow,
reserve_formation_slot, free_formation_slot, cloak, uncloak, remove, evolve, events, check) on numpy arrays in the
reference's layout, with the tick in the C oracle (oracle/flight.cpp's sequential tick with its combat state:
oracle_combat_tick_mt). Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it, as the checker.

The commands restate exact_ballpark/vec_combat.py (VecCombatPark, :172-560) on numpy: the same guards, the same
stores, in their order. Dynamical orientation only (the park it checks has no other path).
"""

from __future__ import annotations

import ctypes

import numpy as np

from .park import FOLLOW, MISSILE, ORBIT, STOP, WARP, OraclePark, _BOOL, _F64, _State, _unit, f32, lib

FORMATION = 12
DSTNORMALCLOAK = 1
FORMATION_MAX_SLOTS = 16
FLAG_DEFENDER, FLAG_UNDEFINED, FLAG_POOL, FLAG_MASSIVE = 1, 2, 16, 32


class _Combat(ctypes.Structure):
    _fields_ = ([(k, ctypes.c_void_p) for k in (
        "exists", "formation_id", "formation_slots", "owner_ptr", "hits_n", "ev_n", "ev_self", "bubble", "cloaked",
        "flags", "formations", "formation_len")]
        + [("n_formations", ctypes.c_int64), ("max_slots", ctypes.c_int64), ("tick_ms", ctypes.c_int64),
           ("do_missiles_off", ctypes.c_int32), ("master", ctypes.c_int32)])


def _char(x) -> np.ndarray:
    return ((np.asarray(x).astype(np.int64) + 128) & 0xFF) - 128


def _f32s(x) -> np.ndarray:
    return np.asarray(x, dtype=np.float32)


def _rotated_vector(q: np.ndarray, v: tuple) -> np.ndarray:
    """GetRotatedVector with dynamical orientation: v turned by RotationMatrix(q) and TransformCoord, in floats."""
    x, y, z, w = (_f32s(q[:, k]) for k in range(4))
    one, two, zero = np.float32(1.0), np.float32(2.0), np.zeros_like(x)
    m = ((one - two * (y * y + z * z), two * (x * y + z * w), two * (x * z - y * w), zero),
         (two * (x * y - z * w), one - two * (x * x + z * z), two * (y * z + x * w), zero),
         (two * (x * z + y * w), two * (y * z - x * w), one - two * (x * x + y * y), zero),
         (zero, zero, zero, zero + one))
    vx, vy, vz = (np.full_like(x, np.float32(c)) for c in v)
    norm = ((m[0][3] * vx + m[1][3] * vy) + m[2][3] * vz) + m[3][3]
    with np.errstate(all="ignore"):
        out = [(((vx * m[0][j] + vy * m[1][j]) + vz * m[2][j]) + m[3][j]) / norm for j in range(3)]
    return np.stack([np.where(norm != 0.0, c, zero) for c in out], axis=1).astype(np.float64)


class OracleCombatPark(OraclePark):
    """The reference combat park's API on the CPU (module docstring)."""

    def __init__(self, n: int, friction: float = 1.0e6, tick_interval_ms: int = 1000, device="cpu",
                 dynamical_orientation: bool = True, use_new_orbit: bool = False, block: int = 128,
                 master: bool = False, disable_do_for_missiles: bool = False, ypr="host"):
        if not dynamical_orientation:
            raise ValueError("the oracle's combat park runs with dynamical orientation")
        super().__init__(n, friction, tick_interval_ms, device, True, use_new_orbit, block, ypr)
        self.tick_ms = int(tick_interval_ms)
        self.tick_interval = int(tick_interval_ms)
        self.master = bool(master)
        self.disable_do_for_missiles = bool(disable_do_for_missiles)
        self.exists = np.ones(n, dtype=bool)
        self.formation_id = np.full(n, -1, dtype=np.int64)
        self.owner_ptr = np.full(n, -1, dtype=np.int64)
        for k in ("formation_slots", "hits_n", "ev_n", "flags"):
            setattr(self, k, np.zeros(n, dtype=np.int64))
        self.ev_self = np.zeros(n, dtype=bool)
        self.load_formations([])

    def __setattr__(self, key, value):
        if hasattr(value, "cpu") and hasattr(value, "numpy"):           # a torch tensor written by a caller
            value = value.detach().cpu().numpy()
        object.__setattr__(self, key, value)

    # ---- loading ----
    def load(self, rows: list) -> None:
        rows = [dict(r) for r in rows]
        for r in rows:
            if not r.get("exists", True):
                r.update(moribund=True, free=False, massive=False, interactive=False, mode=STOP)
        super().load(rows)
        n = self.n
        self.exists = np.array([bool(r.get("exists", True)) for r in rows], dtype=bool)
        self.formation_id = np.full(n, -1, dtype=np.int64)
        self.owner_ptr = np.full(n, -1, dtype=np.int64)
        for k in ("formation_slots", "hits_n", "ev_n", "flags"):
            setattr(self, k, np.zeros(n, dtype=np.int64))
        self.ev_self = np.zeros(n, dtype=bool)
        self.labels = list(dict.fromkeys(self.world.tolist()))
        index = {w: k for k, w in enumerate(self.labels)}
        self.world_index = np.array([index[w] for w in self.world.tolist()], dtype=np.int64)
        groups = [[] for _ in self.labels]
        for r, k in enumerate(self.world_index.tolist()):
            groups[k].append(r)
        width = max((len(g) for g in groups), default=0)
        self.rows_of_world = np.array([g + [-1] * (width - len(g)) for g in groups], dtype=np.int64)

    def lookup(self, rows: np.ndarray, ball: np.ndarray) -> np.ndarray:
        cand = self.rows_of_world[self.world_index[rows]]
        safe = np.maximum(cand, 0)
        hit = (cand >= 0) & self.exists[safe] & (self.ids[safe] == np.asarray(ball, dtype=np.int64)[:, None])
        first = hit.argmax(axis=1)
        return np.where(hit.any(axis=1), cand[np.arange(len(rows)), first], -1)

    def add_balls(self, mask, rows: list) -> None:
        idx = np.nonzero(self._m(mask))[0]
        if len(idx) != len(rows):
            raise ValueError(f"{len(rows)} balls for {len(idx)} rows")
        if not rows:
            return
        ids = np.array([int(r["id"]) for r in rows], dtype=np.int64)
        taken = self.exists[idx] | (self.lookup(idx, ids) >= 0)
        if taken.any():
            self.flags[idx] |= np.where(taken, FLAG_POOL, 0)
            raise ValueError("add_balls: a row is not empty or the id is already in its world")
        sub = OraclePark(len(rows), self.friction, self.tick_ms, "cpu", True, self.use_new_orbit)
        sub.load([{**r, "world": 0, "time": 0} for r in rows])
        names = _F64 + _BOOL + ("ids", "mode", "effect_stamp", "follow_id", "owner_id", "follow_ptr", "cloaked")
        if all("bubble" in r for r in rows):
            names = names + ("bubble",)
        for name in names:
            t = np.array(getattr(self, name), copy=True)
            t[idx] = getattr(sub, name)
            setattr(self, name, t)
        for name, v in (("exists", True), ("formation_id", -1), ("formation_slots", 0), ("owner_ptr", -1)):
            t = np.array(getattr(self, name), copy=True)
            t[idx] = v
            setattr(self, name, t)
        self._refresh_owners()

    def _refresh_owners(self) -> None:
        found = self.lookup(np.arange(self.n), np.abs(self.owner_id))
        self.owner_ptr = np.where(self.exists & (self.mode == MISSILE), found, -1)

    # ---- the follower bookkeeping ----
    def _following(self) -> np.ndarray:
        return (self.mode == FOLLOW) | (self.mode == ORBIT) | (self.mode == MISSILE) | (self.mode == FORMATION)

    def _stop_rows(self, mask: np.ndarray) -> None:
        if self.master:
            self._free_slots(mask & (self.mode == FORMATION) & (self.follow_ptr >= 0))
        self.owner_ptr = np.where(mask & self._following(), -1, self.owner_ptr)
        super()._stop_rows(mask)

    def _formation_len(self, fid: np.ndarray) -> np.ndarray:
        return self.formation_lengths[np.clip(fid, 0, max(0, self.n_formations - 1))]

    def _free_slots(self, rows: np.ndarray) -> None:
        for i in np.nonzero(rows)[0].tolist():                      # one member at a time, as Destiny frees them
            lead = int(self.follow_ptr[i])
            fid = int(self.formation_id[lead])
            if fid == -1 or fid > self.n_formations - 1:
                continue
            if fid < 0:
                self.flags[i] |= FLAG_UNDEFINED
                continue
            slot = int(self.effect_stamp[i]) & ((1 << 64) - 1)
            if slot > ((len(self.formations[fid]) - 1) & ((1 << 64) - 1)):
                continue
            if slot >= FORMATION_MAX_SLOTS:
                self.flags[i] |= FLAG_UNDEFINED
                continue
            self.formation_slots[lead] &= ~(1 << slot)

    def _release_followers(self, rows: np.ndarray) -> None:
        self._release_members(self._members(rows) & self.exists)

    def _release_members(self, f: np.ndarray) -> None:
        missile = f & (self.mode == MISSILE)
        flies = missile | (f & self.interactive & (self.mode == ORBIT))
        self.massive = np.where(missile, False, self.massive)
        self._stop_rows(f & ~flies)
        self.goto_direction(flies, self.vel.copy())

    # ---- missiles ----
    def missile_follow(self, mask, target, owner) -> None:
        m = self._m(mask)
        rows = np.arange(self.n)
        dst, own = self._a(target).astype(np.int64), self._a(owner).astype(np.int64)
        trow = self.lookup(rows, dst)
        tsafe = np.maximum(trow, 0)
        ok = (m & self.exists & (dst >= 0) & (self.ids != dst) & (self.ids != own) & (dst != own) & (trow >= 0)
              & ~self.moribund[tsafe])
        self._stop_rows(ok)
        ok = ok & (self.bubble == self.bubble[tsafe]) & (self.cloaked[tsafe] == 0)
        self.follow_id = np.where(ok, dst, self.follow_id)
        self.follow_ptr = np.where(ok, trow, self.follow_ptr)
        self.follow_range = np.where(ok, -f32(self.radius + self.radius[tsafe]), self.follow_range)
        self.owner_id = np.where(ok, own, self.owner_id)
        self.owner_ptr = np.where(ok, self.lookup(rows, np.abs(own)), self.owner_ptr)
        self.effect_stamp = np.where(ok, self.clock, self.effect_stamp)
        with np.errstate(all="ignore"):
            self.goto = np.where(ok[:, None], _unit(self.vel) * 1.0e16, self.goto)
        self.speed_fraction = np.where(ok, 1.0, self.speed_fraction)
        self.mode = np.where(ok, MISSILE, self.mode)
        self.flags |= np.where(ok & (own < 0), FLAG_DEFENDER, 0)

    def launch_missile(self, mask, target, owner, aimed, massive) -> None:
        m = self._m(mask)
        rows = np.arange(self.n)
        dst, own = self._a(target).astype(np.int64), self._a(owner).astype(np.int64)
        aimed, massive = _char(self._a(aimed)), _char(self._a(massive))
        go = m & (dst >= 0)
        lrow = self.lookup(rows, np.abs(own))
        go = go & (lrow >= 0)
        lsafe = np.maximum(lrow, 0)
        trow = np.where(dst != own, self.lookup(rows, dst), -1)
        has_t = trow >= 0
        tsafe = np.maximum(trow, 0)
        ps = self.pos[lsafe]
        aim = has_t & (aimed == 1) & (self.cloaked[tsafe] == 0)
        with np.errstate(all="ignore"):
            v_aim = _unit(self.pos[tsafe] - ps)
            vs = self.vel[lsafe]
            max_velocity = np.where(aim, 0.0, self.max_vel[lsafe])
            direction = _unit(vs)
            still = (direction[:, 0] * direction[:, 0] + direction[:, 1] * direction[:, 1]
                     + direction[:, 2] * direction[:, 2]) == 0.0
            if (go & ~aim & still).any():
                direction = np.where(still[:, None], _rotated_vector(self.rot[lsafe], (0.0, 0.0, -1.0)), direction)
            speed = np.where(150.0 < max_velocity, max_velocity, 150.0)
            v0 = np.where(aim[:, None], v_aim, vs + direction * speed[:, None])
        here = go & self.exists
        self.massive = np.where(here & (massive != 0), True, self.massive)
        self.pos = np.where(here[:, None], ps, self.pos)
        self.old_pos = np.where(here[:, None], ps, self.old_pos)
        self.set_velocity(here, v0)
        cloaked_t = has_t & (self.cloaked[tsafe] != 0)
        self.goto_direction(here & ~has_t & (max_velocity > 0.0), v0)
        self.missile_follow(go & has_t & ~cloaked_t, dst, own)

    # ---- formations ----
    def load_formations(self, formations: list) -> None:
        f = [[[float(c) for c in v] for v in vectors] for vectors in formations]
        self.formations = f
        self.n_formations = len(f)
        self.max_slots = max([len(v) for v in f] + [1])
        table = np.zeros((max(1, len(f)), self.max_slots, 3))
        for i, vectors in enumerate(f):
            if vectors:
                table[i, :len(vectors)] = vectors
        self.formation_table = table
        self.formation_lengths = np.array([len(v) for v in f] or [0], dtype=np.int64)

    def set_ball_formation(self, mask, formation) -> None:
        m = self._m(mask)
        fid = _char(self._a(formation))
        F = self.n_formations
        ok = m & self.exists & ~(fid > F - 1)
        cur = self.formation_id.copy()
        inside = ok & (cur >= 0)
        leave = inside & (fid == -1)
        self._release_followers(leave)
        self.formation_slots = np.where(leave, 0, self.formation_slots)
        change = inside & (fid != -1) & (fid != cur)
        bad = change & ((fid < 0) | (cur > F - 1))
        self.flags |= np.where(bad, FLAG_UNDEFINED, 0)
        change = change & ~bad
        new_len = self._formation_len(fid)
        shrink = change & (self._formation_len(cur) > new_len)
        safe = np.maximum(self.follow_ptr, 0)
        f = (self.exists & (self.mode == FORMATION) & (self.follow_ptr >= 0) & shrink[safe]
             & (self.effect_stamp > new_len[safe] - 1))
        self._stop_rows(f)
        self.formation_id = np.where(ok & ~bad, fid, self.formation_id)

    def formation_follow(self, mask, leader, slot) -> None:
        m = self._m(mask)
        rows = np.arange(self.n)
        slot, dst = _char(self._a(slot)), self._a(leader).astype(np.int64)
        lrow = self.lookup(rows, dst)
        lsafe = np.maximum(lrow, 0)
        fid = self.formation_id[lsafe]
        ok = (m & self.exists & (self.ids != dst) & (lrow >= 0) & (fid >= 0) & ~(fid > self.n_formations - 1)
              & ~(slot > self._formation_len(fid) - 1))
        self._stop_rows(ok)
        ok = ok & (self.bubble == self.bubble[lsafe]) & (self.cloaked[lsafe] == 0)
        self.follow_id = np.where(ok, dst, self.follow_id)
        self.follow_ptr = np.where(ok, lrow, self.follow_ptr)
        self.effect_stamp = np.where(ok, slot, self.effect_stamp)
        self.mode = np.where(ok, FORMATION, self.mode)
        self.flags |= np.where(ok & (slot < 0), FLAG_UNDEFINED, 0)

    def reserve_formation_slot(self, row: int) -> int:
        fid = int(self.formation_id[row])
        if fid == -1 or fid > self.n_formations - 1:
            return -1
        if fid < 0:
            self.flags[row] |= FLAG_UNDEFINED
            return -1
        n = len(self.formations[fid])
        if n > FORMATION_MAX_SLOTS:
            return -1
        bits = int(self.formation_slots[row])
        for i in range(n):
            if not bits >> i & 1:
                self.formation_slots[row] = bits | (1 << i)
                return i
        return -1

    def free_formation_slot(self, row: int, slot: int) -> None:
        fid = int(self.formation_id[row])
        if fid == -1 or fid > self.n_formations - 1:
            return
        if fid < 0:
            self.flags[row] |= FLAG_UNDEFINED
            return
        full = (1 << 64) - 1
        slot = int(slot) & full
        if slot > ((len(self.formations[fid]) - 1) & full):
            return
        if slot >= FORMATION_MAX_SLOTS:
            self.flags[row] |= FLAG_UNDEFINED
            return
        self.formation_slots[row] = int(self.formation_slots[row]) & ~(1 << slot)

    # ---- cloaking and removal ----
    def cloak(self, mask, mode, range_=None) -> None:
        m = self._m(mask)
        mode = _char(self._a(mode))
        ok = m & self.exists & (mode > 0)
        if self.master:
            rng = f32(np.full(self.n, 2000.0) if range_ is None else self._a(range_).astype(np.float64))
            self.sensor = self.sensor | (ok & (mode == DSTNORMALCLOAK) & ~(f32(self.radius + rng) < 0.0))
        self._release_followers(ok)
        self.cloaked = np.where(ok, mode & 0xFF, self.cloaked)
        self.massive = np.where(ok, False, self.massive)

    def uncloak(self, mask) -> None:
        ok = self._m(mask) & self.exists
        if self.master:
            self.sensor = self.sensor & ~(ok & (self.cloaked == DSTNORMALCLOAK))
        self.cloaked = np.where(ok, 0, self.cloaked)
        warping = (self.mode == WARP) & (self.effect_stamp >= 0)
        self.massive = np.where(ok & ~warping, True, self.massive)

    def remove(self, mask) -> None:
        ok = self._m(mask) & self.exists
        self._stop_rows(ok)
        self._release_followers(ok)
        stale = self._members(ok) & self.exists
        self.follow_ptr = np.where(stale | ok, -1, self.follow_ptr)
        self.exists = self.exists & ~ok
        self.moribund = self.moribund | ok
        for k in ("massive", "interactive", "sensor"):
            setattr(self, k, np.where(ok, False, getattr(self, k)))
        self.formation_id = np.where(ok, -1, self.formation_id)
        self.formation_slots = np.where(ok, 0, self.formation_slots)
        self._refresh_owners()

    # ---- the tick ----
    def evolve(self, lib_=None, active=None, threads: int = 1) -> None:
        if active is not None:
            raise NotImplementedError("the oracle ticks every world")
        self.watch()
        for k in _F64:
            setattr(self, k, np.ascontiguousarray(getattr(self, k), dtype=np.float64))
        for k in ("ids", "world", "mode", "effect_stamp", "follow_id", "owner_id", "follow_ptr", "clock", "cloaked",
                  "bubble", "formation_id", "formation_slots", "owner_ptr", "hits_n", "ev_n", "flags"):
            setattr(self, k, np.ascontiguousarray(getattr(self, k), dtype=np.int64))
        bools = {k: np.ascontiguousarray(getattr(self, k), dtype=np.uint8)
                 for k in _BOOL + ("exists", "ev_self")}
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
        lib().oracle_combat_tick_mt(ctypes.byref(s), ctypes.byref(c), int(threads))
        for k, a in bools.items():
            setattr(self, k, a.astype(bool))
        self.watch()
        self.current_time += 1

    def events(self) -> list:
        sel = (self.ev_n > 0) | self.ev_self
        rows = np.nonzero(sel)[0].tolist()
        order = {w: k for k, w in enumerate(self.labels)}
        out = []
        for r in sorted(rows, key=lambda r: (order[int(self.world[r])], int(self.ids[r]))):
            w, t, i = int(self.world[r]), int(self.clock[r]) - 1, int(self.ids[r])
            out.extend((w, t, i, int(self.follow_id[r])) for _ in range(int(self.ev_n[r])))
            if self.ev_self[r]:
                out.append((w, t, i, i))
        return out

    # ---- the domain ----
    def watch(self) -> None:
        m = self.exists & ~self.moribund & self.massive & (self.mode != MISSILE)
        rw = self.rows_of_world
        two = (m[np.maximum(rw, 0)] & (rw >= 0)).sum(axis=1) > 1
        self.flags = self.flags | np.where(two[self.world_index], FLAG_MASSIVE, 0)

    def world_flags(self) -> list:
        rw = self.rows_of_world
        f = np.where(rw >= 0, self.flags[np.maximum(rw, 0)], 0)
        return [int(np.bitwise_or.reduce(row)) if len(row) else 0 for row in f]

    def check(self) -> None:
        if any(self.world_flags()):
            raise RuntimeError("outside the batched domain")

