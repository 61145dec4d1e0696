"""The combat park on a B200: a drop-in for exact_ballpark.vec_combat.VecCombatPark (missiles, formations, cloaking,
AddBall and RemoveBall mid-run, on the flight park) and its CUDA tick (exact_ballpark.vec_combat_cuda: `tick`,
`CombatGraph`).

The public API is the reference park's (exact_ballpark/vec_combat.py:147-1121): the constructor (with `master` and
`disable_do_for_missiles`), `load(rows)` (a row with "exists": False is an empty row of its world), `add_balls`,
`missile_follow`, `launch_missile`, `load_formations`, `set_ball_formation`, `formation_follow`,
`reserve_formation_slot`, `free_formation_slot`, `cloak`, `uncloak`, `remove`, the flight park's commands and
setters, `evolve()`, `events()`, `check()`, `watch()`, `world_flags()`, `followers(row)`, and the per-row attributes
in the reference's layout (`exists`, `formation_id`, `formation_slots`, `owner_ptr`, `hits_n`, `ev_n`, `ev_self`,
`flags` besides the flight park's).

The commands are the reference's tensor operations in its order, on the device (correctly rounded +, -, *, /, sqrt,
comparisons and selections; floats as float32 operations); the tick is one launch of the native library
(ebb_combat_tick: tiles of whole worlds, one thread block a tile, the records in shared memory, block barriers between
phase 1, the missiles' contacts and the commit). Dynamical orientation is required: the yaw, pitch and roll path the
reference keeps without it (glibc's double atan2, asin and sin on the host every tick) is not built. Not built
either: mushrooms (AddMushroom, BringOutTheDeads). OnTick's per-world mask runs inside the kernel.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _native
from .modes import (FOLLOW, FORMATION, GOTO, MISSILE, ORBIT, STOP, WARP, MINIBALL, VecModesPark, _int_prop,
                    _plane_prop, _unit)
from .tiles import plan_tiles

F64, F32, I64, I32, BOOL = torch.float64, torch.float32, torch.int64, torch.int32, torch.bool

DSTNORMALCLOAK = 1                  # IDstConstants.h: a normal cloak
MISSILE_GOTO = 1.0e16               # MissileFollow: mGoto 1e16 m along the velocity (Ballpark.cpp:3867)
MISSILE_LAUNCH_SPEED = 150.0        # PyLaunchMissile: at least 150 m/s faster than the launcher (Thunkers.cpp:925)
FORMATION_MAX_SLOTS = 16            # Ball::ReserveFormationSlot's bitset<16> (Ball.cpp:2288)
FLAG_DEFENDER, FLAG_UNDEFINED, FLAG_BUBBLES, FLAG_DEAD, FLAG_POOL, FLAG_MASSIVE = 1, 2, 4, 8, 16, 32
FLAG_NAMES = {FLAG_DEFENDER: "a defender missile", FLAG_UNDEFINED: "a call whose result Destiny leaves undefined",
              FLAG_BUBBLES: "more than one bubble in a world", FLAG_DEAD: "a world without an interactive ball",
              FLAG_POOL: "an AddBall the rows cannot take",
              FLAG_MASSIVE: "two massive balls outside MISSILE mode in a world (no collision code for them here)"}
_ADD_FIELDS = ("pos", "vel", "old_pos", "old_vel", "goto", "last_g", "mass", "time_factor", "last_collision",
               "radius", "max_vel", "agility", "speed_fraction", "follow_range", "max_ang_vel", "rot_agility",
               "rot_roll", "rot", "old_rot", "ang_vel", "old_ang_vel", "torque", "ids", "effect_stamp", "follow_id",
               "owner_id", "mode", "follow_ptr", "free", "moribund", "massive", "interactive", "sensor")
_COMBAT_STORAGE = (("exists", BOOL), ("formation_id", I64), ("formation_slots", I64), ("owner_ptr", I64),
                   ("hits_n", I64), ("ev_n", I64), ("ev_self", BOOL), ("flags", I64))


def _char(x: torch.Tensor) -> torch.Tensor:
    """A conversion to (signed) char: 128 to 255 become negative."""
    return ((x.to(I64) + 128) & 0xFF) - 128


def _fmax(a, b):
    """std::max: (a < b) ? b : a."""
    return torch.where(a < b, b, a)


def _rotated_vector(q: torch.Tensor, v: tuple) -> torch.Tensor:
    """Ball::GetRotatedVector (Ball.cpp:2191) with dynamical orientation: the float vector v turned by the rotations
    q [R, 4] (x, y, z, w floats) through RotationMatrix(Quaternion) and TransformCoord, each float operation rounded
    as Destiny's (float32 tensors); [R, 3] float64."""
    x, y, z, w = (q[:, k].to(F32) for k in range(4))
    one, two = torch.ones_like(x), torch.full_like(x, 2.0)
    zero = torch.zeros_like(x)
    m = ((one - two * (y * y + z * z), two * (x * y + z * w), two * (x * z - y * w), zero),
         (two * (x * y - z * w), one - two * (x * x + z * z), two * (y * z + x * w), zero),
         (two * (x * z + y * w), two * (y * z - x * w), one - two * (x * x + y * y), zero),
         (zero, zero, zero, one))
    vx, vy, vz = (torch.full_like(x, float(c)) for c in v)
    norm = ((m[0][3] * vx + m[1][3] * vy) + m[2][3] * vz) + m[3][3]
    out = [(((vx * m[0][j] + vy * m[1][j]) + vz * m[2][j]) + m[3][j]) / norm for j in range(3)]
    return torch.stack([torch.where(norm != 0.0, c, zero) for c in out], dim=1).to(F64)


class VecCombatPark(VecModesPark):
    """VecModesPark with MISSILE and FORMATION, the missiles' contacts and collision events, cloaking at the park,
    AddBall and RemoveBall mid-run (the module's docstring)."""

    def __init__(self, n: int, friction: float = 1.0e6, tick_interval_ms: int = 1000, device="cuda",
                 dynamical_orientation: bool = True, use_new_orbit: bool = False, block: int = 256,
                 master: bool = False, disable_do_for_missiles: bool = False, ypr: str = "host"):
        if not dynamical_orientation:
            raise ValueError("the B200 combat park needs dynamical orientation (the yaw, pitch and roll path is not "
                             "built)")
        super().__init__(n, friction, tick_interval_ms, device, dynamical_orientation, use_new_orbit, block, ypr)
        self.tick_ms = int(tick_interval_ms)
        self.master = bool(master)
        self.disable_do_for_missiles = bool(disable_do_for_missiles)
        for name, dt in _COMBAT_STORAGE:
            setattr(self, "_" + name, torch.zeros(self.n, dtype=dt, device=self.dev))
        self._exists.fill_(True)
        self._formation_id.fill_(-1)
        self._owner_ptr.fill_(-1)
        self._combat_state = None
        self.load_formations([])

    exists, ev_self = (_plane_prop(k, False) for k in ("exists", "ev_self"))
    formation_id, formation_slots, owner_ptr, hits_n, ev_n, flags = (_int_prop(k) for k in (
        "formation_id", "formation_slots", "owner_ptr", "hits_n", "ev_n", "flags"))

    def combat_state(self) -> _native.CombatState:
        """include/ebb.h's EbbCombatState over the storage (the formation table's pointers refreshed by
        load_formations)."""
        if self._combat_state is None:
            c = _native.CombatState()
            c.flight = self.state()
            for name, _ in _COMBAT_STORAGE:
                setattr(c, name, getattr(self, "_" + name).data_ptr())
            c.bubble, c.cloaked = self.bubble.data_ptr(), self.cloaked.data_ptr()
            c.tick_ms, c.do_missiles_off, c.master = self.tick_ms, int(self.disable_do_for_missiles), int(self.master)
            self._combat_state = c
        c = self._combat_state
        c.formations, c.formation_len = self.formation_table.data_ptr(), self.formation_lengths.data_ptr()
        c.n_formations, c.max_slots = self.n_formations, self.max_slots
        return c

    # ---- loading ----

    def load(self, rows: list[dict]) -> None:
        """VecModesPark.load, every row: a ball (as the Python AddBall adds it) or, with "exists": False, an empty row
        of its world (moribund, fixed, inert until `add_balls`); then the world index."""
        rows = [dict(r) for r in rows]
        for r in rows:
            if not r.get("exists", True):
                r.update(moribund=True, free=False, massive=False, interactive=False, mode=STOP)
        super().load(rows)
        self._exists.copy_(torch.tensor([bool(r.get("exists", True)) for r in rows], dtype=BOOL))
        self._formation_id.fill_(-1)
        self._formation_slots.zero_()
        self._owner_ptr.fill_(-1)
        for name in ("hits_n", "ev_n", "ev_self", "flags"):
            getattr(self, "_" + name).zero_()
        self._index_worlds()
        self.plan = plan_tiles(self.world, cap=self.block, block=self.block)

    def _index_worlds(self) -> None:
        """rows_of_world [W, N] (-1 padded, each world's rows in row order, worlds in first-appearance order) and each
        row's world index."""
        labels = self.world.cpu().numpy()
        order, index = np.unique(labels, return_index=True)
        order = order[np.argsort(index, kind="stable")]
        self.labels = order.tolist()
        where = {w: k for k, w in enumerate(self.labels)}
        widx = np.array([where[w] for w in labels.tolist()], dtype=np.int64)
        counts = np.bincount(widx, minlength=len(order)) if len(widx) else np.zeros(0, dtype=np.int64)
        width = int(counts.max()) if len(counts) else 0
        table = np.full((len(order), width), -1, dtype=np.int64)
        fill = np.zeros(len(order), dtype=np.int64)
        for r, k in enumerate(widx.tolist()):
            table[k, fill[k]] = r
            fill[k] += 1
        self.rows_of_world = torch.from_numpy(table).to(self.dev)
        self.world_index = torch.from_numpy(widx).to(self.dev)

    def lookup(self, rows: torch.Tensor, ball: torch.Tensor) -> torch.Tensor:
        """For each row, the row of its own world holding the ball whose id is ball[i] (`balls.get`), or -1."""
        cand = self.rows_of_world[self.world_index[rows.to(I64)]]
        safe = cand.clamp(min=0)
        hit = (cand >= 0) & self._exists[safe] & (self._ids[safe] == ball.to(I64)[:, None])
        first = hit.to(I64).argmax(dim=1)
        return torch.where(hit.any(dim=1), cand.gather(1, first[:, None])[:, 0], -1)

    def add_balls(self, mask: torch.Tensor, rows: list) -> None:
        """The Python AddBall of new balls (Thunkers.cpp:150; MOV-711) into the empty rows in `mask` (one dict a
        masked row, in row order, `load`'s keys, the id new in its world): AddBall's clamps and defaults, the decay
        factor, STOP, the rotation snapped; a missile whose owner is the new ball finds it again."""
        m = self._m(mask)
        idx = m.nonzero().flatten()
        if idx.numel() != len(rows):
            raise ValueError(f"{len(rows)} balls for {idx.numel()} rows")
        if not rows:
            return
        ids = torch.tensor([int(r["id"]) for r in rows], dtype=I64, device=self.dev)
        taken = self._exists[idx] | (self.lookup(idx, ids) >= 0)
        if bool(taken.any()):
            self._flags[idx] |= torch.where(taken, FLAG_POOL, 0)
            raise ValueError("add_balls: a row is not empty or the id is already in its world")
        sub = VecModesPark(len(rows), self.friction, self.tick_interval, self.dev, True, self.use_new_orbit, self.block)
        sub.load([{**r, "world": 0, "time": 0} for r in rows])
        for name in _ADD_FIELDS:
            dst, src = getattr(self, "_" + name), getattr(sub, "_" + name)
            if dst.dim() == 2:
                dst[:, idx] = src
            else:
                dst[idx] = src
        self.cloaked[idx] = sub.cloaked
        if all("bubble" in r for r in rows):
            self.bubble[idx] = sub.bubble
        self._exists[idx] = True
        self._formation_id[idx] = -1
        self._formation_slots[idx] = 0
        self._owner_ptr[idx] = -1
        self._refresh_owners()

    def _refresh_owners(self) -> None:
        """Each missile's owner row (`balls.get(ABS(mOwnerId))`, Ballpark.cpp:633), -1 when it is not in the park."""
        rows = torch.arange(self.n, device=self.dev)
        found = self.lookup(rows, self._owner_id.abs())
        self._owner_ptr.copy_(torch.where(self._exists & (self._mode == MISSILE), found, -1))

    # ---- the follower bookkeeping (followModes: FOLLOW, ORBIT, MISSILE, FORMATION) ----

    def _following(self) -> torch.Tensor:
        m = self._mode
        return (((m == FOLLOW) | (m == ORBIT)) | (m == MISSILE)) | (m == FORMATION)

    def _stop_rows(self, mask: torch.Tensor) -> None:
        """Stop(Ball*) (Ballpark.cpp:4578): on the master a FORMATION follower's slot freed in its leader first
        (4629-4633); a follower's follow fields cleared, its owner row with them; then STOP."""
        if self.master:
            self._free_slots(mask & (self._mode == FORMATION) & (self._follow_ptr >= 0))
        self._owner_ptr.masked_fill_(mask & self._following(), -1)
        super()._stop_rows(mask)

    def _free_slots(self, rows: torch.Tensor) -> None:
        """Ball::FreeFormationSlot((size_t) mEffectStamp) (Ball.cpp:2324) in the leader of each row: nothing without a
        loaded formation or for a slot past its end (unsigned comparisons), a negative formation index or a slot of 16
        or more flagged, the bits cleared per leader."""
        lead = self._follow_ptr.to(I64).clamp(min=0)
        fid = self._formation_id[lead]
        ok = rows & (fid != -1) & ~(fid > self.n_formations - 1)
        bad = ok & (fid < 0)
        sign = torch.iinfo(torch.int64).min
        slot = self._effect_stamp
        past = (slot ^ sign) > ((self._formation_len(fid) - 1) ^ sign)
        go = ok & ~bad & ~past
        wide = go & ((slot < 0) | (slot >= FORMATION_MAX_SLOTS))
        self._flags |= torch.where(bad | wide, FLAG_UNDEFINED, 0)
        clear = go & ~wide
        bit = torch.where(clear, torch.ones_like(slot) << slot.clamp(0, FORMATION_MAX_SLOTS - 1), 0)
        bits = torch.zeros(self.n, dtype=I64, device=self.dev)
        for b in range(FORMATION_MAX_SLOTS):                 # OR per leader: one bit plane at a time
            hit = torch.zeros(self.n, dtype=I64, device=self.dev).index_add_(0, lead, (bit == (1 << b)).to(I64))
            bits |= torch.where(hit > 0, 1 << b, 0)
        self._formation_slots &= ~bits

    def followers(self, row: int) -> list:
        sel = (self._follow_ptr == row) & (self._follow_id == self._ids[row]) & self._exists
        return sorted(self._ids[sel].tolist())

    def _release_followers(self, rows: torch.Tensor) -> None:
        """StopAllFollowers (Ballpark.cpp:5416; MOV-730) of the balls in `rows`."""
        self._release_members(self._members(rows) & self._exists)

    def _release_members(self, f: torch.Tensor) -> None:
        """StopAllFollowers on the members in `f`: a missile is made non-massive and, as an interactive orbiter, flies
        on by GotoDirection along its velocity; every other member stops."""
        missile = f & (self._mode == MISSILE)
        flies = missile | (f & self._interactive & (self._mode == ORBIT))
        self._massive.masked_fill_(missile, False)
        self._stop_rows(f & ~flies)
        self.goto_direction(flies, self.vel.clone())

    # ---- missiles (MOV-723 to MOV-725) ----

    def missile_follow(self, mask: torch.Tensor, target: torch.Tensor, owner: torch.Tensor) -> None:
        """PyMissileFollow and MissileFollow (Ballpark.cpp:3798; MOV-724) for the missiles in `mask`: target is each
        row's target's Destiny id, owner the owner's id (negative: a defender)."""
        m = self._m(mask)
        rows = torch.arange(self.n, device=self.dev)
        dst = torch.as_tensor(target).to(device=self.dev, dtype=I64).reshape(self.n)
        own = torch.as_tensor(owner).to(device=self.dev, dtype=I64).reshape(self.n)
        trow = self.lookup(rows, dst)
        tsafe = trow.clamp(min=0)
        src = self._ids
        ok = (m & self._exists & (dst >= 0) & (src != dst) & (src != own) & (dst != own) & (trow >= 0)
              & ~self._moribund[tsafe])
        self._stop_rows(ok)
        ok = ok & (self.bubble == self.bubble[tsafe]) & (self.cloaked[tsafe] == 0)
        radius = self.radius
        self._follow_id.copy_(torch.where(ok, dst, self._follow_id))
        self._follow_ptr.copy_(torch.where(ok, trow.to(I32), self._follow_ptr))
        self._follow_range.copy_(torch.where(ok, -((radius + radius[tsafe]).to(F32)), self._follow_range))
        self._owner_id.copy_(torch.where(ok, own, self._owner_id))
        self._owner_ptr.copy_(torch.where(ok, self.lookup(rows, own.abs()), self._owner_ptr))
        self._effect_stamp.copy_(torch.where(ok, self._clock, self._effect_stamp))
        self._goto.copy_(torch.where(ok[None, :], (_unit(self.vel) * MISSILE_GOTO).t(), self._goto))
        self._speed_fraction.masked_fill_(ok, 1.0)
        self._mode.masked_fill_(ok, MISSILE)
        self._flags |= torch.where(ok & (own < 0), FLAG_DEFENDER, 0)

    def launch_missile(self, mask: torch.Tensor, target: torch.Tensor, owner: torch.Tensor, aimed: torch.Tensor,
                       massive: torch.Tensor) -> None:
        """PyLaunchMissile (Thunkers.cpp:857; MOV-725) for the missile balls in `mask`: at the launcher (found by
        |owner|), aimed (1 m/s toward an uncloaked target) or not (the launcher's velocity plus max(150, its maximum
        speed) along its velocity, or along its rotated (0, 0, -1) at rest), made massive if asked, its velocity set,
        then MissileFollow, or GotoDirection without a target; target and owner Destiny ids, aimed and massive the
        thunk's chars."""
        m = self._m(mask)
        rows = torch.arange(self.n, device=self.dev)
        dst = torch.as_tensor(target).to(device=self.dev, dtype=I64).reshape(self.n)
        own = torch.as_tensor(owner).to(device=self.dev, dtype=I64).reshape(self.n)
        aimed = _char(torch.as_tensor(aimed).to(self.dev).reshape(self.n))
        massive = _char(torch.as_tensor(massive).to(self.dev).reshape(self.n))
        go = m & (dst >= 0)
        lrow = self.lookup(rows, own.abs())
        go = go & (lrow >= 0)
        lsafe = lrow.clamp(min=0)
        trow = torch.where(dst != own, self.lookup(rows, dst), -1)
        has_t = trow >= 0
        tsafe = trow.clamp(min=0)
        pos, vel = self.pos, self.vel
        ps = pos[lsafe]
        aim = has_t & (aimed == 1) & (self.cloaked[tsafe] == 0)
        v_aim = _unit(pos[tsafe] - ps)
        vs = vel[lsafe]
        max_velocity = torch.where(aim, 0.0, self.max_vel[lsafe])
        direction = _unit(vs)
        still = (direction[:, 0] * direction[:, 0] + direction[:, 1] * direction[:, 1]
                 + direction[:, 2] * direction[:, 2]) == 0.0
        if bool((go & ~aim & still).any()):
            back = _rotated_vector(self.rot[lsafe], (0.0, 0.0, -1.0))
            direction = torch.where(still[:, None], back, direction)
        speed = _fmax(torch.full_like(max_velocity, MISSILE_LAUNCH_SPEED), max_velocity)
        v0 = torch.where(aim[:, None], v_aim, vs + direction * speed[:, None])
        here = go & self._exists
        self._massive.masked_fill_(here & (massive != 0), True)
        self._pos.copy_(torch.where(here[None, :], ps.t(), self._pos))          # SetBallPosition (no partition here)
        self._old_pos.copy_(torch.where(here[None, :], ps.t(), self._old_pos))
        self.set_velocity(here, v0)
        cloaked_t = has_t & (self.cloaked[tsafe] != 0)
        self.goto_direction(here & ~has_t & (max_velocity > 0.0), v0)
        self.missile_follow(go & has_t & ~cloaked_t, dst, own)

    # ---- formations (MOV-726) ----

    def load_formations(self, formations: list) -> None:
        """PyLoadFormations and AddFormation: the slot offsets (doubles), one table for the park."""
        f = [[[float(c) for c in v] for v in vectors] for vectors in formations]
        self.formations = f
        self.n_formations = len(f)
        self.max_slots = max([len(v) for v in f] + [1])
        table = np.zeros((max(1, len(f)), self.max_slots, 3), dtype=np.float64)
        for i, vectors in enumerate(f):
            if vectors:
                table[i, :len(vectors)] = vectors
        self.formation_table = torch.from_numpy(table).to(self.dev).contiguous()
        self.formation_lengths = torch.tensor([len(v) for v in f] or [0], dtype=I64, device=self.dev)

    def _formation_len(self, fid: torch.Tensor) -> torch.Tensor:
        return self.formation_lengths[fid.clamp(0, max(0, self.n_formations - 1))]

    def set_ball_formation(self, mask: torch.Tensor, formation: torch.Tensor) -> None:
        """PySetBallFormation and SetBallFormation (Ballpark.cpp:6673): leaving a formation releases the followers
        and frees every slot; a smaller formation stops the FORMATION followers in the slots it lacks."""
        m = self._m(mask)
        fid = _char(torch.as_tensor(formation).to(self.dev).reshape(self.n))
        F = self.n_formations
        ok = m & self._exists & ~(fid > F - 1)
        cur = self._formation_id.clone()
        inside = ok & (cur >= 0)
        leave = inside & (fid == -1)
        self._release_followers(leave)
        self._formation_slots.masked_fill_(leave, 0)
        change = inside & (fid != -1) & (fid != cur)
        bad = change & ((fid < 0) | (cur > F - 1))
        self._flags |= torch.where(bad, FLAG_UNDEFINED, 0)
        change = change & ~bad
        new_len = self._formation_len(fid)
        shrink = change & (self._formation_len(cur) > new_len)
        fp = self._follow_ptr.to(I64)
        safe = torch.where(fp >= 0, fp, 0)
        f = (self._exists & (self._mode == FORMATION) & (fp >= 0) & shrink[safe]
             & (self._effect_stamp > new_len[safe] - 1))
        self._stop_rows(f)
        self._formation_id.copy_(torch.where(ok & ~bad, fid, self._formation_id))

    def formation_follow(self, mask: torch.Tensor, leader: torch.Tensor, slot: torch.Tensor) -> None:
        """PyFormationFollow and FormationFollow (Ballpark.cpp:3947) for the balls in `mask`: leader is each row's
        leader's Destiny id, slot the thunk's char."""
        m = self._m(mask)
        rows = torch.arange(self.n, device=self.dev)
        slot = _char(torch.as_tensor(slot).to(self.dev).reshape(self.n))
        dst = torch.as_tensor(leader).to(device=self.dev, dtype=I64).reshape(self.n)
        lrow = self.lookup(rows, dst)
        lsafe = lrow.clamp(min=0)
        fid = self._formation_id[lsafe]
        ok = (m & self._exists & (self._ids != dst) & (lrow >= 0) & (fid >= 0) & ~(fid > self.n_formations - 1)
              & ~(slot > self._formation_len(fid) - 1))
        self._stop_rows(ok)
        ok = ok & (self.bubble == self.bubble[lsafe]) & (self.cloaked[lsafe] == 0)
        self._follow_id.copy_(torch.where(ok, dst, self._follow_id))
        self._follow_ptr.copy_(torch.where(ok, lrow.to(I32), self._follow_ptr))
        self._effect_stamp.copy_(torch.where(ok, slot, self._effect_stamp))
        self._mode.masked_fill_(ok, FORMATION)
        self._flags |= torch.where(ok & (slot < 0), FLAG_UNDEFINED, 0)     # EvolveFormation reads a negative slot

    def reserve_formation_slot(self, row: int) -> int:
        """Ball::ReserveFormationSlot (Ball.cpp:2275): the first free slot of at most 16, or -1 (one ball, a rare
        call: on the host)."""
        fid = int(self._formation_id[row])
        if fid == -1 or fid > self.n_formations - 1:
            return -1
        if fid < 0:
            self._flags[row] |= FLAG_UNDEFINED
            return -1
        n = len(self.formations[fid])
        if n > FORMATION_MAX_SLOTS:
            return -1
        bits = int(self._formation_slots[row])
        for i in range(n):
            if not bits >> i & 1:
                self._formation_slots[row] = bits | (1 << i)
                return i
        return -1

    def free_formation_slot(self, row: int, slot: int) -> None:
        """Ball::FreeFormationSlot (Ball.cpp:2324) with a size_t slot (one ball, on the host)."""
        fid = int(self._formation_id[row])
        if fid == -1 or fid > self.n_formations - 1:
            return
        if fid < 0:
            self._flags[row] |= FLAG_UNDEFINED
            return
        mask64 = (1 << 64) - 1
        n = len(self.formations[fid])
        slot = int(slot) & mask64
        if slot > ((n - 1) & mask64):
            return
        if slot >= FORMATION_MAX_SLOTS:
            self._flags[row] |= FLAG_UNDEFINED
            return
        self._formation_slots[row] = int(self._formation_slots[row]) & ~(1 << slot)

    # ---- cloaking (SEN-711) and removal ----

    def cloak(self, mask: torch.Tensor, mode: torch.Tensor, range_: torch.Tensor | None = None) -> None:
        """CloakBall (Ballpark.cpp:5223): refused unless the (signed char) mode is positive; on the master a normal
        cloak sets the sensor flag (refused for float(radius) + float(range) < 0); the followers released; cloaked
        with the mode's byte, non-massive."""
        m = self._m(mask)
        mode = _char(torch.as_tensor(mode).to(self.dev).reshape(self.n))
        ok = m & self._exists & (mode > 0)
        if self.master:
            rng = torch.full((self.n,), 2000.0, dtype=F64, device=self.dev) if range_ is None else \
                torch.as_tensor(range_).to(device=self.dev, dtype=F64).reshape(self.n)
            rng = rng.to(F32).to(F64)
            self._sensor |= ok & (mode == DSTNORMALCLOAK) & ~((self.radius + rng).to(F32) < 0.0)
        self._release_followers(ok)
        self.cloaked.copy_(torch.where(ok, mode & 0xFF, self.cloaked))
        self._massive.masked_fill_(ok, False)

    def uncloak(self, mask: torch.Tensor) -> None:
        """UncloakBall (Ballpark.cpp:5257): the normal cloak's sensor flag cleared (master); uncloaked; massive again
        unless in warp proper."""
        ok = self._m(mask) & self._exists
        if self.master:
            self._sensor &= ~(ok & (self.cloaked == DSTNORMALCLOAK))
        self.cloaked.masked_fill_(ok, 0)
        warping = (self._mode == WARP) & (self._effect_stamp >= 0)
        self._massive.masked_fill_(ok & ~warping, True)

    def remove(self, mask: torch.Tensor) -> None:
        """RemoveBall outside Evolve without a delay (Ballpark.cpp:5471; TIME-711): the ball stopped, its followers
        released (a missile flies off), its row emptied (a missile whose owner it was is orphaned)."""
        ok = self._m(mask) & self._exists
        self._stop_rows(ok)
        self._release_followers(ok)
        stale = self._members(ok) & self._exists       # members out of the follow modes: in no follower set again
        self._follow_ptr.masked_fill_(stale | ok, -1)
        self._exists &= ~ok
        self._moribund |= ok
        for t in (self._massive, self._interactive, self._sensor):
            t.masked_fill_(ok, False)
        self._formation_id.masked_fill_(ok, -1)
        self._formation_slots.masked_fill_(ok, 0)
        self._refresh_owners()

    # ---- the tick ----

    def evolve(self, lib=None, active: torch.Tensor | None = None) -> None:
        """One tick of every world in place (ebb_combat_tick: one launch), the domain watched at its start and end;
        no host synchronisation. `active` [n] (OnTick's per-world mask, a world's rows alike): only those worlds
        tick, inside the kernel; every other row keeps every field (the reference's tick-and-put-back, exact since a
        world's tick reads its own rows only), and `events()` then reports the rows that ticked."""
        act = self._world_mask(active)
        self.watch()
        tick(self, act)
        self.watch()
        self._ticked = (self.current_time, act)
        self.current_time += 1

    def _world_mask(self, active) -> torch.Tensor | None:
        """OnTick's mask as bytes on the device, refused unless a world's rows are alike (one host synchronisation)."""
        if active is None:
            return None
        act = torch.as_tensor(active).to(device=self.dev, dtype=BOOL).reshape(self.n)
        rw = self.rows_of_world
        v = act[rw.clamp(min=0)] | (rw < 0)
        w = act[rw.clamp(min=0)] & (rw >= 0)
        if bool((v.all(dim=1) != w.any(dim=1)).any()):
            raise ValueError("OnTick's mask: a world's rows tick together")
        return act.to(torch.uint8).contiguous()

    def _ticked_rows(self, sel: torch.Tensor) -> torch.Tensor:
        """sel, less the rows outside the last tick's mask when that tick was a masked one."""
        last = getattr(self, "_ticked", None)
        if last is not None and last[0] == self.current_time - 1 and last[1] is not None:
            return sel & (last[1] != 0)
        return sel

    def events(self) -> list:
        """The tick's DoCollision events (COL-719) in Destiny's order, from the dispatch's counts: per world (its label,
        in first-appearance order), the missiles by ascending id, each with its target's id ev_n times, then itself on
        the master when orphaned: (world label, time, missile id, collider id). One host synchronisation."""
        sel = self._ticked_rows((self._ev_n > 0) | self._ev_self)
        rows = sel.nonzero().flatten().tolist()
        if not rows:
            return []
        world, ids = self.world.tolist(), self._ids.tolist()
        ev_n, ev_self, clock = self._ev_n.tolist(), self._ev_self.tolist(), self._clock.tolist()
        follow = self._follow_id.tolist()
        order = {w: k for k, w in enumerate(self.labels)}
        out = []
        for r in sorted(rows, key=lambda r: (order[world[r]], ids[r])):
            out.extend((world[r], clock[r] - 1, ids[r], follow[r]) for _ in range(ev_n[r]))
            if ev_self[r]:
                out.append((world[r], clock[r] - 1, ids[r], ids[r]))
        return out

    # ---- the domain ----

    def watch(self) -> None:
        """A world holding two massive balls outside MISSILE mode is flagged on all its rows: this park computes only
        a normal missile's contact with its target (index work on the device)."""
        m = self._exists & ~self._moribund & self._massive & (self._mode != MISSILE)
        rw = self.rows_of_world
        two = (m[rw.clamp(min=0)] & (rw >= 0)).sum(dim=1) > 1
        self._flags |= torch.where(two[self.world_index], FLAG_MASSIVE, 0)

    def world_flags(self) -> list:
        """Each world's flags (the OR of its rows'), in world label order."""
        rw = self.rows_of_world
        f = torch.where(rw >= 0, self._flags[rw.clamp(min=0)], 0)
        out = torch.zeros(f.shape[0], dtype=I64, device=self.dev)
        for k in range(f.shape[1]):
            out |= f[:, k]
        return out.tolist()

    def check(self) -> None:
        """Raise if any world left the domain: the commands' flags, and on the master a world with balls in more than
        one bubble or without an interactive ball; or a follow target outside its world's tile."""
        flags = 0
        for v in self.world_flags():
            flags |= int(v)
        if self.master:
            rw = self.rows_of_world
            safe = rw.clamp(min=0)
            ok = (rw >= 0) & self._exists[safe]
            b = torch.where(ok, self.bubble[safe], torch.iinfo(torch.int64).max)
            first = b.min(dim=1).values
            if bool((ok & (b != first[:, None])).any()):
                flags |= FLAG_BUBBLES
            if bool((ok.any(dim=1) & ~(ok & self._interactive[safe]).any(dim=1)).any()):
                flags |= FLAG_DEAD
        if flags:
            raise RuntimeError("outside the batched domain: " + ", ".join(v for k, v in FLAG_NAMES.items() if flags & k))
        st = int(self._status[0])
        if st:
            raise RuntimeError(f"the combat tick refused a tile (status {st}: a follow target outside its world's "
                               "tile, or a world wider than the block)")

    def row_tensors(self) -> list:
        return super().row_tensors() + ["_" + name for name, _ in _COMBAT_STORAGE]


def tick(park: VecCombatPark, active: torch.Tensor | None = None) -> None:
    """One tick of a VecCombatPark in place on torch's current stream (the drop-in for
    exact_ballpark.vec_combat_cuda.tick): one launch, tiles of whole worlds; no allocation, no host synchronisation."""
    plan = park.plan
    if plan is None:
        raise ValueError("the combat park's worlds are not contiguous rows: no tile plan")
    if not park.n:
        return
    if plan.cap > plan.block:
        raise ValueError(f"a world of {plan.max_world} rows is wider than the block ({plan.block} threads)")
    tr = plan.tile_rows_on(park.dev)
    c = park.combat_state()
    c.active = None if active is None else active.data_ptr()
    with torch.cuda.device(park.dev):
        rc = _native.lib().ebb_combat_tick(ctypes.byref(c), tr.data_ptr(), plan.tiles, park._status.data_ptr(),
                                           park._stream(), plan.block)
    _native.check(rc, "ebb_combat_tick")


class CombatGraph:
    """The combat park's tick (`evolve`: the domain watch and the one-launch tick) captured as a CUDA graph on the
    park's own buffers (the drop-in for exact_ballpark.vec_combat_cuda.CombatGraph): each `tick()` is one replay; a
    LoadFormations since the capture (a new table) is captured anew first."""

    def __init__(self, park: VecCombatPark):
        self.park = park
        self._capture()

    def _capture(self) -> None:
        park = self.park
        names = [n for n in vars(park) if isinstance(getattr(park, n), torch.Tensor)]
        keep = {n: getattr(park, n).clone() for n in names}
        side = torch.cuda.Stream(device=park.dev)
        side.wait_stream(torch.cuda.current_stream(park.dev))
        with torch.cuda.stream(side):                             # a warm-up tick, undone
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
        self._tables = (park.formation_table, park.formation_lengths)

    def tick(self) -> None:
        park = self.park
        if park.formation_table is not self._tables[0] or park.formation_lengths is not self._tables[1]:
            self._capture()
        self.graph.replay()
        park.current_time += 1
