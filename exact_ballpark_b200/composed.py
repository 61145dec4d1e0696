"""The composed park on a B200: a drop-in for exact_ballpark.vec_composed.VecComposedPark (flight modes, missiles,
formations and ship-to-ship collisions by the gradient method in one park) and its CUDA tick
(exact_ballpark.vec_composed_cuda).

The public API is the reference park's (exact_ballpark/vec_composed.py:189-604): VecCombatPark's (this package's
exact_ballpark_b200.combat) with `collisions`, the per-row collision acceleration `last_c`, the partition's filing
(`level`, `key`, `mod`), the collision lists (`hits`, `hits_n`, `collision_lists()`), the re-filing commands
(AddBall, SetBallRadius, SetMaxSpeed, LaunchMissile at its launcher, SetBallFree(false)) and `events()` from the
missiles' collision lists.

The tick is one launch of the native library (ebb_composed_tick: tiles of whole worlds, one thread block a tile;
phase 1, the warp paths and drop-outs, every live massive ball's Gradient over its world from a view staged in shared
memory, the commit with the re-filings), where the reference takes thirteen. The filings of the commands run in the
native library too (ebb_composed_file). With `collisions=False` the tick is the combat park's, the collision lists
made from its counts as the reference's tick on tensors makes them.

Domain (flags on the rows, raised by `check()`): the combat park's, less its two-massive-balls refusal and, with
collisions, its refusal of defender missiles; no massive ball in warp proper (FLAG_WARP_MASSIVE), no ball at the
partition's edge or wider than a top box (FLAG_PARTITION), on the master no normal cloak (FLAG_SENSOR: its proximity
sensor re-files its ball, which this park does not model). A world holds at most 64 rows.
"""

from __future__ import annotations

import ctypes

import torch

from . import _native
from .combat import FLAG_DEFENDER, FLAG_NAMES, VecCombatPark
from .modes import _int_prop, _plane_prop

F64, F32, I64, BOOL = torch.float64, torch.float32, torch.int64, torch.bool

FLAG_WARP_MASSIVE = 64          # a massive ball in warp proper beside collisions (its state changes mid-tick)
FLAG_PARTITION = 128            # a ball at the partition's edge or wider than a top box
FLAG_SENSOR = 256               # a proximity sensor on the master (a normal cloak's): its re-filing is not modelled
COMPOSED_FLAG_NAMES = {**FLAG_NAMES,
                       FLAG_WARP_MASSIVE: "a massive ball in warp proper beside collisions",
                       FLAG_PARTITION: "a ball at the partition's edge or wider than a top box",
                       FLAG_SENSOR: "a proximity sensor on the master (its re-filing is not modelled)"}
MAX_WORLD_ROWS = 64             # the tick's candidate list: a world's rows at most


class VecComposedPark(VecCombatPark):
    """VecCombatPark with the gradient method's collisions between every massive ball (the module's docstring)."""

    def __init__(self, n: int, friction: float = 1.0e6, tick_interval_ms: int = 1000, device="cuda",
                 dynamical_orientation: bool = True, use_new_orbit: bool = False, block: int = 256,
                 master: bool = False, disable_do_for_missiles: bool = False, collisions: bool = True):
        super().__init__(n, friction, tick_interval_ms, device, dynamical_orientation, use_new_orbit, block, master,
                         disable_do_for_missiles)
        self.collisions = bool(collisions)
        d = self.dev
        self._last_c = torch.zeros(3, self.n, dtype=F64, device=d)
        self._level = torch.zeros(self.n, dtype=I64, device=d)
        self._key = torch.zeros(3, self.n, dtype=I64, device=d)
        self._mod = torch.zeros(3, self.n, dtype=I64, device=d)
        self._hits = torch.full((self.n, 1), -1, dtype=I64, device=d)
        self._composed_state = None

    last_c = _plane_prop("last_c", True)
    key, mod = (_plane_prop(k, False) for k in ("key", "mod"))
    level = _int_prop("level")

    @property
    def hits(self) -> torch.Tensor:
        return self._hits

    @hits.setter
    def hits(self, value) -> None:
        self._hits.copy_(torch.as_tensor(value, device=self.dev))

    def composed_state(self) -> _native.ComposedState:
        """include/ebb.h's EbbComposedState over the storage."""
        if self._composed_state is None:
            x = _native.ComposedState()
            x.world, x.last_c, x.level = self.world.data_ptr(), self._last_c.data_ptr(), self._level.data_ptr()
            x.key, x.mod, x.hits, x.hit_cap = (self._key.data_ptr(), self._mod.data_ptr(), self._hits.data_ptr(),
                                               self._hits.shape[1])
            self._composed_state = x
        x = self._composed_state
        x.combat = self.combat_state()
        return x

    # ---- loading, adding, the setters that re-file ----

    def load(self, rows: list[dict]) -> None:
        """VecCombatPark.load, the collision lists sized for the largest world (three appends a candidate and the
        master's self-collision), then every ball's first filing (AddBall files it)."""
        super().load(rows)
        S = int(self.rows_of_world.shape[1]) if self.rows_of_world.numel() else 1
        if S > MAX_WORLD_ROWS:
            raise ValueError(f"a world of {S} rows: the composed tick takes at most {MAX_WORLD_ROWS}")
        self._hits = torch.full((self.n, max(1, 3 * (S - 1)) + 1), -1, dtype=I64, device=self.dev)
        self._last_c.zero_()
        self._level.zero_()
        self._key.zero_()
        self._mod.zero_()
        self._composed_state = None
        self._file(self._exists & ~self._moribund)

    def add_balls(self, mask: torch.Tensor, rows: list) -> None:
        """VecCombatPark.add_balls, then each new ball's collision state cleared and the ball filed."""
        m = self._m(mask)
        super().add_balls(m, rows)
        new = m & self._exists
        self._last_c.masked_fill_(new[None, :], 0.0)
        self._hits.masked_fill_(new[:, None], -1)
        self._hits_n.masked_fill_(new, 0)
        self._file(new)

    def set_radius(self, mask, r) -> None:
        """SetBallRadius, then the ball re-filed."""
        m, v = self._m(mask), self._vals(r)
        ok = m & ~(v.to(F32) < 0.0) & self._exists
        super().set_radius(m, v)
        self._file(ok)

    def set_max_velocity(self, mask, v) -> None:
        """SetMaxSpeed, then the ball re-filed."""
        m, val = self._m(mask), self._vals(v)
        ok = m & ~(val.to(F32) < 0.0) & self._exists
        super().set_max_velocity(m, val)
        self._file(ok)

    def launch_missile(self, mask, target, owner, aimed, massive) -> None:
        """PyLaunchMissile with SetBallPosition's re-filing at the launcher, from the velocity and speed fraction
        before SetBallVelocity and MissileFollow change them."""
        m = self._m(mask)
        rows = torch.arange(self.n, device=self.dev)
        dst = torch.as_tensor(target).to(device=self.dev, dtype=I64).reshape(self.n)
        own = torch.as_tensor(owner).to(device=self.dev, dtype=I64).reshape(self.n)
        go = m & (dst >= 0) & (self.lookup(rows, own.abs()) >= 0) & self._exists
        vel0, sf0 = self.vel.clone(), self._speed_fraction.clone()
        super().launch_missile(m, dst, own, aimed, massive)
        self._file(go, vel=vel0, sf=sf0)

    def missile_follow(self, mask, target, owner) -> None:
        """MissileFollow; with collisions a defender missile is held (its candidates the gradient's), so the combat
        park's refusal of it is lifted."""
        before = self._flags.clone()
        super().missile_follow(mask, target, owner)
        if self.collisions:
            self._flags.copy_((self._flags & ~FLAG_DEFENDER) | (before & FLAG_DEFENDER))

    def set_free(self, mask, flag) -> None:
        """SetBallFree, then a ball fixed re-filed from its state then."""
        m = self._m(mask)
        f = torch.as_tensor(flag).to(self.dev).reshape(self.n) != 0
        fix = m & (f != self._free) & ~f
        super().set_free(m, f)
        self._file(fix & self._exists)

    def cloak(self, mask, mode, range_=None) -> None:
        """CloakBall; on the master a normal cloak's proximity sensor (not modelled here) flags its world."""
        before = self._sensor.clone()
        super().cloak(mask, mode, range_)
        if self.master and self.collisions:
            self._flags |= torch.where(self._sensor & ~before, FLAG_SENSOR, 0)

    def _file(self, which: torch.Tensor, pos=None, vel=None, sf=None) -> None:
        """Ball::InsertInBoxes for the rows in `which` from each row's state (or the given [n, 3] position, velocity
        and [n] speed fraction), in the native library; a filing the reference refuses raises FLAG_PARTITION."""
        if not self.collisions or not bool(which.any()):
            return
        m = self._mask_bytes(which)
        keep = []

        def planes(t):
            if t is None:
                return None
            a = torch.as_tensor(t).to(device=self.dev, dtype=F64).reshape(self.n, 3).t().contiguous()
            keep.append(a)
            return a.data_ptr()

        def floats(t):
            if t is None:
                return None
            a = torch.as_tensor(t).to(device=self.dev).reshape(self.n).to(F32).contiguous()
            keep.append(a)
            return a.data_ptr()
        with torch.cuda.device(self.dev):
            rc = _native.lib().ebb_composed_file(ctypes.byref(self.composed_state()), m.data_ptr(), planes(pos),
                                                 planes(vel), floats(sf), self._stream())
        _native.check(rc, "ebb_composed_file")

    # ---- the tick ----

    def watch(self) -> None:
        """The combat park's two-massive-balls refusal only with collisions off (with them, they collide here)."""
        if not self.collisions:
            super().watch()

    def evolve(self, lib=None, active: torch.Tensor | None = None) -> None:
        """One tick in place, no host synchronisation: with collisions the composed tick (one launch); without them
        the combat park's tick and the collision lists made from its counts. `active`: OnTick's per-world mask, inside
        the kernel (the combat park's `evolve`)."""
        if not self.collisions:
            follow = self._follow_id.clone()
            hits, hits_n = self._hits.clone(), self._hits_n.clone()
            super().evolve(active=active)
            self._lists_from_counts(follow)
            if active is not None:                                    # the lists of the worlds that did not tick
                act = torch.as_tensor(active).to(device=self.dev, dtype=BOOL).reshape(self.n)
                self._hits.copy_(torch.where(act[:, None], self._hits, hits))
                self._hits_n.copy_(torch.where(act, self._hits_n, hits_n))
            return
        act = self._world_mask(active)
        tick(self, act)
        self._ticked = (self.current_time, act)
        self.current_time += 1

    def _lists_from_counts(self, follow: torch.Tensor) -> None:
        """With collisions off: each row's list its target's id once a contact, then its own id on the master's
        self-collision (vec_composed.py:_lists_from_counts, _list_self_collisions)."""
        width = self._hits.shape[1]
        ar = torch.arange(width, device=self.dev)
        self._hits.copy_(torch.where(ar[None, :] < self._hits_n[:, None], follow[:, None], -1))
        put = (ar[None, :] == self._hits_n.clamp(max=width - 1)[:, None]) & self._ev_self[:, None]
        self._hits.copy_(torch.where(put, self._ids[:, None], self._hits))
        self._hits_n += self._ev_self.to(I64)

    # ---- reading ----

    def collision_lists(self) -> list:
        """Each row's collision list (Ball::mCollisions: the ids Potential appended, in order)."""
        hits, n = self._hits.tolist(), self._hits_n.tolist()
        return [tuple(h[:k]) for h, k in zip(hits, n)]

    def events(self) -> list:
        """The tick's DoCollision events in Destiny's order: per world (label order) the missiles that dispatched by
        ascending id, each with its collision list in order, then itself on the master when orphaned: (world label,
        time, missile id, collider id). One host synchronisation."""
        sel = self._ticked_rows((self._ev_n > 0) | self._ev_self)
        rows = sel.nonzero().flatten().tolist()
        if not rows:
            return []
        world, ids = self.world.tolist(), self._ids.tolist()
        ev_n, ev_self, clock = self._ev_n.tolist(), self._ev_self.tolist(), self._clock.tolist()
        lists = dict(zip(rows, self._hits[sel].tolist()))
        order = {w: k for k, w in enumerate(self.labels)}
        out = []
        for r in sorted(rows, key=lambda r: (order[world[r]], ids[r])):
            out.extend((world[r], clock[r] - 1, ids[r], lists[r][k]) for k in range(ev_n[r]))
            if ev_self[r]:
                out.append((world[r], clock[r] - 1, ids[r], ids[r]))
        return out

    def check(self) -> None:
        """Raise if any world left the domain: this park's flags, then the combat park's."""
        flags = 0
        for v in self.world_flags():
            flags |= int(v)
        extra = flags & (FLAG_WARP_MASSIVE | FLAG_PARTITION | FLAG_SENSOR)
        if extra:
            names = [v for k, v in COMPOSED_FLAG_NAMES.items() if extra & k]
            raise RuntimeError(f"outside the batched domain: {', '.join(names)}")
        if int(self._status[0]) & 4:
            raise RuntimeError(f"a world wider than {MAX_WORLD_ROWS} rows reached the composed tick")
        super().check()

    ROW_MAJOR = ("_hits",)                  # per-row tensors laid out [n, ...] (the others are [k, n] planes)

    def row_tensors(self) -> list:
        return super().row_tensors() + ["_last_c", "_level", "_key", "_mod", "_hits"]


def tick(park: VecComposedPark, active: torch.Tensor | None = None) -> None:
    """One tick of a VecComposedPark with collisions in place on torch's current stream (the drop-in for
    exact_ballpark.vec_composed_cuda.tick): one launch; no allocation, no host synchronisation."""
    plan = park.plan
    if plan is None:
        raise ValueError("the composed park's worlds are not contiguous rows: no tile plan")
    if not park.n:
        return
    if plan.cap > plan.block:
        raise ValueError(f"a world of {plan.max_world} rows is wider than the block ({plan.block} threads)")
    tr = plan.tile_rows_on(park.dev)
    x = park.composed_state()
    x.combat.active = None if active is None else active.data_ptr()
    with torch.cuda.device(park.dev):
        rc = _native.lib().ebb_composed_tick(ctypes.byref(x), tr.data_ptr(), plan.tiles, park._status.data_ptr(),
                                             park._stream(), plan.block)
    _native.check(rc, "ebb_composed_tick")
