"""The flight-mode park on a B200: a drop-in for exact_ballpark.vec_modes.VecModesPark and its CUDA tick
(exact_ballpark.vec_modes_cuda: `tick`, `ModesGraph`, `kernel_info`).

The public API is the reference park's (exact_ballpark/vec_modes.py:193-483, vec_orient.py:296-478): the constructor,
`load(rows)`, the masked commands (stop, goto_point, goto_direction, follow, orbit, warp_to, entity_warp_in,
set_free, set_ball_rigid, set_boid, set_interactive, set_ball_troll) and setters (set_mass, set_agility,
set_max_velocity, set_speed_fraction, set_radius, set_max_angular_speed, set_rot_agility, set_angular_velocity,
set_rotation, set_velocity), `evolve(lib=None, active=None)`, `followers(row)`, and the per-row attributes in the
reference's layout (`pos` [n, 3] float64, `radius` [n] float64, `mode` [n] int64, ...).

The storage is this package's own: structure-of-arrays on the device (a vector field is [3, n] or [4, n] planes),
Destiny's float members stored as float32 and its doubles as float64, modes and follow pointers as int32 (include/ebb.h,
EbbFlightState). The reference-layout attributes are views of the planes (pos, vel, goto, ...: writable views) or
converted copies (the float and int32 fields). Every command writes the storage in place, so a captured CUDA graph's
buffers stay the park's.

The tick is the native library's (libebb.so): with the rows grouped by world (each world's rows contiguous) the tiled
schedule, one thread block a tile of whole worlds with the records in shared memory, otherwise the plain two-launch
schedule with the records in a scratch buffer. There is no CPU tick: a park on another device is refused.

The commands are the reference's own tensor operations in its order (only correctly rounded +, -, *, /, sqrt,
comparisons and selections, which torch's CUDA kernels compute exactly, one operation a kernel); the glibc functions
they need (exp for the decay factor; acosf, atan2f, sinf, cosf for SnapOrientation) run in the native library.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _native
from .tiles import TilePlan, plan_tiles

F64, F32, I64, I32, BOOL = torch.float64, torch.float32, torch.int64, torch.int32, torch.bool

GOTO, FOLLOW, STOP, WARP, ORBIT, MISSILE = 0, 1, 2, 3, 4, 5
MUSHROOM, BOID, TROLL, MINIBALL, FIELD, RIGID, FORMATION = 6, 7, 8, 9, 10, 11, 12
INERT_MODES = (BOID, MINIBALL, FIELD, RIGID)
LOADABLE = (STOP,) + INERT_MODES
AU = .1495978707e12
MIN_WARP_DISTANCE_SQ = 10000000000.0
DIR_DIST = 1.0e17
TROLL_MIN_DELAY = 1

# storage: (name, dtype, planes; 0 for one value a row)
_STORAGE = (
    ("pos", F64, 3), ("vel", F64, 3), ("old_pos", F64, 3), ("old_vel", F64, 3), ("goto", F64, 3),
    ("last_g", F64, 3), ("mass", F64, 0), ("time_factor", F64, 0), ("last_collision", F64, 0),
    ("radius", F32, 0), ("max_vel", F32, 0), ("agility", F32, 0), ("speed_fraction", F32, 0),
    ("follow_range", F32, 0), ("max_ang_vel", F32, 0), ("rot_agility", F32, 0), ("rot_roll", F32, 0),
    ("rot", F32, 4), ("old_rot", F32, 4), ("ang_vel", F32, 3), ("old_ang_vel", F32, 3), ("torque", F32, 3),
    ("ids", I64, 0), ("effect_stamp", I64, 0), ("follow_id", I64, 0), ("owner_id", I64, 0), ("clock", I64, 0),
    ("mode", I32, 0), ("follow_ptr", I32, 0), ("free", BOOL, 0), ("moribund", BOOL, 0), ("massive", BOOL, 0),
    ("interactive", BOOL, 0), ("sensor", BOOL, 0))
_HOST_ONLY = (("world", I64), ("cloaked", I64), ("bubble", I64), ("refiled", I64))
_STATE_FIELD = {"goto": "goto_pt", "free": "free_"}


# load()'s row keys: (key, numpy dtype, default (None: required)); pos and vel are 3-vectors
ROW_COLUMNS = (("id", np.int64, None), ("world", np.int64, 0), ("time", np.int64, 0), ("mass", np.float64, None),
               ("radius", np.float64, None), ("max_vel", np.float64, None), ("agility", np.float64, None),
               ("speed_fraction", np.float64, None), ("free", np.bool_, True), ("massive", np.bool_, False),
               ("interactive", np.bool_, False), ("moribund", np.bool_, False), ("cloaked", np.int64, 0),
               ("bubble", np.int64, -1), ("mode", np.int64, STOP), ("max_ang_vel", np.float64, 1.0),
               ("rot_agility", np.float64, 0.9))


def rows_to_columns(rows: list) -> dict:
    """load()'s rows as columns (numpy arrays), the reference's defaults filled in: what load_columns takes."""
    conv = {np.int64: int, np.float64: float, np.bool_: bool}
    cols = {}
    for key, dt, default in ROW_COLUMNS:
        c = conv[dt]
        if default is None:
            cols[key] = np.array([c(r[key]) for r in rows], dtype=dt)
        else:
            cols[key] = np.array([c(r.get(key, default)) for r in rows], dtype=dt)
    for key in ("pos", "vel"):
        cols[key] = np.array([[float(v) for v in r[key]] for r in rows], dtype=np.float64).reshape(len(rows), 3)
    return cols


def f32(x: torch.Tensor) -> torch.Tensor:
    """A double rounded to the nearest float and held as float64 (a C++ float)."""
    return x.to(F32).to(F64)


def _unit(d: torch.Tensor) -> torch.Tensor:
    """ref.py's _normalized on [n, 3] rows: times the reciprocal of the length; a zero vector as it is."""
    norm = torch.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
    inv = torch.ones_like(norm) / torch.where(norm == 0.0, 1.0, norm)
    return torch.where((norm == 0.0)[:, None], d, d * inv[:, None])


def _plane_prop(name: str, f64: bool):
    """A reference-layout attribute over a storage tensor: [n, k] rows of [k, n] planes, float64."""
    key = "_" + name

    def get(self):
        t = getattr(self, key)
        t = t.t() if t.dim() == 2 else t
        return t if (not f64 or t.dtype == F64) else t.to(F64)

    def set_(self, value):
        t = getattr(self, key)
        v = torch.as_tensor(value, device=self.dev)
        t.copy_((v.t() if t.dim() == 2 else v).to(t.dtype))
    return property(get, set_)


def _int_prop(name: str):
    key = "_" + name

    def get(self):
        t = getattr(self, key)
        return t if t.dtype == I64 else t.to(I64)

    def set_(self, value):
        t = getattr(self, key)
        t.copy_(torch.as_tensor(value, device=self.dev).to(t.dtype))
    return property(get, set_)


class VecModesPark:
    """B balls, one a row, in independent worlds, with Destiny's flight modes and (optionally) dynamical orientation;
    the drop-in for exact_ballpark.vec_modes.VecModesPark (module docstring)."""

    def __init__(self, n: int, friction: float = 1.0e6, tick_interval_ms: int = 1000, device="cuda",
                 dynamical_orientation: bool = False, use_new_orbit: bool = False, block: int = 128,
                 ypr: str = "host"):
        dev = torch.device(device)
        if dev.type != "cuda":
            raise ValueError("the B200 park ticks on a CUDA device only (there is no CPU tick)")
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.n, self.dev = int(n), dev
        self.friction = float(friction)
        self.tick_interval = int(tick_interval_ms)
        self.dt = tick_interval_ms * 0.001
        self.fdt = float(torch.tensor(self.dt, dtype=F64).to(F32).item())
        self.ffriction = float(torch.tensor(self.friction, dtype=F64).to(F32).item())
        self.dynamical_orientation = bool(dynamical_orientation)
        self.use_new_orbit = bool(use_new_orbit)
        self.block = int(block)
        self.ypr = ypr
        self.current_time = 0
        n = self.n
        for name, dt, planes in _STORAGE:
            setattr(self, "_" + name, torch.zeros((planes, n) if planes else (n,), dtype=dt, device=dev))
        for name, dt in _HOST_ONLY:
            setattr(self, name, torch.zeros(n, dtype=dt, device=dev))
        self._rot[3].fill_(1.0)
        self._old_rot[3].fill_(1.0)
        self._last_collision.fill_(-1.0)
        self._follow_range.fill_(10.0)
        self._ids.copy_(torch.arange(1, n + 1, dtype=I64, device=dev))
        self._follow_ptr.fill_(-1)
        self._mode.fill_(STOP)
        self.bubble.fill_(-1)
        self._scratch = None
        self.plan: TilePlan | None = None
        self._status = torch.zeros(1, dtype=I32, device=dev)
        self._state = None

    # ---- the reference layout ----
    pos, vel, old_pos, old_vel, goto, last_g = (_plane_prop(k, True) for k in
                                                ("pos", "vel", "old_pos", "old_vel", "goto", "last_g"))
    mass, time_factor, last_collision = (_plane_prop(k, True) for k in ("mass", "time_factor", "last_collision"))
    radius, max_vel, agility, speed_fraction, follow_range = (_plane_prop(k, True) for k in (
        "radius", "max_vel", "agility", "speed_fraction", "follow_range"))
    max_ang_vel, rot_agility, rot_roll = (_plane_prop(k, True) for k in ("max_ang_vel", "rot_agility", "rot_roll"))
    rot, old_rot, ang_vel, old_ang_vel, torque = (_plane_prop(k, True) for k in (
        "rot", "old_rot", "ang_vel", "old_ang_vel", "torque"))
    ids, effect_stamp, follow_id, owner_id, clock, mode, follow_ptr = (_int_prop(k) for k in (
        "ids", "effect_stamp", "follow_id", "owner_id", "clock", "mode", "follow_ptr"))
    free, moribund, massive, interactive, sensor = (_plane_prop(k, False) for k in (
        "free", "moribund", "massive", "interactive", "sensor"))

    def state(self) -> _native.FlightState:
        """include/ebb.h's EbbFlightState over the storage (the same buffers every tick)."""
        if self._state is None:
            s = _native.FlightState()
            s.n, s.friction, s.dt, s.ffriction, s.fdt = self.n, self.friction, self.dt, self.ffriction, self.fdt
            s.new_orbit, s.dynamical = int(self.use_new_orbit), int(self.dynamical_orientation)
            for name, _, _ in _STORAGE:
                setattr(s, _STATE_FIELD.get(name, name), getattr(self, "_" + name).data_ptr())
            self._state = s
        return self._state

    def _stream(self) -> int:
        return torch.cuda.current_stream(self.dev).cuda_stream

    def _mask_bytes(self, mask: torch.Tensor) -> torch.Tensor:
        return mask.to(device=self.dev, dtype=torch.uint8).contiguous()

    def _decay_rows(self, mask: torch.Tensor) -> None:
        """SetBallTimeFactor for the rows in mask (glibc's exp, in the native library)."""
        m = self._mask_bytes(mask)
        with torch.cuda.device(self.dev):
            rc = _native.lib().ebb_flight_decay(ctypes.byref(self.state()), m.data_ptr(),
                                                -self.friction * self.dt, self._stream(), 256)
        _native.check(rc, "ebb_flight_decay")

    def _snap(self, mask: torch.Tensor, fresh: bool = False) -> None:
        """SnapOrientation of the rows in mask (vec_orient.py:556) in the native library."""
        m = self._mask_bytes(mask)
        with torch.cuda.device(self.dev):
            rc = _native.lib().ebb_flight_snap(ctypes.byref(self.state()), m.data_ptr(), int(fresh),
                                               self._stream(), 128)
        _native.check(rc, "ebb_flight_snap")

    # ---- loading: the Python AddBall (vec_modes.py:221) ----
    def load(self, rows: list[dict]) -> None:
        """Every ball as the Python AddBall adds a new one: AddBall's clamps, the decay factor, STOP or an inert mode,
        Ball::Ball's defaults; with dynamical orientation the turning values and the rotation snapped to the
        velocity. Keys as the reference's: id, world, time, mass, radius, max_vel, pos, vel, agility,
        speed_fraction, free, massive, interactive, cloaked, bubble, moribund, mode, max_ang_vel, rot_agility."""
        if len(rows) != self.n:
            raise ValueError(f"{len(rows)} rows for a park of {self.n}")
        self.load_columns(rows_to_columns(rows))

    def load_columns(self, cols: dict) -> None:
        """`load` with the rows given as columns (numpy arrays, rows_to_columns' keys and dtypes): the same balls."""
        n = len(cols["id"])
        if n != self.n:
            raise ValueError(f"{n} rows for a park of {self.n}")
        mode = np.asarray(cols["mode"])
        if not np.isin(mode, LOADABLE).all():
            raise ValueError(f"a ball starts in STOP or an inert mode, not {int(mode[~np.isin(mode, LOADABLE)][0])}")
        dev = self.dev
        cpu = lambda key, dt=F64: torch.from_numpy(np.ascontiguousarray(cols[key])).to(dt)
        mass = cpu("mass")
        mass = torch.where(mass < 0.0, 0.0, mass)
        radius = f32(cpu("radius"))
        radius = torch.where(radius < 0.0, 0.0, radius)
        max_vel = f32(cpu("max_vel"))
        max_vel = torch.where(max_vel < 0.0, 0.0, max_vel)
        agility = f32(cpu("agility"))
        agility = torch.where(agility <= 0.0, 1.0, agility)
        sf = f32(cpu("speed_fraction"))
        sf = torch.where(sf < 0.0, 0.0, sf)
        pos = cpu("pos").reshape(n, 3)
        vel = cpu("vel").reshape(n, 3)
        self._mass.copy_(mass)
        self._radius.copy_(radius)
        self._max_vel.copy_(max_vel)
        self._agility.copy_(agility)
        self._speed_fraction.copy_(sf)
        self._pos.copy_(pos.t())
        self._vel.copy_(vel.t())
        self._old_pos.copy_((pos.to(dev) - vel.to(dev) * self.dt).t())
        self._old_vel.copy_(vel.t())
        self._goto.zero_()
        self._last_g.zero_()
        for t in (self._rot, self._old_rot):
            t.zero_()
            t[3].fill_(1.0)
        for t in (self._ang_vel, self._old_ang_vel, self._torque, self._rot_roll):
            t.zero_()
        if self.dynamical_orientation:
            mav = f32(cpu("max_ang_vel"))
            rag = f32(cpu("rot_agility"))
            self._max_ang_vel.copy_(torch.where(mav < 0.0, 0.0, mav))
            self._rot_agility.copy_(torch.where(rag <= 0.0, 1.0, rag))
        else:
            self._max_ang_vel.fill_(1.0)
            self._rot_agility.fill_(0.9)
        self._ids.copy_(cpu("id", I64))
        self.world.copy_(cpu("world", I64))
        self._clock.copy_(cpu("time", I64))
        self._mode.copy_(cpu("mode", I32))
        self._free.copy_(cpu("free", BOOL))
        self._massive.copy_(cpu("massive", BOOL))
        self._interactive.copy_(cpu("interactive", BOOL))
        self._moribund.copy_(cpu("moribund", BOOL))
        self.cloaked.copy_(cpu("cloaked", I64))
        self.bubble.copy_(cpu("bubble", I64))
        self._sensor.zero_()
        self._effect_stamp.zero_()
        self._follow_id.zero_()
        self._owner_id.zero_()
        self._follow_ptr.fill_(-1)
        self._follow_range.fill_(10.0)
        self._last_collision.fill_(-1.0)
        self.refiled.zero_()
        every = torch.ones(n, dtype=BOOL, device=dev)
        self._decay_rows(every)
        if self.dynamical_orientation:
            self._snap(every, fresh=True)
        self.plan = plan_tiles(self.world)

    # ---- the follower bookkeeping: Stop(Ball*) (vec_modes.py:289) ----
    def _following(self) -> torch.Tensor:
        """The rows in a follow mode whose Stop clears the follow fields (FOLLOW, ORBIT here)."""
        return (self._mode == FOLLOW) | (self._mode == ORBIT)

    def _stop_rows(self, mask: torch.Tensor) -> None:
        follower = mask & self._following()
        self._effect_stamp.masked_fill_(follower, 0)
        self._follow_ptr.masked_fill_(follower, -1)
        self._follow_id.masked_fill_(follower, 0)
        self._owner_id.masked_fill_(follower, 0)
        self._follow_range.masked_fill_(follower, 0.0)
        self._mode.masked_fill_(mask, STOP)

    def _members(self, rows: torch.Tensor) -> torch.Tensor:
        """The balls in the follower set of a row in `rows` as StopAllFollowers acts on it (vec_modes.py:300)."""
        fp = self._follow_ptr.to(I64)
        safe = torch.where(fp >= 0, fp, 0)
        return (fp >= 0) & (self._follow_id == self._ids[safe]) & rows[safe]

    def followers(self, row: int) -> list:
        sel = (self._follow_ptr == row) & (self._follow_id == self._ids[row])
        return sorted(self._ids[sel].tolist())

    def _m(self, mask) -> torch.Tensor:
        return torch.as_tensor(mask).to(device=self.dev, dtype=BOOL).reshape(self.n)

    # ---- commands (vec_modes.py:315-483) ----
    def stop(self, mask: torch.Tensor) -> None:
        """Stop(const ID&): nothing for a ball already in STOP."""
        m = self._m(mask)
        self._stop_rows(m & (self._mode != STOP))

    def goto_point(self, mask: torch.Tensor, point: torch.Tensor) -> None:
        """GotoPoint: refused for a non-finite point; Stop, the point, a zero speed fraction made 1, GOTO."""
        m = self._m(mask)
        point = torch.as_tensor(point).to(device=self.dev, dtype=F64).reshape(self.n, 3)
        ok = m & torch.isfinite(point).all(dim=1)
        self._stop_rows(ok)
        self._goto.copy_(torch.where(ok[None, :], point.t(), self._goto))
        self._speed_fraction.masked_fill_(ok & (self._speed_fraction == 0.0), 1.0)
        self._mode.masked_fill_(ok, GOTO)

    def goto_direction(self, mask: torch.Tensor, direction: torch.Tensor) -> None:
        """GotoDirection: refused when not finite; a point 1e17 m along the unit direction."""
        m = self._m(mask)
        d = torch.as_tensor(direction).to(device=self.dev, dtype=F64).reshape(self.n, 3)
        ok = m & torch.isfinite(d).all(dim=1)
        self.goto_point(ok, self.pos + _unit(d) * DIR_DIST)

    def _follow(self, mask, target, range_, mode: int) -> None:
        """FollowBall and Orbit (vec_modes.py:341): the guards, then Stop, the follow fields, the mode."""
        m = self._m(mask)
        rng = torch.as_tensor(range_).to(device=self.dev, dtype=F64).reshape(self.n).to(F32)
        target = torch.as_tensor(target).to(device=self.dev, dtype=I64).reshape(self.n)
        inr = (target >= 0) & (target < self.n)
        safe = torch.where(inr, target, 0)
        rows = torch.arange(self.n, device=self.dev)
        ok = (m & torch.isfinite(rng) & inr & (safe != rows) & (self.world[safe] == self.world)
              & ~self._moribund[safe] & (self.bubble[safe] == self.bubble) & (self.cloaked[safe] == 0))
        self._stop_rows(ok)
        self._follow_id.copy_(torch.where(ok, self._ids[safe], self._follow_id))
        self._follow_ptr.copy_(torch.where(ok, safe.to(I32), self._follow_ptr))
        self._follow_range.copy_(torch.where(ok, rng, self._follow_range))
        self._mode.masked_fill_(ok, mode)

    def follow(self, mask, target, range_) -> None:
        """FollowBall: target is each row's target row (-1: missing)."""
        self._follow(mask, target, range_, FOLLOW)

    def orbit(self, mask, target, range_) -> None:
        """Orbit: as FollowBall, in ORBIT."""
        self._follow(mask, target, range_, ORBIT)

    def warp_to(self, mask, point, min_range, warp_factor) -> None:
        """WarpTo (vec_modes.py:367): the short goto within 1e5 m, the repeated no-op, else Stop, the point,
        aligning (-1), the minimum range's bits and the warp factor, WARP."""
        m = self._m(mask)
        point = torch.as_tensor(point).to(device=self.dev, dtype=F64).reshape(self.n, 3)
        mr = torch.as_tensor(min_range).to(device=self.dev, dtype=F64).reshape(self.n)
        wf = torch.as_tensor(warp_factor).to(device=self.dev, dtype=I64).reshape(self.n)
        ok = m & torch.isfinite(point).all(dim=1)
        mr = torch.where(mr < 0.0, 0.0, mr)
        wf = torch.where(wf <= 0, 1, wf)
        d = self.pos - point
        short = ok & ((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]) < MIN_WARP_DISTANCE_SQ)
        self.goto_point(short, point)
        ok = ok & ~short & ~((self._mode == WARP) & (self.goto == point).all(dim=1))
        self._stop_rows(ok)
        self._goto.copy_(torch.where(ok[None, :], point.t(), self._goto))
        self._effect_stamp.masked_fill_(ok, -1)
        self._follow_range.masked_fill_(ok, 0.0)
        self._follow_id.copy_(torch.where(ok, mr.contiguous().view(I64), self._follow_id))
        self._owner_id.copy_(torch.where(ok, wf, self._owner_id))
        self._mode.masked_fill_(ok, WARP)

    def _release_followers(self, warping: torch.Tensor) -> None:
        """StopAllFollowers of the rows in `warping` (vec_modes.py:388)."""
        f = self._members(warping)
        orbiter = f & self._interactive & (self._mode == ORBIT)
        self._stop_rows(f & ~orbiter)
        self.goto_direction(orbiter, self.vel.clone())

    def entity_warp_in(self, mask, point, warp_factor) -> None:
        """EntityWarpIn (vec_modes.py:397): WarpTo with no minimum range, then warp proper at once (RealWarp, its
        followers released), begun five ticks ago, at warp speed along the point's direction from the origin."""
        m = self._m(mask)
        point = torch.as_tensor(point).to(device=self.dev, dtype=F64).reshape(self.n, 3)
        self.warp_to(m, point, torch.zeros_like(point[:, 0]), warp_factor)
        go = m & (self._mode != GOTO)
        self._release_followers(go)
        delta = _unit(self.pos - self.goto)
        mr = self._follow_id.contiguous().view(F64)
        dst = self.goto + delta * mr[:, None]
        self._goto.copy_(torch.where(go[None, :], dst.t(), self._goto))
        self._massive.masked_fill_(go, False)
        self._sensor.masked_fill_(go, False)
        self._vel.copy_(torch.where(go[None, :], (_unit(point) * AU).t(), self._vel))
        if self.dynamical_orientation:
            self._snap(go)
        self._effect_stamp.copy_(torch.where(go, torch.clamp(self._clock - 5, min=0), self._effect_stamp))
        back = self.pos - self.goto
        length = torch.sqrt(back[:, 0] * back[:, 0] + back[:, 1] * back[:, 1] + back[:, 2] * back[:, 2])
        self._last_collision.copy_(torch.where(go, length, self._last_collision))

    def set_velocity(self, mask, v) -> None:
        """SetBallVelocity: the new and old velocity; with dynamical orientation the rotation snapped."""
        m = self._m(mask)
        v = torch.as_tensor(v).to(device=self.dev, dtype=F64).reshape(self.n, 3)
        self._vel.copy_(torch.where(m[None, :], v.t(), self._vel))
        self._old_vel.copy_(torch.where(m[None, :], v.t(), self._old_vel))
        if self.dynamical_orientation:
            self._snap(m)

    def set_free(self, mask, flag) -> None:
        """SetBallFree (vec_modes.py:438)."""
        m = self._m(mask)
        flag = torch.as_tensor(flag).to(self.dev).reshape(self.n) != 0
        change = m & (flag != self._free)
        fix = change & ~flag
        self._free.copy_(torch.where(change, flag, self._free))
        self._stop_rows(fix)
        self.set_velocity(fix, torch.zeros(self.n, 3, dtype=F64, device=self.dev))
        self._last_g.masked_fill_(fix[None, :], 0.0)

    def set_ball_rigid(self, mask) -> None:
        """SetBallRigid: Stop(Ball*), then RIGID."""
        m = self._m(mask)
        self._stop_rows(m)
        self._mode.masked_fill_(m, RIGID)

    def set_boid(self, mask, on) -> None:
        """The Python SetBoid: BOID without a Stop, or a Stop."""
        m = self._m(mask)
        on = torch.as_tensor(on).to(self.dev).reshape(self.n) != 0
        self._mode.masked_fill_(m & on, BOID)
        self._stop_rows(m & ~on)

    def set_interactive(self, mask, flag) -> None:
        m = self._m(mask)
        flag = torch.as_tensor(flag).to(self.dev).reshape(self.n) != 0
        self._interactive.copy_(torch.where(m, flag, self._interactive))

    def set_ball_troll(self, mask, delay) -> None:
        """SetBallTroll (vec_modes.py:472): a delay below 1 made 1; Stop; free; interactive; due at the clock plus
        the delay; TROLL (petrified in the tick it is due)."""
        m = self._m(mask)
        d = torch.as_tensor(delay).to(device=self.dev, dtype=I64).reshape(self.n)
        d = torch.where(d < TROLL_MIN_DELAY, TROLL_MIN_DELAY, d)
        self._stop_rows(m)
        self.set_free(m, torch.ones_like(m))
        self.set_interactive(m, torch.ones_like(m))
        self._effect_stamp.copy_(torch.where(m, self._clock + d, self._effect_stamp))
        self._mode.masked_fill_(m, TROLL)

    # ---- setters (vec_orient.py:403-465) ----
    def _vals(self, x) -> torch.Tensor:
        return torch.as_tensor(x).to(device=self.dev, dtype=F64).reshape(self.n)

    def set_mass(self, mask, mass) -> None:
        """SetBallMass: ignored unless positive (a NaN is stored); the decay factor refreshed."""
        m, v = self._m(mask), self._vals(mass)
        ok = m & ~(v <= 0.0)
        self._mass.copy_(torch.where(ok, v, self._mass))
        self._decay_rows(ok)

    def set_agility(self, mask, a) -> None:
        """SetBallAgility: the float ignored unless positive; the decay factor refreshed."""
        m, v = self._m(mask), self._vals(a).to(F32)
        ok = m & ~(v <= 0.0)
        self._agility.copy_(torch.where(ok, v, self._agility))
        self._decay_rows(ok)

    def set_max_velocity(self, mask, v) -> None:
        """SetMaxSpeed: the float ignored if negative (Destiny re-files the ball: counted in `refiled`)."""
        m, v = self._m(mask), self._vals(v).to(F32)
        ok = m & ~(v < 0.0)
        self._max_vel.copy_(torch.where(ok, v, self._max_vel))
        self.refiled += ok.to(I64)

    def set_speed_fraction(self, mask, s) -> None:
        """SetSpeedFraction: the float refused unless finite, clamped to [0, 1]."""
        m, s = self._m(mask), self._vals(s).to(F32)
        ok = m & torch.isfinite(s)
        s = torch.where(s < 0.0, 0.0, torch.where(s > 1.0, 1.0, s))
        self._speed_fraction.copy_(torch.where(ok, s, self._speed_fraction))

    def set_radius(self, mask, r) -> None:
        """SetBallRadius: the float ignored if negative (re-filing counted)."""
        m, r = self._m(mask), self._vals(r).to(F32)
        ok = m & ~(r < 0.0)
        self._radius.copy_(torch.where(ok, r, self._radius))
        self.refiled += ok.to(I64)

    def set_max_angular_speed(self, mask, w) -> None:
        m, w = self._m(mask), self._vals(w).to(F32)
        ok = m & ~(w < 0.0)
        self._max_ang_vel.copy_(torch.where(ok, w, self._max_ang_vel))

    def set_rot_agility(self, mask, a) -> None:
        m, a = self._m(mask), self._vals(a).to(F32)
        ok = m & ~(a <= 0.0)
        self._rot_agility.copy_(torch.where(ok, a, self._rot_agility))

    def set_angular_velocity(self, mask, w) -> None:
        """SetBallAngularVelocity: the new and old angular velocity, as floats."""
        m = self._m(mask)
        w = torch.as_tensor(w).to(device=self.dev, dtype=F64).reshape(self.n, 3).to(F32).t()
        self._ang_vel.copy_(torch.where(m[None, :], w, self._ang_vel))
        self._old_ang_vel.copy_(torch.where(m[None, :], w, self._old_ang_vel))

    def set_rotation(self, mask, q) -> None:
        """SetBallRotation: normalised when longer than 1e-20 (else ignored), the rotation stopped."""
        m = self._m(mask)
        q = torch.as_tensor(q).to(device=self.dev, dtype=F64).reshape(self.n, 4).to(F32)
        l2 = ((q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1]) + q[:, 2] * q[:, 2]) + q[:, 3] * q[:, 3]
        length = torch.sqrt(l2)
        ok = m & (length.to(F64) > 1e-20)
        d = torch.ones_like(length) / torch.where(ok, length, torch.ones_like(length))
        rot = (q * d[:, None]).t()
        for t in (self._rot, self._old_rot):
            t.copy_(torch.where(ok[None, :], rot, t))
        for t in (self._ang_vel, self._old_ang_vel):
            t.masked_fill_(ok[None, :], 0.0)

    # ---- the tick ----
    def scratch(self) -> torch.Tensor:
        """The plain schedule's records buffer (device bytes, made once)."""
        need = int(_native.lib().ebb_flight_scratch_bytes(self.n))
        if self._scratch is None or self._scratch.numel() < need:
            self._scratch = torch.empty(max(need, 256), dtype=torch.uint8, device=self.dev)
        return self._scratch

    def evolve(self, lib=None, active: torch.Tensor | None = None) -> None:
        """One tick of every world, in place, on the device, no host synchronisation. `active` [n] (OnTick's
        per-world mask): only those rows tick, every other row keeps its state bit for bit (inside the listed-worlds
        kernel when the worlds are contiguous rows, else by a save and put-back around the tick)."""
        if active is not None:
            act = torch.as_tensor(active).to(device=self.dev, dtype=BOOL).reshape(self.n).contiguous()
            if _worlds_plan_ok(self):
                tick_worlds(self, act)
            else:
                masked_tick(self, act, lambda: tick(self, self.block))
        else:
            tick(self, self.block)
        self.current_time += 1

    def row_tensors(self) -> list:
        return ["_" + name for name, _, _ in _STORAGE] + ["refiled"]


# ================================================================================================= the schedules

def tick_plain(park: VecModesPark, block: int = 128) -> None:
    """The plain schedule: the records pass and the tick, two launches, records in the park's scratch."""
    if not park.n:
        return
    sc = park.scratch()
    with torch.cuda.device(park.dev):
        rc = _native.lib().ebb_flight_tick(ctypes.byref(park.state()), sc.data_ptr(), sc.numel(), park._stream(),
                                           int(block))
    _native.check(rc, "ebb_flight_tick")


def tick_tiled(park: VecModesPark, plan: TilePlan | None = None) -> None:
    """The tiled schedule: one launch, the records in shared memory (the rows grouped by world)."""
    plan = plan or park.plan
    if plan is None:
        raise ValueError("the park's worlds are not contiguous rows: no tile plan")
    if not park.n:
        return
    tr = plan.tile_rows_on(park.dev)
    with torch.cuda.device(park.dev):
        rc = _native.lib().ebb_flight_tick_tiled(ctypes.byref(park.state()), tr.data_ptr(), plan.tiles, plan.cap,
                                                 park._status.data_ptr(), park._stream(), plan.block, plan.grid)
    _native.check(rc, "ebb_flight_tick_tiled")


WORLDS_MAX_TILE = 1024          # include/ebb.h: EBB_WORLDS_MAX_TILE


def _worlds_plan_ok(park: VecModesPark) -> bool:
    return park.plan is not None and park.plan.cap <= WORLDS_MAX_TILE and len(park.plan.world_rows) > 1


def tick_worlds(park: VecModesPark, active: torch.Tensor | None = None, plan=None) -> None:
    """The listed-worlds schedule over the park's own worlds (its tile plan as a world list, or a best-fit
    tiles.WorldsPlan), with OnTick's row mask `active` (a contiguous bool tensor [n], or None for every row) applied
    inside the kernel."""
    plan = plan or park.plan
    if plan is None:
        raise ValueError("the park's worlds are not contiguous rows: no tile plan")
    if not park.n:
        return
    worlds, tile_worlds = plan.worlds_on(park.dev)
    act = 0 if active is None else active.data_ptr()
    with torch.cuda.device(park.dev):
        rc = _native.lib().ebb_flight_tick_worlds(ctypes.byref(park.state()), worlds.data_ptr(), tile_worlds.data_ptr(),
                                                  plan.tiles, plan.cap, act, park._status.data_ptr(), park._stream(),
                                                  plan.block, plan.grid)
    _native.check(rc, "ebb_flight_tick_worlds")


def tick(park: VecModesPark, block: int = 128, lib=None) -> None:
    """One tick in place on torch's current stream (the drop-in for exact_ballpark.vec_modes_cuda.tick): the tiled
    schedule when the park's worlds are contiguous rows, the plain one otherwise."""
    if park.plan is not None:
        tick_tiled(park)
    else:
        tick_plain(park, block)


def masked_tick(park: VecModesPark, active: torch.Tensor, run) -> None:
    """OnTick's per-world mask (vec_orient.py:217): `run()` ticks every row, then the rows outside `active` get
    their state back bit for bit (every world's reads stay in its world)."""
    act = torch.as_tensor(active).to(device=park.dev, dtype=BOOL).reshape(park.n)
    names = park.row_tensors()
    before = {k: getattr(park, k).clone() for k in names}
    run()
    row_major = getattr(park, "ROW_MAJOR", ())
    for k, old in before.items():
        cur = getattr(park, k)
        sel = act if cur.dim() == 1 else (act[:, None] if k in row_major else act[None, :])
        cur.copy_(torch.where(sel, cur, old))


def kernel_info(device=None) -> dict:
    """The kernels as loaded on a device: registers, local memory, binary and PTX versions."""
    out = {}
    for which, name in ((0, "tick"), (1, "records"), (2, "tiled"), (3, "worlds"), (4, "move")):
        vals = [ctypes.c_int() for _ in range(5)]
        with torch.cuda.device(torch.device(device or "cuda")):
            rc = _native.lib().ebb_kernel_info(which, *[ctypes.byref(v) for v in vals])
        _native.check(rc, "ebb_kernel_info")
        regs, local, binary, ptx, threads = (v.value for v in vals)
        out[name] = {"registers": regs, "local_bytes": local, "binary_version": binary, "ptx_version": ptx,
                     "max_threads_per_block": threads}
    return out


LIBM_FUNCS = {"sin": 0, "cos": 1, "log": 2, "exp": 3, "sincos_sin": 4, "sincos_cos": 5, "pow": 6, "expf": 10,
              "logf": 11, "sinf": 12, "cosf": 13, "acosf": 14, "atanf": 15, "atan2f": 16, "powf": 17}


def libm(name: str, x: torch.Tensor, y: torch.Tensor | None = None, block: int = 128) -> torch.Tensor:
    """The device's glibc function `name` on a CUDA float64 tensor (floats held in doubles for the float ones)."""
    x = x.to(F64).contiguous()
    y = (x if y is None else y.to(F64)).contiguous()
    out = torch.empty_like(x)
    with torch.cuda.device(x.device):
        rc = _native.lib().ebb_libm(LIBM_FUNCS[name], x.numel(), x.data_ptr(), y.data_ptr(), out.data_ptr(),
                                    torch.cuda.current_stream(x.device).cuda_stream, int(block))
    _native.check(rc, "ebb_libm")
    return out


class ModesGraph:
    """A park's tick captured once as a CUDA graph on the park's own buffers (the drop-in for
    exact_ballpark.vec_modes_cuda.ModesGraph): each `tick()` is one replay. The commands write the buffers in place,
    so nothing is re-bound between replays. With `masked=True` OnTick's mask is a device buffer in the graph."""

    def __init__(self, park: VecModesPark, block: int | None = None, lib=None, masked: bool = False):
        self.park = park
        self.block = park.block if block is None else int(block)
        self.masked = masked
        self.mask = torch.ones(park.n, dtype=BOOL, device=park.dev)
        if park.plan is None:
            park.scratch()
        else:
            park.plan.tile_rows_on(park.dev)
        names = park.row_tensors()
        self.in_kernel = masked and _worlds_plan_ok(park)            # OnTick's mask inside the listed-worlds kernel
        if self.in_kernel:
            park.plan.worlds_on(park.dev)
        self.saved = {k: torch.empty_like(getattr(park, k)) for k in names} if masked and not self.in_kernel else {}
        keep = {k: getattr(park, k).clone() for k in names}      # the warm-up tick is undone
        side = torch.cuda.Stream(device=park.dev)
        side.wait_stream(torch.cuda.current_stream(park.dev))
        with torch.cuda.stream(side):                                # a warm-up launch of every kernel
            if self.in_kernel:
                tick_worlds(park, self.mask)
            else:
                tick(park, self.block)
            for k, v in keep.items():
                getattr(park, k).copy_(v)
        torch.cuda.current_stream(park.dev).wait_stream(side)
        torch.cuda.synchronize(park.dev)
        del keep
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            if self.in_kernel:
                tick_worlds(park, self.mask)
            else:
                if masked:
                    self._save()
                tick(park, self.block)
                if masked:
                    self._put_back()

    def _save(self) -> None:
        for k, b in self.saved.items():
            b.copy_(getattr(self.park, k))

    def _put_back(self) -> None:
        for k, b in self.saved.items():
            cur = getattr(self.park, k)
            sel = self.mask if cur.dim() == 1 else self.mask[None, :]
            cur.copy_(torch.where(sel, cur, b))

    def tick(self, active: torch.Tensor | None = None) -> None:
        if active is not None and not self.masked:
            raise ValueError("a graph made without OnTick's mask (masked=True) ticks every row")
        if self.masked:
            if active is None:
                self.mask.fill_(True)
            else:
                self.mask.copy_(torch.as_tensor(active).to(device=self.park.dev, dtype=BOOL).reshape(self.park.n))
        self.graph.replay()
        self.park.current_time += 1
