"""The server layer over the flight-mode park on a B200: a drop-in for exact_ballpark.vec_server's VecServer and
ModesAdapter (exact_ballpark/vec_server.py:197-1080): Destiny's net/server layer batched for many worlds, each world one
bubble with its pilots.

Per tick, as Destiny's test helper drives the layer: `push` queues an Actions call for every masked world (TIME-709,
TIME-710: stamped, and dropped when it equals the world's last queued call — same kind, ball, target, floats by value
(a NaN equals nothing), ints and the local argument exactly); `pre_tick` moves the stamp, flushes the queue and applies
every queued call but CloakBall through the park in queue order (the j-th calls of every world together, each world's
in its own order), updates the bubble's additions (BubbleUpdater: a user ball seen for the first time gets every
uncloaked ball of its bubble), then walks the history: CloakBall applied there and its event sent to the bubble it
was queued in, UncloakBall's event to its own character with an AddBallsToPark to every other interactive pilot, a
local SetBallPosition sent nowhere, every other event to the bubble, or to the ball's character while it is cloaked;
`evolve` is the park's tick (a world whose bubble is dead at an evolve is refused by `check`); `post_tick` sets, per
pilot, whether it gets the bubble's narrowcast and a character update (ParkUpdateBatcher.send_batch). `batch` holds the
tick's update batch as tensors: the stamps, the queued calls, their routes, the uncloaks' recipients, the additions
and the flags, with the park's fields where the streams would be written (`stream_fields`).

Two paths with one result, bit for bit. kernel="torch": every park write is the park's own command or setter
(exact_ballpark_b200.modes, on the device) over all worlds at once, one queued call after another; the layer adds only
index work (masks, gathers, comparisons) and the cloak's float sum radius + range as float32, as the C++ does.
kernel="cuda": the native library's server kernel (ebb_server_tick), one thread a world walking its own queue, every
command restated for one row; one launch for the whole pre-tick (or one per history segment when the park's fields are
recorded for the streams), one for the dead-bubble test before the park's tick (fused into the pre-tick's launch in a
graph, where nothing comes between them) and one for the send flags after it.
`ServerGraph` captures a kernel-path tick with a fixed schedule of pushes as one CUDA graph.

The pending queries and the undo of a pending cloak (Actions, _actions.py:686-766) answer from the queue on both paths;
OnTick's per-world intervals (`on_tick`, the masks of `pre_tick`, `evolve` and `post_tick`) run on both paths.

`decode` turns a batch into what Destiny's network sends each client: its singlecast and the bubble's narrowcast, with
the events, the AddBallsToPark streams in WriteBallToStream's layout and the packaged additions.

`CollideAdapter` puts the layer over the collision park (torch path). `ClientView` keeps what each pilot's client
holds, `down` ticks behind the server.

Not built: the orientation and combat parks' adapters, bubbles other than one a world.
"""

from __future__ import annotations

import copy
import ctypes
import struct
from dataclasses import dataclass, field
from enum import IntEnum

import torch

from . import _native
from .modes import WARP, tick as _park_tick

F64, F32, I64, BOOL = torch.float64, torch.float32, torch.int64, torch.bool

# the queued actions by the event the server sends (the index is the kind's code; 0 no action)
KINDS = ("", "GotoPoint", "GotoDirection", "Stop", "FollowBall", "Orbit", "WarpTo", "EntityWarpIn", "SetSpeedFraction",
         "SetMaxSpeed", "SetBallMass", "SetBallAgility", "SetBallRadius", "SetBallVelocity", "SetBallMassive",
         "SetBallInteractive", "SetBallPosition", "CloakBall", "UncloakBall", "SetMaxAngularSpeed",
         "SetBallAngularVelocity", "SetBallRotation", "SetBallAngularAgility", "SetMaxAngularVelocity",
         "LaunchMissile", "SetBallTroll", "SetBallFree", "AddBallsToPark", "BallNotGlobal")
CODE = {name: k for k, name in enumerate(KINDS) if name}
DYNAMICAL_ONLY = frozenset(CODE[k] for k in ("SetBallAngularVelocity", "SetMaxAngularVelocity", "SetBallRotation",
                                             "SetBallAngularAgility", "SetMaxAngularSpeed"))
NONE, BUBBLE, CHARACTER = 0, 1, 2                   # where an event goes
MAX_CATCH_UP_TICKS = 5                              # OnTick's backlog on the master (Ballpark.cpp:248, TIME-703)
DSTNORMALCLOAK = 1
CLOAK, UNCLOAK, SETPOS, INTERACTIVE = CODE["CloakBall"], CODE["UncloakBall"], CODE["SetBallPosition"], \
    CODE["SetBallInteractive"]
FOLLOWS = (CODE["FollowBall"], CODE["Orbit"])
TROLL = CODE["SetBallTroll"]
# applied by the parks with missiles, and by the partition layer's server: not by the flight park
NOT_APPLIED = frozenset(CODE[k] for k in ("LaunchMissile", "AddBallsToPark", "BallNotGlobal"))


def _char(x: torch.Tensor) -> torch.Tensor:
    return ((x.to(I64) + 128) & 0xFF) - 128


class _Worlds:
    """The rows of a park grouped into worlds: `world` [R] (0 .. W-1), `rows_of_world` [W, width] (in the order the
    balls were added, -1 padded) with `ids_of_world` (0 padded), and the lookups the layer makes."""

    def _index_worlds(self, labels: list) -> None:
        order, groups = [], {}
        for r, w in enumerate(labels):
            if w not in groups:
                groups[w] = []
                order.append(w)
            groups[w].append(r)
        self.labels, self.W = order, len(order)
        width = max((len(g) for g in groups.values()), default=0)
        table = [g + [-1] * (width - len(g)) for g in (groups[w] for w in order)]
        self.rows_of_world = torch.tensor(table, dtype=I64, device=self.dev).reshape(self.W, width)
        index = {w: k for k, w in enumerate(order)}
        self.world = torch.tensor([index[w] for w in labels], dtype=I64, device=self.dev)
        self._ids_of_rows()
        self.arange = torch.arange(self.R, device=self.dev)

    def _ids_of_rows(self) -> None:
        safe = self.rows_of_world.clamp(min=0)
        self.ids_of_world = torch.where(self.rows_of_world >= 0, self.ids[safe], 0)

    def lookup(self, ball: torch.Tensor) -> torch.Tensor:
        """Each world's row of the ball whose Destiny id is ball[w], or -1."""
        hit = self.ids_of_world == ball.to(I64)[:, None]
        first = hit.to(I64).argmax(dim=1)
        return torch.where(hit.any(dim=1), self.rows_of_world.gather(1, first[:, None])[:, 0], -1)

    def any_in_world(self, flag: torch.Tensor) -> torch.Tensor:
        safe = self.rows_of_world.clamp(min=0)
        return (flag[safe] & (self.rows_of_world >= 0)).any(dim=1)


class ModesAdapter(_Worlds):
    """The flight-mode park (exact_ballpark_b200.VecModesPark) as the server layer sees it: its rows grouped by world
    label (first appearance order; a world's rows in the order its balls were added, the bubble's dictionary order),
    the Destiny ids, the flags the layer routes by, and each kind applied through the park's command or setter."""

    master = True

    def __init__(self, park, master: bool = True):
        self.park, self.R, self.dev, self.master = park, park.n, park.dev, bool(master)
        self.ids = park.ids
        self.exists = torch.ones(self.R, dtype=BOOL, device=self.dev)
        self._index_worlds(park.world.tolist())
        do = park.dynamical_orientation
        self.kinds = frozenset(k for k in range(1, len(KINDS))
                               if (do or k not in DYNAMICAL_ONLY) and k not in NOT_APPLIED)

    interactive = property(lambda s: s.park.interactive, lambda s, v: setattr(s.park, "interactive", v))
    massive = property(lambda s: s.park.massive, lambda s, v: setattr(s.park, "massive", v))

    @property
    def cloaked(self) -> torch.Tensor:
        return self.park.cloaked

    @cloaked.setter
    def cloaked(self, v) -> None:
        self.park.cloaked.copy_(torch.as_tensor(v, device=self.dev))

    def radius(self) -> torch.Tensor:
        return self.park.radius

    def clock(self) -> torch.Tensor:
        """Each world's mCurrentTime (its rows share one clock)."""
        return self.park.clock[self.rows_of_world[:, 0]]

    def warping(self) -> torch.Tensor:
        return (self.park.mode == WARP) & (self.park.effect_stamp >= 0)

    def cloak(self, m: torch.Tensor, mode: torch.Tensor, rng: torch.Tensor) -> None:
        """CloakBall (Ballpark.cpp:5223): refused unless the signed char mode is positive; on the master a normal cloak
        adds a proximity sensor (unless float(radius) + float(range) < 0); the followers released; cloaked with the
        mode's byte, non-massive."""
        mode = _char(mode)
        ok = m & self.exists & (mode > 0)
        if self.master:
            rng32 = rng.to(F64).to(F32).to(F64)
            sense = ok & (mode == DSTNORMALCLOAK) & ~((self.radius() + rng32).to(F32) < 0.0)
            self.park.sensor = self.park.sensor | sense
        self.park._release_followers(ok)
        self.cloaked = torch.where(ok, mode & 0xFF, self.cloaked)
        self.massive = torch.where(ok, False, self.massive)

    def uncloak(self, m: torch.Tensor) -> None:
        """UncloakBall (Ballpark.cpp:5257): a normal cloak's sensor removed (master); uncloaked; massive again unless
        in warp proper."""
        ok = m & self.exists
        if self.master:
            self.park.sensor = self.park.sensor & ~(ok & (self.cloaked == DSTNORMALCLOAK))
        self.cloaked = torch.where(ok, 0, self.cloaked)
        self.massive = torch.where(ok & ~self.warping(), True, self.massive)

    def apply(self, kind: int, m: torch.Tensor, trow: torch.Tensor, f: torch.Tensor, n: torch.Tensor) -> None:
        """One kind on the rows in m, each row's arguments: the park's own command or setter."""
        p, name = self.park, KINDS[kind]
        xyz = f[:, :3].contiguous()
        one = f[:, 0].contiguous()
        if name == "GotoPoint":
            p.goto_point(m, xyz)
        elif name == "GotoDirection":
            p.goto_direction(m, xyz)
        elif name == "Stop":
            p.stop(m)
        elif name == "FollowBall":
            p.follow(m, trow, one)
        elif name == "Orbit":
            p.orbit(m, trow, one)
        elif name == "WarpTo":
            p.warp_to(m, xyz, f[:, 3].contiguous(), n)
        elif name == "EntityWarpIn":
            p.entity_warp_in(m, xyz, n)
        elif name == "SetSpeedFraction":
            p.set_speed_fraction(m, one)
        elif name == "SetMaxSpeed":
            p.set_max_velocity(m, one)
        elif name == "SetBallMass":
            p.set_mass(m, one)
        elif name == "SetBallAgility":
            p.set_agility(m, one)
        elif name == "SetBallRadius":
            p.set_radius(m, one)
        elif name == "SetBallVelocity":
            p.set_velocity(m, xyz)
        elif name == "SetBallMassive":
            p.massive = torch.where(m, n != 0, p.massive)
        elif name == "SetBallInteractive":
            p.interactive = torch.where(m, n != 0, p.interactive)
        elif name == "SetBallPosition":                 # the new and old position
            p.pos = torch.where(m[:, None], xyz, p.pos)
            p.old_pos = torch.where(m[:, None], xyz, p.old_pos)
        elif name == "UncloakBall":
            self.uncloak(m)
        elif name == "SetMaxAngularSpeed":
            p.set_max_angular_speed(m, one)
        elif name == "SetBallAngularVelocity":
            p.set_angular_velocity(m, xyz)
        elif name == "SetBallRotation":
            p.set_rotation(m, f)
        elif name == "SetBallAngularAgility":
            p.set_rot_agility(m, one)
        elif name == "SetMaxAngularVelocity":
            pass                                        # the park has no such method: never applied
        elif name == "SetBallTroll":
            p.set_ball_troll(m, n)
        elif name == "SetBallFree":                     # a flag != 0 frees
            p.set_free(m, n)
        else:
            raise ValueError(f"{name} is not applied by the flight park's server layer")

    def evolve(self, worlds: torch.Tensor | None = None) -> None:
        """The park's tick; `worlds` [W] (OnTick's mask): those worlds' rows alone."""
        self.park.evolve(active=None if worlds is None else worlds[self.world])

    def stream_fields(self) -> dict:
        """The fields WriteBallToStream writes (Thunkers.cpp:3180-3377), every row, copied to the host (a snapshot: later
        writes to the park do not reach it)."""
        p = self.park
        out = {k: getattr(p, k).detach().to("cpu", copy=True) for k in ("ids", "mode", "radius", "pos", "free", "massive",
                                                          "interactive", "mass", "cloaked", "max_vel", "vel",
                                                          "agility", "speed_fraction", "goto", "follow_id",
                                                          "follow_range", "effect_stamp", "last_collision",
                                                          "owner_id", "rot", "max_ang_vel", "ang_vel",
                                                          "rot_agility")}
        out["dynamical"] = bool(p.dynamical_orientation)
        return out


class CollideAdapter(_Worlds):
    """The collision park (exact_ballpark_b200.VecCollidePark: W worlds of N slots, GOTO and STOP with Destiny's
    collisions) as the server layer sees it (vec_server.py:491-580): row w N + slot, a world's balls in its first
    slots; the park's exists, ids, massive flag and cloak flag (the cloak's mode kept here), the interactive flags
    kept here (given at the construction, all interactive by default), each world's park time kept here; GotoPoint,
    GotoDirection, Stop, SetSpeedFraction, SetBallMassive, SetBallInteractive, CloakBall and UncloakBall. A normal
    cloak's proximity sensor is not modelled by this park. The server kernel does not take this adapter."""

    master = True

    def __init__(self, park, interactive=None, master: bool = True):
        self.park, self.dev, self.master = park, park.dev, bool(master)
        W, N = park.W, park.N
        self.R = W * N
        self.ids = park.id.reshape(-1)
        self.exists = park.exists.reshape(-1)
        self._index_worlds([r // N for r in range(self.R)])
        self.rows_of_world = torch.where(park.exists, self.rows_of_world, -1)
        self._ids_of_rows()
        given = [True] * self.R if interactive is None else [bool(x) for x in interactive]
        self.interactive = torch.tensor(given, dtype=BOOL, device=self.dev) & self.exists
        self._cloaked = torch.where(park.cloaked.reshape(-1), 1, 0).to(I64)
        self.time = torch.full((self.W,), int(park.current_time), dtype=I64, device=self.dev)
        self.kinds = frozenset(CODE[k] for k in ("GotoPoint", "GotoDirection", "Stop", "SetSpeedFraction",
                                                  "SetBallMassive", "SetBallInteractive", "CloakBall", "UncloakBall"))

    @property
    def massive(self) -> torch.Tensor:
        return self.park.massive.reshape(-1)

    @massive.setter
    def massive(self, v) -> None:
        self.park.massive.copy_(torch.as_tensor(v, device=self.dev).reshape(self.park.W, self.park.N))

    @property
    def cloaked(self) -> torch.Tensor:
        return self._cloaked

    @cloaked.setter
    def cloaked(self, v) -> None:
        self._cloaked = torch.as_tensor(v, device=self.dev).to(I64)
        self.park.cloaked.copy_((self._cloaked != 0).reshape(self.park.W, self.park.N))

    def radius(self) -> torch.Tensor:
        return self.park.radius.reshape(-1)

    def clock(self) -> torch.Tensor:
        return self.time

    def cloak(self, m: torch.Tensor, mode: torch.Tensor, rng: torch.Tensor) -> None:
        """CloakBall: refused unless the signed char mode is positive; cloaked with the mode's byte, non-massive (no
        followers and no sensor in this park)."""
        mode = _char(mode)
        ok = m & self.exists & (mode > 0)
        self.cloaked = torch.where(ok, mode & 0xFF, self.cloaked)
        self.massive = torch.where(ok, False, self.massive)

    def uncloak(self, m: torch.Tensor) -> None:
        """UncloakBall: uncloaked and massive again (no ball of this park is in warp)."""
        ok = m & self.exists
        self.cloaked = torch.where(ok, 0, self.cloaked)
        self.massive = torch.where(ok, True, self.massive)

    def apply(self, kind: int, m: torch.Tensor, trow: torch.Tensor, f: torch.Tensor, n: torch.Tensor) -> None:
        p, name, W, N = self.park, KINDS[kind], self.park.W, self.park.N
        mm = m.reshape(W, N)
        xyz = f[:, :3].reshape(W, N, 3)
        if name == "GotoPoint":
            p.goto_point(mm, xyz)
        elif name == "GotoDirection":
            p.goto_direction(mm, xyz)
        elif name == "Stop":
            p.stop(mm)
        elif name == "SetSpeedFraction":
            p.set_speed_fraction(mm, f[:, 0].reshape(W, N))
        elif name == "SetBallMassive":
            self.massive = torch.where(m, n != 0, self.massive)
        elif name == "SetBallInteractive":
            self.interactive = torch.where(m & self.exists, n != 0, self.interactive)
        elif name == "UncloakBall":
            self.uncloak(m)
        else:
            raise ValueError(f"{name} is not applied by the collision park's server layer")

    def evolve(self, worlds: torch.Tensor | None = None) -> None:
        """The park's tick and each world's park time; `worlds` [W] (OnTick's mask): those worlds alone."""
        if worlds is None:
            self.park.evolve()
            self.time.add_(1)
            return
        self.park.evolve(active=worlds)
        self.time.add_(worlds.to(I64))

    def stream_fields(self) -> dict:
        p, R = self.park, self.R
        host = lambda t: t.detach().to("cpu", copy=True)                     # noqa: E731  (a snapshot)
        zero = torch.zeros(R, dtype=I64)
        out = {k: host(getattr(p, k).reshape(R, *getattr(p, k).shape[2:]))
               for k in ("mode", "radius", "pos", "free", "mass", "max_vel", "vel", "agility", "speed_fraction", "goto",
                         "last_collision")}
        out.update(ids=host(self.ids), massive=host(self.massive), interactive=host(self.interactive),
                   cloaked=host(self.cloaked), follow_id=zero, owner_id=zero, effect_stamp=zero,
                   follow_range=torch.zeros(R, dtype=F64), dynamical=False)
        return out


@dataclass
class Slot:
    """One push: one Actions call for every masked world."""
    kind: int
    ok: torch.Tensor                    # [W] queued
    ball: torch.Tensor                  # [W] Destiny id
    row: torch.Tensor                   # [W] the ball's row, or -1
    target: torch.Tensor                # [W] the target's id (FollowBall, Orbit)
    trow: torch.Tensor                  # [W] the target's row, or -1
    f: torch.Tensor                     # [W, 4] the float arguments
    n: torch.Tensor                     # [W] the int argument
    loc: torch.Tensor                   # [W] SetBallPosition: is local; CloakBall: its bubble (0, or -1)


@dataclass
class Batch:
    """One tick's update batches, every world (the fields of exact_ballpark.vec_server.Batch)."""
    stamp: torch.Tensor
    clock: torch.Tensor
    slots: list
    route: torch.Tensor                 # [W, J] NONE, BUBBLE or CHARACTER
    notices: list = field(default_factory=list)     # (slot j, recipients [R], the park's fields there or None)
    additions: tuple | None = None      # (fresh [R], listed [R], the park's fields or None)
    gets_bubble: torch.Tensor | None = None
    has_character: torch.Tensor | None = None
    ticked: torch.Tensor | None = None


class VecServer:
    """The server layer over an adapter (the module's docstring): kernel "torch" or "cuda"."""

    def __init__(self, adapter: ModesAdapter, pilots=None, kernel: str = "torch", block: int = 128):
        if kernel not in ("torch", "cuda"):
            raise ValueError(f"kernel {kernel!r}: 'torch' or 'cuda'")
        self.a = A = adapter
        self.W, self.R, self.dev = A.W, A.R, A.dev
        self.kernel, self.block = kernel, int(block)
        self.pilot = (torch.full((self.R,), -1, dtype=I64, device=self.dev) if pilots is None
                      else torch.as_tensor(pilots, dtype=I64).to(self.dev))
        clock = A.clock()
        self.stamp_for_system = torch.where(clock == 0, 0, clock + 1)     # Actions' first stamp
        self.settled = torch.zeros(self.R, dtype=BOOL, device=self.dev)   # the old bubble is the bubble
        self.dead = torch.zeros(self.W, dtype=BOOL, device=self.dev)
        self._bubble_time = torch.full((self.W,), -1, dtype=I64, device=self.dev)
        self._fresh = torch.zeros(self.R, dtype=BOOL, device=self.dev)
        self._listed = torch.zeros(self.R, dtype=BOOL, device=self.dev)
        self._seen_first = False
        self.slots: list = []
        self._reset_last()
        self.batch: Batch | None = None
        self._q = None
        if kernel == "cuda":
            if self.dev.type != "cuda" or not isinstance(adapter, ModesAdapter):
                raise ValueError("the server kernel runs the flight park's layer (a ModesAdapter) on a CUDA device")
            self._state = self._server_state()

    def _reset_last(self) -> None:
        W, d = self.W, self.dev
        self.last = {"kind": torch.zeros(W, dtype=I64, device=d), "ball": torch.zeros(W, dtype=I64, device=d),
                     "target": torch.zeros(W, dtype=I64, device=d), "f": torch.zeros(W, 4, dtype=F64, device=d),
                     "n": torch.zeros(W, dtype=I64, device=d), "loc": torch.zeros(W, dtype=I64, device=d)}

    # ---- the kernel's state and queue (include/ebb.h: EbbServerState, EbbServerQueue) ----
    def _server_state(self) -> _native.ServerState:
        A, p = self.a, self.a.park
        self._const = {"world_rows": A.rows_of_world.contiguous(), "world_ids": A.ids_of_world.contiguous(),
                       "pilot": self.pilot.contiguous(), "exists": A.exists.contiguous()}
        st = _native.ServerState()
        st.flight = p.state()
        st.worlds, st.width = self.W, A.rows_of_world.shape[1]
        for k, t in self._const.items():
            setattr(st, k, t.data_ptr())
        for k, t in (("label", p.world), ("cloaked", p.cloaked), ("bubble", p.bubble), ("refiled", p.refiled),
                     ("stamp_for_system", self.stamp_for_system), ("bubble_time", self._bubble_time),
                     ("dead", self.dead), ("settled", self.settled), ("fresh", self._fresh),
                     ("listed", self._listed)):
            if not t.is_contiguous() or t.device != self.dev:
                raise ValueError(f"the server kernel writes {k} in place: a contiguous tensor on {self.dev}")
            setattr(st, k, t.data_ptr())
        st.neg_kdt = -p.friction * p.dt
        st.master = int(A.master)
        return st

    def _queue(self, kinds: list, cols: dict | None = None) -> dict:
        """The queue's tensors for kinds [J]: the pushes' columns ([J, W] stacks, given or zeros) and the outputs."""
        J, W, R, d = len(kinds), self.W, self.R, self.dev
        z = lambda *shape, dt=I64: torch.zeros(*shape, dtype=dt, device=d)          # noqa: E731
        q = {"kinds": torch.tensor(kinds, dtype=torch.int32).to(d), "mask": z(J, W, dt=torch.uint8), "ball": z(J, W),
             "target": z(J, W), "f": z(J, W, 4, dt=F64), "n": z(J, W), "loc_in": z(J, W),
             "ok": z(J, W, dt=BOOL), "row": z(J, W), "trow": z(J, W), "loc": z(J, W),
             "route": z(W, J, dt=torch.int8), "notice": z(J, R, dt=BOOL), "stamp": z(W), "clock": z(W),
             "has_character": z(R, dt=BOOL), "gets_bubble": z(R, dt=BOOL)}
        if cols is not None:
            for k, v in cols.items():
                q[k].copy_(v)
        qs = _native.ServerQueue()
        qs.slots = J
        for k in ("kinds", "mask", "ball", "target", "n", "loc_in", "f", "ok", "row", "trow", "loc", "route",
                  "notice", "stamp", "clock", "has_character", "gets_bubble"):
            setattr(qs, k, q[k].data_ptr())
        q["struct"] = qs
        return q

    def _launch(self, q: dict, phase: int, j0: int = 0, j1: int = 0) -> None:
        with torch.cuda.device(self.dev):
            stream = torch.cuda.current_stream(self.dev).cuda_stream
            rc = _native.lib().ebb_server_tick(ctypes.byref(self._state), ctypes.byref(q["struct"]), int(phase),
                                               int(j0), int(j1), stream, self.block)
        _native.check(rc, "ebb_server_tick")

    # ---- the queue ----
    def push(self, kind, mask, ball, target=None, f=None, n=None, loc=None) -> Slot:
        """An Actions call (a kind's code or event name) for every world in mask [W]: ball [W] ids, target [W] ids
        (FollowBall, Orbit), f [W, k<=4] floats, n [W] the int argument, loc [W] SetBallPosition's is_local_ball.
        CloakBall captures the ball's bubble (0, or -1 before its old bubble is its bubble) and is not queued for a
        ball not in the park; a call equal to the world's last queued call is dropped. On the kernel path the call is
        recorded as given and tested in the pre-tick's launch (its flags and rows filled in there)."""
        k = CODE[kind] if isinstance(kind, str) else int(kind)
        if k not in self.a.kinds:
            raise ValueError(f"{KINDS[k] or kind} is not applied by this park")
        W, d = self.W, self.dev
        z = lambda dt: torch.zeros(W, dtype=dt, device=d)                    # noqa: E731
        mask = torch.as_tensor(mask).to(device=d, dtype=BOOL)
        ball = torch.as_tensor(ball).to(device=d, dtype=I64)
        target = z(I64) if target is None else torch.as_tensor(target).to(device=d, dtype=I64)
        ff = torch.zeros(W, 4, dtype=F64, device=d)
        if f is not None:
            f = torch.as_tensor(f).to(device=d, dtype=F64).reshape(W, -1)
            ff[:, :f.shape[1]] = f
        n = z(I64) if n is None else torch.as_tensor(n).to(device=d, dtype=I64)
        loc = z(I64) if loc is None else torch.as_tensor(loc).to(device=d, dtype=I64)
        if self.kernel == "cuda":
            slot = Slot(k, None, ball, None, target, None, ff, n, loc)
            slot.mask = mask
            self.slots.append(slot)
            return slot
        row = self.a.lookup(ball)
        trow = self.a.lookup(target) if k in FOLLOWS else z(I64) - 1
        if k == CLOAK:
            loc = torch.where(self.settled[row.clamp(min=0)], 0, -1)
            mask = mask & (row >= 0)
        last = self.last
        dup = ((last["kind"] == k) & (last["ball"] == ball) & (last["target"] == target)
               & (last["f"] == ff).all(dim=1) & (last["n"] == n) & (last["loc"] == loc))
        ok = mask & ~dup
        for key, val in (("kind", torch.full((W,), k, dtype=I64, device=d)), ("ball", ball), ("target", target),
                         ("n", n), ("loc", loc)):
            last[key] = torch.where(ok, val, last[key])
        last["f"] = torch.where(ok[:, None], ff, last["f"])
        slot = Slot(k, ok, ball, row, target, trow, ff, n, loc)
        self.slots.append(slot)
        return slot

    # ---- the pending queries and the undo of a pending cloak (_actions.py:686-766) ----
    #
    # Destiny's game code asks the queue between ticks what is pending and may undo a pending cloak. On the torch path
    # each call was tested at its push; on the kernel path the calls are tested here, in queue order, as the kernel
    # would test them, and an undo hands the kernel the tested calls (`resolved`: bit 1 of the kernel's mask byte,
    # bit 0 then the queued flag and `loc` CloakBall's tested bubble) so that it does not test them again.

    def _deferred(self) -> bool:
        return self.kernel == "cuda"

    def _zero_last(self) -> dict:
        W, d = self.W, self.dev
        return {"kind": torch.zeros(W, dtype=I64, device=d), "ball": torch.zeros(W, dtype=I64, device=d),
                "target": torch.zeros(W, dtype=I64, device=d), "f": torch.zeros(W, 4, dtype=F64, device=d),
                "n": torch.zeros(W, dtype=I64, device=d), "loc": torch.zeros(W, dtype=I64, device=d)}

    @staticmethod
    def _become_last(last: dict, s: Slot, queued: torch.Tensor, loc: torch.Tensor) -> None:
        for key, val in (("kind", torch.full_like(last["kind"], s.kind)), ("ball", s.ball), ("target", s.target),
                         ("n", s.n), ("loc", loc)):
            last[key] = torch.where(queued, val, last[key])
        last["f"] = torch.where(queued[:, None], s.f, last["f"])

    def _test_pending(self, commit: bool = False) -> list:
        """The kernel path's pending calls tested as the kernel tests them (the resolved prefix taken as it is): each
        call's queued flag [W]; `commit` makes every call resolved."""
        last = self._zero_last()
        out = []
        for s in self.slots:
            if getattr(s, "resolved", False):
                queued, loc = s.mask, s.loc
            else:
                row = self.a.lookup(s.ball)
                queued, loc = s.mask, s.loc
                if s.kind == CLOAK:
                    loc = torch.where(self.settled[row.clamp(min=0)], 0, -1)
                    queued = queued & (row >= 0)
                dup = ((last["kind"] == s.kind) & (last["ball"] == s.ball) & (last["target"] == s.target)
                       & (last["f"] == s.f).all(dim=1) & (last["n"] == s.n) & (last["loc"] == loc))
                queued = queued & ~dup
            self._become_last(last, s, queued, loc)
            out.append(queued)
            if commit:
                s.mask, s.loc, s.resolved = queued, loc, True
        return out

    def _queued(self) -> list:
        return self._test_pending() if self._deferred() else [s.ok for s in self.slots]

    def _last_pending(self, kind: int, mask, ball) -> tuple:
        """Actions._get_pending_actions for one kind in every world of mask: (found [W], the last such call's slot
        index [W], -1 for none)."""
        mask = torch.as_tensor(mask).to(device=self.dev, dtype=BOOL)
        ball = torch.as_tensor(ball).to(device=self.dev, dtype=I64)
        found = torch.zeros(self.W, dtype=BOOL, device=self.dev)
        at = torch.full((self.W,), -1, dtype=I64, device=self.dev)
        for j, (s, queued) in enumerate(zip(self.slots, self._queued())):
            if s.kind == kind:
                hit = mask & queued & (s.ball == ball)
                found = found | hit
                at = torch.where(hit, j, at)
        return found, at

    def _pending_value(self, at: torch.Tensor, attr: str, col: int | None = None) -> torch.Tensor:
        if not self.slots:
            return torch.zeros(self.W, dtype=F64 if col is not None else I64, device=self.dev)
        vals = torch.stack([getattr(s, attr) if col is None else getattr(s, attr)[:, col] for s in self.slots])
        return vals.gather(0, at.clamp(min=0)[None, :])[0]

    def _pending_else_current(self, kind: int, mask, ball, attr: str, col, current: torch.Tensor) -> tuple:
        """The last pending call's argument as pushed, else the ball's current value, else nothing: (value, known)."""
        found, at = self._last_pending(kind, mask, ball)
        row = self.a.lookup(torch.as_tensor(ball).to(device=self.dev, dtype=I64))
        pending = self._pending_value(at, attr, col)
        now = current[row.clamp(min=0)].to(pending.dtype)
        value = torch.where(found, pending, torch.where(row >= 0, now, torch.zeros_like(pending)))
        known = torch.as_tensor(mask).to(device=self.dev, dtype=BOOL) & (found | (row >= 0))
        return value, known

    def has_pending_cloak(self, mask, ball) -> torch.Tensor:
        """Actions.has_pending_cloak, every world of mask: [W] bool."""
        return self._last_pending(CLOAK, mask, ball)[0]

    def has_pending_uncloak(self, mask, ball) -> torch.Tensor:
        """Actions.has_pending_uncloak, every world of mask: [W] bool."""
        return self._last_pending(UNCLOAK, mask, ball)[0]

    def get_pending_cloak_mode(self, mask, ball) -> tuple:
        """Actions.get_pending_cloak_mode: the last pending CloakBall's mode as pushed, else the ball's cloak byte, else
        None: (value [W] int64, known [W] bool)."""
        return self._pending_else_current(CLOAK, mask, ball, "n", None, self.a.cloaked)

    def get_pending_interactive_state(self, mask, ball) -> tuple:
        """Actions.get_pending_interactive_state: the last pending SetBallInteractive's flag, else the ball's, else
        None: (value [W] bool, known [W] bool)."""
        value, known = self._pending_else_current(INTERACTIVE, mask, ball, "n", None, self.a.interactive.to(I64))
        return value != 0, known

    def get_pending_speed_fraction(self, mask, ball) -> tuple:
        """Actions.get_pending_speed_fraction: the last pending SetSpeedFraction's value as pushed, else the ball's
        speed fraction, else None: (value [W] float64, known [W] bool)."""
        return self._pending_else_current(CODE["SetSpeedFraction"], mask, ball, "f", 0, self.a.park.speed_fraction)

    def _pending_free(self, mask, ball, value: int) -> tuple:
        found, at = self._last_pending(CODE["SetBallFree"], mask, ball)
        return found & (self._pending_value(at, "n") == value), found

    def has_pending_set_free(self, mask, ball) -> tuple:
        """Actions.has_pending_set_free: whether the last pending SetBallFree's flag is 1: (answer, pending) [W]; where
        nothing is pending Destiny answers the int 0 (`pending` False)."""
        return self._pending_free(mask, ball, 1)

    def has_pending_set_not_free(self, mask, ball) -> tuple:
        """Actions.has_pending_set_not_free: whether the last pending SetBallFree's flag is 0: (answer, pending)."""
        return self._pending_free(mask, ball, 0)

    def undo_pending_cloak(self, mask, ball) -> None:
        """Actions.undo_pending_cloak, every world of mask: every pending CloakBall of the ball taken out of the
        world's queue; the calls pushed later are tested against the queue's last call as it then stands."""
        mask = torch.as_tensor(mask).to(device=self.dev, dtype=BOOL)
        ball = torch.as_tensor(ball).to(device=self.dev, dtype=I64)
        deferred = self._deferred()
        if deferred:
            self._test_pending(commit=True)
        for s in self.slots:
            if s.kind != CLOAK:
                continue
            out = mask & (s.ball == ball)
            if deferred:
                s.mask = s.mask & ~out
            else:
                s.ok = s.ok & ~out
        if not deferred:                                  # the torch path's queue: its last call again
            last = self._zero_last()
            for s in self.slots:
                self._become_last(last, s, s.ok, s.loc)
            self.last = last

    def _rows(self, slot: Slot) -> tuple:
        """The call as per-row masks and arguments: a row is commanded iff its world's call is queued for it."""
        A = self.a
        w = A.world
        m = slot.ok[w] & (slot.row[w] == A.arange)
        return m, slot.trow[w], slot.f[w], slot.n[w]

    # ---- OnTick's per-world mask: the queue split, the last call, a world's first pre-tick ----
    def _split_queue(self, on: torch.Tensor, flag: str) -> list:
        """The queue split by the worlds that tick (`on` [W]): each call's flag (`ok` on the torch path, the pushed
        `mask` on the kernel path) restricted to them for this pre-tick; the calls still held by a world without a
        tick kept, in queue order, with the flag of those worlds (the calls no world holds dropped)."""
        slots, self.slots = self.slots, []
        if not slots:
            return []

        def restricted(s, keep):
            t = copy.copy(s)
            setattr(t, flag, getattr(s, flag) & keep)
            return t
        kept = [restricted(s, ~on) for s in slots]
        held = torch.stack([getattr(s, flag) for s in kept]).any(dim=1).tolist()
        self.slots = [s for s, h in zip(kept, held) if h]
        return [restricted(s, on) for s in slots]

    def _keep_last(self, on: torch.Tensor) -> None:
        """The duplicate test's last call after a masked pre-tick: none for the worlds that ticked, kept for the rest."""
        zero = self._zero_last()
        self.last = {k: torch.where(on.reshape(self.W, *([1] * (v.dim() - 1))), zero[k], v)
                     for k, v in self.last.items()}

    def _first_pre_tick(self, on: torch.Tensor) -> bool:
        """Whether a world in `on` has its first pre-tick now (its additions' fields are then recorded); every world
        seen once, the layer's first pre-tick is over."""
        seen = getattr(self, "_seen_w", None)
        if seen is None:
            seen = torch.full((self.W,), bool(self._seen_first), dtype=BOOL, device=self.dev)
        first, every = torch.stack(((on & ~seen).any(), (seen | on).all())).tolist()
        self._seen_w = seen | on
        self._seen_first = bool(every)
        return bool(first)

    def _snapshot(self, kinds, snapshot, on=None) -> bool:
        first = (not self._seen_first) if on is None else self._first_pre_tick(on)
        if on is None:
            self._seen_first = True
            if getattr(self, "_seen_w", None) is not None:
                self._seen_w = torch.ones_like(self._seen_w)
        if snapshot is None:
            snapshot = (UNCLOAK in kinds) or (INTERACTIVE in kinds) or (TROLL in kinds) or first
        return snapshot

    def _mask(self, mask):
        return None if mask is None else torch.as_tensor(mask).to(device=self.dev, dtype=BOOL).reshape(self.W)

    # ---- the tick ----
    def pre_tick(self, snapshot: bool | None = None, mask=None) -> None:
        """The Ticker's tick (TIME-712): the stamp moves, the queue is flushed and applied (CloakBall after the bubble
        update), the events routed. `snapshot`: record the park's fields where the streams would be written (by
        default when an uncloak, a SetBallInteractive, a SetBallTroll or a world's first pre-tick can send one).
        `mask` [W] (OnTick's): the worlds that tick; every other world keeps its queue, its stamp, its last call and
        its bubble update's lists, and routes nothing (`Batch.ticked`)."""
        on = self._mask(mask)
        if self.kernel == "cuda":
            return self._pre_tick_kernel(snapshot, on)
        A = self.a
        clock = A.clock().clone()
        stamp = self.stamp_for_system
        if on is None:
            self.stamp_for_system = clock + 1
            slots, self.slots = self.slots, []
            self._reset_last()
        else:
            self.stamp_for_system = torch.where(on, clock + 1, stamp)
            slots = self._split_queue(on, "ok")
            self._keep_last(on)
        snapshot = self._snapshot({s.kind for s in slots}, snapshot, on)
        for s in slots:                                     # every queued call but CloakBall, in queue order
            if s.kind != CLOAK:
                A.apply(s.kind, *self._rows(s))
        # BubbleUpdater: the additions once per park time (a second pre-tick at the same time reuses the lists)
        user = A.interactive & A.exists
        fresh = user & ~self.settled
        listed = A.exists & (A.cloaked == 0)
        fresh = fresh & A.any_in_world(listed)[A.world]
        again = (clock == self._bubble_time)[A.world]
        if on is not None:                                  # a world without a tick keeps its lists
            again = again | ~on[A.world]
        fresh = torch.where(again, self._fresh, fresh)
        listed = torch.where(again, self._listed, listed)
        self.settled = torch.where(again, self.settled, self.settled | user)
        self._bubble_time = clock if on is None else torch.where(on, clock, self._bubble_time)
        self._fresh, self._listed = fresh, listed
        additions = (fresh if on is None else fresh & on[A.world], listed, A.stream_fields() if snapshot else None)
        live = A.any_in_world(A.interactive & A.exists)
        route = torch.zeros(self.W, len(slots), dtype=torch.int8, device=self.dev)
        notices = []
        for j, s in enumerate(slots):                       # the history
            valid = s.ok & (s.row >= 0)
            safe = s.row.clamp(min=0)
            if s.kind == CLOAK:                             # to the bubble it was queued in; then applied
                r = torch.where(s.ok & (s.loc == 0), BUBBLE, NONE)
                m, _, f, n = self._rows(s)
                A.cloak(m, n, f[:, 0])
            elif s.kind == UNCLOAK:                         # to its own character; AddBallsToPark to the others
                own = valid & A.interactive[safe] & (self.pilot[safe] >= 0) & live
                r = torch.where(own, CHARACTER, NONE)
                rec = ((valid & live)[A.world] & A.interactive & A.exists & (A.arange != s.row[A.world])
                       & (self.pilot >= 0))
                notices.append((j, rec, A.stream_fields() if snapshot else None))
            elif s.kind == SETPOS:                          # a local ball's move is sent nowhere
                go = valid & (s.loc == 0) & live
                r = torch.where(go, torch.where(A.cloaked[safe] == 0, BUBBLE,
                                                torch.where(self.pilot[safe] >= 0, CHARACTER, NONE)), NONE)
            else:
                go = valid & live & (s.ball > 0)
                r = torch.where(go, torch.where(A.cloaked[safe] == 0, BUBBLE,
                                                torch.where(self.pilot[safe] >= 0, CHARACTER, NONE)), NONE)
            route[:, j] = r.to(torch.int8)
        self.batch = Batch(stamp=stamp, clock=clock, slots=slots, route=route, notices=notices, additions=additions,
                           ticked=on)

    def _pre_tick_kernel(self, snapshot, on=None) -> None:
        """The pre-tick as the kernel: one launch, or, with the park's fields recorded, the queue and bubble update,
        then the history split at each UncloakBall (the fields its notices send are read there). With OnTick's mask
        the worlds without a tick have no pushed call in the launch (no park write) and get their stamp and bubble
        update's state back after it."""
        A = self.a
        if on is None:
            slots, self.slots = self.slots, []
        else:                                               # tested first (as the kernel tests them), so that a
            self._test_pending(commit=True)                 # world without a tick keeps its queued calls alone
            slots = self._split_queue(on, "mask")
            saved = [t.clone() for t in (self.stamp_for_system, self._bubble_time, self.settled, self._fresh,
                                         self._listed)]
        kinds = [s.kind for s in slots]
        J = len(slots)
        snapshot = self._snapshot(set(kinds), snapshot, on)
        cols = None
        if J:
            cols = {"mask": torch.stack([s.mask.to(torch.uint8) | (2 if getattr(s, "resolved", False) else 0)
                                         for s in slots]),
                    "ball": torch.stack([s.ball for s in slots]),
                    "target": torch.stack([s.target for s in slots]), "f": torch.stack([s.f for s in slots]),
                    "n": torch.stack([s.n for s in slots]), "loc_in": torch.stack([s.loc for s in slots])}
        q = self._queue(kinds, cols)
        notices, fields = [], None
        if not snapshot:
            self._launch(q, 0)
            notices = [(j, q["notice"][j], None) for j, k in enumerate(kinds) if k == UNCLOAK]
        else:
            self._launch(q, 1)
            fields = A.stream_fields()
            j0 = 0
            for j in [j for j, k in enumerate(kinds) if k == UNCLOAK]:
                self._launch(q, 2, j0, j)
                notices.append((j, q["notice"][j], A.stream_fields()))
                j0 = j
            self._launch(q, 2, j0, J)
        if on is not None:                                  # the worlds without a tick as they were
            ron = on[A.world]
            for cur, old, sel in zip((self.stamp_for_system, self._bubble_time, self.settled, self._fresh,
                                      self._listed), saved, (on, on, ron, ron, ron)):
                cur.copy_(torch.where(sel, cur, old))
        self._finish(q, slots, notices, fields, on=on)

    def _finish(self, q: dict, slots: list, notices: list, fields, live: bool = False, on=None) -> None:
        """The Batch over the queue's tensors; the additions copied (an eager tick) or the live lists (a graph's)."""
        for j, s in enumerate(slots):                       # the slots as the torch path holds them
            s.ok, s.row, s.trow, s.loc = q["ok"][j], q["row"][j], q["trow"][j], q["loc"][j]
        self._q = q
        lists = (self._fresh, self._listed) if live else (self._fresh.clone(), self._listed.clone())
        if on is not None:
            lists = (lists[0] & on[self.a.world], lists[1])
        self.batch = Batch(stamp=q["stamp"], clock=q["clock"], slots=slots, route=q["route"], notices=notices,
                           additions=(*lists, fields),
                           gets_bubble=q["gets_bubble"], has_character=q["has_character"], ticked=on)

    def evolve(self, mask=None) -> None:
        """The park's tick; a world whose bubble is dead is recorded (refused by `check`). `mask` [W] (OnTick's):
        those worlds alone, every other world's balls and clock kept bit for bit."""
        A = self.a
        on = self._mask(mask)
        if on is not None:
            self.dead = self.dead | (on & ~A.any_in_world(A.interactive & A.exists))
            A.evolve(on)
            return
        if self.kernel == "cuda":
            self._launch(self._q if self._q is not None else self._queue([]), 4)
        else:
            self.dead = self.dead | ~A.any_in_world(A.interactive & A.exists)
        A.evolve()

    def post_tick(self, mask=None) -> None:
        """send_batch: per row (its pilot), whether it gets the bubble's narrowcast and a character update. `mask` [W]
        (OnTick's; by default the pre-tick's, `Batch.ticked`): the worlds that ticked; the others send nothing."""
        on = self._mask(mask)
        if on is None and self.batch is not None:
            on = self.batch.ticked
        A = self.a
        if self.kernel == "cuda":                           # the flags' phase, in place in the batch
            self._launch(self._q, 3)
            if on is not None:
                ron = on[A.world]
                self._q["has_character"].logical_and_(ron)
                self._q["gets_bubble"].logical_and_(ron)
            return
        b = self.batch
        bubble = ((b.route == BUBBLE).any(dim=1) if b.route.shape[1]
                  else torch.zeros(self.W, dtype=BOOL, device=self.dev))
        has = torch.zeros(self.R, dtype=BOOL, device=self.dev)
        for j, s in enumerate(b.slots):
            has = has | (s.ok[A.world] & (s.row[A.world] == A.arange) & (b.route[:, j] == CHARACTER)[A.world])
        for _, rec, _ in b.notices:
            has = has | rec
        has = has | b.additions[0]
        pilot = self.pilot >= 0
        if on is not None:
            pilot = pilot & on[A.world]
        b.has_character = has & pilot
        b.gets_bubble = bubble[A.world] & A.interactive & A.exists & pilot

    def on_tick(self, sim_time) -> list:
        """Ballpark::OnTick on the master for every world, each at its own simulation time (sim_time [W], 100 ns
        units; Ballpark.cpp:219-330, TIME-702 to TIME-705), with the Ticker's tick at DoPreTick and send_batch at
        DoPostTick: less than a whole interval since the world's time, nothing (its time and queue kept); on the master
        a backlog of more than five intervals cut to one; a world's first call evolves once without the tick's events
        (its queue kept); every other world runs its whole intervals, each a pre-tick, the park's tick and a
        post-tick, the worlds with an interval left ticking together under a mask (a round of every world unmasked),
        the remainder carried in its time. `time` [W] and `first_time` [W] are made at the first call. Returns the
        batches of the rounds run, in order (a world's sends are in those whose `ticked` holds it); `tick_counts` holds
        the call's counts."""
        A, W, d = self.a, self.W, self.dev
        if getattr(self, "time", None) is None:
            self.time = torch.zeros(W, dtype=I64, device=d)
            self.first_time = torch.ones(W, dtype=BOOL, device=d)
        sim = torch.as_tensor(sim_time, dtype=I64).to(d).reshape(W)
        interval = int(round(A.park.dt * 1000.0)) * 10000
        since = sim - self.time
        go = ~(since < interval)
        n = torch.where(go, torch.div(since, interval, rounding_mode="floor"), 0)
        resync = go & (n > MAX_CATCH_UP_TICKS) & bool(A.master)
        since = torch.where(resync, interval, since)
        n = torch.where(resync, 1, n)
        first = go & self.first_time
        rest = go & ~first
        runs = torch.where(rest, n, 0)
        counts = torch.stack(((~go).sum(), first.sum(), first.all().to(I64), resync.sum(), runs.sum(),
                              (rest & (since - n * interval > 0)).sum(), runs.max() if W else runs.sum())).tolist()
        self.tick_counts = {"worlds too early": counts[0], "first calls": counts[1], "resynchronisations": counts[3],
                            "intervals run": counts[4], "remainders carried": counts[5]}
        if counts[1]:
            self.evolve(mask=None if counts[2] else first)
        self.first_time = self.first_time & ~first
        batches = []
        for k in range(counts[6]):
            m = rest & (n > k)
            mm = None if bool(m.all()) else m
            self.pre_tick(mask=mm)
            self.evolve(mask=mm)
            self.post_tick(mask=mm)
            self.batch.ticked = m
            batches.append(self.batch)
        self.time = torch.where(go, sim - torch.where(rest, since - n * interval, 0), self.time)
        return batches

    def tick(self) -> None:
        self.pre_tick()
        self.evolve()
        self.post_tick()

    def check(self) -> None:
        if bool(self.dead.any()):
            bad = torch.nonzero(self.dead).flatten().tolist()
            raise RuntimeError(f"worlds {bad[:8]} had no interactive ball at an evolve: on the master their balls "
                               "would not be evolved (TIME-714), which the batched park does not model")


class ServerGraph:
    """A kernel-path VecServer's tick with a fixed schedule of pushes, captured once as a CUDA graph (the drop-in for
    exact_ballpark.vec_server.ServerGraph, vec_server.py:1200): before each replay the caller writes each push's
    arguments into `inputs[j]` (mask, ball, target, f, n, loc: views of the queue's [J, W] buffers) and `tick()`
    replays the pre-tick with the dead-bubble test (one launch), the park's tick and the send flags, and returns the graph's
    Batch (its tensors refilled in place; no park fields recorded). Every state tensor is written in place by its
    kernel, so nothing is re-bound between replays and eager setters between ticks are seen by the next replay."""

    def __init__(self, server: VecServer, schedule: list):
        if server.kernel != "cuda":
            raise ValueError("a ServerGraph captures the kernel path (VecServer(..., kernel='cuda'))")
        if server.slots:
            raise ValueError("pushes are queued: tick them eagerly first")
        self.server = srv = server
        self.schedule = [CODE[k] if isinstance(k, str) else int(k) for k in schedule]
        for k in self.schedule:
            if k not in srv.a.kinds:
                raise ValueError(f"{KINDS[k]} is not applied by this park")
        p, d = srv.a.park, srv.dev
        self.q = q = srv._queue(self.schedule)
        self.inputs = [{"mask": q["mask"][j].view(BOOL), "ball": q["ball"][j], "target": q["target"][j], "f": q["f"][j],
                        "n": q["n"][j], "loc": q["loc_in"][j]} for j in range(len(self.schedule))]
        if p.plan is None:
            p.scratch()
        else:
            p.plan.tile_rows_on(d)
        keep = [(t, t.clone()) for t in self._state_tensors()]
        side = torch.cuda.Stream(device=d)                 # a warm-up of every launch, undone
        side.wait_stream(torch.cuda.current_stream(d))
        with torch.cuda.stream(side):
            self._body()
        torch.cuda.current_stream(d).wait_stream(side)
        torch.cuda.synchronize(d)
        for t, v in keep:
            t.copy_(v)
        del keep
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._body()
        srv._seen_first = True
        slots = [Slot(k, None, q["ball"][j], None, q["target"][j], None, q["f"][j], q["n"][j], q["loc_in"][j])
                 for j, k in enumerate(self.schedule)]
        notices = [(j, q["notice"][j], None) for j, k in enumerate(self.schedule) if k == UNCLOAK]
        srv._finish(q, slots, notices, None, live=True)
        self.out = srv.batch

    def _state_tensors(self) -> list:
        srv, p = self.server, self.server.a.park
        return ([getattr(p, k) for k in p.row_tensors()] + [p.cloaked, p.bubble]
                + [srv.stamp_for_system, srv._bubble_time, srv.dead, srv.settled, srv._fresh, srv._listed]
                + [self.q[k] for k in ("ok", "row", "trow", "loc", "route", "notice", "stamp", "clock",
                                       "has_character", "gets_bubble")])

    def _body(self) -> None:
        srv, p = self.server, self.server.a.park
        srv._launch(self.q, 5)                             # the pre-tick and the dead-bubble test, one launch
        _park_tick(p, p.block)
        srv._launch(self.q, 3)

    def tick(self) -> Batch:
        if self.server.slots:
            raise RuntimeError("eager pushes before a graph tick: the graph's tick pushes its own schedule")
        self.graph.replay()
        self.server.a.park.current_time += 1
        self.server.batch = self.out
        return self.out


# ================================================================================ what each client holds

class ClientView:
    """What each pilot's client holds after each tick (vec_server.py:1292-1340): the server's state `down` ticks back (a
    client applies each update at its stamp, so its park settles `down` ticks behind the server's), kept as a ring of
    the last `down` + 1 recorded states of the observed fields; another pilot's cloaked ship is absent from a client's
    park (its CloakBall removed it there), the client's own ship is present, and a client's park holds its own world
    only. `record(time)` after each server tick; `view()` the state each client holds and its park time."""

    def __init__(self, server: VecServer, down: int, fields: tuple = ("pos", "vel", "mode")):
        if down < 0:
            raise ValueError("down: whole ticks, at least 0")
        self.server, self.down, self.fields = server, int(down), tuple(fields)
        self.depth = self.down + 1
        self.ring: dict = {}
        self.times = torch.full((self.depth,), -1, dtype=I64)
        self.k = 0

    def _field(self, name: str) -> torch.Tensor:
        a = self.server.a
        if name == "cloaked":
            return a.cloaked
        t = getattr(a.park, name)
        return t.reshape(a.R, *t.shape[2:]) if isinstance(a, CollideAdapter) else t

    def record(self, time: int) -> None:
        """Keep the server's state at park time `time` (the time the park has reached)."""
        slot = self.k % self.depth
        for name in self.fields + ("cloaked",):
            t = self._field(name)
            if name not in self.ring:
                self.ring[name] = torch.zeros((self.depth, *t.shape), dtype=t.dtype, device=t.device)
            self.ring[name][slot].copy_(t)
        self.times[slot] = int(time)
        self.k += 1

    def view(self) -> tuple:
        """(time, {field: [R, ...]}, present [R, R]: row r is in the park of the pilot whose ship is row c), the state
        `down` ticks before the latest recorded one; time -1 (and nothing) until that state was recorded."""
        if self.k <= self.down:
            return -1, {}, None
        slot = (self.k - 1 - self.down) % self.depth
        out = {name: self.ring[name][slot] for name in self.fields}
        cloaked = self.ring["cloaked"][slot]
        a = self.server.a
        own_world = a.world[:, None] == a.world[None, :]
        mine = torch.eye(a.R, dtype=BOOL, device=cloaked.device)
        return int(self.times[slot]), out, own_world & ((cloaked == 0)[:, None] | mine)


# ================================================================================ the batches as Destiny sends them

class ClientUpdateCountThisTick(IntEnum):
    """How many DoDestinyUpdate calls a client gets this tick (net/const.py:6-8)."""
    ONE = 1
    TWO = 2


class Marshalled:
    """A marshalled payload (blue.marshal.Save) kept as the value it encodes: equal when the values are equal."""
    __slots__ = ("value",)

    def __init__(self, value):
        self.value = copy.deepcopy(value)

    def __eq__(self, other):
        return isinstance(other, Marshalled) and self.value == other.value

    def __repr__(self):
        return f"Marshalled({self.value!r})"

    __hash__ = None


_XYZ_EVENTS = ("GotoPoint", "GotoDirection", "SetBallVelocity", "SetBallAngularVelocity", "SetMaxAngularVelocity",
               "SetBallPosition")
_ONE_FLOAT_EVENTS = ("SetSpeedFraction", "SetMaxSpeed", "SetBallMass", "SetBallAgility", "SetBallRadius",
                     "SetMaxAngularSpeed", "SetBallAngularAgility")
_MODE_TAIL = {0: "goto", 1: "follow", 3: "warp", 4: "follow", 5: "missile", 6: "mushroom", 8: "troll", 12: "formation"}


def _int32(v: int) -> int:
    v &= 0xFFFFFFFF
    return v - (1 << 32) if v >= (1 << 31) else v


def _pack_ball(fields: dict, r: int, out: list) -> None:
    """One ball as WriteBallToStream writes it (Thunkers.cpp:3180-3377), from a row of the park's fields: the head (id,
    mode, radius, position, the flags free, global, massive, interactive), the mass block (not for RIGID), the motion
    block of a free ball (with the orientation block under dynamical orientation), the formation id, then the mode's
    own tail."""
    mode = int(fields["mode"][r]) & 0xFF
    is_global = bool(fields["global"][r]) if "global" in fields else False
    flags = (int(bool(fields["free"][r])) | (2 if is_global else 0) | (4 if bool(fields["massive"][r]) else 0)
             | (8 if bool(fields["interactive"][r]) else 0))
    out.append(struct.pack("<qBf3dB", int(fields["ids"][r]), mode, float(fields["radius"][r]),
                           *(float(x) for x in fields["pos"][r].tolist()), flags))
    if mode != 11:
        cloak = int(fields["cloaked"][r]) & 0xFF
        out.append(struct.pack("<dbqii", float(fields["mass"][r]), cloak - 256 if cloak >= 128 else cloak, -1, -1, -1))
    if flags & 1:
        out.append(struct.pack("<f3dff", float(fields["max_vel"][r]), *(float(x) for x in fields["vel"][r].tolist()),
                               float(fields["agility"][r]), float(fields["speed_fraction"][r])))
        if fields["dynamical"]:
            out.append(struct.pack("<4ff3ff", *(float(x) for x in fields["rot"][r].tolist()),
                                   float(fields["max_ang_vel"][r]), *(float(x) for x in fields["ang_vel"][r].tolist()),
                                   float(fields["rot_agility"][r])))
    formation = int(fields["formation_id"][r]) if "formation_id" in fields else -1
    out.append(struct.pack("<b", ((formation + 128) & 0xFF) - 128))
    stamp = _int32(int(fields["effect_stamp"][r]))
    goto = [float(x) for x in fields["goto"][r].tolist()]
    tail = _MODE_TAIL.get(mode)
    if tail == "follow":
        out.append(struct.pack("<qf", int(fields["follow_id"][r]), float(fields["follow_range"][r])))
    elif tail == "goto":
        out.append(struct.pack("<3d", *goto))
    elif tail == "warp":
        out.append(struct.pack("<3didqq", *goto, stamp, float(fields["last_collision"][r]),
                               int(fields["follow_id"][r]), int(fields["owner_id"][r])))
    elif tail == "missile":
        out.append(struct.pack("<qfqi3d", int(fields["follow_id"][r]), float(fields["follow_range"][r]),
                               int(fields["owner_id"][r]), stamp, *goto))
    elif tail == "formation":
        out.append(struct.pack("<qfi", int(fields["follow_id"][r]), float(fields["follow_range"][r]), stamp))
    elif tail == "mushroom":
        out.append(struct.pack("<fdiq", float(fields["follow_range"][r]), goto[0], stamp, int(fields["owner_id"][r])))
    elif tail == "troll":
        out.append(struct.pack("<i", stamp))


def ball_stream(fields: dict, rows: list, time: int) -> bytes:
    """WriteBallsToStream (Thunkers.cpp:2202-2257): the DESTINY_BALLS tag, the time as an int32, then each ball."""
    out = [struct.pack("<Bi", 1, _int32(int(time)))]
    for r in rows:
        _pack_ball(fields, r, out)
    return b"".join(out)


def event_of(slot: Slot, w: int) -> tuple:
    """The event (name, args) Destiny queued for world w's call in this slot, local arguments dropped: floats for the
    float arguments, ints for ids and the int arguments."""
    name = KINDS[slot.kind]
    ball, f, n = int(slot.ball[w]), [float(x) for x in slot.f[w].tolist()], int(slot.n[w])
    if name in _XYZ_EVENTS:
        return name, (ball, f[0], f[1], f[2])
    if name in _ONE_FLOAT_EVENTS:
        return name, (ball, f[0])
    if name in ("Stop", "UncloakBall"):
        return name, (ball,)
    if name in ("FollowBall", "Orbit"):
        return name, (ball, int(slot.target[w]), f[0])
    if name == "WarpTo":
        return name, (ball, f[0], f[1], f[2], f[3], n)
    if name == "EntityWarpIn":
        return name, (ball, f[0], f[1], f[2], n)
    if name in ("SetBallMassive", "SetBallInteractive", "SetBallTroll", "SetBallFree"):
        return name, (ball, n)
    if name == "CloakBall":
        return name, (ball, n, f[0])
    if name == "SetBallRotation":
        return name, (ball, f[0], f[1], f[2], f[3])
    if name == "LaunchMissile":
        return name, (ball, int(slot.target[w]), n, int(f[0]), int(f[1]))
    raise ValueError(f"no event for {name}")


def decode(server: VecServer, batch: Batch | None = None, client_base: int = 10000) -> list:
    """The batch as Destiny's network sends it, per world: {client id: [(kind, method, state, wait_for_bubble,
    count)]} in the order the client receives them (its singlecast, then the bubble's narrowcast). A client is
    client_base + its pilot. The singlecast's state is, in order, the uncloaks' AddBallsToPark (the latest first), the
    bubble's additions as a PackagedAction and the events routed to the client's character; the narrowcast's the
    events routed to the bubble, each as (stamp, (name, args)). Host work only; the streams need the park's fields
    recorded at the pre-tick (`snapshot`)."""
    A, b = server.a, batch if batch is not None else server.batch
    pilot = server.pilot.tolist()
    rows_of = [[r for r in rw if r >= 0] for rw in A.rows_of_world.tolist()]
    route = b.route.cpu().tolist()
    stamp, clock = b.stamp.tolist(), b.clock.tolist()
    queued = [s.ok.tolist() for s in b.slots]
    has, gets = b.has_character.tolist(), b.gets_bubble.tolist()
    fresh, listed, add_fields = b.additions
    fresh, listed = fresh.tolist(), listed.tolist()
    notices = [(j, rec.tolist(), fl) for j, rec, fl in b.notices]
    out = []
    for w in range(A.W):
        to_bubble, to_character = [], {}
        for j, s in enumerate(b.slots):
            if not queued[j][w]:
                continue
            if route[w][j] == BUBBLE:
                to_bubble.append((stamp[w], event_of(s, w)))
            elif route[w][j] == CHARACTER:
                to_character.setdefault(pilot[int(s.row[w])], []).append((stamp[w], event_of(s, w)))
        uncloaks = {}
        for j, rec, fl in notices:                         # each uncloak's AddBallsToPark, the latest in front
            row = int(b.slots[j].row[w])
            if not queued[j][w] or row < 0 or not any(rec[r] for r in rows_of[w]):
                continue
            if fl is None:
                raise ValueError("this tick ran without the park's fields recorded: its uncloaks' streams are missing")
            payload = ("AddBallsToPark", (ball_stream(fl, [row], clock[w]),))
            for r in rows_of[w]:
                if rec[r]:
                    uncloaks.setdefault(pilot[r], []).insert(0, (stamp[w], payload))
        additions = {}
        listing = [r for r in rows_of[w] if listed[r]]
        for r in rows_of[w]:
            if fresh[r] and pilot[r] >= 0 and listing:
                if add_fields is None:
                    raise ValueError("this tick ran without the park's fields recorded: its additions are missing")
                package = Marshalled([(clock[w], ("AddBallsToPark", (ball_stream(add_fields, listing, clock[w]),)))])
                additions[pilot[r]] = [(clock[w], ("PackagedAction", package))]
        per = {}
        for r in rows_of[w]:
            p = pilot[r]
            if p < 0:
                continue
            sends = []
            if has[r]:
                state = uncloaks.get(p, []) + additions.get(p, []) + to_character.get(p, [])
                sends.append(("single", "DoDestinyUpdate", state, bool(gets[r]),
                              ClientUpdateCountThisTick.TWO if gets[r] else ClientUpdateCountThisTick.ONE))
            if gets[r]:
                sends.append(("narrow", "DoDestinyUpdate", to_bubble, False,
                              ClientUpdateCountThisTick.TWO if has[r] else ClientUpdateCountThisTick.ONE))
            if sends:
                per[client_base + p] = sends
        out.append(per)
    return out
