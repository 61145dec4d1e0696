"""The master's partition and bubble partition over the flight park, on the device: the drop-in for the reference's
`exact_ballpark.vec_space.VecSpace` layer (vec_space.py:777) over `VecModesPark`, in this build's slice: each ball's
filing (the level of its inflated radius, the key of its box, the sides its sphere reaches), the partition's boxes
(made with their parents, released when empty, BoxAllocator's kept count, the reads of a released box), the top boxes'
bubbles (a neighbour's or a new id), the bubble dictionaries (+1, 0, -1 in insertion order), the interactive and
keep-alive sets, InitializeBubbles, CopyBubbles, the dead-bubble rows the park's tick skips (TIME-714) and the tick's
re-filings (a warp's drop-out nearly at rest, at its drop-out point; every ball that moved at least sqrt(0.1) m, in
ascending id), as the reference's `SpaceBallpark` on the master runs them (space.py:596-1319).

Beside the filing: the proximity sensors, notification ranges and target tracking with their events,
HandleProximities, and the queries (CheckVisibility, GetBallIdsInRange, GetBubbleAtCoordinates, GetNearbyBalls).

The layer is one sequential program a world, one CUDA thread or one warp a world (csrc/ebb_space.cuh): an operation
is a tape, per world K operations applied in order, one launch for all worlds (`tape`, `ops`, `broadcast`), with the
reference's operation names (`OP`). Its state is tensors indexed [entry, world]: stored interleaved (a warp's 32
worlds read consecutive words; a thread a world) or world-major (a world's entries consecutive, every world `pitch`
bytes apart in one arena; the form for a warp a world, whose lanes then read a world's slots together). A world that
leaves the layer's domain (a table full, the grid's edge, an operation outside this slice) is flagged and left alone;
`check()` raises for it. Not in this slice: the collision park's view and the delayed removal.
"""

from __future__ import annotations

import ctypes
import math

import torch

from . import _native
from .modes import VecModesPark, WARP

I64, U8, BOOL = torch.int64, torch.uint8, torch.bool

OPS = ("NONE", "ADD", "REFILE", "INIT_BUBBLES", "COPY_BUBBLES", "KEEP_ALIVE", "SET_INTERACTIVE", "ADD_SENSOR",
       "REMOVE_SENSOR", "NOTIFY_RANGE", "TRACK", "REMOVE_BALL", "DEAD", "AFTER_EVOLVE", "CLEAR_EVENTS")
OP = {name: k for k, name in enumerate(OPS)}
OP.update(HANDLE_PROXIMITIES=18, SET_CLOAKED=19)            # this build's own (no number in the reference's OPS)
EVENTS = ("", "DoProximity", "DoRange", "DoTargetTracking")
QUERIES = ("NONE", "VISIBILITY", "RANGE_BALL", "RANGE_POINT", "BUBBLE_AT", "NEARBY")
Q = {name: k for k, name in enumerate(QUERIES)}
FLAGS = ("EVENTS", "TOPS", "EDGE", "BOXES", "DICTS", "ENTRIES", "PROXIMITY", "SENSOR_LIST", "HUGE", "BAD_OP", "SETS",
         "UNDEFINED")
FLAG = {name: 1 << k for k, name in enumerate(FLAGS)}
BLOCK = 128


def state_spec(N: int, B: int, D: int, E: int, S: int, U: int, M: int) -> list:
    """The layer's arrays a world (include/ebb.h's EbbSpaceState, `rnd` aside): (name, shape, dtype, initial value)
    for N slots, B box-table entries, D dictionaries, E entries, S set members, U keys a map and M events."""
    F64, I32 = torch.float64, torch.int32
    return [("rows", (N,), I64, 0), ("level", (N,), I64, -1), ("key", (3, N), I64, 0), ("mod", (3, N), I64, -2),
            ("active", (N,), I64, 0), ("bubble", (N,), I64, -1), ("old_bubble", (N,), I64, -1),
            ("seq", (N,), I64, 0), ("my_box", (N,), I64, -1), ("my_top", (N,), I64, -1),
            ("in_park", (N,), U8, 0), ("keep_alive", (N,), U8, 0), ("dead", (N,), U8, 0),
            ("dropped", (N,), U8, 0), ("box_level", (B,), I64, -1), ("box_key", (3, B), I64, 0),
            ("box_balls", (B,), I64, 0), ("box_kids", (B,), I64, 0), ("box_bubble", (B,), I64, -1),
            ("stack", (B,), I64, 0), ("box_n", (), I64, 0), ("free_boxes", (), I64, 0),
            ("box_hash", (2 * B,), I64, 0), ("box_free", (B,), I64, 0), ("box_free_n", (), I64, 0),
            ("dict_bubble", (D,), I64, 0), ("dict_n", (), I64, 0), ("entry_bubble", (E,), I64, 0),
            ("entry_id", (E,), I64, 0), ("entry_value", (E,), I64, 0), ("entry_n", (), I64, 0),
            ("inter_bubble", (S,), I64, 0), ("inter_id", (S,), I64, 0), ("inter_n", (), I64, 0),
            ("keep_bubble", (S,), I64, 0), ("keep_id", (S,), I64, 0), ("keep_n", (), I64, 0),
            ("bubble_id", (), I64, 0), ("seq_next", (), I64, 0), ("flags", (), I64, 0),
            ("srange", (N,), F64, 0), ("speriod", (N,), F64, 2.0), ("selapsed", (N,), F64, 0),
            ("ntf_range", (N,), F64, 0), ("trk_range", (N,), F64, 0), ("trk", (N,), I64, -1),
            ("cloaked", (N,), I64, 0), ("sonly", (N,), U8, 0), ("has_prox", (N,), U8, 0),
            ("ntf_in", (N,), U8, 0), ("trk_in", (N,), U8, 0), ("slist", (U, N), U8, 0), ("slen", (N,), I32, 0),
            ("sbkt", (N,), I32, 1), ("pmap", (U,), U8, 0), ("pn", (), I32, 0), ("pbkt", (), I32, 1),
            ("ev", (max(M, 1),), I32, 0), ("evn", (), I64, 0), ("smask", (2, N), I64, 0),
            ("pmask", (2,), I64, 0), ("box_parent", (B,), I64, -1), ("box_top", (B,), I64, -1),
            ("box_home", (B,), I64, 0), ("box_slot", (B,), I64, 0), ("fbox", (8, N), I64, -1)]


# the box table's per-entry fields in a world-major arena: records of BOX_RECORD int64 words an entry (the word of
# each field; box_key takes three)
BOX_RECORD = 16
BOX_WORDS = {"box_level": 0, "box_key": 1, "box_balls": 4, "box_kids": 5, "box_bubble": 6, "box_parent": 7,
             "box_top": 8, "box_home": 9, "box_slot": 10}


def allocate_state(spec, W: int, dev, world_major: bool):
    """The layer's arrays, each a tensor [*shape, W] (its entries, then the world). Interleaved: each its own
    contiguous tensor. World-major: views into one arena [W][pitch bytes], each array at its own offset a world (16-byte
    aligned), the world's row of the arena holding its copy of every array, the box table's per-entry fields as
    records of BOX_RECORD words an entry (one 128-byte line). Returns (arrays, pitch; 0 interleaved)."""
    if not world_major:
        return {name: torch.full((*shape, W), fill, dtype=dt, device=dev) for name, shape, dt, fill in spec}, 0
    at, off, rec, boxes = [], 0, None, None
    for name, shape, dt, fill in spec:
        if name in BOX_WORDS:
            at.append(None)
            boxes = shape[-1]
            continue
        size = math.prod(shape) * torch.empty((), dtype=dt).element_size()
        at.append(off)
        off += (size + 15) // 16 * 16
    if boxes is not None:
        rec = (off + 127) // 128 * 128
        off = rec + boxes * BOX_RECORD * 8
    pitch = (off + 127) // 128 * 128
    arena = torch.zeros(W, pitch, dtype=U8, device=dev)
    words = arena.view(torch.int64)                        # [W, pitch / 8]
    out = {}
    for (name, shape, dt, fill), o in zip(spec, at):
        if o is None:                                      # a record field: its word of each entry's record
            first = rec // 8 + BOX_WORDS[name]
            if len(shape) == 1:
                t = words.as_strided((shape[0], W), (BOX_RECORD, pitch // 8), first)
            else:
                t = words.as_strided((shape[0], shape[1], W), (1, BOX_RECORD, pitch // 8), first)
        else:
            n = math.prod(shape)
            size = n * torch.empty((), dtype=dt).element_size()
            t = arena[:, o:o + size].view(dt).reshape(W, *shape).movedim(0, -1)
        if fill:
            t.fill_(fill)
        out[name] = t
    return out, pitch


class VecSpace:
    """The layer for W worlds of N slots over a flight park's rows. `rows` [W, N]: the park's row of each slot (-1 for
    none), each world's slots in the order its balls are added. Capacities a world: `boxes` box-table entries,
    `dicts` bubble dictionaries, `entries` dictionary entries, `sets` members of each of the interactive and keep-alive
    set families (defaults from N). `lanes`: 1 (a thread a world) or 32 (a warp a world); `world_major`: the
    state's arrangement (default: world-major for a warp a world, interleaved for a thread a world)."""

    def __init__(self, park: VecModesPark, rows, boxes: int | None = None, dicts: int | None = None,
                 entries: int | None = None, sets: int | None = None, block: int = BLOCK, events: int = 256,
                 umap_cap: int | None = None, seed=1, lanes: int = 1, world_major: bool | None = None):
        if not isinstance(park, VecModesPark):
            raise TypeError("the space layer runs over the flight park (exact_ballpark_b200.VecModesPark)")
        self.park, self.dev, self.block = park, park.dev, int(block)
        rows = torch.as_tensor(rows, dtype=I64)
        if rows.dim() != 2:
            raise ValueError("rows: [W, N]")
        self.W, self.N = int(rows.shape[0]), int(rows.shape[1])
        if not 1 <= self.N <= _native.SPACE_MAX_SLOTS:
            raise ValueError(f"{self.N} slots a world: from 1 to {_native.SPACE_MAX_SLOTS}")
        if bool(((rows < -1) | (rows >= park.n)).any()):
            raise ValueError("rows: a park row or -1 for each slot")
        N, W, d = self.N, self.W, self.dev
        self.B = int(boxes) if boxes is not None else 16 * N + 64
        self.D = int(dicts) if dicts is not None else 8 * N + 16
        self.E = int(entries) if entries is not None else 4 * N + 8
        self.S = int(sets) if sets is not None else 2 * N + 8
        self.M = int(events)
        self.U = N if umap_cap is None else int(umap_cap)
        if not 1 <= self.U <= _native.SPACE_MAX_SLOTS or self.M < 0:
            raise ValueError(f"umap_cap {self.U}: from 1 to {_native.SPACE_MAX_SLOTS}; events >= 0")
        if lanes not in (1, 32):
            raise ValueError("lanes: 1 (a thread a world) or 32 (a warp a world)")
        self.lanes = int(lanes)
        self.world_major = (self.lanes == 32) if world_major is None else bool(world_major)
        spec = state_spec(N, self.B, self.D, self.E, self.S, self.U, self.M)
        self.st, self.pitch = allocate_state(spec, W, d, self.world_major)
        self.st["rows"].copy_(rows.t())
        self.rows = self.st.pop("rows")                              # [N][W]
        self.st["rnd"] = torch.zeros(W, _native.RAND_WORDS, dtype=torch.int32, device=d)
        seeds = torch.as_tensor(seed, dtype=I64).reshape(-1)
        seeds = (seeds.expand(W) if seeds.numel() == 1 else seeds).contiguous().to(d)
        if seeds.numel() != W:
            raise ValueError(f"seed: an int or one a world ({W})")
        _native.check(_native.lib().ebb_glibc_srand(seeds.data_ptr(), W, self.st["rnd"].data_ptr(),
                                                     park._stream()), "ebb_glibc_srand")
        self._flat = torch.where(self.rows >= 0, self.rows, park.n).t().flatten()   # [W N] slot -> row, n for none
        self._state = None
        self.last_dead = None

    # ---- plumbing ----

    def state(self) -> _native.SpaceState:
        """include/ebb.h's EbbSpaceState over the layer's tensors."""
        if self._state is None:
            s = _native.SpaceState()
            s.worlds, s.slots, s.boxes, s.dicts, s.entries, s.sets = self.W, self.N, self.B, self.D, self.E, self.S
            s.umap_cap, s.events, s.lanes, s.pitch = self.U, self.M, self.lanes, self.pitch
            s.rows = self.rows.data_ptr()
            for name, t in self.st.items():
                setattr(s, name, t.data_ptr())
            self._state = s
        return self._state

    def tape(self, code, a=None, b=None, f=None) -> None:
        """Per world, K operations in order: code [W, K] (OP), a [W, K] (a slot), b [W, K] (an integer), f [W, K, 4]
        (floating-point arguments: ADD_SENSOR's range and period, NOTIFY_RANGE's range, TRACK's range and whether
        the target's id is 0)."""
        code = torch.as_tensor(code, dtype=I64).to(self.dev).reshape(self.W, -1)
        K = int(code.shape[1])
        if K == 0:
            return
        a = (torch.full_like(code, -1) if a is None else torch.as_tensor(a, dtype=I64).to(self.dev).reshape(self.W, K))
        b = (torch.zeros_like(code) if b is None else torch.as_tensor(b, dtype=I64).to(self.dev).reshape(self.W, K))
        code_t, a_t, b_t = (x.t().contiguous() for x in (code, a, b))    # [K][W]
        f_t = None
        if f is not None:
            f_t = torch.as_tensor(f, dtype=torch.float64).to(self.dev).reshape(self.W, K, 4).permute(1, 2, 0) \
                .contiguous()                                               # [K][4][W]
        t = _native.SpaceTape(K, code_t.data_ptr(), a_t.data_ptr(), b_t.data_ptr(),
                              f_t.data_ptr() if f_t is not None else None)
        rc = _native.lib().ebb_space_tape(ctypes.byref(self.park.state()), ctypes.byref(self.state()), ctypes.byref(t),
                                          self.park._stream(), self.block)
        _native.check(rc, "ebb_space_tape")
        self._keep = (code_t, a_t, b_t, f_t)                # alive until the stream has run the launch

    def ops(self, per_world: list) -> None:
        """A tape from per-world lists of (op name, slot, int, floats)."""
        K = max((len(x) for x in per_world), default=0)
        if K == 0:
            return
        code = torch.zeros(self.W, K, dtype=I64)
        a = torch.full((self.W, K), -1, dtype=I64)
        b = torch.zeros(self.W, K, dtype=I64)
        f = torch.zeros(self.W, K, 4, dtype=torch.float64)
        for w, lst in enumerate(per_world):
            for k, op in enumerate(lst):
                code[w, k] = OP[op[0]]
                a[w, k] = int(op[1]) if len(op) > 1 else -1
                b[w, k] = int(op[2]) if len(op) > 2 else 0
                for c, x in enumerate(op[3] if len(op) > 3 else ()):
                    f[w, k, c] = float(x)
        self.tape(code, a, b, f)

    def query(self, kind: str, a=None, b=None, f=None) -> tuple:
        """One query a world (the reference's VecSpace.query, vec_space.py:938): kind in QUERIES (NEARBY, GetNearbyBalls,
        is this build's own), a [W] (a slot), b [W] (a slot or flags), f [W, <=5]. Returns (out [W, 1 + N] int64: the
        answer, then the balls' ids; outd [W, N]: their squared distances). No host synchronisation."""
        W, N, d = self.W, self.N, self.dev
        a = torch.full((W,), -1, dtype=I64, device=d) if a is None else torch.as_tensor(a, dtype=I64).to(d).reshape(W)
        b = torch.zeros(W, dtype=I64, device=d) if b is None else torch.as_tensor(b, dtype=I64).to(d).reshape(W)
        ff = torch.zeros(5, W, dtype=torch.float64, device=d)
        if f is not None:
            f = torch.as_tensor(f, dtype=torch.float64).to(d).reshape(W, -1)
            ff[:f.shape[1]] = f.t()
        a, b = a.contiguous(), b.contiguous()
        out = torch.zeros(1 + N, W, dtype=I64, device=d)
        outd = torch.zeros(N, W, dtype=torch.float64, device=d)
        q = _native.SpaceQuery(Q[kind], a.data_ptr(), b.data_ptr(), ff.data_ptr(), out.data_ptr(), outd.data_ptr())
        rc = _native.lib().ebb_space_query(ctypes.byref(self.park.state()), ctypes.byref(self.state()), ctypes.byref(q),
                                           self.park._stream(), self.block)
        _native.check(rc, "ebb_space_query")
        self._keep_query = (a, b, ff)
        return out.t(), outd.t()

    def broadcast(self, name: str, mask: torch.Tensor | None = None) -> None:
        """One operation without arguments for every world (or the worlds in mask [W]), on the device."""
        code = torch.full((self.W, 1), OP[name], dtype=I64, device=self.dev)
        if mask is not None:
            code = torch.where(mask.to(self.dev).reshape(self.W, 1), code, torch.zeros_like(code))
        self.tape(code)

    # ---- the load and the tick ----

    def load(self) -> None:
        """AddBall's filing of every ball, each world's slots in order: one tape, made on the device."""
        code = torch.where(self.rows.t() >= 0, OP["ADD"], OP["NONE"]).to(I64)
        slots = torch.arange(self.N, dtype=I64, device=self.dev).expand(self.W, self.N).contiguous()
        self.tape(code, slots)

    def dead_rows(self, worlds: torch.Tensor | None = None) -> torch.Tensor:
        """Phase 1's dead-bubble flags [n] (TIME-714) for the park's tick to skip, no host synchronisation."""
        self.broadcast("DEAD", worlds)
        out = torch.zeros(self.park.n + 1, dtype=BOOL, device=self.dev)
        out.scatter_(0, self._flat, self.st["dead"].t().flatten().to(BOOL))
        return out[:self.park.n]

    def after_evolve(self, dropped_rows: torch.Tensor | None = None, worlds: torch.Tensor | None = None) -> None:
        """After the park's tick: the warp drop-outs' re-filings, then the commits' (no host synchronisation)."""
        dr = self.st["dropped"]
        if dropped_rows is None:
            dr.zero_()
        else:
            pad = torch.cat([dropped_rows.to(self.dev).to(U8), torch.zeros(1, dtype=U8, device=self.dev)])
            dr.copy_(pad[self._flat].reshape(self.W, self.N).t())
        self.broadcast("AFTER_EVOLVE", worlds)

    def tick(self) -> None:
        """One tick of the park with the layer, as Destiny's Evolve runs it on the master: the dead bubbles' balls left
        out of the park's tick (flagged moribund for the call, which every phase skips), then the re-filings."""
        park = self.park
        dead = self.dead_rows()
        self.last_dead = dead
        warp_proper = ((park._mode == WARP) & (park._effect_stamp >= 0) & park._free & ~park._moribund & ~dead)
        saved = park._moribund.clone()
        park._moribund.logical_or_(dead)
        try:
            park.evolve()
        finally:
            park._moribund.copy_(saved)
        self.after_evolve(warp_proper & (park._mode != WARP))

    def check(self) -> None:
        """Raise on a world flagged outside this layer's domain (a deleted box read included)."""
        bad = torch.nonzero(self.st["flags"]).flatten().tolist()
        if bad:
            fl = int(self.st["flags"][bad[0]])
            names = [n for n, bit in FLAG.items() if fl & bit]
            raise RuntimeError(f"worlds {bad[:8]} left the space layer's domain (world {bad[0]}: {names})")

    # ---- readers (host) ----

    def world(self, w: int) -> dict:
        """World w's state on the host: each tensor's column for the world."""
        out = {}
        for name, t in self.st.items():
            out[name] = t[..., w].cpu() if t.dim() > 1 else t[w].cpu()
        return out

    def events(self, w: int) -> list:
        """World w's events since the last CLEAR_EVENTS, in order: (name, ball id, other id, value) for DoProximity,
        (name, ball id, value) for DoRange and DoTargetTracking."""
        n = min(int(self.st["evn"][w]), self.M)
        raw = self.st["ev"][:n, w].cpu().tolist()
        rows = self.rows[:, w].cpu().tolist()
        ids = self.park._ids.cpu().tolist()
        out = []
        for e in raw:
            kind, value, ball, other = e & 15, (e >> 4) & 15, (e >> 8) & 255, (e >> 16) & 255
            if kind == 1:
                out.append((EVENTS[kind], ids[rows[ball]], ids[rows[other]], value))
            else:
                out.append((EVENTS[kind], ids[rows[ball]], value))
        return out

    def clear_events(self) -> None:
        self.st["evn"].zero_()

    def dicts(self, w: int) -> dict:
        """World w's bubble dictionaries: {bubble: [(ball id, +1 | 0 | -1), ...] in insertion order}."""
        st = self.world(w)
        out = {int(b): [] for b in st["dict_bubble"][:int(st["dict_n"])].tolist()}
        for e in range(int(st["entry_n"])):
            out.setdefault(int(st["entry_bubble"][e]), []).append((int(st["entry_id"][e]), int(st["entry_value"][e])))
        return out
