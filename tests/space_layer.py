"""Test harness of the space layer (exact_ballpark_b200.space, csrc/ebb_space.cuh): the golden streams of
tests/golden/space_trace.py driven through the layer, one world a stream, and the layer's state written as the
oracle's state text (oracle/space.cpp's `state`) less what the layer does not hold (the sensors' lines, each ball's
flight-state line, the queries' answers), so that it compares line for line with the oracle's text of the same
operations.

Two backends: "host", the layer's per-world program compiled for the host (tests/native/space_host.cpp: the same
source the device runs), and "cuda", the product's VecSpace over a VecModesPark on the device. A stream's ball ids
are 1 to N (the largest in the streams) and ball id b sits in slot b - 1 of its world, row w N + b - 1 of the park;
the streams' setters are applied to the park's rows and their re-filings are the layer's operations."""

from __future__ import annotations

import ctypes
import math
import struct
import subprocess
from pathlib import Path

import numpy as np

import space_trace as sp

ROOT = Path(__file__).resolve().parent.parent
NATIVE = Path(__file__).resolve().parent / "native"
HOST_LIB = NATIVE / "_build" / "libspace_host.so"
FRICTION, DT = 1.0e6, 1.0
_host = None


def host_lib() -> ctypes.CDLL:
    """The host build of the layer's program (g++, the device build's arithmetic flags)."""
    global _host
    if _host is not None:
        return _host
    src = NATIVE / "space_host.cpp"
    deps = [src, ROOT / "exact_ballpark_b200/csrc/ebb_space.cuh", ROOT / "exact_ballpark_b200/csrc/ebb_arith.cuh",
            ROOT / "include/ebb.h"]
    if not HOST_LIB.exists() or HOST_LIB.stat().st_mtime < max(d.stat().st_mtime for d in deps):
        HOST_LIB.parent.mkdir(parents=True, exist_ok=True)
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
                        "-o", str(HOST_LIB), str(src)], check=True)
    from exact_ballpark_b200 import _native
    L = ctypes.CDLL(str(HOST_LIB))
    L.space_tape_host.argtypes = [ctypes.POINTER(_native.FlightState), ctypes.POINTER(_native.SpaceState),
                                  ctypes.POINTER(_native.SpaceTape)]
    L.space_query_host.argtypes = [ctypes.POINTER(_native.FlightState), ctypes.POINTER(_native.SpaceState),
                                   ctypes.POINTER(_native.SpaceQuery)]
    _host = L
    return L


def srand(seed: int) -> np.ndarray:
    """A world's rand() state after srand(seed) (EBB_RAND_WORDS int32: the table, then the front and rear indices),
    from the oracle's statement of glibc's generator (oracle/grand.py)."""
    from oracle.grand import Rand
    return np.array(Rand(int(seed)).state(), dtype=np.int32)


def f32(x: float) -> float:
    return struct.unpack("<f", struct.pack("<f", float(x)))[0]


class HostPark:
    """The park's rows the layer reads, as numpy arrays in include/ebb.h's EbbFlightState layout."""

    def __init__(self, n: int):
        self.n = n
        self.pos, self.vel = np.zeros((3, n)), np.zeros((3, n))
        self.old_pos, self.old_vel = np.zeros((3, n)), np.zeros((3, n))
        self.mass, self.time_factor = np.zeros(n), np.zeros(n)
        self.radius, self.max_vel = np.zeros(n, np.float32), np.zeros(n, np.float32)
        self.agility, self.speed_fraction = np.ones(n, np.float32), np.ones(n, np.float32)
        self.ids = np.arange(1, n + 1, dtype=np.int64)
        self.mode = np.full(n, 2, np.int32)
        self.free, self.interactive = np.zeros(n, np.uint8), np.zeros(n, np.uint8)
        self.goto_pt, self.follow_ptr = np.zeros((3, n)), np.full(n, -1, np.int32)
        self.follow_range = np.full(n, 10.0, np.float32)
        self.massive, self.sensor = np.zeros(n, np.uint8), np.zeros(n, np.uint8)

    def struct(self):
        from exact_ballpark_b200 import _native
        s = _native.FlightState()
        s.n, s.friction, s.dt = self.n, FRICTION, DT
        for name in ("pos", "vel", "old_pos", "old_vel", "mass", "time_factor", "radius", "max_vel", "agility",
                     "speed_fraction", "ids", "mode", "interactive", "goto_pt", "follow_ptr", "follow_range",
                     "massive", "sensor"):
            setattr(s, name, getattr(self, name).ctypes.data)
        s.free_ = self.free.ctypes.data
        return s

    def add(self, r: int, a: list) -> None:
        """AddBall's values for row r (space.py:1097): float parameters as floats, the clamps, the time factor."""
        mass, radius, max_vel = a[0], f32(a[1]), f32(a[2])
        self.free[r], self.interactive[r] = int(bool(a[3])), int(bool(a[4]))
        self.pos[:, r], self.vel[:, r] = a[5:8], a[8:11]
        self.old_pos[:, r] = [a[5 + i] - a[8 + i] * DT for i in range(3)]
        self.old_vel[:, r] = a[8:11]
        self.radius[r] = 0.0 if radius < 0.0 else radius
        self.mass[r] = 0.0 if mass < 0.0 else mass
        self.max_vel[r] = 0.0 if max_vel < 0.0 else max_vel
        ag, sf = f32(a[11]), f32(a[12])
        self.agility[r] = 1.0 if ag <= 0.0 else ag
        self.speed_fraction[r] = 0.0 if sf < 0.0 else sf
        m = float(self.mass[r]) * float(self.agility[r])
        self.time_factor[r] = 0.0 if m <= 0.0 else math.exp(-FRICTION * DT / m)
        self.mode[r] = 2
        self.massive[r] = int(bool(a[13]))


class HostLayer:
    """The layer's state as numpy arrays (VecSpace's tensors, the same shapes), run by the host build."""

    def __init__(self, W: int, n: int, boxes: int | None = None, seeds=None, events: int | None = None,
                 world_major: bool = False):
        from exact_ballpark_b200.space import allocate_state, state_spec
        self.W, self.N = W, n
        self.M = n * (n + 2) if events is None else events     # a tick's most: every pair entering, each range
        self.B, self.D, self.E, self.S = (boxes or 16 * n + 64), 8 * n + 16, 4 * n + 8, 2 * n + 8
        st, self.pitch = allocate_state(state_spec(n, self.B, self.D, self.E, self.S, n, self.M), W, "cpu",
                                        world_major)
        self._keep = st                                        # the tensors the numpy views below share memory with
        self.st = {k: v.numpy() for k, v in st.items()}
        self.rows = self.st.pop("rows")
        self.rows[...] = np.array([[w * n + j for w in range(W)] for j in range(n)], dtype=np.int64)
        self.st["rnd"] = np.stack([srand(seed) for seed in (seeds if seeds is not None else [1] * W)])

    def _state(self):
        from exact_ballpark_b200 import _native
        s = _native.SpaceState()
        s.worlds, s.slots, s.boxes, s.dicts, s.entries, s.sets = self.W, self.N, self.B, self.D, self.E, self.S
        s.umap_cap, s.events, s.lanes, s.pitch = self.N, self.M, 1, self.pitch
        s.rows = self.rows.ctypes.data
        for name, arr in self.st.items():
            setattr(s, name, arr.ctypes.data)
        return s

    def query(self, park: HostPark, kind: int, a, b, f) -> tuple:
        """One query a world on the host build: (out [1 + N][W], outd [N][W])."""
        from exact_ballpark_b200 import _native
        s = self._state()
        a, b = (np.ascontiguousarray(np.asarray(x, dtype=np.int64).reshape(self.W)) for x in (a, b))
        f = np.ascontiguousarray(np.asarray(f, dtype=np.float64).reshape(5, self.W))
        out = np.zeros((1 + self.N, self.W), dtype=np.int64)
        outd = np.zeros((self.N, self.W))
        q = _native.SpaceQuery(kind, a.ctypes.data, b.ctypes.data, f.ctypes.data, out.ctypes.data, outd.ctypes.data)
        ps = park.struct()
        host_lib().space_query_host(ctypes.byref(ps), ctypes.byref(s), ctypes.byref(q))
        return out, outd

    def tape(self, park: HostPark, code, a, b, f=None) -> None:
        from exact_ballpark_b200 import _native
        s = self._state()
        code, a, b = (np.ascontiguousarray(np.asarray(x, dtype=np.int64).reshape(-1, self.W)) for x in (code, a, b))
        K = code.shape[0]
        f = np.zeros((K, 4, self.W)) if f is None else np.ascontiguousarray(np.asarray(f, np.float64).reshape(K, 4,
                                                                                                           self.W))
        t = _native.SpaceTape(K, code.ctypes.data, a.ctypes.data, b.ctypes.data, f.ctypes.data)
        ps = park.struct()
        host_lib().space_tape_host(ctypes.byref(ps), ctypes.byref(s), ctypes.byref(t))


def translate(park: HostPark, w: int, op, n: int) -> tuple:
    """One golden operation of world w: its effect on the park's rows, and the layer's operation (code, slot, b, f)."""
    from exact_ballpark_b200.space import OP
    code, bid = int(op[0]), int(op[1])
    a = [float(x) for x in op[2:]]
    j = bid - 1
    r = w * n + j
    none = (OP["NONE"], -1, 0, (0.0, 0.0, 0.0, 0.0))
    if code == sp.ADD:
        park.add(r, a)
        return OP["ADD"], j, 0, none[3]
    if code == sp.POS:
        park.pos[:, r] = a[0:3]
        park.old_pos[:, r] = a[0:3]
        return OP["REFILE"], j, 0, none[3]
    if code == sp.RADIUS:
        v = f32(a[0])
        if v < 0.0:
            return none
        park.radius[r] = v
        return OP["REFILE"], j, 0, none[3]
    if code == sp.MAXVEL:
        v = f32(a[0])
        if v < 0.0:
            return none
        park.max_vel[r] = v
        return OP["REFILE"], j, 0, none[3]
    if code == sp.REMOVE:
        return OP["REMOVE_BALL"], j, 0, none[3]
    if code == sp.INIT:
        return OP["INIT_BUBBLES"], -1, 0, none[3]
    if code == sp.COPY:
        return OP["COPY_BUBBLES"], -1, 0, none[3]
    if code == sp.INTERACTIVE:
        return OP["SET_INTERACTIVE"], j, int(bool(a[0])), none[3]
    if code == sp.KEEPALIVE:
        return OP["KEEP_ALIVE"], j, 0, none[3]
    if code == sp.CLOAKED:
        return OP["SET_CLOAKED"], j, int(a[0]), none[3]
    if code == sp.SENSOR:                                 # range, period, only interactives, shuffled
        return OP["ADD_SENSOR"], j, int(bool(a[2])) | (2 if a[3] else 0), (a[0], a[1], 0.0, 0.0)
    if code == sp.UNSENSOR:
        return OP["REMOVE_SENSOR"], j, 0, none[3]
    if code == sp.NOTIFY:
        return OP["NOTIFY_RANGE"], j, 0, (a[0], 0.0, 0.0, 0.0)
    if code == sp.TRACK:                                  # the target's slot, or -1 when its id is none of the world's
        t = int(a[0])
        slot = t - 1 if 1 <= t <= n else -1
        return OP["TRACK"], j, slot, (a[1], 1.0 if t == 0 else 0.0, 0.0, 0.0)
    if code == sp.PROXIMITIES:
        return OP["HANDLE_PROXIMITIES"], -1, 0, none[3]
    if code == sp.GOTO and all(math.isfinite(x) for x in a[0:3]):   # GotoPoint: a speed fraction of 0 becomes 1
        if park.speed_fraction[r] == 0.0:
            park.speed_fraction[r] = 1.0
        park.mode[r] = 0
        park.goto_pt[:, r] = a[0:3]
        return none
    if code == sp.STOP:
        park.mode[r] = 2
        return none
    return none                                           # the queries: not the layer's


QUERY_OPS = (sp.VISIBILITY, sp.RANGE_BALL, sp.RANGE_POINT, sp.BUBBLE_AT, sp.NEARBY)


def query_of(op, n: int) -> tuple:
    """A golden query operation as the layer's query: (kind, a, b, f[5]); ids outside 1..n are no ball's."""
    from exact_ballpark_b200.space import Q
    code, bid = int(op[0]), int(op[1])
    a = [float(x) for x in op[2:]]
    slot = lambda i: int(i) - 1 if 1 <= int(i) <= n else -1      # noqa: E731
    if code == sp.VISIBILITY:
        return Q["VISIBILITY"], slot(bid), slot(a[0]), [0.0] * 5
    if code == sp.RANGE_BALL:
        return Q["RANGE_BALL"], slot(bid), int(bool(a[1])), [a[0], 0.0, 0.0, 0.0, 0.0]
    if code == sp.RANGE_POINT:
        return Q["RANGE_POINT"], -1, int(bool(a[4])), [a[0], a[1], a[2], a[3], 0.0]
    if code == sp.BUBBLE_AT:
        return Q["BUBBLE_AT"], -1, 0, [a[0], a[1], a[2], 0.0, 0.0]
    return Q["NEARBY"], slot(bid), int(bool(a[0])) | (2 if a[1] else 0) | (4 if a[2] else 0), [0.0] * 5


def answer_text(op, out, outd, w: int) -> str:
    """The layer's answer to world w's query as the oracle writes it."""
    code = int(op[0])
    v = int(out[0, w])
    if code == sp.VISIBILITY:
        return f"Q {v}\n"
    if code == sp.BUBBLE_AT:
        return "Q None\n" if v == -2 else f"Q {v}\n"
    if code == sp.RANGE_BALL and v == -1:
        return "Q None\n"
    dist = code in (sp.RANGE_BALL, sp.RANGE_POINT) and bool(op[4] if code == sp.RANGE_BALL else op[7])
    items = []
    for i in range(max(v, 0)):
        bid = int(out[1 + i, w])
        if dist:
            bits = "%016x" % struct.unpack("<Q", struct.pack("<d", float(outd[i, w])))[0]
            items.append(f" {bits}:{bid}")
        else:
            items.append(f" {bid}")
    return "Q" + "".join(items) + "\n"


def text(st: dict, park_ids, park_mode, w: int, park_sensor=None) -> str:
    """World w's layer state as the oracle's state text (the lines the layer holds)."""
    n = st["level"].shape[0]
    col = lambda name: st[name][..., w]                   # noqa: E731
    level, key, mod, active = col("level"), col("key"), col("mod"), col("active")
    bubble, old_bubble, in_park = col("bubble"), col("old_bubble"), col("in_park")
    inter = {}
    for e in range(int(st["inter_n"][w])):
        inter.setdefault(int(st["inter_bubble"][e, w]), set()).add(int(st["inter_id"][e, w]))
    keep = {}
    for e in range(int(st["keep_n"][w])):
        keep.setdefault(int(st["keep_bubble"][e, w]), set()).add(int(st["keep_id"][e, w]))
    out = []
    slots = sorted((int(park_ids[w * n + j]), j) for j in range(n) if in_park[j])
    for bid, j in slots:
        dead = 0 if int(park_mode[w * n + j]) == 3 else int(not inter.get(int(bubble[j])) and
                                                             not keep.get(int(bubble[j])))
        act = int(active[j])
        if level[j] >= 0:
            head = (f"B {bid} {bubble[j]} {old_bubble[j]} {level[j]} {key[0, j]} {key[1, j]} {key[2, j]} "
                    f"{mod[0, j]} {mod[1, j]} {mod[2, j]} {act} {dead}")
            boxes = sorted((key[0, j] + x, key[1, j] + y, key[2, j] + z) for z in (-1, 0, 1) for y in (-1, 0, 1)
                           for x in (-1, 0, 1) if (act >> (13 + x + 3 * y + 9 * z)) & 1)
        else:
            head = f"B {bid} {bubble[j]} {old_bubble[j]} - {mod[0, j]} {mod[1, j]} {mod[2, j]} {act} {dead}"
            boxes = []
        out.append(head + "".join(f" {k[0]},{k[1]},{k[2]}" for k in boxes) + "\n")
    lv = col("box_level")[:int(st["box_n"][w])]
    out.append("L" + "".join(f" {int((lv == i).sum())}" for i in range(8)) + "\n")
    undefined = 1 if int(st["flags"][w]) & (1 << 11) else 0
    out.append(f"F {int(st['free_boxes'][w])} {int(st['bubble_id'][w])} {undefined}\n")
    if "pn" in st:
        pid = lambda k: int(park_ids[w * n + int(k)])     # noqa: E731
        pn = int(st["pn"][w])
        if pn:
            out.append("P" + "".join(f" {pid(k)}" for k in st["pmap"][:pn, w]) + "\n")
        for bid, j in slots:
            on, ln, hp = int(park_sensor[w * n + j]) if park_sensor is not None else 0, int(st["slen"][j, w]), \
                int(st["has_prox"][j, w])
            if not on and not ln and not hp:
                continue
            trk = int(st["trk"][j, w])
            bits = "%016x" % struct.unpack("<Q", struct.pack("<d", float(st["selapsed"][j, w])))[0]
            out.append(f"S {bid} {on} {bits} {hp} {int(st['ntf_in'][j, w])} {int(st['trk_in'][j, w])} "
                       f"{pid(trk) if trk >= 0 else 0}" + "".join(f" {pid(k)}" for k in st["slist"][:ln, j, w])
                       + "\n")
    dicts = {int(b): [] for b in col("dict_bubble")[:int(st["dict_n"][w])]}
    for e in range(int(st["entry_n"][w])):
        dicts.setdefault(int(st["entry_bubble"][e, w]), []).append((int(st["entry_id"][e, w]),
                                                                     int(st["entry_value"][e, w])))
    for bub in sorted(dicts):
        out.append(f"U {bub}" + "".join(f" {k}:{v}" for k, v in dicts[bub]) + "\n")
    for tag, m in (("I", inter), ("K", keep)):
        for bub in sorted(m):
            out.append(f"{tag} {bub}" + "".join(f" {i}" for i in sorted(m[bub])) + "\n")
    return "".join(out)


def oracle_lines(t: str, code: int = 0) -> str:
    """The oracle's state text less the lines the layer does not hold (the flight states, the queries' answers):
    the answer kept for HandleProximities and a tick (their events)."""
    keep = ("B", "L", "F", "P", "S", "U", "I", "K") + (("Q",) if code in (sp.PROXIMITIES, sp.TICK) + QUERY_OPS
                                                         else ())
    return "".join(line + "\n" for line in t.splitlines() if line[:1] in keep)


def events_text(st: dict, park_ids, w: int, n: int) -> str:
    """World w's events as the oracle writes a HandleProximities answer."""
    out = []
    for e in st["ev"][:int(st["evn"][w]), w]:
        e = int(e)
        kind, value, ball, other = e & 15, (e >> 4) & 15, (e >> 8) & 255, (e >> 16) & 255
        b = int(park_ids[w * n + ball])
        if kind == 1:
            out.append(f" {b}:{int(park_ids[w * n + other])}:{value}")
        else:
            out.append(f" {'R' if kind == 2 else 'T'}{b}:{value}")
    return "Q" + "".join(out) + "\n"


def drive(streams: list, kernel: str = "host", device=None, lanes: int = 1, world_major: bool | None = None) -> tuple:
    """Every stream through the layer, one world each, one operation a launch: (texts [world][op], flags [W]); a
    HandleProximities operation's text ends with its events. `world_major`: the state's arrangement (None: the
    layer's default for `lanes`; interleaved on the host)."""
    W = len(streams)
    seeds = [int(s[1]) if isinstance(s, tuple) else 1 for s in streams]
    streams = [s[0] if isinstance(s, tuple) else s for s in streams]
    N = int(max(int(np.max(np.asarray(s)[:, 1])) for s in streams))
    park = HostPark(W * N)
    park.ids[:] = np.tile(np.arange(1, N + 1, dtype=np.int64), W)       # world w's ball b at row w N + b - 1
    K = max(len(s) for s in streams)
    texts = [[] for _ in range(W)]
    if kernel == "host":
        layer = HostLayer(W, N, seeds=seeds, world_major=bool(world_major))

        def run(code, a, b, f):
            layer.st["evn"][:] = 0
            layer.tape(park, code, a, b, f)

        read = lambda: layer.st                                                     # noqa: E731
        sensor = lambda: park.sensor                                                # noqa: E731
        ask = lambda kind, a, b, f: layer.query(park, kind, a, b, f)                # noqa: E731
    else:
        import torch
        from exact_ballpark_b200.modes import VecModesPark
        from exact_ballpark_b200.space import VecSpace
        dpark = VecModesPark(W * N, friction=FRICTION, tick_interval_ms=1000, device=device or "cuda")
        layer = VecSpace(dpark, np.arange(W * N, dtype=np.int64).reshape(W, N), events=N * (N + 2), seed=seeds,
                         lanes=lanes, world_major=world_major)

        def run(code, a, b, f):
            for name in ("pos", "vel", "old_pos", "old_vel", "mass", "time_factor", "radius", "max_vel", "agility",
                         "speed_fraction", "ids", "mode", "follow_ptr", "follow_range"):
                getattr(dpark, "_" + name).copy_(torch.from_numpy(getattr(park, name)).to(getattr(dpark, "_" + name)))
            dpark._goto.copy_(torch.from_numpy(park.goto_pt).to(dpark._goto))
            for name in ("free", "interactive", "massive"):
                getattr(dpark, "_" + name).copy_(torch.from_numpy(getattr(park, name).astype(bool)).to(dpark.dev))
            layer.clear_events()
            layer.tape(torch.from_numpy(np.asarray(code, dtype=np.int64).reshape(W, 1)),
                       torch.from_numpy(np.asarray(a, dtype=np.int64).reshape(W, 1)),
                       torch.from_numpy(np.asarray(b, dtype=np.int64).reshape(W, 1)),
                       torch.from_numpy(np.asarray(f, dtype=np.float64).reshape(W, 1, 4)))
            park.interactive[:] = dpark._interactive.cpu().numpy().astype(np.uint8)
            park.radius[:] = dpark._radius.cpu().numpy()

        read = lambda: {k: v.cpu().numpy() for k, v in layer.st.items()}            # noqa: E731
        sensor = lambda: dpark._sensor.cpu().numpy().astype(np.uint8)                # noqa: E731

        def ask(kind, a, b, f):
            from exact_ballpark_b200.space import QUERIES
            out, outd = layer.query(QUERIES[kind], torch.from_numpy(a), torch.from_numpy(b),
                                    torch.from_numpy(np.ascontiguousarray(f.T)))
            return out.t().cpu().numpy(), outd.t().cpu().numpy()
    for k in range(K):
        code, a, b = np.zeros(W, np.int64), np.full(W, -1, np.int64), np.zeros(W, np.int64)
        f = np.zeros((W, 4))
        for w, ops in enumerate(streams):
            if k < len(ops):
                code[w], a[w], b[w], f[w] = translate(park, w, ops[k], N)
        run(code, a, b, f.T.copy() if kernel == "host" else f)
        st = read()
        sens = sensor()
        answers, asked = {}, {}
        for w, ops in enumerate(streams):
            if k < len(ops) and int(ops[k][0]) in QUERY_OPS:
                asked.setdefault(query_of(ops[k], N)[0], []).append(w)
        for kind, worlds in asked.items():                # one query launch a kind, every world asking it
            qa, qb, qf = np.full(W, -1, np.int64), np.zeros(W, np.int64), np.zeros((5, W))
            for w in worlds:
                _, qa[w], qb[w], qf[:, w] = query_of(streams[w][k], N)
            out, outd = ask(kind, qa, qb, qf)
            for w in worlds:
                answers[w] = answer_text(streams[w][k], out, outd, w)
        for w, ops in enumerate(streams):
            if k < len(ops):
                t = text(st, park.ids, park.mode, w, sens)
                if int(ops[k][0]) == sp.PROXIMITIES:
                    t += events_text(st, park.ids, w, N)
                t += answers.get(w, "")
                texts[w].append(t)
    return texts, read()["flags"].copy()


def drive_ticks(ops, device="cuda", seed: int = 1, lanes: int = 1, world_major: bool | None = None) -> list:
    """One ticking or mode stream (tests/golden/space_trace.py's tick_ops and mode_ops) through VecSpace over a
    VecModesPark on the device, its ticks the layer's `tick` (dead bubbles skipped, the re-filings and
    HandleProximities after): the texts after every operation, a tick's and HandleProximities' with their events. The
    park owns the rows: AddBall writes a row, GotoPoint, Stop, FollowBall and Orbit (their same-bubble test reading
    the layer's bubbles), WarpTo and RemoveBall's Stop and StopAllFollowers are its commands; the sensors' operations
    are the layer's."""
    import torch
    from exact_ballpark_b200.modes import VecModesPark
    from exact_ballpark_b200.space import OP, VecSpace
    n = int(np.max(np.asarray(ops)[:, 1]))
    park = VecModesPark(n, friction=FRICTION, tick_interval_ms=1000, device=device)
    layer = VecSpace(park, np.arange(n, dtype=np.int64).reshape(1, n), events=n * (n + 2), seed=seed, lanes=lanes,
                     world_major=world_major)
    out = []
    dev = park.dev
    for op in ops:
        code, bid = int(op[0]), int(op[1])
        a = [float(x) for x in op[2:]]
        j = bid - 1
        mask = torch.zeros(n, dtype=torch.bool, device=dev)
        if 0 <= j < n:
            mask[j] = True
        live = 0 <= j < n and bool(layer.st["in_park"][j, 0])
        layer.clear_events()
        if code in (sp.SENSOR, sp.UNSENSOR, sp.NOTIFY, sp.TRACK, sp.CLOAKED, sp.PROXIMITIES):
            h = HostPark(n)
            lc, la, lb, lf = translate(h, 0, op, n)
            if lc:
                name = next(k for k, v in OP.items() if v == lc)
                layer.ops([[(name, la, lb, lf)]])
        elif code == sp.TICK:
            layer.tick()
        elif code == sp.ADD:
            h = HostPark(n)
            h.add(j, a)
            names = ("pos", "vel", "mass", "time_factor", "radius", "max_vel", "agility", "speed_fraction")
            for name in names if live else names + ("old_pos", "old_vel"):
                getattr(park, "_" + name)[..., j] = torch.as_tensor(getattr(h, name)[..., j]).to(
                    getattr(park, "_" + name))
            park._free[j], park._interactive[j] = bool(h.free[j]), bool(h.interactive[j])
            park._massive[j] = bool(a[13])
            park._effect_stamp[j] = park._owner_id[j] = park._follow_id[j] = 0
            park._follow_range[j], park._mode[j] = 10.0, 2          # a re-added ball keeps its target pointer
            if not live:
                park._follow_ptr[j], park._last_g[:, j], park._last_collision[j] = -1, 0.0, -1.0
            layer.ops([[("ADD", j)]])
        elif not live and code in (sp.GOTO, sp.STOP, sp.REMOVE, sp.FOLLOW, sp.ORBIT, sp.WARP):
            pass                                          # a command to a ball not in the world does nothing
        elif code in (sp.FOLLOW, sp.ORBIT):
            t = int(a[0]) - 1
            park.bubble.copy_(layer.st["bubble"][:, 0].to(park.bubble))   # FollowBall's same-bubble test
            saved = park._moribund.clone()
            park._moribund.logical_or_(~layer.st["in_park"][:, 0].to(torch.bool))   # a target not in the world
            target = torch.full((n,), t if 0 <= t < n else -1, dtype=torch.int64, device=dev)
            (park.follow if code == sp.FOLLOW else park.orbit)(mask, target, torch.full((n,), a[1], device=dev,
                                                                                          dtype=torch.float64))
            park._moribund.copy_(saved)
        elif code == sp.WARP:
            park.warp_to(mask, torch.tensor([a[0:3]] * n, dtype=torch.float64, device=dev),
                         torch.full((n,), a[3], dtype=torch.float64, device=dev),
                         torch.full((n,), int(a[4]), dtype=torch.int64, device=dev))
        elif code == sp.POS:
            park._pos[:, j] = torch.tensor(a[0:3], dtype=torch.float64, device=dev)
            park._old_pos[:, j] = torch.tensor(a[0:3], dtype=torch.float64, device=dev)
            layer.ops([[("REFILE", j)]])
        elif code == sp.GOTO:
            park.goto_point(mask, torch.tensor([a[0:3]] * n, dtype=torch.float64, device=dev))
        elif code == sp.STOP:
            park.stop(mask)
        elif code == sp.REMOVE:                           # RemoveBall: Stop, then StopAllFollowers
            park.stop(mask)
            park._release_followers(mask)
            layer.ops([[("REMOVE_BALL", j)]])
        elif code == sp.INIT:
            layer.ops([[("INIT_BUBBLES",)]])
        elif code == sp.COPY:
            layer.ops([[("COPY_BUBBLES",)]])
        elif code == sp.INTERACTIVE:
            layer.ops([[("SET_INTERACTIVE", j, int(bool(a[0])))]])
        elif code == sp.KEEPALIVE:
            layer.ops([[("KEEP_ALIVE", j)]])
        st = {k: v.cpu().numpy() for k, v in layer.st.items()}
        ids = park._ids.cpu().numpy()
        t = text(st, ids, park._mode.cpu().numpy(), 0, park._sensor.cpu().numpy().astype(np.uint8))
        if code in (sp.TICK, sp.PROXIMITIES):
            t += events_text(st, ids, 0, n)
        if code in QUERY_OPS:
            from exact_ballpark_b200.space import QUERIES
            kind, qa, qb, qf = query_of(op, n)
            qo, qd = layer.query(QUERIES[kind], [qa], [qb], torch.tensor([qf], dtype=torch.float64))
            t += answer_text(op, qo.t().cpu().numpy(), qd.t().cpu().numpy(), 0)
        out.append(t)
    return out


def drive_ticks_host(ops, seed: int = 1, world_major: bool = False) -> list:
    """drive_ticks on the CPU, for the ticking and the mode streams: the flight oracle's park (oracle/park.py's
    OraclePark, its tick the C++ oracle) owns the rows (AddBall, GotoPoint, Stop, FollowBall and Orbit with the
    layer's bubbles for their same-bubble test, WarpTo, RemoveBall's Stop and StopAllFollowers) and ticks them with
    the dead rows flagged moribund for the call; the layer's host build runs DEAD and AFTER_EVOLVE around the tick (the
    warp drop-outs among its re-filings), as VecSpace.tick does on the device."""
    from exact_ballpark_b200.space import OP
    from oracle.park import OraclePark
    n = int(np.max(np.asarray(ops)[:, 1]))
    op = OraclePark(n, friction=FRICTION, tick_interval_ms=1000)
    host, layer = HostPark(n), HostLayer(1, n, seeds=[seed], world_major=world_major)

    def pull() -> None:                                   # the layer's view of the oracle park's rows
        for name in ("pos", "vel", "old_pos", "old_vel"):
            getattr(host, name)[:] = getattr(op, name).T
        for name in ("mass", "time_factor"):
            getattr(host, name)[:] = getattr(op, name)
        for name in ("radius", "max_vel", "agility", "speed_fraction"):
            getattr(host, name)[:] = getattr(op, name).astype(np.float32)
        host.ids[:] = op.ids
        host.mode[:] = op.mode.astype(np.int32)
        host.free[:] = op.free.astype(np.uint8)
        host.interactive[:] = op.interactive.astype(np.uint8)
        host.massive[:] = op.massive.astype(np.uint8)
        host.goto_pt[:] = op.goto.T
        host.follow_ptr[:] = op.follow_ptr.astype(np.int32)
        host.follow_range[:] = op.follow_range.astype(np.float32)
        host.sensor[:] = op.sensor.astype(np.uint8)

    def run(name: str, j: int = -1, b: int = 0, f=(0.0, 0.0, 0.0, 0.0)) -> None:
        pull()
        layer.tape(host, [OP[name]], [j], [b], np.asarray(f, dtype=np.float64).reshape(1, 4, 1))
        op.interactive = host.interactive.astype(bool)
        op.sensor = host.sensor.astype(bool)               # the layer's sensor flags (AddProximitySensor's)

    out = []
    for row in ops:
        code, bid = int(row[0]), int(row[1])
        a = [float(x) for x in row[2:]]
        j = bid - 1
        mask = np.zeros(n, dtype=bool)
        if 0 <= j < n:
            mask[j] = True
        layer.st["evn"][:] = 0
        sensor_op = code in (sp.SENSOR, sp.UNSENSOR, sp.NOTIFY, sp.TRACK, sp.CLOAKED, sp.PROXIMITIES)
        if sensor_op:
            lc, la, lb, lf = translate(host, 0, row, n)
            if lc:
                run(next(k for k, v in OP.items() if v == lc), la, lb, lf)
        elif code == sp.TICK:
            run("DEAD")
            dead = layer.st["dead"][:, 0].astype(bool)
            warp_proper = (op.mode == 3) & (op.effect_stamp >= 0) & op.free & ~op.moribund & ~dead
            saved = op.moribund.copy()
            op.moribund = saved | dead
            op.evolve()
            op.moribund = saved
            layer.st["dropped"][:, 0] = (warp_proper & (op.mode != 3)).astype(np.uint8)
            run("AFTER_EVOLVE")
        elif code == sp.ADD:
            h = HostPark(n)
            h.add(j, a)
            again = bool(layer.st["in_park"][j, 0])
            for name in ("pos", "vel") if again else ("pos", "vel", "old_pos", "old_vel"):
                getattr(op, name)[j] = getattr(h, name)[:, j]
            for name in ("mass", "time_factor", "radius", "max_vel", "agility", "speed_fraction"):
                getattr(op, name)[j] = float(getattr(h, name)[j])
            op.free[j], op.interactive[j], op.massive[j] = bool(h.free[j]), bool(h.interactive[j]), bool(a[13])
            op.effect_stamp[j] = op.owner_id[j] = op.follow_id[j] = 0
            op.follow_range[j], op.mode[j] = 10.0, 2         # a re-added ball keeps its target pointer
            if not again:
                op.follow_ptr[j], op.last_g[j], op.last_collision[j] = -1, 0.0, -1.0
            run("ADD", j)
        elif not (0 <= j < n and layer.st["in_park"][j, 0]) and code in (sp.GOTO, sp.STOP, sp.REMOVE, sp.FOLLOW,
                                                                           sp.ORBIT, sp.WARP):
            pass                                          # a command to a ball not in the world does nothing
        elif code in (sp.FOLLOW, sp.ORBIT):
            t = int(a[0]) - 1
            op.bubble = layer.st["bubble"][:, 0].copy()  # FollowBall's same-bubble test reads the layer's bubbles
            saved = op.moribund.copy()
            op.moribund = saved | ~layer.st["in_park"][:, 0].astype(bool)   # a target not in the world is refused
            (op.follow if code == sp.FOLLOW else op.orbit)(mask, np.full(n, t if 0 <= t < n else -1), np.full(n, a[1]))
            op.moribund = saved
        elif code == sp.WARP:
            op.warp_to(mask, np.array([a[0:3]] * n), np.full(n, a[3]), np.full(n, int(a[4]), dtype=np.int64))
        elif code == sp.POS:
            op.pos[j] = a[0:3]
            op.old_pos[j] = a[0:3]
            run("REFILE", j)
        elif code == sp.GOTO:
            op.goto_point(mask, np.array([a[0:3]] * n))
        elif code == sp.STOP:
            op.stop(mask)
        elif code == sp.REMOVE:                           # RemoveBall: Stop, then StopAllFollowers
            op.stop(mask)
            members = op._members(mask)
            orbiter = members & op.interactive & (op.mode == 4)
            op._stop_rows(members & ~orbiter)
            op.goto_direction(orbiter, op.vel.copy())
            run("REMOVE_BALL", j)
        elif code == sp.INIT:
            run("INIT_BUBBLES")
        elif code == sp.COPY:
            run("COPY_BUBBLES")
        elif code == sp.INTERACTIVE:
            run("SET_INTERACTIVE", j, int(bool(a[0])))
        elif code == sp.KEEPALIVE:
            run("KEEP_ALIVE", j)
        t = text(layer.st, op.ids, op.mode, 0, op.sensor.astype(np.uint8))
        if code in (sp.TICK, sp.PROXIMITIES):
            t += events_text(layer.st, op.ids, 0, n)
        if code in QUERY_OPS:
            pull()
            kind, qa, qb, qf = query_of(row, n)
            qo, qd = layer.query(host, kind, [qa], [qb], np.asarray(qf).reshape(5, 1))
            t += answer_text(row, qo, qd, 0)
        out.append(t)
    return out


def partition_world_ops(pw, w: int, goto: np.ndarray, ticks: int) -> np.ndarray:
    """World w of the partition worlds as a golden-style stream: AddBall of each ship, its sensor, its goto point,
    then the ticks."""
    c = pw.cols
    s0, k = int(pw.starts[w]), int(pw.sizes[w])
    ops = []
    for j in range(k):
        r = s0 + j
        ops.append(sp._op(sp.ADD, j + 1, c["mass"][r], c["radius"][r], c["max_vel"][r], 1.0, 1.0, *c["pos"][r],
                          0.0, 0.0, 0.0, c["agility"][r], 1.0, 0.0))
    for j in range(k):
        ops.append(sp._op(sp.SENSOR, j + 1, pw.sensor_range[s0 + j], 1.0, 0.0, 0.0))
    for j in range(k):
        ops.append(sp._op(sp.GOTO, j + 1, *goto[s0 + j]))
    ops += [sp._op(sp.TICK) for _ in range(ticks)]
    return np.array(ops)
