"""Golden traces of the flight-mode park: a scenario as the calls a caller makes on the park's public API, and the
park's state after every tick as digests.

A trace holds the constructor's arguments, the `load` rows, and a list of events: a command call (its name, the rows
its mask selects, and each further argument's values at those rows) or a tick. `make_golden.py` records traces by
running the reference's own batched park (exact_ballpark.vec_modes.VecModesPark, its CPU tick, which the reference
holds bit for bit to its scalar ModeBallpark and FullBallpark) with a recording subclass; the tests replay them on
this package's park and compare the state digests tick by tick.

A state digest covers every per-row field a tick or a command may change (FIELDS), each canonicalised: floats as
float64 bit patterns with every NaN made one quiet NaN (the reference compares NaN equal to NaN), integers and flags
as int64. Each field has its own 8-byte digest (a mismatch names the field), and the tick's digest is the SHA-256 of
them all.
"""

from __future__ import annotations

import gzip
import hashlib
import json
from pathlib import Path

import numpy as np
import torch

GOLDEN = Path(__file__).resolve().parent

FIELDS = ("pos", "vel", "old_pos", "old_vel", "goto", "last_g", "ang_vel", "old_ang_vel", "torque", "rot", "old_rot",
          "mass", "radius", "max_vel", "agility", "speed_fraction", "follow_range", "last_collision", "time_factor",
          "max_ang_vel", "rot_roll", "rot_agility", "mode", "effect_stamp", "follow_id", "owner_id", "ids",
          "follow_ptr", "clock", "world", "cloaked", "bubble", "free", "moribund", "massive", "interactive", "sensor",
          "refiled")
COMMANDS = ("stop", "goto_point", "goto_direction", "follow", "orbit", "warp_to", "entity_warp_in",
            "set_speed_fraction", "set_mass", "set_agility", "set_max_velocity", "set_radius", "set_velocity",
            "set_max_angular_speed", "set_rot_agility", "set_angular_velocity", "set_rotation", "set_free",
            "set_ball_rigid", "set_boid", "set_interactive", "set_ball_troll")
_QNAN = np.uint64(0x7FF8000000000000)


def canonical(t) -> np.ndarray:
    """A field as canonical numpy: float64 with one NaN pattern, or int64."""
    a = t.detach().cpu() if isinstance(t, torch.Tensor) else torch.as_tensor(t)
    if a.dtype in (torch.float64, torch.float32, torch.float16):
        x = np.ascontiguousarray(a.to(torch.float64).numpy())
        bits = x.view(np.uint64).copy()
        bits[np.isnan(x)] = _QNAN
        return bits.view(np.float64)
    return np.ascontiguousarray(a.to(torch.int64).numpy())


def field_digests(park) -> np.ndarray:
    """[len(FIELDS)] uint64: each field's digest."""
    out = np.zeros(len(FIELDS), dtype=np.uint64)
    for i, f in enumerate(FIELDS):
        a = canonical(getattr(park, f))
        h = hashlib.sha256(f.encode() + str(a.shape).encode() + a.tobytes()).digest()
        out[i] = np.frombuffer(h[:8], dtype=np.uint64)[0]
    return out


def state_digest(fd: np.ndarray) -> bytes:
    return hashlib.sha256(fd.tobytes()).digest()


def snapshot(park) -> dict:
    return {f: canonical(getattr(park, f)) for f in FIELDS}


# ---- recording ----

def _arg(a, rows: np.ndarray):
    t = torch.as_tensor(a).detach().cpu()
    vals = t[torch.as_tensor(rows, dtype=torch.long)] if t.dim() >= 1 and t.shape[0] > 0 else t
    if t.dtype in (torch.float64, torch.float32):
        return {"k": "f", "cols": (t.shape[1] if t.dim() == 2 else 0),
                "v": [float(x).hex() for x in vals.reshape(-1).tolist()]}
    return {"k": "i", "cols": (t.shape[1] if t.dim() == 2 else 0), "v": [int(x) for x in vals.reshape(-1).tolist()]}


def recording(park_cls):
    """A subclass of park_cls that records every top-level command, load and tick into self.trace."""

    class Recording(park_cls):
        def __init__(self, n, *args, **kw):
            super().__init__(n, *args, **kw)
            self._depth = 0
            self.trace = {"ctor": {"n": n, **_ctor_kw(args, kw)}, "rows": None, "events": [], "digests": [],
                          "field_digests": []}

        def load(self, rows):
            self.trace["rows"] = [_row_json(r) for r in rows]
            self._depth += 1
            try:
                super().load(rows)
            finally:
                self._depth -= 1

        def evolve(self, *a, **k):
            self._depth += 1                # the tick's own command calls (a follower's release) are not events
            try:
                super().evolve(*a, **k)
            finally:
                self._depth -= 1
            fd = field_digests(self)
            self.trace["events"].append({"tick": 1})
            self.trace["field_digests"].append(fd)
            self.trace["digests"].append(state_digest(fd))

    def make(name):
        base = getattr(park_cls, name)

        def wrapped(self, mask, *args):
            if self._depth == 0:
                m = torch.as_tensor(mask).detach().cpu().to(torch.bool)
                rows = torch.nonzero(m).reshape(-1).numpy()
                self.trace["events"].append({"call": name, "rows": rows.tolist(),
                                             "args": [_arg(a, rows) for a in args]})
            self._depth += 1
            try:
                return base(self, mask, *args)
            finally:
                self._depth -= 1
        wrapped.__name__ = name
        return wrapped

    for name in COMMANDS:
        if hasattr(park_cls, name):
            setattr(Recording, name, make(name))
    return Recording


_CTOR_NAMES = ("friction", "tick_interval_ms", "device", "dynamical_orientation", "use_new_orbit", "block", "ypr")


def _ctor_kw(args, kw) -> dict:
    out = dict(zip(_CTOR_NAMES, args))
    out.update(kw)
    out.pop("device", None)
    out.pop("block", None)
    return out


def _jf(x):
    return float(x).hex() if isinstance(x, float) else x


def _row_json(r: dict) -> dict:
    out = {}
    for k, v in r.items():
        if isinstance(v, (list, tuple)):
            out[k] = [_jf(float(c)) for c in v]
        elif isinstance(v, bool):
            out[k] = v
        elif isinstance(v, float):
            out[k] = _jf(v)
        else:
            out[k] = v
    return out


def save(traces: list, path: Path, finals: list | None = None) -> None:
    """Write a bundle of traces (one per park) as path.json.gz (the calls) and path.npz (digests, final states)."""
    bodies = [{k: v for k, v in t.items() if k not in ("digests", "field_digests")} for t in traces]
    with gzip.open(str(path) + ".json.gz", "wt") as f:
        json.dump({"groups": bodies}, f)
    arrays = {}
    for i, t in enumerate(traces):
        arrays[f"g{i}_digests"] = np.array([np.frombuffer(d, dtype=np.uint8) for d in t["digests"]],
                                           dtype=np.uint8).reshape(-1, 32)
        arrays[f"g{i}_field_digests"] = np.array(t["field_digests"], dtype=np.uint64).reshape(-1, len(FIELDS))
        for k, v in ((finals or [None] * len(traces))[i] or {}).items():
            arrays[f"g{i}_final_{k}"] = v
    np.savez_compressed(str(path) + ".npz", **arrays)


# ---- loading and replay ----

def _unhex(x):
    return float.fromhex(x) if isinstance(x, str) else x


def load(path: Path) -> list:
    """A bundle's traces, each with its rows, events, digests, field digests and final state."""
    with gzip.open(str(path) + ".json.gz", "rt") as f:
        groups = json.load(f)["groups"]
    z = np.load(str(path) + ".npz")
    for i, body in enumerate(groups):
        body["rows"] = [{k: ([_unhex(c) for c in v] if isinstance(v, list) else _unhex(v)) for k, v in r.items()}
                        for r in body["rows"]]
        body["digests"] = z[f"g{i}_digests"]
        body["field_digests"] = z[f"g{i}_field_digests"]
        pre = f"g{i}_final_"
        body["final"] = {k[len(pre):]: z[k] for k in z.files if k.startswith(pre)}
    return groups


def _rebuild(arg: dict, rows: list, n: int, dev):
    cols = arg["cols"]
    shape = (n, cols) if cols else (n,)
    if arg["k"] == "f":
        full = torch.zeros(shape, dtype=torch.float64)
        vals = torch.tensor([_unhex(v) for v in arg["v"]], dtype=torch.float64)
    else:
        full = torch.zeros(shape, dtype=torch.int64)
        vals = torch.tensor(arg["v"], dtype=torch.int64)
    if rows:
        full[torch.tensor(rows, dtype=torch.long)] = vals.reshape((len(rows),) + shape[1:])
    return full.to(dev)


def replay(trace: dict, park, tick=None, on_tick=None) -> None:
    """Apply the trace's load and events to `park` (constructed by the caller from trace["ctor"]); `tick()` defaults
    to park.evolve(); `on_tick(k, park)` is called after the k-th tick (0-based)."""
    park.load(trace["rows"])
    n, dev = park.n, park.dev
    k = 0
    tick = tick or park.evolve
    for ev in trace["events"]:
        if "tick" in ev:
            tick()
            if on_tick is not None:
                on_tick(k, park)
            k += 1
            continue
        mask = torch.zeros(n, dtype=torch.bool)
        if ev["rows"]:
            mask[torch.tensor(ev["rows"], dtype=torch.long)] = True
        args = [_rebuild(a, ev["rows"], n, dev) for a in ev["args"]]
        getattr(park, ev["call"])(mask.to(dev), *args)


def first_mismatch(trace: dict, k: int, fd: np.ndarray):
    """None if tick k's field digests match, else the names of the fields that differ."""
    want = trace["field_digests"][k]
    if np.array_equal(want, fd):
        return None
    return [FIELDS[i] for i in range(len(FIELDS)) if want[i] != fd[i]]
