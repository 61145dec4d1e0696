"""Golden traces of the collision park: a scenario as the calls a caller makes on the park's public API (the
constructor's worlds x slots and tick, the load's worlds, GotoPoint / GotoDirection / Stop / SetSpeedFraction calls
with their [W, N] masks), and the park's state after every tick as digests.

`make_golden.py --only collide` records them on the reference's batched collision park
(exact_ballpark.vec_collide.VecCollidePark, its torch tick on the CPU, which the reference holds bit for bit to its
scalar SpaceBallpark and to Destiny's code) with a recording subclass; the tests replay them on this package's park.
A digest covers every [W, N] field the tick or a command writes (FIELDS), floats by their float64 bits with one NaN.
"""

from __future__ import annotations

import gzip
import hashlib
import json
from pathlib import Path

import numpy as np
import torch

from trace import canonical

GOLDEN = Path(__file__).resolve().parent

FIELDS = ("pos", "vel", "old_pos", "old_vel", "goto", "last_g", "last_c", "last_collision", "mode", "level", "key",
          "mod", "speed_fraction", "hits", "hits_n", "imp_slot", "imp_s", "imp_closing", "imp_n", "time_factor",
          "mass", "radius", "max_vel", "agility", "id", "exists", "free", "massive", "junk", "cloaked")
COMMANDS = ("goto_point", "goto_direction", "stop", "set_speed_fraction")


def field_digests(park) -> np.ndarray:
    out = np.zeros(len(FIELDS), dtype=np.uint64)
    for i, f in enumerate(FIELDS):
        a = canonical(getattr(park, f))
        h = hashlib.sha256(f.encode() + str(a.shape).encode() + a.tobytes()).digest()
        out[i] = np.frombuffer(h[:8], dtype=np.uint64)[0]
    return out


def _jf(x):
    return float(x).hex() if isinstance(x, float) else x


def _ball_json(b: dict) -> dict:
    return {k: ([_jf(float(c)) for c in v] if isinstance(v, (list, tuple)) else
                (v if isinstance(v, bool) else _jf(v))) for k, v in b.items()}


def _unhex(x):
    """A float written by float.hex() back to its value; any other string (a static collidable's kind) as it is."""
    if isinstance(x, str) and (x.lstrip("-").startswith("0x") or x in ("inf", "-inf", "nan")):
        return float.fromhex(x)
    return x


def recording(park_cls):
    """A subclass of park_cls recording its load, its commands (masks and values at the masked slots) and a digest
    after every tick into self.trace."""

    class Recording(park_cls):
        def __init__(self, worlds, slots, *args, **kw):
            super().__init__(worlds, slots, *args, **kw)
            self._depth = 0
            self.trace = {"W": int(worlds), "N": int(slots), "S": int(kw.get("statics", 0)),
                          "friction": float(self.friction), "tick_interval_ms": int(round(self.dt * 1000)),
                          "worlds": None, "statics": None, "events": [], "field_digests": []}

        def load(self, worlds, statics=None):
            self.trace["worlds"] = [[_ball_json(b) for b in w] for w in worlds]
            if statics is not None:
                self.trace["statics"] = [[_ball_json(x) for x in w] for w in statics]
                super().load(worlds, statics)
                self.trace["filing"] = {"s_geo": self.s_geo.cpu().numpy().copy(),
                                        "s_int": self.s_int.cpu().numpy().copy(),
                                        "s_keys": self.s_keys.cpu().numpy().copy(),
                                        "s_exists": self.s_exists.cpu().numpy().copy()}
            else:
                super().load(worlds)

        def evolve(self, *a, **k):
            if a or k:
                raise ValueError("a masked or skipping tick is not recorded")
            super().evolve()
            self.trace["events"].append({"tick": 1})
            self.trace["field_digests"].append(field_digests(self))

    def make(name):
        base = getattr(park_cls, name)

        def wrapped(self, mask, *args):
            if self._depth == 0:                     # a command's own inner calls (GotoDirection's GotoPoint) are not
                m = torch.as_tensor(mask).detach().cpu().to(torch.bool)     # events
                idx = torch.nonzero(m).tolist()
                vals, cols = [], []
                for a in args:
                    t = torch.as_tensor(a).detach().cpu().to(torch.float64)
                    cols.append(int(t.shape[2]) if t.dim() == 3 else 0)
                    vals.append([[float(x).hex() for x in t[w, j].reshape(-1).tolist()] for w, j in idx])
                self.trace["events"].append({"call": name, "at": idx, "args": vals, "cols": cols})
            self._depth += 1
            try:
                return base(self, mask, *args)
            finally:
                self._depth -= 1
        wrapped.__name__ = name
        return wrapped

    for name in COMMANDS:
        setattr(Recording, name, make(name))
    return Recording


def save(traces: list, path: Path) -> None:
    bodies = [{k: v for k, v in t.items() if k not in ("field_digests", "filing")} for t in traces]
    with gzip.open(str(path) + ".json.gz", "wt") as f:
        json.dump({"groups": bodies}, f)
    arrays = {f"g{i}_field_digests": np.array(t["field_digests"], dtype=np.uint64).reshape(-1, len(FIELDS))
              for i, t in enumerate(traces)}
    for i, t in enumerate(traces):
        for k, v in (t.get("filing") or {}).items():
            arrays[f"g{i}_{k}"] = v
    np.savez_compressed(str(path) + ".npz", **arrays)


def load(path: Path) -> list:
    with gzip.open(str(path) + ".json.gz", "rt") as f:
        groups = json.load(f)["groups"]
    z = np.load(str(path) + ".npz")
    for i, g in enumerate(groups):
        g["worlds"] = [[{k: ([_unhex(c) for c in v] if isinstance(v, list) else _unhex(v)) for k, v in b.items()}
                        for b in w] for w in g["worlds"]]
        g["field_digests"] = z[f"g{i}_field_digests"]
        g["statics"] = [[{k: ([_unhex(c) for c in v] if isinstance(v, list) else _unhex(v)) for k, v in x.items()}
                         for x in w] for w in g["statics"]] if g.get("statics") else None
        g["filing"] = {k: z[f"g{i}_{k}"] for k in ("s_geo", "s_int", "s_keys", "s_exists") if f"g{i}_{k}" in z.files}
    return groups


def replay(g: dict, park, on_tick) -> None:
    """Drive `park` (already constructed with g's W, N and tick) through the trace: the load, then every event;
    on_tick(k, park) after tick k."""
    if g.get("statics"):
        park.load(g["worlds"], g["statics"])
    else:
        park.load(g["worlds"])
    dev = park.dev
    k = 0
    for ev in g["events"]:
        if "tick" in ev:
            park.evolve()
            on_tick(k, park)
            k += 1
            continue
        mask = torch.zeros(g["W"], g["N"], dtype=torch.bool)
        args = [torch.zeros(g["W"], g["N"], c, dtype=torch.float64) if c else
                torch.zeros(g["W"], g["N"], dtype=torch.float64) for c in ev["cols"]]
        for n, (w, j) in enumerate(ev["at"]):
            mask[w, j] = True
            for t, a in zip(args, ev["args"]):
                vals = [float.fromhex(x) for x in a[n]]
                if t.dim() == 3:
                    t[w, j] = torch.tensor(vals, dtype=torch.float64)
                else:
                    t[w, j] = vals[0]
        getattr(park, ev["call"])(mask.to(dev), *[t.to(dev) for t in args])


def first_mismatch(g: dict, k: int, fd: np.ndarray) -> list:
    want = g["field_digests"][k]
    return [FIELDS[i] for i in range(len(FIELDS)) if want[i] != fd[i]]
