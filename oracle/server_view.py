"""TEST INFRASTRUCTURE, NOT THE PRODUCT. The CPU oracle's parks (oracle/park.py's OraclePark, oracle/collide_park.py's
OracleCollidePark, their ticks the C++ oracle) seen through torch: every array as a CPU tensor sharing its memory, every
assignment of a tensor stored back as numpy, so that the server layer's torch path (exact_ballpark_b200.server's
VecServer with its ModesAdapter or CollideAdapter) runs on the CPU over the oracle's park, and its replays of the
reference's server goldens check the layer's logic without a GPU. Only tests/ use it.

Two things the oracle's flight park does not carry are stated here from the reference park's API: StopAllFollowers of a set of
rows (`_release_followers`, vec_modes.py:388: a member's Stop, an interactive orbiter sent along its velocity) and
OnTick's per-world mask on the flight park's tick (`evolve(active=...)`: every row ticked, then the rows outside the
mask given back their state, as the reference's masked tick does, vec_orient.py:217; the collision oracle masks its
worlds itself).
"""

from __future__ import annotations

import numpy as np
import torch

from .park import ORBIT


class OracleParkView:
    """An OraclePark whose arrays read as CPU tensors (module docstring)."""

    def __init__(self, park, threads: int = 1):
        object.__setattr__(self, "_park", park)
        object.__setattr__(self, "_threads", int(threads))

    def __getattr__(self, name):
        v = getattr(self._park, name)
        if isinstance(v, np.ndarray):
            return torch.from_numpy(np.ascontiguousarray(v))
        return v

    def __setattr__(self, name, value):
        if torch.is_tensor(value):
            value = value.detach().cpu().numpy().copy()
        setattr(self._park, name, value)

    @property
    def dev(self):
        return torch.device("cpu")

    def _release_followers(self, rows) -> None:
        p = self._park
        rows = np.asarray(rows.cpu() if torch.is_tensor(rows) else rows, dtype=bool)
        members = p._members(rows)
        orbiter = members & p.interactive & (p.mode == ORBIT)
        p._stop_rows(members & ~orbiter)
        p.goto_direction(orbiter, p.vel.copy())

    def evolve(self, lib=None, active=None) -> None:
        p = self._park
        if active is None:
            p.evolve(threads=self._threads)
            return
        if hasattr(p, "W"):                                 # the collision oracle masks its worlds itself
            p.evolve(active=np.asarray(active.cpu() if torch.is_tensor(active) else active, dtype=bool),
                     threads=self._threads)
            return
        act = np.asarray(active.cpu() if torch.is_tensor(active) else active, dtype=bool).reshape(p.n)
        names = [k for k, v in vars(p).items() if isinstance(v, np.ndarray) and v.shape[:1] == (p.n,)]
        before = {k: getattr(p, k).copy() for k in names}
        p.evolve(threads=self._threads)
        for k, old in before.items():
            cur = getattr(p, k)
            sel = act.reshape((p.n,) + (1,) * (cur.ndim - 1))
            setattr(p, k, np.where(sel, cur, old).astype(old.dtype))
