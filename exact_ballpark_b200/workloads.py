"""Seeded synthetic worlds for the flight-mode park: the batched destiny tick's benchmark and parity workloads.

`flight_worlds` builds W independent worlds of S ships each, every world from its own seed (base seed + world
index), in the shape the flight-mode benchmark is quoted on: positions uniform in a +-50 km cube, at rest; maximum
velocity log-uniform in [100, 3000] m/s; mass log-uniform in [1e6, 1e9] kg; agility uniform in [0.1, 5]; radius
uniform in [20, 500] m; each ship FOLLOW, ORBIT or WARP uniformly at random. A follower or orbiter targets a uniform
other ship of its world at a range uniform in [500, 30,000] m; a warper aims at a point 10^U(8, 11) m away in a
uniform direction, with the thunker's minimum range (20 km) and a warp factor uniform in [3000, 10000] (the
reference's flight benchmark's span). Half the ships are interactive (an interactive orbiter flies on when its
target warps off). Dynamical orientation's turning values are Destiny's defaults.

The worlds are plain data (`rows`, and the commands as row masks and values), applied through the park's public
API (`apply`), so the same world can be run by any implementation of that API.
"""

from __future__ import annotations

import math
import random
from dataclasses import dataclass

import numpy as np
import torch

FOLLOW, ORBIT, WARP = 1, 4, 3          # Destiny's DSTBALL_FOLLOW, DSTBALL_ORBIT, DSTBALL_WARP


@dataclass
class FlightWorlds:
    rows: list                          # load() rows, world-major, ships in id order
    follow_mask: list
    orbit_mask: list
    warp_mask: list
    target: list                        # the target's row (followers and orbiters), -1 otherwise
    range_: list
    point: list                         # the warp point ([x, y, z]), zeros otherwise
    warp_factor: list
    worlds: int
    ships: int

    def apply(self, park) -> None:
        """The initial commands, through the park's API: FollowBall, Orbit and WarpTo on their rows."""
        self.packed().apply(park)

    def packed(self) -> "PackedWorlds":
        """The same worlds as numpy columns (made once): what a park's load_columns and the commands take."""
        if getattr(self, "_packed", None) is None:
            from .modes import rows_to_columns
            n = len(self.rows)
            self._packed = PackedWorlds(
                rows_to_columns(self.rows), np.array(self.follow_mask, dtype=bool).reshape(n),
                np.array(self.orbit_mask, dtype=bool).reshape(n), np.array(self.warp_mask, dtype=bool).reshape(n),
                np.array(self.target, dtype=np.int64).reshape(n), np.array(self.range_, dtype=np.float64).reshape(n),
                np.array(self.point, dtype=np.float64).reshape(n, 3),
                np.array(self.warp_factor, dtype=np.int64).reshape(n), self.worlds)
        return self._packed

    @property
    def sizes(self) -> list:
        """Each world's rows, in order."""
        out = []
        for r in self.rows:
            if not out or r["world"] != last:
                out.append(0)
                last = r["world"]
            out[-1] += 1
        return out

    @staticmethod
    def concat(parts: list) -> "FlightWorlds":
        """Several FlightWorlds as one: worlds renumbered in order, targets moved with their rows. Each world loads
        and takes its commands as it does alone (a park's load and commands act on each world's own rows)."""
        rows, fm, om, wm, tgt, rg, pt, wf = [], [], [], [], [], [], [], []
        world = 0
        for part in parts:
            base = len(rows)
            first = part.rows[0]["world"] if part.rows else 0
            for r in part.rows:
                q = dict(r)
                q["world"] = world + (r["world"] - first)
                rows.append(q)
            world += part.worlds
            fm += part.follow_mask
            om += part.orbit_mask
            wm += part.warp_mask
            tgt += [t + base if t >= 0 else -1 for t in part.target]
            rg += part.range_
            pt += part.point
            wf += part.warp_factor
        ships = max((p.ships for p in parts), default=0)
        return FlightWorlds(rows, fm, om, wm, tgt, rg, pt, wf, world, ships)


@dataclass
class PackedWorlds:
    """Worlds as columns: the load columns (exact_ballpark_b200.modes.rows_to_columns) and the initial commands as
    arrays, one entry a row. `concat` joins several (worlds renumbered, targets moved with their rows) with numpy
    alone, and `load` + `apply` give a park the same state as FlightWorlds.rows and FlightWorlds.apply."""
    cols: dict
    follow_mask: np.ndarray
    orbit_mask: np.ndarray
    warp_mask: np.ndarray
    target: np.ndarray
    range_: np.ndarray
    point: np.ndarray
    warp_factor: np.ndarray
    worlds: int

    @property
    def n(self) -> int:
        return len(self.target)

    def load(self, park) -> None:
        park.load_columns(self.cols)

    def apply(self, park) -> None:
        dev = park.dev
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        rng = t(self.range_)
        park.follow(t(self.follow_mask), t(self.target), rng)
        park.orbit(t(self.orbit_mask), t(self.target), rng)
        park.warp_to(t(self.warp_mask), t(self.point), torch.full_like(rng, 20000.0), t(self.warp_factor))

    @staticmethod
    def concat(parts: list) -> "PackedWorlds":
        sizes = [p.n for p in parts]
        base = np.concatenate(([0], np.cumsum(sizes)[:-1])).astype(np.int64)
        wbase = np.concatenate(([0], np.cumsum([p.worlds for p in parts])[:-1])).astype(np.int64)
        cols = {}
        for key in parts[0].cols:
            if key == "world":
                cols[key] = np.concatenate([p.cols[key] - (p.cols[key][0] if p.n else 0) + wb
                                            for p, wb in zip(parts, wbase)])
            else:
                cols[key] = np.concatenate([p.cols[key] for p in parts])
        target = np.concatenate([np.where(p.target >= 0, p.target + b, -1) for p, b in zip(parts, base)])
        cat = lambda k: np.concatenate([getattr(p, k) for p in parts])
        return PackedWorlds(cols, cat("follow_mask"), cat("orbit_mask"), cat("warp_mask"), target, cat("range_"),
                            cat("point"), cat("warp_factor"), int(sum(p.worlds for p in parts)))


def _unit(r: random.Random) -> list:
    while True:
        v = [r.gauss(0.0, 1.0) for _ in range(3)]
        n = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
        if n > 1e-9:
            return [c / n for c in v]


def flight_worlds(seed: int, worlds: int, ships: int = 4) -> FlightWorlds:
    """W worlds of S ships (module docstring); world w is drawn from random.Random(seed * 1_000_003 + w)."""
    rows, fm, om, wm, tgt, rg, pt, wf = [], [], [], [], [], [], [], []
    for w in range(worlds):
        r = random.Random(seed * 1_000_003 + w)
        base = w * ships
        for j in range(ships):
            rows.append({
                "id": base + j + 1, "world": w, "time": 0,
                "mass": 10.0 ** r.uniform(6.0, 9.0), "radius": r.uniform(20.0, 500.0),
                "max_vel": 10.0 ** r.uniform(2.0, math.log10(3000.0)),
                "pos": [r.uniform(-5e4, 5e4) for _ in range(3)], "vel": [0.0, 0.0, 0.0],
                "agility": r.uniform(0.1, 5.0), "speed_fraction": 1.0, "free": True, "massive": False,
                "interactive": r.random() < 0.5,
            })
            mode = r.choice((FOLLOW, ORBIT, WARP)) if ships > 1 else WARP
            fm.append(mode == FOLLOW)
            om.append(mode == ORBIT)
            wm.append(mode == WARP)
            if mode in (FOLLOW, ORBIT):
                other = r.randrange(ships - 1)
                tgt.append(base + (other if other < j else other + 1))
                rg.append(r.uniform(500.0, 30000.0))
                pt.append([0.0, 0.0, 0.0])
                wf.append(0)
            else:
                d = 10.0 ** r.uniform(8.0, 11.0)
                u = _unit(r)
                p = rows[-1]["pos"]
                tgt.append(-1)
                rg.append(0.0)
                pt.append([p[0] + u[0] * d, p[1] + u[1] * d, p[2] + u[2] * d])
                wf.append(r.randint(3000, 10000))
    return FlightWorlds(rows, fm, om, wm, tgt, rg, pt, wf, worlds, ships)


def ragged_flight_worlds(seed: int, worlds: int, max_ships: int = 128) -> FlightWorlds:
    """W flight-mode worlds of ragged size (ship counts log-uniform in [1, max_ships], the ragged benchmark's shape;
    world w drawn as flight_worlds(seed * 1_000_003 + w, 1, size)), concatenated with ids restarting in each world."""
    r = random.Random(seed)
    return FlightWorlds.concat([flight_worlds(seed * 1_000_003 + w, 1, ragged_ships(r, max_ships))
                                for w in range(worlds)])


def ragged_ships(r: random.Random, max_ships: int) -> int:
    """A world's ship count, log-uniform in [1, max_ships] (floor of 10^U(0, log10 max_ships))."""
    return max(1, min(max_ships, int(10.0 ** r.uniform(0.0, math.log10(max_ships)))))


# ============================================================================ collisions with static spheres

@dataclass
class CollideWorlds:
    """Worlds for the collision park (exact_ballpark_b200.collide.VecCollidePark): `worlds` (each a list of the
    load's ball dicts), `collidables` (each world's capsules and oriented boxes, or None) and the ships' GOTO aims,
    {step: [(world, ball id, point)]} (step 1 is before the first tick)."""
    worlds: list
    aims: dict
    ships: int
    spheres: int
    statics: int
    collidables: list | None = None

    def apply(self, park, step: int) -> None:
        """The aims of `step` through the park's API: one GotoPoint call with every aimed ship's point."""
        todo = self.aims.get(step)
        if not todo:
            return
        mask = torch.zeros(park.W, park.N, dtype=torch.bool)
        point = torch.zeros(park.W, park.N, 3, dtype=torch.float64)
        ids = torch.as_tensor(park.id).detach().cpu()
        for w, bid, p in todo:
            j = int((ids[w] == bid).nonzero()[0, 0])
            mask[w, j] = True
            point[w, j] = torch.tensor(p, dtype=torch.float64)
        if isinstance(park.id, torch.Tensor):
            park.goto_point(mask.to(park.dev), point.to(park.dev))
        else:                                    # a numpy park (the CPU oracle)
            park.goto_point(mask.numpy(), point.numpy())


def collide_worlds(seed: int, worlds: int, ships: int = 4, spheres: int = 4, statics: int = 8, ticks: int = 500,
                   reaim: int = 25) -> CollideWorlds:
    """W worlds of `ships` ships, `spheres` free massive spheres and `statics` fixed spheres, everything in a +-20 km
    cube, each world from random.Random(seed * 1_000_003 + w). Ships as the flight-mode benchmark draws them (mass
    log-uniform 1e6-1e9 kg, radius 20-500 m, max velocity log-uniform 100-3000 m/s, agility 0.1-5); spheres of radius
    log-uniform 10 m-5 km, mass log-uniform 1e6-1e10 kg (the free ones; a fixed sphere is immovable whatever its
    mass); free balls start with a velocity of uniform direction and a speed uniform up to their maximum. Every ship
    flies GOTO at a sphere's centre, re-aimed at another random sphere every `reaim` ticks (the aims are harness
    choices), so that overlaps and gradient pushes occur every tick."""
    out, aims = [], {}
    lg = math.log10
    for w in range(worlds):
        r = random.Random(seed * 1_000_003 + w)
        balls = []
        bid = 0
        for kind, count in (("ship", ships), ("sphere", spheres), ("static", statics)):
            for _ in range(count):
                bid += 1
                free = kind != "static"
                if kind == "ship":
                    mass, radius = 10.0 ** r.uniform(6.0, 9.0), r.uniform(20.0, 500.0)
                    max_vel, agility = 10.0 ** r.uniform(2.0, lg(3000.0)), r.uniform(0.1, 5.0)
                else:
                    mass, radius = 10.0 ** r.uniform(6.0, 10.0), 10.0 ** r.uniform(1.0, lg(5000.0))
                    max_vel, agility = 10.0 ** r.uniform(2.0, lg(3000.0)), 1.0
                pos = [r.uniform(-2e4, 2e4) for _ in range(3)]
                vel = [0.0, 0.0, 0.0]
                if free:
                    u = _unit(r)
                    sp = r.uniform(0.0, max_vel)
                    vel = [c * sp for c in u]
                balls.append({"id": bid, "mass": mass, "radius": radius, "max_vel": max_vel, "agility": agility,
                              "speed_fraction": 1.0, "pos": pos, "vel": vel, "free": free, "massive": True})
        out.append(balls)
        targets = [b for b in balls if b["id"] > ships]
        for step in range(1, ticks + 1, reaim):
            for s in range(ships):
                t = r.choice(targets)
                aims.setdefault(step, []).append((w, s + 1, list(t["pos"])))
    return CollideWorlds(out, aims, ships, spheres, statics)


def _frame(r: random.Random) -> tuple:
    """Three orthonormal directions, uniformly oriented (Gram-Schmidt of two random unit vectors)."""
    u = _unit(r)
    while True:
        v = _unit(r)
        d = sum(u[i] * v[i] for i in range(3))
        w = [v[i] - d * u[i] for i in range(3)]
        n = math.sqrt(sum(c * c for c in w))
        if n > 1e-3:
            w = [c / n for c in w]
            break
    x = [u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]]
    return u, w, x


def collide_statics_worlds(seed: int, worlds: int, ships: int = 4, spheres: int = 4, statics: int = 8,
                           ticks: int = 500, reaim: int = 25) -> CollideWorlds:
    """The collision benchmark's static-collidable shape: W worlds of `ships` ships and `spheres` fixed spheres (the
    balls), and `statics` static collidables, half capsules and half oriented boxes, in a +-20 km cube, world w from
    random.Random(seed * 1_000_003 + w). Ships as collide_worlds draws them; fixed spheres of radius log-uniform
    10 m - 5 km; a capsule of radius log-uniform 30-500 m along a uniform direction, 100 m - 2 km long; a box of
    edges log-uniform 100 m - 5 km on a uniformly oriented frame. Every ship flies GOTO at a static collidable's
    centre or a sphere's, re-aimed every `reaim` ticks (harness choices, as in collide_worlds)."""
    out, coll, aims = [], [], {}
    lg = math.log10
    for w in range(worlds):
        r = random.Random(seed * 1_000_003 + w)
        balls, items, centres = [], [], []
        bid = 0
        for kind, count in (("ship", ships), ("sphere", spheres)):
            for _ in range(count):
                bid += 1
                if kind == "ship":
                    mass, radius = 10.0 ** r.uniform(6.0, 9.0), r.uniform(20.0, 500.0)
                    max_vel, agility = 10.0 ** r.uniform(2.0, lg(3000.0)), r.uniform(0.1, 5.0)
                else:
                    mass, radius, max_vel, agility = 10.0 ** r.uniform(6.0, 10.0), 10.0 ** r.uniform(1.0, lg(5000.0)), \
                        0.0, 1.0
                pos = [r.uniform(-2e4, 2e4) for _ in range(3)]
                vel = [0.0, 0.0, 0.0]
                if kind == "ship":
                    u = _unit(r)
                    sp = r.uniform(0.0, max_vel)
                    vel = [c * sp for c in u]
                else:
                    centres.append(pos)
                balls.append({"id": bid, "mass": mass, "radius": radius, "max_vel": max_vel, "agility": agility,
                              "speed_fraction": 1.0, "pos": pos, "vel": vel, "free": kind == "ship", "massive": True})
        for k in range(statics):
            sid = 1000 + k
            c = [r.uniform(-1.8e4, 1.8e4) for _ in range(3)]
            if k % 2 == 0:
                u = _unit(r)
                half = r.uniform(100.0, 2000.0) / 2.0
                a = [c[i] - u[i] * half for i in range(3)]
                b = [c[i] + u[i] * half for i in range(3)]
                items.append({"kind": "capsule", "id": sid, "parent": 0, "a": a, "b": b,
                              "radius": 10.0 ** r.uniform(lg(30.0), lg(500.0))})
            else:
                f = _frame(r)
                e = [10.0 ** r.uniform(2.0, lg(5000.0)) for _ in range(3)]
                edges = [[f[j][i] * e[j] for i in range(3)] for j in range(3)]
                corner = [c[i] - (edges[0][i] + edges[1][i] + edges[2][i]) / 2.0 for i in range(3)]
                items.append({"kind": "box", "id": sid, "parent": 0, "corner": corner, "lx": edges[0],
                              "ly": edges[1], "lz": edges[2]})
            centres.append(c)
        out.append(balls)
        coll.append(items)
        for step in range(1, ticks + 1, reaim):
            for s in range(ships):
                aims.setdefault(step, []).append((w, s + 1, list(r.choice(centres))))
    return CollideWorlds(out, aims, ships, spheres, statics, coll)


# ============================================================================ the combat park

GOTO, FORMATION_MODE = 0, 12
COMBAT_FORMATIONS = [[[0.0, 0.0, -1.0], [1.0, 0.0, -1.0], [-1.0, 0.0, -1.0], [0.0, 1.0, -2.0]],
                     [[3.0, 0.0, 0.0], [-3.0, 0.0, 0.0], [0.0, 3.0, 0.0]]]


@dataclass
class CombatWorlds:
    """Worlds for the combat park (exact_ballpark_b200.combat.VecCombatPark): each world its ships (ids 1 .. S) and
    its missile rows (ids 101 .., empty until the set-up adds them), as `load` rows; the set-up's commands as row
    arrays, applied through the park's public API by `apply` (so any implementation of it runs the same worlds):
    the ships' modes (FOLLOW, ORBIT or GOTO; in half the worlds ship 1 leads formation 0 or 1 with ship 2 in a slot),
    then each missile added at its launcher and launched (aimed, massive) at another ship of its world."""
    rows: list
    worlds: int
    ships: int
    missiles: int
    follow: np.ndarray
    orbit: np.ndarray
    goto: np.ndarray
    target: np.ndarray              # a follower's or orbiter's target row
    range_: np.ndarray
    point: np.ndarray
    leader: np.ndarray              # rows that lead a formation, with its index in `formation`
    formation: np.ndarray
    member: np.ndarray              # rows that follow their world's leader (its id in `leader_id`) in slot `slot`
    leader_id: np.ndarray
    slot: np.ndarray
    missile: np.ndarray             # the missile rows
    missile_balls: list             # their AddBall dicts, in row order
    launch_target: np.ndarray       # target and owner ids (per row)
    launch_owner: np.ndarray

    def apply(self, park) -> None:
        dev = park.dev
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        park.load_formations(COMBAT_FORMATIONS)
        park.follow(t(self.follow), t(self.target), t(self.range_))
        park.orbit(t(self.orbit), t(self.target), t(self.range_))
        park.goto_point(t(self.goto), t(self.point))
        park.set_ball_formation(t(self.leader), t(self.formation))
        park.formation_follow(t(self.member), t(self.leader_id), t(self.slot))
        park.add_balls(t(self.missile), self.missile_balls)
        one = torch.ones(len(self.rows), dtype=torch.int64, device=dev)
        park.launch_missile(t(self.missile), t(self.launch_target), t(self.launch_owner), one, one)


def combat_worlds(seed: int, worlds: int, ships: int = 4, missiles: int = 4, spheres: int = 0,
                  massive: bool = False, cube: float = 2e4) -> CombatWorlds:
    """W combat worlds (CombatWorlds); world w drawn from random.Random(seed * 1_000_003 + w): ships as the flight
    benchmark's (positions in a +-20 km cube, at rest, maximum velocity log-uniform in [100, 3000] m/s, mass
    log-uniform in [1e6, 1e9] kg, agility uniform in [0.1, 5], radius uniform in [20, 500] m, non-massive), each
    FOLLOW or ORBIT of another ship at 500 - 30,000 m or GOTO a point in the cube; missiles of mass 10^U(3, 5) kg,
    radius U(1, 6) m, maximum velocity U(3000, 8000) m/s, agility U(0.01, 0.2), each launched by a random ship at a
    random other one. For the composed park: `massive` ships, `spheres` fixed massive spheres a world (ids after the
    ships; radius log-uniform in [10, 5000] m, mass log-uniform in [1e8, 1e11] kg) and a smaller `cube`."""
    n = worlds * (ships + spheres + missiles)
    rows = []
    follow, orbit, goto = (np.zeros(n, dtype=bool) for _ in range(3))
    target = np.full(n, -1, dtype=np.int64)
    range_ = np.zeros(n)
    point = np.zeros((n, 3))
    leader, member, missile = (np.zeros(n, dtype=bool) for _ in range(3))
    formation, leader_id, slot = (np.zeros(n, dtype=np.int64) for _ in range(3))
    launch_target, launch_owner = np.zeros(n, dtype=np.int64), np.zeros(n, dtype=np.int64)
    balls = []
    for w in range(worlds):
        r = random.Random(seed * 1_000_003 + w)
        base = len(rows)
        for j in range(ships):
            rows.append({"id": j + 1, "world": w, "time": 0, "mass": 10.0 ** r.uniform(6.0, 9.0),
                         "radius": r.uniform(20.0, 500.0), "max_vel": 10.0 ** r.uniform(2.0, math.log10(3000.0)),
                         "pos": [r.uniform(-cube, cube) for _ in range(3)], "vel": [0.0, 0.0, 0.0],
                         "agility": r.uniform(0.1, 5.0), "speed_fraction": 1.0, "free": True, "massive": massive,
                         "interactive": j == 0 or r.random() < 0.5})
            k = base + j
            mode = r.choice((FOLLOW, ORBIT, GOTO)) if ships > 1 else GOTO
            if mode == GOTO:
                goto[k] = True
                point[k] = [r.uniform(-cube, cube) for _ in range(3)]
            else:
                other = r.randrange(ships - 1)
                target[k] = base + (other if other < j else other + 1)
                range_[k] = r.uniform(500.0, 30000.0)
                (follow if mode == FOLLOW else orbit)[k] = True
        if ships > 1 and r.random() < 0.5:                 # ship 1 leads a formation, ship 2 flies in a slot
            leader[base] = True
            formation[base] = r.randrange(len(COMBAT_FORMATIONS))
            member[base + 1] = True
            leader_id[base + 1] = 1
            slot[base + 1] = r.randrange(len(COMBAT_FORMATIONS[formation[base]]))
        for q in range(spheres):
            rows.append({"id": ships + q + 1, "world": w, "time": 0, "mass": 10.0 ** r.uniform(8.0, 11.0),
                         "radius": 10.0 ** r.uniform(1.0, math.log10(5000.0)), "max_vel": 0.0,
                         "pos": [r.uniform(-cube, cube) for _ in range(3)], "vel": [0.0, 0.0, 0.0], "agility": 1.0,
                         "speed_fraction": 0.0, "free": False, "massive": True, "interactive": False})
        for m in range(missiles):
            k = len(rows)
            owner = r.randrange(ships)
            other = r.randrange(ships - 1) if ships > 1 else 0
            tgt = (other if other < owner else other + 1) if ships > 1 else owner
            ball = {"id": 101 + m, "mass": 10.0 ** r.uniform(3.0, 5.0), "radius": r.uniform(1.0, 6.0),
                    "max_vel": r.uniform(3000.0, 8000.0), "free": True, "massive": False, "interactive": False,
                    "pos": [0.0, 0.0, 0.0], "vel": [0.0, 0.0, 0.0], "agility": r.uniform(0.01, 0.2),
                    "speed_fraction": 1.0, "max_ang_vel": r.uniform(0.5, 3.0), "rot_agility": r.uniform(0.2, 1.0)}
            rows.append({"id": 101 + m, "world": w, "time": 0, "exists": False, "mass": 1.0, "radius": 1.0,
                         "max_vel": 1.0, "pos": [0.0, 0.0, 0.0], "vel": [0.0, 0.0, 0.0], "agility": 1.0,
                         "speed_fraction": 1.0})
            missile[k] = True
            balls.append(ball)
            launch_target[k] = tgt + 1
            launch_owner[k] = owner + 1
    return CombatWorlds(rows, worlds, ships, missiles, follow, orbit, goto, target, range_, point, leader, formation,
                        member, leader_id, slot, missile, balls, launch_target, launch_owner)


def composed_worlds(seed: int, worlds: int, ships: int = 6, missiles: int = 2, spheres: int = 1) -> CombatWorlds:
    """The composed benchmark's worlds (its shape: 6 ships, 2 missiles and 1 sphere a world): combat_worlds with
    massive ships in a +-5 km cube and fixed massive spheres among them, so ships, spheres and missiles meet."""
    return combat_worlds(seed, worlds, ships, missiles, spheres, massive=True, cube=5e3)


# ============================================================================ the partition's ragged worlds

@dataclass
class PartitionWorlds:
    """Ragged worlds for the partition layer over the flight park (bubbles, the spatial partition and proximity
    sensors, a pilot a ship): `cols` the park's load columns (world-major, each world's ships in id order from 1),
    `sizes` each world's ship count, `sensor_range` each ship's sensor radius (m), `direction` and `speed` each ship's
    pilot's GotoDirection and SetSpeedFraction (drawn once; a pilot sends them every tick)."""
    cols: dict
    sizes: np.ndarray
    sensor_range: np.ndarray
    direction: np.ndarray
    speed: np.ndarray

    @property
    def n(self) -> int:
        return int(self.sizes.sum())

    @property
    def starts(self) -> np.ndarray:
        return np.concatenate(([0], np.cumsum(self.sizes)[:-1])).astype(np.int64)


def partition_worlds(seed: int, worlds: int, max_ships: int = 128) -> PartitionWorlds:
    """W worlds of ragged size (ship counts floor(10^U(0, log10 max_ships)), clipped to [1, max_ships]; mean about 20
    for 128) with the ships clustered as 1 to 5 Gaussian blobs (sigma 10 km) a world around centres uniform in
    +-1,000 km; ship parameters as the flight benchmark draws them (mass log-uniform 1e6-1e9 kg, radius uniform
    20-500 m, maximum velocity log-uniform 100-3000 m/s, agility uniform 0.1-5), at rest, free, interactive (each has
    a pilot), not massive; a proximity sensor on every ship with a radius log-uniform in [1 km, 250 km], period 1 s.
    Numpy draws from one seeded generator, so a million ships take a second."""
    g = np.random.default_rng(seed)
    sizes = np.clip(np.floor(10.0 ** g.uniform(0.0, math.log10(max_ships), worlds)), 1, max_ships).astype(np.int64)
    n = int(sizes.sum())
    world = np.repeat(np.arange(worlds, dtype=np.int64), sizes)
    starts = np.concatenate(([0], np.cumsum(sizes)[:-1]))
    ids = np.arange(n, dtype=np.int64) - np.repeat(starts, sizes) + 1
    blobs = g.integers(1, 6, worlds)
    centres = g.uniform(-1e6, 1e6, (worlds, 5, 3))
    pick = (g.random(n) * blobs[world]).astype(np.int64)
    pos = centres[world, pick] + g.normal(0.0, 1e4, (n, 3))
    cols = {"id": ids, "world": world, "time": np.zeros(n, np.int64),
            "mass": 10.0 ** g.uniform(6.0, 9.0, n), "radius": g.uniform(20.0, 500.0, n),
            "max_vel": 10.0 ** g.uniform(2.0, math.log10(3000.0), n), "agility": g.uniform(0.1, 5.0, n),
            "speed_fraction": np.ones(n), "free": np.ones(n, bool), "massive": np.zeros(n, bool),
            "interactive": np.ones(n, bool), "moribund": np.zeros(n, bool), "cloaked": np.zeros(n, np.int64),
            "bubble": np.full(n, -1, np.int64), "mode": np.full(n, 2, np.int64),
            "max_ang_vel": np.ones(n), "rot_agility": np.full(n, 0.9), "pos": pos, "vel": np.zeros((n, 3))}
    rng = 10.0 ** g.uniform(3.0, math.log10(2.5e5), n)
    d = g.normal(0.0, 1.0, (n, 3))
    d /= np.maximum(np.linalg.norm(d, axis=1, keepdims=True), 1e-9)
    return PartitionWorlds(cols, sizes, rng, d, g.uniform(0.2, 1.0, n))


def face_worlds(seed: int, worlds: int) -> PartitionWorlds:
    """The reference's space benchmark shape (benchmarks/space_speed.py:31-56): worlds of four ships within 4 km
    (each axis uniform in +-4 km) of a point on the face between two top boxes (x at one top box's width, y and z at
    +-0.3 of it), the first ship moved half a box deeper into the first top so that its bubble comes first; mass 1e7
    kg, radius 50 m, maximum velocity 300 m/s, agility 0.5, at rest (STOP), free, interactive, not massive; a 5 km proximity
    sensor on every ship (period 1 s); GotoDirection along (1, 0.2, 0.1) for the odd ships and (-1, -0.1, 0.2) for
    the even ones, so every ship re-files every tick and crosses the face. Ids 1-4 in each world (the reference's
    101-104: the order is the same). The offsets come from this module's seeded generator, not the reference's."""
    from .statics import LEVEL_WIDTH
    top = LEVEL_WIDTH[0]
    g = np.random.default_rng(seed)
    n = 4 * worlds
    k = np.tile(np.arange(4), worlds)
    pos = np.array([top, 0.3 * top, -0.3 * top]) + g.uniform(-4000.0, 4000.0, (n, 3))
    pos[k == 0, 0] -= 0.5 * top
    cols = {"id": 1 + k, "world": np.repeat(np.arange(worlds, dtype=np.int64), 4), "time": np.zeros(n, np.int64),
            "mass": np.full(n, 1e7), "radius": np.full(n, 50.0), "max_vel": np.full(n, 300.0),
            "agility": np.full(n, 0.5), "speed_fraction": np.ones(n), "free": np.ones(n, bool),
            "massive": np.zeros(n, bool), "interactive": np.ones(n, bool), "moribund": np.zeros(n, bool),
            "cloaked": np.zeros(n, np.int64), "bubble": np.full(n, -1, np.int64), "mode": np.full(n, 2, np.int64),
            "max_ang_vel": np.ones(n), "rot_agility": np.full(n, 0.9), "pos": pos, "vel": np.zeros((n, 3))}
    d = np.where((k % 2 == 1)[:, None], np.array([1.0, 0.2, 0.1]), np.array([-1.0, -0.1, 0.2]))
    return PartitionWorlds(cols, np.full(worlds, 4, np.int64), np.full(n, 5000.0), d, np.ones(n))
