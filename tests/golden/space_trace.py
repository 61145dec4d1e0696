"""Golden traces of the master's partition and bubble partition of one world (the space layer's first slice): seeded
streams of operations (AddBall, SetBallPosition, SetBallRadius, SetMaxSpeed, RemoveBall, SetBallInteractive, a
keep-alive ball, the cloak attribute, InitializeBubbles, CopyBubbles, and the queries GetNearbyBalls, CheckVisibility,
GetBallIdsInRange from a ball or a point, GetBubbleAtCoordinates) and, after each one, the world's state as a text: each
ball's bubble, old bubble, filing box, sides, active neighbours, dead-bubble flag and boxes; the live boxes per level;
the kept boxes, the next bubble id; each bubble's dictionary in its order; the interactive and keep-alive sets; the
query's answer.

`make_golden.py` records the texts' digests by running the reference's own SpaceBallpark (exact_ballpark.space, the
master's view; its scalar transcription of Destiny's Partition and Ballpark); the tests run the same operations on the
CPU oracle (oracle/space.cpp) and compare, operation by operation.
"""

from __future__ import annotations

import hashlib
import math
import random
import struct
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent
STRIDE = 16
ADD, POS, RADIUS, MAXVEL, REMOVE, INIT, COPY, INTERACTIVE, KEEPALIVE = range(1, 10)
CLOAKED, VISIBILITY, RANGE_BALL, RANGE_POINT, BUBBLE_AT, NEARBY = range(10, 16)
SENSOR, UNSENSOR, PROXIMITIES, NOTIFY, TRACK, GOTO, STOP, TICK = range(16, 24)
FOLLOW, ORBIT, WARP = range(24, 27)
TOP = 7864320.0                                           # a top box's width (m)


def _op(code: int, bid: int = 0, *args) -> list:
    row = [float(code), float(bid)] + [float(a) for a in args]
    return row + [0.0] * (STRIDE - len(row))


def ops_for(seed: int, n_ops: int = 60) -> list:
    """One world's operations: balls added around a few centres near top-box faces and corners, moved within and
    across top boxes (joining, splitting and re-forming bubbles), resized up to huge, sped up, removed and re-added,
    made interactive or not, kept alive, and the bubble partition re-initialised and copied now and then."""
    r = random.Random(f"space-bubbles-{seed}")
    centres = [[r.choice((-1.0, 0.0, 1.0)) * TOP * r.choice((0.5, 1.0)) + r.uniform(-2e4, 2e4) for _ in range(3)]
               for _ in range(r.randint(1, 3))]
    ids, live, ops = list(range(1, 13)), [], []

    def where() -> list:
        c = r.choice(centres)
        k = r.random()
        if k < 0.5:
            return [x + r.uniform(-3e4, 3e4) for x in c]
        if k < 0.8:                                        # near a face of a finer box
            return [x + r.choice((-1.0, 1.0)) * r.uniform(0.0, 2e3) for x in c]
        return [x + r.uniform(-1.2 * TOP, 1.2 * TOP) for x in c]

    def radius() -> float:
        return r.choice([r.uniform(5.0, 300.0), r.uniform(300.0, 5e4), r.uniform(5e4, 2e6), r.uniform(4e6, 6e6)])

    for _ in range(n_ops):
        k = r.random()
        free = [b for b in ids if b not in live]
        if (k < 0.3 or not live) and free:
            b = r.choice(free)
            vel = [r.uniform(-300.0, 300.0) for _ in range(3)] if r.random() < 0.6 else [0.0, 0.0, 0.0]
            ops.append(_op(ADD, b, 10 ** r.uniform(5.0, 9.0), radius(), r.uniform(0.0, 3000.0),
                           1.0 if r.random() < 0.8 else 0.0, 1.0 if r.random() < 0.75 else 0.0, *where(), *vel,
                           r.uniform(0.05, 3.0), r.choice((0.0, 0.5, 1.0)), 1.0 if r.random() < 0.7 else 0.0))
            live.append(b)
        elif k < 0.4 and live:                             # a query
            q = r.random()
            a, c = r.choice(live), r.choice(ids)
            if q < 0.3:
                ops.append(_op(NEARBY, a, float(r.random() < 0.5), float(r.random() < 0.3), float(r.random() < 0.5)))
            elif q < 0.5:
                ops.append(_op(VISIBILITY, a, c))
            elif q < 0.7:
                ops.append(_op(RANGE_BALL, a, r.choice((1e3, 3e4, 1e6, 1e7)), float(r.random() < 0.5),
                               float(r.random() < 0.5)))
            elif q < 0.85:
                ops.append(_op(RANGE_POINT, 0, *where(), r.choice((1e3, 3e4, 1e6, 1e7)), float(r.random() < 0.5),
                               float(r.random() < 0.5)))
            else:
                ops.append(_op(BUBBLE_AT, 0, *where()))
        elif k < 0.43 and live:
            ops.append(_op(CLOAKED, r.choice(live), r.choice((0.0, 1.0, 2.0, 200.0))))
        elif k < 0.47 and live:                            # a proximity sensor on, or off
            if r.random() < 0.8:
                ops.append(_op(SENSOR, r.choice(live), r.choice((100.0, 3e4, 1e6, 5e6, -1e7)), r.choice((0.5, 1.0, 3.0)),
                               float(r.random() < 0.3), float(r.random() < 0.3)))
            else:
                ops.append(_op(UNSENSOR, r.choice(live)))
        elif k < 0.49 and live:                            # a notification range, a tracked target, a goto, a stop
            q, a = r.random(), r.choice(live)
            if q < 0.3:
                if r.random() < 0.6:
                    ops.append(_op(GOTO, a, *where()))
                ops.append(_op(NOTIFY, a, r.choice((0.0, 500.0, 5e4, 1e7, 1e7, -1.0))))
            elif q < 0.6:
                target = r.choice(live) if r.random() < 0.85 else r.choice(ids + [0])
                ops.append(_op(TRACK, a, target, r.choice((0.0, 1e3, 1e5, 1e7, 1e7))))
            elif q < 0.85:
                ops.append(_op(GOTO, a, *where()))
            else:
                ops.append(_op(STOP, a))
        elif k < 0.53:
            ops.append(_op(PROXIMITIES))
        elif k < 0.55:
            ops.append(_op(POS, r.choice(live), *where()))
        elif k < 0.62:
            ops.append(_op(RADIUS, r.choice(live), radius() if r.random() < 0.9 else -1.0))
        elif k < 0.67:
            ops.append(_op(MAXVEL, r.choice(live), r.uniform(0.0, 1e5)))
        elif k < 0.74:
            b = r.choice(live)
            ops.append(_op(REMOVE, b))
            live.remove(b)
        elif k < 0.82:
            ops.append(_op(INTERACTIVE, r.choice(live), float(r.random() < 0.5)))
        elif k < 0.86:
            ops.append(_op(KEEPALIVE, r.choice(ids)))
        elif k < 0.93:
            ops.append(_op(COPY))
        else:
            ops.append(_op(INIT))
    return ops


def sweep_ops(seed: int) -> list:
    """A world that releases more boxes than BoxAllocator keeps: a dozen huge balls (27 top boxes each) far apart,
    a few small ones among them, then every huge ball removed (past 256 kept boxes the released ones are deleted), new
    balls added (taking kept boxes), the partition re-initialised and copied."""
    r = random.Random(f"space-sweep-{seed}")
    ops = []
    for b in range(1, 13):
        c = [(b - 6) * 4.0 * TOP, r.uniform(-TOP, TOP), r.uniform(-TOP, TOP)]
        ops.append(_op(ADD, b, 1e8, r.uniform(4.0e6, 4.5e6), 0.0, 0.0, float(b % 3 == 0), *c, 0.0, 0.0, 0.0, 1.0,
                       1.0))
    for b in range(20, 26):
        c = [r.uniform(-20.0, 20.0) * TOP, r.uniform(-TOP, TOP), r.uniform(-TOP, TOP)]
        ops.append(_op(ADD, b, 1e7, r.uniform(10.0, 500.0), 200.0, 1.0, 1.0, *c, 50.0, 0.0, 0.0, 1.0, 1.0))
    ops.append(_op(COPY))
    for b in r.sample(range(1, 13), 12):
        ops.append(_op(REMOVE, b))
    for b in range(30, 36):
        c = [r.uniform(-20.0, 20.0) * TOP, r.uniform(-TOP, TOP), r.uniform(-TOP, TOP)]
        ops.append(_op(ADD, b, 1e7, r.choice((100.0, 3e5, 4.2e6)), 200.0, 1.0, 1.0, *c, 0.0, 0.0, 0.0, 1.0, 1.0))
    ops += [_op(INIT), _op(COPY)]
    for b in (20, 21, 30):
        ops.append(_op(POS, b, r.uniform(-20.0, 20.0) * TOP, 0.0, 0.0))
    return ops


def _bits(x: float) -> str:
    return "%016x" % struct.unpack("<Q", struct.pack("<d", float(x)))[0]


def tick_ops(seed: int, n_ops: int = 80) -> list:
    """A world that ticks: up to 10 non-massive ships near top-box faces (so that they cross top boxes within a few
    ticks), flying GOTO legs at up to 3 km/s across boxes and bubbles, stopped, moved, with sensors, tracked targets
    and notification ranges, the bubble partition re-initialised and copied, balls made interactive or not and
    removed; a tick between most operations."""
    r = random.Random(f"space-tick-{seed}")
    centres = [[r.choice((-1.0, 0.0, 1.0)) * TOP + r.uniform(-4e3, 4e3) for _ in range(3)] for _ in range(r.randint(1, 3))]
    ids, live, ops = list(range(1, 11)), [], []

    def near() -> list:
        return [x + r.uniform(-6e3, 6e3) for x in r.choice(centres)]

    def add(b: int) -> None:
        vel = [r.uniform(-300.0, 300.0) for _ in range(3)] if r.random() < 0.6 else [0.0, 0.0, 0.0]
        ops.append(_op(ADD, b, 10 ** r.uniform(5.0, 9.0), r.choice((r.uniform(5.0, 300.0), r.uniform(300.0, 3e4),
                                                                     r.uniform(3e4, 1e6))),
                       r.uniform(50.0, 3000.0), 1.0 if r.random() < 0.9 else 0.0, 1.0 if r.random() < 0.75 else 0.0,
                       *near(), *vel, r.uniform(0.1, 3.0), r.choice((0.5, 1.0)), 0.0))
        live.append(b)
    for b in r.sample(ids, r.randint(3, 8)):
        add(b)
    for _ in range(n_ops):
        k = r.random()
        free = [b for b in ids if b not in live]
        a = r.choice(live) if live else None
        if k < 0.45 or a is None:
            ops.append(_op(TICK))
        elif k < 0.6:
            far = [x + r.choice((-1.0, 1.0)) * r.uniform(1e5, 3e7) for x in near()]
            ops.append(_op(GOTO, a, *far))
        elif k < 0.63:
            ops.append(_op(STOP, a))
        elif k < 0.7:
            ops.append(_op(SENSOR, a, r.choice((100.0, 3e4, 1e6)), r.choice((0.5, 1.0, 3.0)), float(r.random() < 0.3),
                           float(r.random() < 0.3)))
        elif k < 0.74:
            ops.append(_op(TRACK, a, r.choice(live), r.choice((1e3, 1e5, 1e7))))
        elif k < 0.78:
            ops.append(_op(NOTIFY, a, r.choice((500.0, 5e4, 1e7))))
        elif k < 0.81:
            ops.append(_op(POS, a, *near()))
        elif k < 0.84:
            ops.append(_op(INIT))
        elif k < 0.88:
            ops.append(_op(COPY))
        elif k < 0.92:
            ops.append(_op(INTERACTIVE, a, float(r.random() < 0.6)))
        elif k < 0.95 and free:
            add(r.choice(free))
        elif k < 0.97:
            ops.append(_op(REMOVE, a))
            live.remove(a)
        else:
            ops.append(_op(NEARBY, a, 1.0, 0.0, 0.0))
    return ops


def mode_ops(seed: int, n_ops: int = 110) -> list:
    """A world of the follow, orbit and warp modes: up to 10 light non-massive ships (a time constant of 0.01 to 10 s,
    some with a top speed under 0.6 m/s, so that their warps drop out nearly at rest and are re-filed there) around
    one or two centres near top-box faces, following and orbiting one another, warping 0.3 to 30 Mm at warp factors
    of 1,000 to 30,000 (a few tens of ticks a warp), sent along GOTO legs, stopped, re-added (which keeps a follower's
    target pointer), removed (which releases its followers), with sensors, notification ranges and the bubble partition
    re-initialised;
    runs of ticks between the commands."""
    r = random.Random(f"space-modes-{seed}")
    centres = [[r.choice((-1.0, 0.0, 1.0)) * TOP + r.uniform(-4e3, 4e3) for _ in range(3)] for _ in range(r.randint(1, 2))]
    ids, live, ops = list(range(1, 11)), [], []

    def near() -> list:
        return [x + r.uniform(-5e3, 5e3) for x in r.choice(centres)]

    def add(b: int) -> None:
        vel = [r.uniform(-100.0, 100.0) for _ in range(3)] if r.random() < 0.5 else [0.0, 0.0, 0.0]
        max_vel = r.uniform(0.2, 0.6) if r.random() < 0.2 else r.uniform(50.0, 500.0)
        ops.append(_op(ADD, b, 10 ** r.uniform(5.0, 7.0), r.uniform(5.0, 3e3), max_vel,
                       1.0 if r.random() < 0.9 else 0.0, 1.0 if r.random() < 0.6 else 0.0, *near(), *vel,
                       r.uniform(0.1, 1.0), 1.0 if r.random() < 0.8 else 0.5, 0.0))
        if b not in live:
            live.append(b)
    for b in r.sample(ids, r.randint(3, 8)):
        add(b)
    for _ in range(n_ops):
        k = r.random()
        a = r.choice(live) if live else None
        if k < 0.4 or a is None:
            ops.extend(_op(TICK) for _ in range(r.choice((1, 1, 3, 10))))
        elif k < 0.52:
            ops.append(_op(FOLLOW, a, r.choice(live), r.choice((0.0, 50.0, 2e3))))
        elif k < 0.62:
            ops.append(_op(ORBIT, a, r.choice(live), r.choice((0.0, 500.0, 5e3))))
        elif k < 0.74:
            d = [r.gauss(0.0, 1.0) for _ in range(3)]
            n = sum(x * x for x in d) ** 0.5 or 1.0
            dist = 10 ** r.uniform(5.5, 7.5)
            origin = near()
            ops.append(_op(WARP, a, *[origin[i] + d[i] / n * dist for i in range(3)],
                           r.choice((0.0, 2e4, 1e5)), r.choice((1000, 3000, 10000, 30000))))
        elif k < 0.8:
            far = [x + r.choice((-1.0, 1.0)) * r.uniform(1e4, 1e6) for x in near()]
            ops.append(_op(GOTO, a, *far))
        elif k < 0.84:
            ops.append(_op(STOP, a))
        elif k < 0.88:
            add(r.choice(ids))
        elif k < 0.9:
            ops.append(_op(REMOVE, a))
            live.remove(a)
        elif k < 0.92:
            ops.append(_op(SENSOR, a, r.choice((1e3, 3e4)), r.choice((1.0, 2.0)), 0.0, float(r.random() < 0.3)))
        elif k < 0.94:
            ops.append(_op(NOTIFY, a, r.choice((100.0, 2e3, 1e5))))
        elif k < 0.96:
            ops.append(_op(INTERACTIVE, a, float(r.random() < 0.6)))
        else:
            ops.append(_op(INIT))
    return ops


def collide_ops(seed: int, n_ops: int = 100) -> list:
    """A world of collisions inside the tick: up to 10 massive balls packed within a few kilometres of a top-box face,
    free ships (masses 1e4 to 1e8 kg, so that light balls meet heavy ones) and fixed rocks up to 3 km across, many
    overlapping from the start, some placed on one another (coincident centres), sent at one another along GOTO legs
    through the crowd, following one another, cloaked (no longer a candidate), made non-massive by re-adding, warping
    out (a drop-out is massive again) and re-added; runs of ticks between the commands."""
    r = random.Random(f"space-collide-{seed}")
    centre = [r.choice((-1.0, 0.0, 1.0)) * TOP + r.uniform(-2e3, 2e3) for _ in range(3)]
    ids, live, ops = list(range(1, 11)), [], []

    def near(spread: float = 3e3) -> list:
        return [x + r.uniform(-spread, spread) for x in centre]

    def add(b: int) -> None:
        rock = r.random() < 0.25
        vel = [0.0, 0.0, 0.0] if rock or r.random() < 0.4 else [r.uniform(-200.0, 200.0) for _ in range(3)]
        ops.append(_op(ADD, b, 10 ** r.uniform(9.0, 11.0) if rock else 10 ** r.uniform(4.0, 8.0),
                       r.uniform(200.0, 3e3) if rock else r.uniform(20.0, 800.0), 0.0 if rock else r.uniform(50.0, 400.0),
                       0.0 if rock else 1.0, 1.0 if (not rock and r.random() < 0.8) else 0.0, *near(), *vel,
                       r.uniform(0.2, 2.0), 1.0, 1.0 if r.random() < 0.9 else 0.0))
        if b not in live:
            live.append(b)
    for b in r.sample(ids, r.randint(4, 9)):
        add(b)
    for _ in range(n_ops):
        k = r.random()
        a = r.choice(live) if live else None
        if k < 0.4 or a is None:
            ops.extend(_op(TICK) for _ in range(r.choice((1, 1, 2, 5))))
        elif k < 0.56:
            ops.append(_op(GOTO, a, *near(r.choice((50.0, 3e3, 2e4)))))
        elif k < 0.64:
            ops.append(_op(FOLLOW, a, r.choice(live), r.choice((0.0, 100.0))))
        elif k < 0.7:
            ops.append(_op(POS, a, *near(r.choice((10.0, 1e3)))))
        elif k < 0.72 and len(live) > 1:                   # onto where another ball was last placed
            other = r.choice([b for b in live if b != a])
            start = next(op for op in reversed(ops) if op[0] in (ADD, POS) and int(op[1]) == other)
            ops.append(_op(POS, a, *(start[7:10] if start[0] == ADD else start[2:5])))
        elif k < 0.76:
            ops.append(_op(CLOAKED, a, float(r.random() < 0.6)))
        elif k < 0.8:
            d = [r.gauss(0.0, 1.0) for _ in range(3)]
            n = sum(x * x for x in d) ** 0.5 or 1.0
            dist = 10 ** r.uniform(5.5, 6.5)
            ops.append(_op(WARP, a, *[centre[i] + d[i] / n * dist for i in range(3)], r.choice((0.0, 1e3)),
                           r.choice((3000, 30000))))
        elif k < 0.86:
            add(r.choice(ids))
        elif k < 0.88:
            ops.append(_op(STOP, a))
        elif k < 0.9:
            ops.append(_op(REMOVE, a))
            live.remove(a)
        elif k < 0.95:
            ops.append(_op(INTERACTIVE, a, float(r.random() < 0.6)))
        else:
            ops.append(_op(INIT))
    return ops


def crowd_ops(seed: int, n_ticks: int = 12) -> list:
    """A crowded world of config 3's shape at a golden's size: 16 to 128 ships (free, interactive, not massive) in 1
    to 3 Gaussian blobs (sigma 10 km) around centres within +-1,000 km, every ship with a proximity sensor of 1 to
    250 km (log-uniform; period 1 s, some shuffled), so that the sensors' lists and the proximity map grow past 13,
    29, 59 and 127 keys (the rehash policy's growths); GOTO legs of up to 3 km/s, a few notification ranges, tracked
    targets, removals, InitializeBubbles and CopyBubbles between the ticks."""
    r = random.Random(f"space-crowd-{seed}")
    n = r.choice((16, 40, 70, 128)) if seed > 4 else (16, 40, 70, 128)[seed - 1]
    centres = [[r.uniform(-1e6, 1e6) for _ in range(3)] for _ in range(r.randint(1, 3))]
    ops, live = [], []
    for b in range(1, n + 1):
        c = r.choice(centres)
        p = [x + r.gauss(0.0, 1e4) for x in c]
        max_vel = 10 ** r.uniform(2.0, math.log10(3000.0))
        ops.append(_op(ADD, b, 10 ** r.uniform(6.0, 9.0), r.uniform(20.0, 500.0), max_vel, 1.0, 1.0, *p, 0.0, 0.0,
                       0.0, r.uniform(0.1, 5.0), 1.0, 0.0))
        live.append(b)
    for b in live:
        ops.append(_op(SENSOR, b, 10 ** r.uniform(3.0, math.log10(2.5e5)), 1.0, 0.0, float(r.random() < 0.3)))
    for t in range(n_ticks):
        for b in r.sample(live, max(1, len(live) // 4)):
            c = r.choice(centres)
            ops.append(_op(GOTO, b, *[x + r.gauss(0.0, 2e4) for x in c]))
        k = r.random()
        if k < 0.2:
            ops.append(_op(NOTIFY, r.choice(live), r.choice((500.0, 5e3, 5e4))))
        elif k < 0.4:
            ops.append(_op(TRACK, r.choice(live), r.choice(live), r.choice((1e3, 2e4, 1e5))))
        elif k < 0.5 and len(live) > 4:
            b = r.choice(live)
            ops.append(_op(REMOVE, b))
            live.remove(b)
        elif k < 0.55:
            ops.append(_op(INIT))
        elif k < 0.6:
            ops.append(_op(COPY))
        ops.append(_op(TICK))
    return ops


def apply(park, op: list) -> str:
    """One operation on the reference's SpaceBallpark; a query's answer as the oracle writes it ("" for the others)."""
    code, bid = int(op[0]), int(op[1])
    a = [float(x) for x in op[2:]]
    if code == CLOAKED:
        park.set_cloaked(bid, int(a[0]))
    elif code == VISIBILITY:
        return f"Q {park.check_visibility(bid, int(a[0]))}\n"
    elif code in (RANGE_BALL, RANGE_POINT):
        if code == RANGE_BALL:
            got = park.ball_ids_in_range(bid, a[0], int(a[1]), include_dist=bool(a[2]))
        else:
            got = park.ball_ids_in_range(a[0], a[1], a[2], a[3], int(a[4]), include_dist=bool(a[5]))
        if got is None:
            return "Q None\n"
        return "Q" + "".join(f" {_bits(x[0])}:{x[1]}" if isinstance(x, tuple) else f" {x}" for x in got) + "\n"
    elif code == BUBBLE_AT:
        top = park.bubble_at(a[0], a[1], a[2])
        return "Q None\n" if top is None else f"Q {top}\n"
    elif code == NEARBY:
        b = park.balls.get(bid)
        got = [] if b is None else park._nearby_balls(b, bool(a[0]), bool(a[1]), False, bool(a[2]), False)
        return "Q" + "".join(f" {o.id}" for o in got) + "\n"
    elif code == SENSOR:
        park.add_proximity_sensor(bid, a[0], a[1], int(a[3]), bool(a[2]))
    elif code == NOTIFY:
        park.set_notification_range(bid, a[0])
    elif code == TRACK:
        park.set_target_tracking(bid, int(a[0]), a[1])
    elif code == GOTO:
        park.goto_point(bid, a[0], a[1], a[2])
    elif code == STOP:
        park.stop(bid)
    elif code == FOLLOW:
        park.follow_ball(bid, int(a[0]), a[1])
    elif code == ORBIT:
        park.orbit(bid, int(a[0]), a[1])
    elif code == WARP:
        park.warp_to(bid, a[0], a[1], a[2], a[3], int(a[4]))
    elif code == UNSENSOR:
        park.remove_proximity_sensor(bid)
    elif code in (PROXIMITIES, TICK):
        park.events = []
        if code == TICK:
            park.evolve()
        else:
            park._handle_proximities()
        out = []
        for e in park.events:
            if e[1] == "DoProximity":
                out.append(f" {e[2]}:{e[3]}:{e[4]}")
            elif e[1] == "DoRange":
                out.append(f" R{e[2]}:{e[3]}")
            elif e[1] == "DoTargetTracking":
                out.append(f" T{e[2]}:{e[3]}")
        return "Q" + "".join(out) + "\n"
    if code == ADD:
        park.add_ball(bid, a[0], a[1], a[2], is_free=bool(a[3]), is_interactive=bool(a[4]), x=a[5], y=a[6], z=a[7],
                      vx=a[8], vy=a[9], vz=a[10], agility=a[11], speed_fraction=a[12], is_massive=bool(a[13]))
    elif code == POS:
        park.set_position(bid, a[0], a[1], a[2])
    elif code == RADIUS:
        park.set_radius(bid, a[0])
    elif code == MAXVEL:
        park.set_max_velocity(bid, a[0])
    elif code == REMOVE:
        park.remove_ball(bid)
    elif code == INIT:
        park.initialize_bubbles(0)
    elif code == COPY:
        park.copy_bubbles()
    elif code == INTERACTIVE:
        park.set_interactive(bid, bool(a[0]))
    elif code == KEEPALIVE:
        park.add_keep_alive_ball(bid)
    return ""


def state_text(park) -> str:
    """The reference world's state in the oracle's text (oracle/space.cpp's `state`)."""
    out = []
    for bid in sorted(park.balls):
        b = park.balls[bid]
        active = sum(1 << i for i in range(27) if b.active[i])
        dead = 1 if park.in_dead_bubble(b) else 0
        if b.my_box is not None:
            head = (f"B {b.id} {b.bubble} {b.old_bubble} {b.my_box.level} {b.my_box.key[0]} {b.my_box.key[1]} "
                    f"{b.my_box.key[2]} {b.mod[0]} {b.mod[1]} {b.mod[2]} {active} {dead}")
        else:
            head = f"B {b.id} {b.bubble} {b.old_bubble} - {b.mod[0]} {b.mod[1]} {b.mod[2]} {active} {dead}"
        out.append(head + "".join(f" {k[0]},{k[1]},{k[2]}" for k in sorted(b.boxes)) + "\n")
    out.append("L" + "".join(f" {len(lv)}" for lv in park.levels) + "\n")
    out.append(f"F {park.free_boxes} {park.bubble_id} 0\n")
    if len(park.proximity_balls):
        out.append("P" + "".join(f" {i}" for i in park.proximity_balls.keys()) + "\n")
    for bid in sorted(park.balls):
        b = park.balls[bid]
        if not b.sensor_active and len(b.sensor_balls) == 0 and not b.has_proximity:
            continue
        tracked = b.tracking_ptr.id if b.tracking_ptr is not None else 0
        out.append(f"S {b.id} {int(b.sensor_active)} {_bits(b.sensor_elapsed)} {int(b.has_proximity)} "
                   f"{int(b.within_range)} {int(b.within_tracking_range)} {tracked}"
                   + "".join(f" {i}" for i in b.sensor_balls.keys()) + "\n")
    for bub in sorted(park.bubbles):
        out.append(f"U {bub}" + "".join(f" {k}:{v}" for k, v in park.bubbles[bub].items()) + "\n")
    for tag, m in (("I", park.bubble_interactives), ("K", park.bubble_keep_alives)):
        for bub in sorted(m):
            out.append(f"{tag} {bub}" + "".join(f" {i}" for i in sorted(m[bub])) + "\n")
    for bid in sorted(park.balls):
        b = park.balls[bid]
        out.append(f"M {b.id} {b.mode} {int(b.is_massive)} {b.follow_ptr or 0}"
                   + "".join(f" {_bits(x)}" for x in (*b.pos, *b.vel)) + " :"
                   + "".join(f" {i}" for i in b.followers.ordered()) + "\n")
    return "".join(out)


def digest(text: str) -> np.uint64:
    return np.frombuffer(hashlib.sha256(text.encode()).digest()[:8], dtype=np.uint64)[0]


def save(path: Path, scenarios: list) -> None:
    """scenarios: [{"seed", "ops" [n][STRIDE], "digests" [n] uint64}], as one compressed archive."""
    arrays = {"names": np.array([s["seed"] for s in scenarios]),
              "rand_seeds": np.array([s.get("rand_seed", 1) for s in scenarios], dtype=np.int64)}
    for i, sc in enumerate(scenarios):
        arrays[f"ops{i}"] = np.array(sc["ops"], dtype=np.float64)
        arrays[f"digests{i}"] = np.array(sc["digests"], dtype=np.uint64)
    np.savez_compressed(str(path) + ".npz", **arrays)


def load(path: Path) -> list:
    z = np.load(str(path) + ".npz")
    return [{"seed": str(name), "ops": z[f"ops{i}"], "digests": z[f"digests{i}"], "rand_seed": int(z["rand_seeds"][i])}
            for i, name in enumerate(z["names"])]
