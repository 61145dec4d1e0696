"""Static collidables (capsules and oriented boxes) of the collision park: each one's record, made once on the host
at the load in the reference's double arithmetic, as AddCapsule and AddOrientedBox make it (Capsule.cpp,
OrientedBox.cpp, BoxShape.cpp; the reference's exact_ballpark/vec_collide.py:261-369 and full.py's Capsule,
OrientedBox, BoxShape, RectangleShape, AABB), with its filing in the partition (InsertInBoxes: its level and its
boxes' keys). A static collidable never moves; the tick's tests read these values on the device.

A record is G_SIZE doubles and I_SIZE integers, laid out as the reference's park keeps them (so that a park's records
compare field for field with the reference's): a capsule's A, B, B - A and radius (a float); a box's centre, its
AABB's corners, its edge vectors, each normalised, half their lengths and their squared lengths, its eight corners,
its six sides' corners, each side's normal ((b - a) x (c - a) normalised: the triangle (a, b, c)'s) and the normal of
its triangle (a, c, d); then kind, id, parent id, level and the number of boxes.
"""

from __future__ import annotations

import itertools
import math
import struct

import numpy as np

STATIC_CAPSULE, STATIC_BOX = 0, 1
G_A, G_B, G_AB, G_RAD = 0, 3, 6, 9
G_CENTER, G_LO, G_HI = 10, 13, 16
G_AXES, G_UNIT, G_HALF, G_LENSQ = 19, 28, 37, 40
G_CORNERS, G_RECT, G_RNORM, G_TNORM = 43, 67, 139, 157
G_SIZE = 175
I_KIND, I_ID, I_PARENT, I_LEVEL, I_NBOX = range(5)
I_SIZE = 5
SIDE_FRONT, SIDE_BACK, SIDE_LEFT, SIDE_RIGHT, SIDE_TOP, SIDE_BOTTOM = range(6)
# BoxShape's corners A .. H as the edges (x, y, z) each adds to A, and its sides' rectangles (a, b, c, d) as corner
# indices, in the side order above (OrientedBox.cpp's SetCorners and its rectangles)
_CORNER_BITS = ((0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (0, 1, 1), (1, 0, 1), (1, 1, 1))
_SIDE_CORNERS = ((7, 5, 3, 6), (2, 4, 1, 0), (5, 2, 0, 3), (4, 7, 6, 1), (2, 5, 7, 4), (1, 6, 3, 0))

NUM_LEVELS = 8
LEVEL_WIDTH = tuple(7864320.0 / (1 << 2 * i) for i in range(NUM_LEVELS))          # 480 m x 4^(7 - level)
LEVEL_GRID = tuple(1 << (2 * i + 23) for i in range(NUM_LEVELS))


def _f32(x: float) -> float:
    try:
        return struct.unpack("f", struct.pack("f", x))[0]
    except OverflowError:
        return math.copysign(math.inf, x)


def _add(u, v) -> list:
    return [u[0] + v[0], u[1] + v[1], u[2] + v[2]]


def _sub(u, v) -> list:
    return [u[0] - v[0], u[1] - v[1], u[2] - v[2]]


def _scale(u, c: float) -> list:
    return [u[0] * c, u[1] * c, u[2] * c]


def _lensq(v) -> float:
    return v[0] * v[0] + v[1] * v[1] + v[2] * v[2]


def _length(v) -> float:
    return math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])


def _normalized(v) -> list:
    """Vector3d::Normalize: times the reciprocal of the length; a zero vector stays zero."""
    n = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    if n == 0.0:
        return list(v)
    inv = 1.0 / n
    return [v[0] * inv, v[1] * inv, v[2] * inv]


def _cross(u, v) -> list:
    """Vector3d::Cross: components in Destiny's order."""
    return [u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]]


def _int64(x: float) -> int:
    """int64_t(x) as aarch64's fcvtzs: toward zero, saturating, NaN to 0."""
    if x != x:
        return 0
    if x >= 9223372036854775808.0:
        return 9223372036854775807
    if x < -9223372036854775808.0:
        return -9223372036854775808
    return int(x)


def level_for(radius: float) -> int:
    """Partition::GetBox(radius, pos)'s level: the finest whose width is at least three radii. The widths shrink with
    the level, so the levels whose width three radii do not exceed are a prefix; the level is its last (0 when even
    the top is exceeded; 7 for a NaN, which exceeds nothing)."""
    return max(sum(1 for w in LEVEL_WIDTH if not 3.0 * radius > w) - 1, 0)


def key_for(level: int, pos) -> tuple:
    """The box key holding pos at a level (before the grid's clamp)."""
    w = LEVEL_WIDTH[level]
    fac, half = 1.0 / w, 0.5 * w * LEVEL_GRID[level]
    return tuple(_int64((pos[i] + half) * fac) for i in range(3))


def bounds(level: int, key) -> tuple:
    """A box's low and high corners."""
    w, n = LEVEL_WIDTH[level], LEVEL_GRID[level]
    center = w * n * 0.5
    return [key[i] * w - center for i in range(3)], [(key[i] + 1) * w - center for i in range(3)]


def with_sides(key, mod) -> set:
    """The box and the adjacent boxes an InsertInBoxes reaches: per axis the key alone, or the key and its neighbour
    on the side `mod` gives (-1, 0, +1), and every combination of those."""
    options = [(key[q],) if mod[q] == 0 else (key[q], key[q] + mod[q]) for q in range(3)]
    return set(itertools.product(*options))


def static_record(s: dict) -> tuple:
    """(doubles [G_SIZE], integers [I_SIZE], the boxes' keys sorted) of {"kind": "capsule", "id", "parent", "a", "b",
    "radius"} or {"kind": "box", "id", "parent", "corner", "lx", "ly", "lz"}. A capsule is filed at its radius's level
    along its segment, sampled every 2r from A while the float length lasts, each sample's box with the adjacent boxes
    its radius reaches (none for a radius <= 0); a box at half its AABB's longest width, with the adjacent boxes its
    AABB reaches, or all 27 top boxes around it when its bounding diameter exceeds a top box. Refused (ValueError): an
    unknown kind, a box at the grid's edge, a capsule whose walk never ends (Destiny's result undefined)."""
    geo, ints = [0.0] * G_SIZE, [0] * I_SIZE
    ints[I_ID], ints[I_PARENT] = int(s["id"]), int(s["parent"])
    kind = s["kind"]
    if kind == "capsule":
        ints[I_KIND] = STATIC_CAPSULE
        a, b, radius = [float(x) for x in s["a"]], [float(x) for x in s["b"]], _f32(s["radius"])
        ab = _sub(b, a)
        geo[G_A:G_A + 3], geo[G_B:G_B + 3], geo[G_AB:G_AB + 3], geo[G_RAD] = a, b, ab, radius
        boxes: set = set()
        level = level_for(radius)
        if radius > 0.0:
            at = list(a)
            left = _f32(_length(ab))
            step_v = [x * float(radius) * 2.0 for x in _normalized(ab)]
            step = _f32(radius * 2.0)
            while left >= 0.0:
                key = key_for(level, at)
                lo, hi = bounds(level, key)
                mod = [0, 0, 0]
                for q in range(3):
                    if lo[q] + float(radius) - at[q] > 0.0:
                        mod[q] = -1
                    elif hi[q] - float(radius) - at[q] < 0.0:
                        mod[q] = 1
                boxes |= with_sides(key, mod)
                at = _add(at, step_v)
                shorter = _f32(left - step)
                if shorter == left:
                    raise ValueError("Capsule::InsertInBoxes never ends (twice the radius is below half a float ulp "
                                     "of the length left): Destiny's result is undefined")
                left = shorter
    elif kind == "box":
        ints[I_KIND] = STATIC_BOX
        A = np.array([float(x) for x in s["corner"]])
        edges = np.array([[float(x) for x in s[k]] for k in ("lx", "ly", "lz")])
        # corner i = A plus the edges its bits name, added x, then y, then z (BoxShape's A .. H: A, A+x, A+y, A+z,
        # A+x+y, A+y+z, A+x+z, A+x+y+z); an absent edge is not added (A + 0 would turn a -0 into +0)
        corners = np.empty((8, 3))
        for i, bits in enumerate(_CORNER_BITS):
            v = A.copy()
            for e in range(3):
                if bits[e]:
                    v = v + edges[e]
            corners[i] = v
        center = corners[0] + (corners[7] - corners[0]) * (1.0 / 2.0)
        # the AABB: on each axis the first corner holding the extreme (the strict-comparison scan's choice)
        low = corners[np.argmin(corners, axis=0), [0, 1, 2]]
        high = corners[np.argmax(corners, axis=0), [0, 1, 2]]
        geo[G_CENTER:G_CENTER + 3], geo[G_LO:G_LO + 3], geo[G_HI:G_HI + 3] = center, low, high
        lengths = np.sqrt(edges[:, 0] * edges[:, 0] + edges[:, 1] * edges[:, 1] + edges[:, 2] * edges[:, 2])
        inv = np.where(lengths == 0.0, 0.0, 1.0 / np.where(lengths == 0.0, 1.0, lengths))
        units = np.where(lengths[:, None] == 0.0, edges, edges * inv[:, None])
        geo[G_AXES:G_AXES + 9] = edges.reshape(-1)
        geo[G_UNIT:G_UNIT + 9] = units.reshape(-1)
        geo[G_HALF:G_HALF + 3] = lengths / 2.0
        geo[G_LENSQ:G_LENSQ + 3] = edges[:, 0] * edges[:, 0] + edges[:, 1] * edges[:, 1] + edges[:, 2] * edges[:, 2]
        geo[G_CORNERS:G_CORNERS + 24] = corners.reshape(-1)
        quads = corners[np.array(_SIDE_CORNERS)]                                 # [6 sides][4 corners][3]
        geo[G_RECT:G_RECT + 72] = quads.reshape(-1)
        ra, rb, rc, rd = (quads[:, k] for k in range(4))
        geo[G_RNORM:G_RNORM + 18] = np.array([_normalized(_cross(u, v)) for u, v in zip(rb - ra, rc - ra)]).reshape(-1)
        geo[G_TNORM:G_TNORM + 18] = np.array([_normalized(_cross(u, v)) for u, v in zip(rc - ra, rd - ra)]).reshape(-1)
        H = corners[7]
        low, high = [float(x) for x in low], [float(x) for x in high]
        center = [float(x) for x in center]
        dx, dy, dz = high[0] - low[0], high[1] - low[1], high[2] - low[2]
        inner = dz if dy < dz else dy
        r = (inner if dx < inner else dx) / 2.0
        level = level_for(r)
        key = key_for(level, center)
        lo, hi = bounds(level, key)
        mod = [0, 0, 0]
        for q in range(3):
            if lo[q] - low[q] > 0.0:
                mod[q] = -1
            elif hi[q] - high[q] < 0.0:
                mod[q] = 1
        bounding = _f32(_length(_sub(H, A)) / 2.0)
        if level == 0 and _f32(bounding * 2.0) > LEVEL_WIDTH[0]:
            boxes = {(key[0] + x, key[1] + y, key[2] + z) for x in (-1, 0, 1) for y in (-1, 0, 1) for z in (-1, 0, 1)}
        else:
            boxes = with_sides(key, mod)
    else:
        raise ValueError(f"a static collidable's kind is 'capsule' or 'box', not {kind!r}")
    n = LEVEL_GRID[level]
    keys = sorted(boxes)
    if any(not 0 < k[q] < n - 1 for k in keys for q in range(3)):
        raise ValueError(f"static collidable {ints[I_ID]}: a box at the partition's edge (not in this park)")
    ints[I_LEVEL], ints[I_NBOX] = level, len(keys)
    return geo, ints, keys
