"""Generates the golden fixtures under tests/golden/ from the reference itself (run where the reference is checked
out; nothing on a GPU box runs this):

    EXACT_BALLPARK_REF=<checkout of exact-ballpark> python tests/golden/make_golden.py [--only libm|libm_dense|traces|collide]

1. libm.npz: inputs and outputs of glibc 2.34 aarch64's functions as the reference transcribes them (dlibm.sin,
   cos, sincos, log; vec_exp.exp; vec_libm.expf, logf, sinf, cosf, acosf, atanf, atan2f, pow), on seeded random
   arguments over each function's branches plus the edge cases (zeros, infinities, NaN, subnormals, the branch
   bounds, sincos's odd point +-0x1.ad1fb54442d18p+0); libm_dense.npz: the double functions densely around their
   branch bounds (make_libm_dense).
2. trace_*.json.gz / .npz: the flight-mode park's scenarios as golden traces (tests/golden/trace.py), recorded on
   the reference's batched park (VecModesPark, CPU tick):
   - mc{1,2}: the reference's own mode_cases scenarios (tests/mode_cases.py; seed 1 development, 2 held out),
     driven by its own modes_batch.batched_modes: FOLLOW, ORBIT under both laws, WARP and its transitions,
     EntityWarpIn, the guards, mixed worlds (no dynamical orientation);
   - fc{1,2}: the reference's flight_cases scenarios (tests/flight_cases.py) driven by modes_batch.batched_full:
     the modes with dynamical orientation on and off and every setter in flight;
   - w0_*: flight_worlds(seed, 64 worlds x 4 ships), 200 ticks, dynamical orientation on, each orbit law, and one
     run without dynamical orientation.
   Before recording, a sample of each scenario family is checked against the reference's scalar transcriptions
   (ModeBallpark, FullBallpark) with the reference's own comparison (modes_batch.differences): the batched CPU park
   the traces come from is bit-exact to the scalar reference on it.
"""

from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent.parent))

import refshim  # noqa: E402

refshim.install()

import torch  # noqa: E402

import trace as tr  # noqa: E402

torch.set_num_threads(8)


# ============================================================================================ libm vectors

def make_libm(rng: np.random.Generator, n: int = 3000) -> None:
    from exact_ballpark import dlibm, vec_exp, vec_libm as L

    H = float.fromhex
    f32 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)
    dbl_edges = [0.0, -0.0, 1.0, -1.0, 0.5, 2.0, 1e-310, -1e-310, 5e-324, 1e-300, 1e300, -1e300, np.inf, -np.inf,
                 np.nan, H("0x1.ad1fb54442d18p+0"), -H("0x1.ad1fb54442d18p+0"), H("0x1.921fb54442d18p+0"),
                 0.855469, 2.426265, 105414350.0, 105414351.0, 1e9, 1e15, 1e22, 1e100, 2 ** -27, 2 ** -26,
                 0.126, 0.12599999999999997, 65535.999, 0.001, 0.9375, 1.0625, 0.93749999, 1.06445312]
    big = rng.uniform(-1, 1, n) * np.exp(rng.uniform(-60, 250, n))
    dx = np.concatenate([rng.uniform(-4, 4, n), rng.uniform(-7e4, 7e4, n), big, np.array(dbl_edges)])
    out = {}
    out["sin_x"] = dx
    out["sin_y"] = np.array([dlibm.sin(float(v)) for v in dx])
    out["cos_y"] = np.array([dlibm.cos(float(v)) for v in dx])
    sc = [dlibm.sincos(float(v)) for v in dx]
    out["sincos_s"] = np.array([s for s, _ in sc])
    out["sincos_c"] = np.array([c for _, c in sc])
    lx = np.concatenate([rng.uniform(0.9, 1.1, n), np.exp(rng.uniform(-700, 700, n)), rng.uniform(0, 10, n),
                         np.array([0.0, -0.0, 1.0, -1.0, 1e-310, 5e-324, np.inf, -np.inf, np.nan, 0.001,
                                   H("0x1.e000000000000p-1"), H("0x1.0900000000000p+0"), 0.9375 - 1e-17])])
    out["log_x"] = lx
    out["log_y"] = np.array([dlibm.log(float(v)) if v > 0 or np.isnan(v) else
                             (-np.inf if v == 0 else np.nan) for v in lx])
    ex = np.concatenate([rng.uniform(-30, 10, n), rng.uniform(-746, 710, n), rng.uniform(-1e-16, 1e-16, 50),
                         np.array([0.0, -0.0, 709.78, 709.79, 710.0, -745.13, -745.14, -708.4, -708.39, -720.0,
                                   512.0, -512.0, 1024.0, -1024.0, np.inf, -np.inf, np.nan, 1e-20, -1e-20])])
    out["exp_x"] = ex
    out["exp_y"] = vec_exp.exp(torch.tensor(ex)).numpy()
    fx = f32(np.concatenate([rng.uniform(-10, 10, n), rng.uniform(-130, 130, n), rng.uniform(-1.05, 1.05, n),
                             rng.uniform(-1, 1, n) * np.exp(rng.uniform(-100, 88, n)), rng.uniform(-1e9, 1e9, n // 4)]))
    fedges = f32([0.0, -0.0, 1.0, -1.0, 0.5, -0.5, np.inf, -np.inf, np.nan, 88.72, 88.73, -103.28, -103.97, -104.0,
                  1e-40, -1e-40, 1e-45, 120.0, 119.99, 0.7853981, 2 ** -12, 2 ** -26, 2 ** -29, 2 ** 25, 0.4375,
                  0.6875, 1.1875, 2.4375, 3e38, 1.17549435e-38])
    fx = np.concatenate([fx, fedges])
    T = torch.tensor(fx)
    out["f_x"] = fx
    out["expf_y"] = L.expf(T).numpy()
    out["sinf_y"] = L.sinf(T).numpy()
    out["cosf_y"] = L.cosf(T).numpy()
    out["atanf_y"] = L.atanf(T).numpy()
    ax = np.abs(fx)
    out["logf_x"] = np.concatenate([ax, f32([-1.0, -0.0, -np.inf])])
    out["logf_y"] = L.logf(torch.tensor(out["logf_x"])).numpy()
    cx = f32(np.concatenate([rng.uniform(-1, 1, 2 * n), rng.uniform(-1.1, 1.1, n),
                             np.array([0.0, -0.0, 1.0, -1.0, 0.5, -0.5, 2 ** -26, -2 ** -26, 1.0000001, np.nan,
                                       np.inf, 0.49999997, -0.49999997])]))
    out["acosf_x"] = cx
    out["acosf_y"] = L.acosf(torch.tensor(cx)).numpy()
    yy = f32(np.concatenate([rng.uniform(-10, 10, len(fx) - 16), np.array([0.0, -0.0, np.inf, -np.inf, 1.0, -1.0,
                                                                           0.0, np.nan, 1e30, -1e-30, 5.0, -5.0,
                                                                           np.inf, -np.inf, 0.0, -0.0])]))
    out["atan2f_y"] = yy
    out["atan2f_out"] = L.atan2f(torch.tensor(yy), T).numpy()
    px = np.concatenate([rng.uniform(0, 1, n), rng.uniform(0.9, 1.1, n), rng.uniform(0, 1e3, n),
                         -rng.uniform(0, 10, 200),
                         np.array([0.0, -0.0, 1.0, -1.0, np.inf, -np.inf, np.nan, 1e-310, 2.0, 0.5, -2.0, -0.5,
                                   10.0, 0.999999, 1e300, 1e-300])])
    py = np.concatenate([rng.integers(0, 100, n).astype(float), rng.uniform(-1e4, 1e4, n), rng.uniform(-300, 300, n),
                         rng.integers(-7, 7, 200).astype(float),
                         np.array([3.0, -3.0, 2.0, np.inf, 0.5, 1e30, 0.0, 1.0, 1e-30, -1e-30, 3.0, -3.0, 1e19,
                                   -1e19, 2.0, 0.5])])
    out["pow_x"], out["pow_y"] = px, py
    out["pow_out"] = L.pow(torch.tensor(px), torch.tensor(py)).numpy()
    np.savez_compressed(HERE / "libm.npz", **out)
    print("libm.npz", {k: v.shape for k, v in out.items()})


def _around(points, ulps: int = 24, rel=(1e-15, 1e-12, 1e-9, 1e-6)) -> np.ndarray:
    """Each point, its neighbours up to `ulps` representable steps either way, and relative nudges either way."""
    out = []
    for p in points:
        p = float(p)
        lo = hi = p
        out.append(p)
        for _ in range(ulps):
            lo, hi = np.nextafter(lo, -np.inf), np.nextafter(hi, np.inf)
            out += [lo, hi]
        out += [p * (1.0 + r) for r in rel] + [p * (1.0 - r) for r in rel]
    return np.array(out, dtype=np.float64)


def make_libm_dense(rng: np.random.Generator) -> None:
    """libm_dense.npz: the double functions (dlibm.sin, cos, sincos, log; vec_exp.exp; vec_libm.pow) densely around
    glibc 2.34's branch bounds, as its sources state them: sin and cos at |x| = 2^-26, 0.126 (the Taylor step),
    0.855469, 2.426265, 105414350 (the reduction's switch) and 2^48, and near multiples of pi/2 (the reduced
    argument's cancellation) up to 10^8; exp at 2^-54, +-512 (the scaled path), 709.78 (overflow), -708.39 (the
    subnormal results) and -745.13 (underflow); log near 1 (the 0.9375 and 1.0644531 bounds of its polynomial path),
    near the smallest normal and through the subnormals; pow at x near 1 with large |y|, at results near the overflow
    and underflow bounds, at negative x with integer and half-integer y, and at tiny |y|."""
    from exact_ballpark import dlibm, vec_exp, vec_libm as L

    sc_bounds = [2.0 ** -26, 0.126, 0.855469, 2.426265, 105414350.0, 2.0 ** 48]
    k = np.concatenate([np.arange(1, 400), rng.integers(400, 10 ** 8, 600)]).astype(np.float64)
    halfpi = np.pi / 2.0
    sx = np.concatenate([_around(sc_bounds), -_around(sc_bounds), _around(k * halfpi, ulps=6, rel=()),
                         -_around(k[:200] * halfpi, ulps=6, rel=())])
    out = {"sin_x": sx}
    out["sin_y"] = np.array([dlibm.sin(float(v)) for v in sx])
    out["cos_y"] = np.array([dlibm.cos(float(v)) for v in sx])
    pairs = [dlibm.sincos(float(v)) for v in sx]
    out["sincos_s"] = np.array([a for a, _ in pairs])
    out["sincos_c"] = np.array([b for _, b in pairs])
    ex = np.concatenate([_around([2.0 ** -54, -2.0 ** -54, 512.0, -512.0, 709.782712893384, -708.3964185322641,
                                  -745.1332191019411, -745.1332191019412, 1024.0, -1024.0], ulps=40),
                         rng.uniform(-746.0, -700.0, 2000), rng.uniform(700.0, 710.0, 1000)])
    out["exp_x"] = ex
    out["exp_y"] = vec_exp.exp(__import__("torch").tensor(ex)).numpy()
    lx = np.concatenate([_around([1.0, 0.9375, 1.0644531250000000, float.fromhex("0x1.0p-1022")], ulps=40),
                         np.exp(rng.uniform(-745.0, -708.0, 2000)), rng.uniform(0.93, 1.07, 3000)])
    out["log_x"] = lx
    out["log_y"] = np.array([dlibm.log(float(v)) for v in lx])
    n = 1500
    px = np.concatenate([1.0 + rng.uniform(-1e-9, 1e-9, n), rng.uniform(0.5, 2.0, n), -rng.integers(1, 50, n) * 1.0,
                         -rng.uniform(0.1, 10.0, n), rng.uniform(0.0, 1e-300, 200), rng.uniform(1.0, 10.0, n)])
    py = np.concatenate([rng.uniform(-1e12, 1e12, n),
                         np.log(2.0) * rng.choice([1024.0, -1022.0, -1074.0], n) / np.log(rng.uniform(0.5, 2.0, n))
                         * (1.0 + rng.uniform(-1e-12, 1e-12, n)),
                         rng.integers(-60, 60, n).astype(np.float64) + rng.choice([0.0, 0.5], n),
                         rng.integers(-9, 9, n).astype(np.float64),
                         rng.uniform(-2.0, 2.0, 200), rng.uniform(-1.0, 1.0, n) * 2.0 ** -rng.uniform(60.0, 70.0, n)])
    out["pow_x"], out["pow_y"] = px, py
    torch = __import__("torch")
    out["pow_out"] = L.pow(torch.tensor(px), torch.tensor(py)).numpy()
    np.savez_compressed(HERE / "libm_dense.npz", **out)
    print("libm_dense.npz", {k: v.shape for k, v in out.items()})


# ============================================================================================ traces

def _recorded(fn, *args, **kw) -> list:
    """Run one of modes_batch's drivers with the reference's VecModesPark replaced by a recording subclass; the
    parks it made (one per group), in order."""
    import modes_batch as mb
    from exact_ballpark.vec_modes import VecModesPark

    made = []
    Rec = tr.recording(VecModesPark)

    class Collect(Rec):
        def __init__(self, *a, **k):
            super().__init__(*a, **k)
            made.append(self)

    old = mb.VecModesPark
    mb.VecModesPark = Collect
    try:
        fn(*args, **kw)
    finally:
        mb.VecModesPark = old
    return made


def _check_scalar(kind: str, cs: list) -> None:
    """The batched CPU park against the reference's scalar transcription on the scenarios cs (the reference's own
    comparison); raises on any difference."""
    import modes_batch as mb
    t = time.time()
    if kind == "modes":
        want = mb.reference_modes(cs)
        got = mb.batched_modes(cs, device="cpu")
        bad = mb.differences(want, got, mb.FIELDS_MODES)
    else:
        want = mb.reference_full(cs)
        got = mb.batched_full(cs, device="cpu")
        bad = mb.differences(want, got, mb.FIELDS_FULL)
    if bad:
        raise RuntimeError(f"the batched CPU park differs from the scalar reference: {bad[:10]}")
    print(f"  scalar check ({kind}, {len(cs)} scenarios): 0 differences, {time.time() - t:.0f} s")


def _sample(cs: list, per_kind: int) -> list:
    seen, out = {}, []
    for c in cs:
        k = (c["kind"], bool(c.get("do", False)), bool(c["new_orbit"]))
        if seen.get(k, 0) < per_kind:
            seen[k] = seen.get(k, 0) + 1
            out.append(c)
    return out


def _save_parks(prefix: str, parks: list) -> None:
    name = f"trace_{prefix}"
    tr.save([p.trace for p in parks], HERE / name, [tr.snapshot(p) for p in parks])
    print(f"  {name}: {len(parks)} parks, {sum(p.n for p in parks)} rows, "
          f"{sum(len(p.trace['digests']) for p in parks)} ticks")


def make_powf(rng: np.random.Generator, n: int = 4000) -> None:
    """powf's vectors (dlibm_powf.powf, glibc 2.34 aarch64's powf as the reference transcribes it), added to libm.npz
    beside the others (their arrays kept as they are): floats from every range the function branches on (near 1, small,
    subnormal, large, negative with integer and non-integer exponents, the over- and underflow thresholds, mushroom
    growth's range ** 0.25) and every pair of special values."""
    from exact_ballpark import dlibm_powf
    f32 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)   # noqa: E731
    xs = [rng.uniform(0, 2, n), rng.uniform(0.99, 1.01, n), 10.0 ** rng.uniform(-30, 30, n),
          10.0 ** rng.uniform(-45, -38, 400), -rng.uniform(0, 20, n), rng.uniform(0, 1, n)]
    ys = [rng.uniform(-10, 10, n), rng.uniform(-3e3, 3e3, n), rng.uniform(-4, 4, n),
          rng.uniform(-2, 2, 400), rng.integers(-12, 12, n).astype(float) + (rng.random(n) < 0.2) * 0.5,
          np.full(n, 0.25)]
    special = np.array([0.0, -0.0, 1.0, -1.0, 2.0, -2.0, 0.5, -0.5, 3.0, -3.0, np.inf, -np.inf, np.nan, 1e-45, -1e-45,
                        1.17549435e-38, 3.4028235e38, -3.4028235e38, 1.0000001, 0.99999994, 16777216.0, 16777217.0,
                        -16777216.0, 149.0, -150.0, 128.0, -126.0, 0.25])
    sx, sy = np.meshgrid(special, special)
    px = f32(np.concatenate(xs + [sx.ravel()]))
    py = f32(np.concatenate(ys + [sy.ravel()]))
    out = np.array([dlibm_powf.powf(float(a), float(b)) for a, b in zip(px, py)])
    have = dict(np.load(HERE / "libm.npz"))
    have.update(powf_x=px, powf_y=py, powf_out=out)
    np.savez_compressed(HERE / "libm.npz", **have)
    print("libm.npz powf", px.shape)


def make_traces(sample: int) -> None:
    import flight_cases as flc
    import mode_cases as mc
    import modes_batch as mb

    for seed in (1, 2):
        t = time.time()
        cs = mc.cases(seed)
        if sample:
            _check_scalar("modes", _sample(cs, sample))
        parks = _recorded(mb.batched_modes, cs, device="cpu")
        _save_parks(f"mc{seed}", parks)
        print(f"mode_cases({seed}): {len(cs)} scenarios, {time.time() - t:.0f} s")
    for seed in (1, 2):
        t = time.time()
        cs = flc.cases(seed)
        if sample:
            _check_scalar("full", _sample(cs, max(1, sample // 2)))
        parks = _recorded(mb.batched_full, cs, device="cpu")
        _save_parks(f"fc{seed}", parks)
        print(f"flight_cases({seed}): {len(cs)} scenarios, {time.time() - t:.0f} s")


def make_workload_traces() -> None:
    from exact_ballpark.vec_modes import VecModesPark
    from exact_ballpark_b200.workloads import flight_worlds

    Rec = tr.recording(VecModesPark)
    for name, seed, do, new in (("w0_do_new", 1, True, True), ("w0_do_old", 2, True, False),
                                ("w0_nodo_new", 3, False, True)):
        t = time.time()
        w = flight_worlds(seed, 64, 4)
        park = Rec(len(w.rows), device="cpu", dynamical_orientation=do, use_new_orbit=new)
        park.load(w.rows)
        w.apply(park)
        for _ in range(200):
            park.evolve()
        tr.save([park.trace], HERE / f"trace_{name}", [tr.snapshot(park)])
        print(f"  trace_{name}: n={park.n} 200 ticks, {time.time() - t:.0f} s")


def make_collide_traces(sample: int) -> None:
    """The collision park's traces: the reference's collide_cases scenarios (seed 1 development, 2 held out; the
    gradient method, a client's view) driven by its own collide_cases.batched, and the collision benchmark's worlds
    (workloads.collide_worlds: 64 worlds of 4 ships, 4 free spheres and 8 fixed spheres, 100 ticks). Before
    recording, each seed's scenarios are checked against the scalar SpaceBallpark (collide_cases.reference_rows)
    with the reference's own comparison (collide_cases.differences)."""
    import collide_cases as cc
    import collide_trace as ct
    from exact_ballpark.vec_collide import VecCollidePark
    from exact_ballpark_b200.workloads import collide_worlds

    Rec = ct.recording(VecCollidePark)
    for seed in (1, 2):
        t = time.time()
        cs = cc.cases(seed)
        if sample:
            sub = cs[:max(1, sample) * 20]
            want, undefined = cc.reference_rows(sub)
            got = cc.batched(sub, "cpu")
            bad = cc.differences(want, {k: v for k, v in got.items() if k[0] not in undefined})
            if bad:
                raise RuntimeError(f"the batched CPU collision park differs from the scalar reference: {bad[:10]}")
            print(f"  scalar check (collide seed {seed}, {len(sub)} scenarios): 0 differences")
        parks = []

        def make(*a, **k):
            parks.append(Rec(*a, **k))
            return parks[-1]
        cc.batched(cs, "cpu", park_cls=make)
        ct.save([p.trace for p in parks], HERE / f"collide_cc{seed}")
        ticks = sum(len(p.trace["field_digests"]) for p in parks)
        print(f"  collide_cc{seed}: {len(cs)} scenarios in {len(parks)} parks, {ticks} ticks, {time.time() - t:.0f} s")
    import exact_ballpark.vec_collide as VC
    import static_cases as stc
    for seed in (1, 2):
        t = time.time()
        cs = stc.cases(seed, n=200)
        if sample:
            want, _, _, undefined = stc.reference(cs)
            got = stc.batched(cs, "cpu")
            bad = stc.differences(want, {k: v for k, v in got.items() if k[0] not in undefined})
            if bad:
                raise RuntimeError(f"the batched CPU statics park differs from the scalar reference: {bad[:10]}")
            print(f"  scalar check (statics seed {seed}, {len(cs)} scenarios): 0 differences")
        parks = []
        real = VC.VecCollidePark

        def make_s(*a, **k):
            parks.append(Rec(*a, **k))
            return parks[-1]
        VC.VecCollidePark = make_s
        try:
            stc.batched(cs, "cpu")
        finally:
            VC.VecCollidePark = real
        ct.save([p.trace for p in parks], HERE / f"collide_st{seed}")
        ticks = sum(len(p.trace["field_digests"]) for p in parks)
        print(f"  collide_st{seed}: {len(cs)} scenarios in {len(parks)} parks, {ticks} ticks, {time.time() - t:.0f} s")
    t = time.time()
    w = collide_worlds(1, 64, ticks=100)
    park = Rec(64, 16, friction=1.0e6, tick_interval_ms=1000, device="cpu")
    park.load(w.worlds)
    for step in range(1, 101):
        w.apply(park, step)
        park.evolve()
    ct.save([park.trace], HERE / "collide_w0")
    print(f"  collide_w0: 64 worlds x 16 balls, 100 ticks, {time.time() - t:.0f} s")
    from exact_ballpark_b200.workloads import collide_statics_worlds
    t = time.time()
    w = collide_statics_worlds(1, 64, ticks=100)
    park = Rec(64, 8, friction=1.0e6, tick_interval_ms=1000, device="cpu", statics=8)
    park.load(w.worlds, w.collidables)
    for step in range(1, 101):
        w.apply(park, step)
        park.evolve()
    ct.save([park.trace], HERE / "collide_s0")
    print(f"  collide_s0: 64 worlds x (8 balls + 8 static collidables), 100 ticks, {time.time() - t:.0f} s")


def make_collide_crowd() -> None:
    """collide_crowd: the reference's collision park on crowded worlds of 48 and 64 slots (the park's largest),
    workloads.collide_worlds with 8 ships and 16 or 24 free and 24 or 32 fixed spheres, 16 worlds each, 60 ticks,
    the ships re-aimed every 20 ticks: the worlds the GPU tick's largest shared-memory tables serve."""
    import collide_trace as ct
    from exact_ballpark.vec_collide import VecCollidePark
    from exact_ballpark_b200.workloads import collide_worlds

    Rec = ct.recording(VecCollidePark)
    traces = []
    for ships, spheres, fixed in ((8, 16, 24), (8, 24, 32)):
        t = time.time()
        n = ships + spheres + fixed
        w = collide_worlds(31 + n, 16, ships=ships, spheres=spheres, statics=fixed, ticks=60, reaim=20)
        park = Rec(16, n, friction=1.0e6, tick_interval_ms=1000, device="cpu")
        park.load(w.worlds)
        for step in range(1, 61):
            w.apply(park, step)
            park.evolve()
        traces.append(park.trace)
        print(f"  collide_crowd: 16 worlds x {n} balls, 60 ticks, {time.time() - t:.0f} s")
    ct.save(traces, HERE / "collide_crowd")


def make_rand() -> None:
    """rand.npz: glibc's rand() after srand(seed) from the reference's own generator (exact_ballpark.space's
    GlibcRandom, glibc_rand.py), 2000 draws for each of 40 seeds (edge seeds included: 0, 1, 2^31 - 1, 2^31, 2^32 - 1,
    2^32, a negative one), and the state after srand."""
    from exact_ballpark.space import GlibcRandom
    r = np.random.default_rng(7)
    seeds = [0, 1, 2, 2 ** 31 - 1, 2 ** 31, 2 ** 32 - 1, 2 ** 32, -5, 123456789] + \
        [int(x) for x in r.integers(0, 2 ** 40, 31)]
    draws = np.zeros((len(seeds), 2000), dtype=np.int64)
    states = np.zeros((len(seeds), 33), dtype=np.int64)
    for i, sd in enumerate(seeds):
        g = GlibcRandom(sd)
        states[i] = list(g.s) + [g.f, g.r]
        draws[i] = [g.next() for _ in range(2000)]
    np.savez_compressed(HERE / "rand.npz", seeds=np.array(seeds, dtype=np.int64), draws=draws, states=states)
    print(f"  rand.npz: {len(seeds)} seeds x 2000 draws")


# ============================================================================================ combat

def _combat_batches(seed: int) -> list:
    """The reference's combat scenarios of a seed (tests/destiny_combat_cases.py, 12 batches of 12 worlds, as its own
    tests run them), the batches with dynamical orientation, each world checked on the scalar FullBallpark first: the
    worlds outside the reference's domain (Destiny's result undefined, or balls in two bubbles) left out."""
    import destiny_combat_cases as dc
    out = []
    for cfg in dc.batches(seed, 12, 12):
        if not cfg["do"]:
            continue
        refs = [dc.reference(cfg, w) for w in cfg["worlds"]]
        keep = [w for w, r in zip(cfg["worlds"], refs) if dc.in_domain(r)]
        out.append(({**cfg, "worlds": keep}, [r for r in refs if dc.in_domain(r)]))
    return out


def make_combat() -> None:
    """combat_{1,2}: the reference's combat scenarios (seed 1 development, 2 held out), batches with dynamical
    orientation (its missile exclusion on and off, master and client, every tick length and orbit law), recorded on
    the reference's VecCombatPark (its tick on tensors, CPU) by tests/golden/combat_trace.py's driver. Each batch is
    first run by the reference's own harness (destiny_combat_cases.batched) and compared with the scalar FullBallpark
    by its own comparison (destiny_combat_cases.differences): 0 differences, or the generator stops. Worlds the batch
    flags (outside its domain) are left out; the driver's run then gives the same events, answers and final state as
    the reference's harness."""
    import combat_trace as ct
    import destiny_combat_cases as dc
    import exact_ballpark.vec_combat as vc
    for seed in (1, 2):
        t = time.time()
        batches = []
        for cfg, refs in _combat_batches(seed):
            outs, park = dc.batched(cfg, "cpu", path="torch")
            flags = park.world_flags()
            keep = [k for k in range(len(cfg["worlds"])) if not flags[k]]
            for k in keep:
                bad = dc.differences(refs[k], outs[k])
                if bad:
                    raise RuntimeError(f"seed {seed}: the reference's batch differs from FullBallpark: {bad[:4]}")
            cfg = {**cfg, "worlds": [cfg["worlds"][k] for k in keep]}
            outs, park = dc.batched(cfg, "cpu", path="torch")
            if any(park.world_flags()):
                raise RuntimeError("a world flagged once its neighbours were left out")
            digests = []
            p, where = ct.make_park(vc.VecCombatPark, cfg, dc.FORMATIONS, "cpu")
            got = ct.drive(p, cfg, where, lambda s, q: digests.append(ct.field_digests(q)))
            want_e = [(wl, *e) for wl, o in enumerate(outs) for e in o["E"]]
            if sorted(got["E"]) != sorted(want_e) or got["A"] != [o["A"] for o in outs]:
                raise RuntimeError("the driver's run differs from the reference harness's (events or answers)")
            for f in ct.FIELDS + ("exists",):
                a, b = ct.canonical(getattr(p, f)), ct.canonical(getattr(park, f))
                if a.shape != b.shape or not (a.view(np.uint64) == b.view(np.uint64)).all():
                    raise RuntimeError(f"the driver's final {f} differs from the reference harness's")
            batches.append({"cfg": cfg, "digests": np.array(digests, dtype=np.uint64), "events": got["E"],
                            "answers": got["A"]})
        ct.save(HERE / f"combat_{seed}", dc.FORMATIONS, batches)
        print(f"  combat_{seed}: {len(batches)} batches, {sum(len(b['cfg']['worlds']) for b in batches)} worlds, "
              f"{sum(len(b['events']) for b in batches)} events, {time.time() - t:.0f} s")


def make_composed() -> None:
    """composed_{1,2}: the reference's composed-park scenarios (tests/park_cases.py: ship clusters with fixed spheres,
    GOTO, FOLLOW and ORBIT at short range, warps into and out of the cluster with their drop-outs, the setters,
    cloaks, formations, missiles launched at the ships; seed 1 development, 2 held out; 16 batches of 16 worlds as its
    own tests run them), the batches with dynamical orientation, recorded on the reference's VecComposedPark (its
    tick on tensors, CPU) by tests/golden/combat_trace.py's driver with the composed fields (the collision
    acceleration, the filing, the collision list). Each batch is first run by the reference's own harness
    (park_cases.batched) and compared with the scalar FullBallpark by its own comparison: 0 differences, or the
    generator stops. Worlds outside the reference's domain or flagged by the batch are left out."""
    import combat_trace as ct
    import destiny_combat_cases as dc
    import park_cases as pc
    import exact_ballpark.vec_composed as vp
    for seed in (1, 2):
        t = time.time()
        batches = []
        for cfg in pc.batches(seed, 16, 16):
            if not cfg["do"]:
                continue
            refs = [pc.reference(cfg, w) for w in cfg["worlds"]]
            outs, park = pc.batched(cfg, "cpu")
            flags = park.world_flags()
            keep = [k for k in range(len(cfg["worlds"])) if dc.in_domain(refs[k]) and not flags[k]]
            for k in keep:
                bad = pc.differences(refs[k], outs[k])
                if bad:
                    raise RuntimeError(f"seed {seed}: the reference's batch differs from FullBallpark: {bad[:4]}")
            if not keep:
                continue
            cfg = {**cfg, "worlds": [cfg["worlds"][k] for k in keep]}
            outs, park = pc.batched(cfg, "cpu")
            if any(park.world_flags()):
                raise RuntimeError("a world flagged once its neighbours were left out")
            digests = []
            p, where = ct.make_park(vp.VecComposedPark, cfg, pc.FORMATIONS, "cpu")
            got = ct.drive(p, cfg, where, lambda s, q: digests.append(ct.field_digests(q, ct.COMPOSED_FIELDS)))
            want_e = [(wl, *e) for wl, o in enumerate(outs) for e in o["E"]]
            if sorted(got["E"]) != sorted(want_e) or got["A"] != [o["A"] for o in outs]:
                raise RuntimeError("the driver's run differs from the reference harness's (events or answers)")
            for f in ct.COMPOSED_FIELDS + ("exists",):
                a, b = ct._field(p, f), ct._field(park, f)
                if a.shape != b.shape or not (a.view(np.uint64) == b.view(np.uint64)).all():
                    raise RuntimeError(f"the driver's final {f} differs from the reference harness's")
            batches.append({"cfg": cfg, "digests": np.array(digests, dtype=np.uint64), "events": got["E"],
                            "answers": got["A"]})
            print(f"    batch: {len(keep)} worlds, {len(got['E'])} events, {time.time() - t:.0f} s", flush=True)
        ct.save(HERE / f"composed_{seed}", pc.FORMATIONS, batches)
        print(f"  composed_{seed}: {len(batches)} batches, {sum(len(b['cfg']['worlds']) for b in batches)} worlds, "
              f"{sum(len(b['events']) for b in batches)} events, {time.time() - t:.0f} s", flush=True)


def make_server() -> None:
    """server_{modes,modes_do}: the reference's server-layer scenarios over the flight-mode park (tests/server_cases.py:
    40 worlds of one bubble with their pilots, 14 ticks of Actions calls each: conflicting commands, duplicates dropped
    and kept, cloaks and uncloaks in both orders, local and non-local SetBallPosition, follows and orbits of a
    cloaking ship, warps and warp-ins with followers, every setter, refused values; seeds 1 and 2; without and with
    dynamical orientation), recorded on the reference's VecServer (torch path, over its VecModesPark on the CPU) by
    tests/golden/server_trace.py's driver, with the digest of what every client is sent (the reference's decode). Each
    scenario set is first run by the reference's own comparison against its scalar server layer (server_cases.run:
    every ball's state and every client's update list): 0 differences."""
    import server_cases as S
    import server_trace as st
    import exact_ballpark.vec_server as VS
    from exact_ballpark.vec_modes import VecModesPark
    for do in (False, True):
        t = time.time()
        runs = []
        for seed in (1, 2):
            cs = S.cases(seed, 40, "modes", do=do, ticks=14)
            res = S.run(cs, "modes", "cpu", do=do, evolve=True)
            if res["rows"] or res["sends"] or not res["compared"]:
                raise RuntimeError(f"seed {seed}: the reference's server layer differs from its scalar one")
            parks, batches, sends = [], [], []

            def on_tick(tk, server):
                parks.append(tr.field_digests(server.a.park))
                batches.append(st.batch_digests(server))
                sends.append(st.decode_digest(VS.decode(server)))
            server, _ = st.build(VS, VecModesPark, cs, do, "cpu")
            st.drive(server, cs, True, "cpu", on_tick)
            runs.append({"cases": cs, "do": do, "evolve": True, "park": np.array(parks, dtype=np.uint64),
                         "batch": batches, "decode": sends})
        name = "server_modes_do" if do else "server_modes"
        st.save(HERE / name, runs)
        print(f"  {name}: {len(runs)} runs of {len(runs[0]['cases'])} worlds, {time.time() - t:.0f} s", flush=True)


def make_server_collide() -> None:
    """server_collide: the reference's server scenarios over the collision park (tests/server_cases.py with park
    "collide": 40 worlds of 2 to 5 massive balls within 3 km that meet, GotoPoint, GotoDirection, Stop, the speed
    fraction, SetBallMassive, SetBallInteractive, the cloaks; seeds 1 and 2, 14 ticks), recorded on the reference's
    VecServer over its CollideAdapter (torch path, its VecCollidePark on the CPU) by server_trace's driver: the park's
    fields (collide_trace's), the update batch and what every client is sent, after every tick. Each scenario set is
    first run by the reference's own comparison against its scalar server layer: 0 differences."""
    import server_cases as S
    import server_trace as st
    import exact_ballpark.vec_server as VS
    from exact_ballpark.vec_collide import VecCollidePark
    t0 = time.time()
    runs = []
    for seed in (1, 2):
        cs = S.cases(seed, 40, "collide", ticks=14)
        res = S.run(cs, "collide", "cpu", evolve=True)
        if res["rows"] or res["sends"] or not res["compared"]:
            raise RuntimeError(f"seed {seed}: the reference's server layer differs from its scalar one")
        parks, batches, sends = [], [], []

        def on_tick(tk, server):
            parks.append(st.park_digests("collide", server.a.park))
            batches.append(st.batch_digests(server))
            sends.append(st.decode_digest(VS.decode(server)))
        server, _ = st.build(VS, VecCollidePark, cs, False, "cpu", park="collide")
        st.drive(server, cs, True, "cpu", on_tick)
        runs.append({"cases": cs, "do": False, "evolve": True, "park": np.array(parks, dtype=np.uint64),
                     "batch": batches, "decode": sends, "park_kind": "collide"})
    st.save(HERE / "server_collide", runs)
    print(f"  server_collide: {len(runs)} runs of 40 worlds, {time.time() - t0:.0f} s", flush=True)


def make_server_pending() -> None:
    """server_pending: the reference's pending-query scenarios over the flight-mode park (tests/server_pending_cases.py's
    augment over tests/server_cases.py's worlds: 40 worlds of one bubble, 12 ticks, the game's queries of every kind at
    any place among the calls, undos of a pending cloak, a cloak pushed twice then undone, undone then pushed again with
    another mode, the prune's edge X, CloakBall, X, undo; seeds 101 and held-out 117), recorded on the reference's
    VecServer (torch path, over its VecModesPark on the CPU) by server_trace's driver with every answer's digest. Each
    scenario set is first run by the reference's own comparison against its scalar server layer (every answer, every
    client's update list, every ship's state): 0 differences."""
    import server_cases as S
    import server_pending_cases as P
    import server_trace as st
    import exact_ballpark.vec_server as VS
    from exact_ballpark.vec_modes import VecModesPark
    t0 = time.time()
    runs = []
    for seed in (101, 117):
        cs = P.augment(S.cases(seed, 40, "modes", ticks=12), "server", f"modes-{seed}", P.MODES["server"]["modes"])
        server, index = S.build(cs, "modes", "cpu")
        res = P.run(cs, "modes", "cpu", server, index, [S.ScalarWorld(w) for w in cs])
        if res["answers"] or res["sends"] or res["rows"] or res["flagged"]:
            raise RuntimeError(f"seed {seed}: the reference's server layer differs from its scalar one")
        cs = P.augment(S.cases(seed, 40, "modes", ticks=12), "server", f"modes-{seed}", P.MODES["server"]["modes"])
        parks, batches, answers, sends = [], [], [], []

        def on_tick(tk, server, ans):
            parks.append(tr.field_digests(server.a.park))
            batches.append(st.batch_digests(server))
            answers.append(ans)
            sends.append(st.decode_digest(VS.decode(server)))
        server, _ = st.build(VS, VecModesPark, cs, False, "cpu")
        st.drive_pending(server, cs, "cpu", on_tick)
        runs.append({"cases": cs, "do": False, "evolve": True, "park": np.array(parks, dtype=np.uint64),
                     "batch": batches, "answers": answers, "decode": sends})
        print(f"  seed {seed}: {res['volumes']['answers']} answers, {res['volumes']['undos']} undos", flush=True)
    st.save(HERE / "server_pending", runs)
    print(f"  server_pending: {len(runs)} runs of 40 worlds, {time.time() - t0:.0f} s", flush=True)


def make_server_ontick() -> None:
    """server_ontick: the reference's OnTick scenarios over the flight-mode park (tests/server_ontick_cases.py's
    server_cases: 32 worlds, 14 OnTick calls, each world's own simulation clock: calls too early, a world's first call,
    one interval, remainders carried, several intervals, the master's resynchronisation, the last call pushed again
    across a kept queue; seed 1 development and 31 held out, dynamical orientation off and on), recorded on the
    reference's VecServer (torch path, over its VecModesPark on the CPU) by server_trace's driver: after every call the
    park's fields, each world's clocks and every round's worlds and update batch. Each scenario set is first run by
    the reference's own comparison against its scalar server layer under OnTick (every send, every ship's fields,
    the clocks): 0 differences."""
    import server_ontick_cases as O
    import server_trace as st
    import exact_ballpark.vec_server as VS
    from exact_ballpark.vec_modes import VecModesPark
    t0 = time.time()
    runs = []
    for do in (False, True):
        for seed in (1, 31):
            res = O.run(O.server_cases(seed, 32, "modes", do, 14), "modes", "cpu", do=do)
            if res["sends"] or res["rows"] or res["clocks"]:
                raise RuntimeError(f"seed {seed}: the reference's OnTick differs from its scalar one")
            cs = O.server_cases(seed, 32, "modes", do, 14)
            parks, calls, sends = [], [], []

            def on_call(tk, server, batches):
                parks.append(tr.field_digests(server.a.park))
                calls.append(st.ontick_digests(server, batches))
                sends.append(st.decode_digest([VS.decode(server, b) for b in batches]))
            server, _ = st.build(VS, VecModesPark, cs, do, "cpu")
            st.drive_ontick(server, cs, "cpu", on_call)
            runs.append({"cases": cs, "do": do, "evolve": True, "ontick": True,
                         "park": np.array(parks, dtype=np.uint64), "batch": calls, "decode": sends})
            print(f"  do={do} seed {seed}: {res['coverage']}, {len(res['out'])} worlds left the domain", flush=True)
    st.save(HERE / "server_ontick", runs)
    print(f"  server_ontick: {len(runs)} runs, {time.time() - t0:.0f} s", flush=True)


def make_server_collide_more() -> None:
    """server_collide_ontick: the reference's OnTick scenarios over the collision park (tests/server_ontick_cases.py's
    server_cases with park "collide", seed 1: 32 worlds, 14 calls), recorded on the reference's VecServer over its
    CollideAdapter (torch path, its VecCollidePark on the CPU) by server_trace's driver, after the set is first run by
    the reference's own comparison against its scalar server layer under OnTick: 0 differences. (Its pending queries
    do not run over the collision park: the reference reads the park's [W, N] speed fraction by row.)"""
    import server_ontick_cases as O
    import server_trace as st
    import exact_ballpark.vec_server as VS
    from exact_ballpark.vec_collide import VecCollidePark
    t0 = time.time()
    seed = 1
    res = O.run(O.server_cases(seed, 32, "collide", False, 14), "collide", "cpu")
    if res["sends"] or res["rows"] or res["clocks"]:
        raise RuntimeError("the reference's collision server layer differs from its scalar one (OnTick)")
    cs = O.server_cases(seed, 32, "collide", False, 14)
    parks, calls, sends = [], [], []

    def on_call(tk, server, batches):
        parks.append(st.park_digests("collide", server.a.park))
        calls.append(st.ontick_digests(server, batches))
        sends.append(st.decode_digest([VS.decode(server, b) for b in batches]))
    server, _ = st.build(VS, VecCollidePark, cs, False, "cpu", park="collide")
    st.drive_ontick(server, cs, "cpu", on_call)
    st.save(HERE / "server_collide_ontick", [{"cases": cs, "do": False, "evolve": True, "ontick": True,
                                              "park_kind": "collide", "park": np.array(parks, dtype=np.uint64),
                                              "batch": calls, "decode": sends}])
    print(f"  server_collide_ontick: {res['coverage']}, {time.time() - t0:.0f} s", flush=True)


def make_space_bubbles() -> None:
    """space_bubbles: the master's partition and bubble partition of one world (tests/golden/space_trace.py's streams:
    60 worlds of 60 mixed operations, 6 of 600, 6 sweeps past BoxAllocator's 256 kept boxes, 40 ticking worlds of 80
    operations with ships flying across top boxes, 40 worlds of the follow, orbit and warp modes, 40 worlds of
    collisions inside the tick), each operation's state
    digest recorded on the reference's own SpaceBallpark (exact_ballpark.space, is_master). A stream whose reference run
    reads a deleted box (DestinyUndefined) is left out."""
    import space_trace as sp
    from exact_ballpark.space import DestinyUndefined, SpaceBallpark
    t0 = time.time()
    scenarios, dropped = [], 0
    streams = ([("mixed", s, sp.ops_for(s)) for s in range(1, 61)]
               + [("long", s, sp.ops_for(s, n_ops=600)) for s in range(1000, 1006)]
               + [("sweep", s, sp.sweep_ops(s)) for s in range(1, 7)]
               + [("tick", s, sp.tick_ops(s)) for s in range(1, 41)]
               + [("modes", s, sp.mode_ops(s)) for s in range(1, 41)]
               + [("collide", s, sp.collide_ops(s)) for s in range(1, 41)])
    for family, seed, ops in streams:
        park = SpaceBallpark(1.0e6, 1000, is_master=True, seed=seed)
        digests = []
        try:
            for op in ops:
                answer = sp.apply(park, op)
                digests.append(sp.digest(sp.state_text(park) + answer))
        except DestinyUndefined:
            dropped += 1
            continue
        scenarios.append({"seed": f"{family}-{seed}", "ops": ops, "digests": digests, "rand_seed": seed})
    sp.save(HERE / "space_bubbles", scenarios)
    print(f"  space_bubbles: {len(scenarios)} worlds, {sum(len(s['ops']) for s in scenarios)} operations, "
          f"{dropped} left out, {time.time() - t0:.0f} s", flush=True)


def make_space_crowd() -> None:
    """space_crowd: crowded worlds of 16 to 128 sensing ships (tests/golden/space_trace.py's crowd_ops: the sensors'
    lists and the proximity map past the rehash policy's growths), each operation's state digest recorded on the
    reference's own SpaceBallpark (is_master)."""
    import space_trace as sp
    from exact_ballpark.space import SpaceBallpark
    t0 = time.time()
    scenarios = []
    for seed in range(1, 9):
        ops = sp.crowd_ops(seed)
        park = SpaceBallpark(1.0e6, 1000, is_master=True, seed=seed)
        digests = []
        for op in ops:
            answer = sp.apply(park, op)
            digests.append(sp.digest(sp.state_text(park) + answer))
        scenarios.append({"seed": f"crowd-{seed}", "ops": ops, "digests": digests, "rand_seed": seed})
        print(f"    crowd-{seed}: {int(max(op[1] for op in ops))} ships, {len(ops)} operations, "
              f"{time.time() - t0:.0f} s", flush=True)
    sp.save(HERE / "space_crowd", scenarios)
    print(f"  space_crowd: {len(scenarios)} worlds, {time.time() - t0:.0f} s", flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=("libm", "libm_dense", "powf", "traces", "workload", "collide", "collide_crowd", "rand", "combat", "composed", "server", "server_pending", "server_ontick",
                                       "server_collide", "server_collide_more", "space_bubbles", "space_crowd"),
                    default=None)
    ap.add_argument("--sample", type=int, default=3, help="scenarios per family checked against the scalar reference")
    a = ap.parse_args()
    if a.only in (None, "libm"):
        make_libm(np.random.default_rng(20261203))
    if a.only in (None, "powf"):
        make_powf(np.random.default_rng(20261204))
    if a.only in (None, "libm_dense"):
        make_libm_dense(np.random.default_rng(20261205))
    if a.only in (None, "workload"):
        make_workload_traces()
    if a.only in (None, "traces"):
        make_traces(a.sample)
    if a.only in (None, "collide"):
        make_collide_traces(a.sample)
    if a.only in (None, "collide_crowd"):
        make_collide_crowd()
    if a.only in (None, "rand"):
        make_rand()
    if a.only in (None, "combat"):
        make_combat()
    if a.only in (None, "composed"):
        make_composed()
    if a.only in (None, "server"):
        make_server()
    if a.only in (None, "server_pending"):
        make_server_pending()
    if a.only in (None, "server_ontick"):
        make_server_ontick()
    if a.only in (None, "server_collide"):
        make_server_collide()
    if a.only in (None, "server_collide_more"):
        make_server_collide_more()
    if a.only in (None, "space_bubbles"):
        make_space_bubbles()
    if a.only in (None, "space_crowd"):
        make_space_crowd()


if __name__ == "__main__":
    main()
