// SPDX-License-Identifier: MIT
// One ship's flight tick on the device: Destiny's flight-mode laws and dynamical orientation as per-ship device
// functions, each expression in the order of the reference's scalar transcription (exact_ballpark/modes.py for the
// modes, exact_ballpark/full.py for dynamical orientation; Carbon's destiny at 114e89fa, Ballpark.cpp), with every
// rounding pinned (ebb_arith.cuh) and glibc 2.34 aarch64's libm (ebb_libm.cuh). Floats are computed in float where
// Destiny's members are floats, doubles in double.
#pragma once

#include "ebb_libm.cuh"
#include "ebb_vec.cuh"

namespace ebb {
namespace flight {

// Destiny's DSTBALLMODE (IDstConstants.h; modes.py:65-67)
enum : int32_t { GOTO = 0, FOLLOW = 1, STOP = 2, WARP = 3, ORBIT = 4, MISSILE = 5, MUSHROOM = 6, BOID = 7, TROLL = 8,
                 MINIBALL = 9, FIELD = 10, RIGID = 11, FORMATION = 12 };

// Destiny's constants, as the reference states them (modes.py:72-78, vec_modes.py:95-109)
constexpr double AU = .1495978707e12;
constexpr double ORBITAL_PRECESSION = 0.001;
constexpr double WARP_AU_PER_S = 0.001;
constexpr double WARP_ACC = 1.0 / 1000;
constexpr double WARP_DEC = 1.0 / 3000;
constexpr int64_t MAX_ALIGN_TICKS = 180;
constexpr double STOP_DECAY = 0.07;
constexpr double STOP_DAMP = 0.9345794392523364485981308411215;
constexpr double TRUNC7 = 10000000.0;
constexpr double RF_SCALE = 40000.0;
constexpr double GOTO_FAR = 10.0;                   // x AU: the old orbit's goto point
constexpr double NORMAL_MIN = 1e-12;
constexpr double ANGLE_SCALE = 0.1;
constexpr double ANGLE_ZERO = 1e-10;
constexpr double FACTOR_FLOOR = -0.999;
constexpr double LOG_FLOOR = 0.001;
constexpr double SLOW_TARGET = 5e-2;
constexpr double THRUST_OFF = 0.1;
constexpr double ALIGN_COS = 0.01;
constexpr double ALIGN_SPEED2 = 0.5625;
constexpr double DROP_SPEED = 100.0;
constexpr double DIR_DIST = 1.0e17;
constexpr double TAYLOR_LIMIT = 1e-10;
constexpr double DO_THRUST = 1e-2;
constexpr int TORQUE_STEPS = 100;                   // n1 = 1 .. 99
constexpr int TORQUE_ROUNDS = 5;

// The tick's scalars
struct Cfg {
    double friction, dt;
    float ffriction, fdt;
    int new_orbit, dynamical;
};

// One ship as its thread holds it
struct Ship {
    D3 pos, vel, gp, last_g;
    double mass, tf, last_collision;
    float radius, max_vel, agility, sf, follow_range;
    int64_t id, effect_stamp, follow_id, owner_id, clock;
    int32_t mode, follow_ptr;
    bool massive, interactive, sensor;
};

// ============================================================================================ thrust laws

// GotoThrust (ref.py:343; Ballpark.cpp:1397): maxThrust along the unit vector to the target, tapered by
// (L^2 / D^2)^2 inside one tick's distance D
__device__ __forceinline__ D3 goto_thrust(const Ship& s, D3 target, const Cfg& c) {
    const D3 a = d3_sub(target, s.pos);
    const double length2 = d3_lensq(a);
    const double sf = tod(s.sf), mv = tod(s.max_vel);
    const double dist = dmul(dmul(sf, mv), c.dt);
    const double max_thrust = ddiv(dmul(dmul(c.friction, sf), mv), dmul(s.mass, tod(s.agility)));
    const D3 unit = d3_unit(a);
    const double dd = dmul(dist, dist);
    if (length2 < dd) {
        const double coff = ddiv(length2, dd);
        return d3_mul(unit, dmul(dmul(max_thrust, coff), coff));
    }
    return d3_mul(unit, max_thrust);
}

// EvolveFollow (modes.py:428): the point at followRange + both radii from the target, on the line from it
__device__ __forceinline__ D3 follow_thrust(Ship& s, D3 tpos, float tradius, const Cfg& c) {
    const D3 delta = d3_sub(s.pos, tpos);
    const double dist = d3_len(delta);
    const double r = dadd(dadd(tod(s.follow_range), tod(s.radius)), tod(tradius));
    if (dist == 0.0) {
        s.gp = D3{dadd(tpos.x, dmul(1.0, r)), dadd(tpos.y, dmul(0.0, r)), dadd(tpos.z, dmul(0.0, r))};
    } else {
        const double inv = ddiv(1.0, dist);
        s.gp = D3{dadd(tpos.x, dmul(dmul(delta.x, r), inv)), dadd(tpos.y, dmul(dmul(delta.y, r), inv)),
                  dadd(tpos.z, dmul(dmul(delta.z, r), inv))};
    }
    return goto_thrust(s, s.gp, c);
}

// (double)((int64_t)(x 1e7)) / 1e7 (modes.py:94)
__device__ __forceinline__ double trunc7(double x) { return ddiv(i2d(to_i64(dmul(x, TRUNC7))), TRUNC7); }

// DefaultOrbitalNormal (modes.py:480): the precessing w, truncated to 7 decimals, not normalised
inline __device__ __noinline__ D3 precessing_w(int64_t clock, int64_t id) {
    const double t = i2d(clock);
    const double phi1 = dmul(t, ORBITAL_PRECESSION);
    const double phi2 = dadd(i2d(id & 0xFFFFLL), dmul(t, ORBITAL_PRECESSION));
    const lm::SinCos a = lm::sincos_v(phi1), b = lm::sincos_v(phi2);
    return D3{trunc7(dmul(a.c, b.c)), trunc7(b.s), trunc7(dmul(a.s, b.c))};
}
__device__ __forceinline__ D3 precessing_normal(const Ship& s) { return precessing_w(s.clock, s.id); }

// EvolveOldStyleOrbit (modes.py:444)
__device__ __forceinline__ D3 old_orbit_thrust(Ship& s, D3 tpos, float tradius, const Cfg& c) {
    const double cruise = dmul(tod(s.sf), tod(s.max_vel));
    const double max_thrust = ddiv(dmul(c.friction, cruise), dmul(s.mass, tod(s.agility)));
    const double r = dadd(dadd(tod(s.follow_range), tod(s.radius)), tod(tradius));
    D3 to = d3_sub(tpos, s.pos);
    const double dist = d3_len(to);
    to = d3_unit(to);
    const D3 w = d3_unit(d3_cross(precessing_normal(s), to));
    const double to_comp = dsub(dmul(dist, dist), dmul(r, r));
    if (to_comp >= 0.0) {
        const double rad_comp = ddiv(dmul(r, dsqrt(to_comp)), dist);
        const double sc = ddiv(to_comp, dist);
        to = d3_unit(D3{dadd(dmul(to.x, sc), dmul(w.x, rad_comp)), dadd(dmul(to.y, sc), dmul(w.y, rad_comp)),
                        dadd(dmul(to.z, sc), dmul(w.z, rad_comp))});
    }
    const double dr = dsub(r, dist);
    const double rf = trunc7(lm::exp(ddiv(dmul(dneg(dr), dr), RF_SCALE)));
    const double phi = dadd(dadd(dmul(dneg(to.x), w.x), dmul(dneg(to.y), w.y)), dmul(dneg(to.z), w.z));
    double k = dadd(1.0, dmul(dmul(rf, rf), dsub(dmul(phi, phi), 1.0)));
    k = (k > 0.0) ? dadd(dmul(rf, phi), dsqrt(k)) : dmul(rf, phi);
    k = dmul(k, dsub(dist, r) >= 0.0 ? 1.0 : -1.0);
    const D3 a = D3{dmul(dadd(dmul(w.x, rf), dmul(to.x, k)), max_thrust),
                    dmul(dadd(dmul(w.y, rf), dmul(to.y, k)), max_thrust),
                    dmul(dadd(dmul(w.z, rf), dmul(to.z, k)), max_thrust)};
    s.gp = d3_add(s.pos, d3_mul(a, dmul(GOTO_FAR, AU)));
    return a;
}

// OrbitThrust (modes.py:586): brake toward the point, zero below a tenth of the maximum acceleration
__device__ __forceinline__ D3 brake_thrust(const Ship& s, D3 target, const Cfg& c) {
    const double fom = ddiv(c.friction, dmul(s.mass, tod(s.agility)));
    const double max_accel = dmul(dmul(fom, tod(s.sf)), tod(s.max_vel));
    if (max_accel <= 0.0) return D3{0.0, 0.0, 0.0};
    D3 a = D3{dsub(dmul(dsub(target.x, s.pos.x), fom), s.vel.x), dsub(dmul(dsub(target.y, s.pos.y), fom), s.vel.y),
              dsub(dmul(dsub(target.z, s.pos.z), fom), s.vel.z)};
    const double tacc = ddiv(d3_len(a), max_accel);
    if (tacc > 1.0) a = d3_mul(a, ddiv(1.0, tacc));
    if (tacc < THRUST_OFF) return D3{0.0, 0.0, 0.0};
    return a;
}

// GotoThrustFollow (modes.py:557) with weight 1: reach the point and match the velocity, capped
__device__ __forceinline__ D3 match_thrust(const Ship& s, D3 target, D3 tv, const Cfg& c) {
    const double sf = tod(s.sf), mv = tod(s.max_vel);
    if (d3_len(tv) < dmul(dmul(SLOW_TARGET, mv), sf)) {
        if (c.new_orbit && s.mode == ORBIT) return brake_thrust(s, target, c);
        return goto_thrust(s, s.gp, c);
    }
    const double fom = ddiv(c.friction, dmul(s.mass, tod(s.agility)));
    const double max_accel = dmul(dmul(fom, sf), mv);
    if (max_accel <= 0.0) return D3{0.0, 0.0, 0.0};
    const double one_minus = dsub(1.0, s.tf);
    double inv = ddiv(1.0, dsub(dmul(c.dt, fom), one_minus));
    D3 a = D3{dmul(dmul(dsub(dmul(dsub(target.x, s.pos.x), fom), dmul(s.vel.x, one_minus)), fom), inv),
              dmul(dmul(dsub(dmul(dsub(target.y, s.pos.y), fom), dmul(s.vel.y, one_minus)), fom), inv),
              dmul(dmul(dsub(dmul(dsub(target.z, s.pos.z), fom), dmul(s.vel.z, one_minus)), fom), inv)};
    inv = ddiv(1.0, dsub(1.0, s.tf));
    const D3 av = D3{dmul(dmul(dsub(tv.x, dmul(s.vel.x, s.tf)), fom), inv),
                     dmul(dmul(dsub(tv.y, dmul(s.vel.y, s.tf)), fom), inv),
                     dmul(dmul(dsub(tv.z, dmul(s.vel.z, s.tf)), fom), inv)};
    const double weight = 1.0;
    inv = ddiv(1.0, dadd(1.0, weight));
    a = D3{dmul(dadd(a.x, dmul(av.x, weight)), inv), dmul(dadd(a.y, dmul(av.y, weight)), inv),
           dmul(dadd(a.z, dmul(av.z, weight)), inv)};
    const double acc2 = d3_lensq(a);
    if (acc2 > dmul(max_accel, max_accel)) a = d3_mul(a, ddiv(max_accel, dsqrt(acc2)));
    return a;
}

// EvolveNewStyleOrbit (modes.py:509) with GetOrbitalNormal (modes.py:488; with dynamical orientation the heading's
// fallback, full.py:2385): a logarithmic spiral toward the orbit radius. tvel is the target's velocity as this ship
// sees it at its own turn; rot its rotation at the start of the tick.
__device__ __forceinline__ D3 new_orbit_thrust(Ship& s, D3 tpos, D3 tvel, float tradius, const Cfg& c, F4 rot) {
    const double cruise = dmul(tod(s.sf), tod(s.max_vel));
    const double tau = ddiv(dmul(s.mass, tod(s.agility)), c.friction);
    const double max_thrust = ddiv(cruise, tau);
    const double r = dadd(dadd(tod(s.follow_range), tod(s.radius)), tod(tradius));
    D3 to = d3_sub(tpos, s.pos);
    to = D3{dadd(to.x, dmul(tvel.x, c.dt)), dadd(to.y, dmul(tvel.y, c.dt)), dadd(to.z, dmul(tvel.z, c.dt))};
    double dist = d3_len(to);
    to = (dist > 0.0) ? d3_mul(to, ddiv(1.0, dist)) : D3{0.0, 0.0, 1.0};
    D3 o = d3_cross(to, s.vel);
    double l2 = d3_lensq(o);
    D3 normal;
    if (l2 > NORMAL_MIN) {
        normal = d3_mul(o, ddiv(1.0, dsqrt(l2)));
    } else if (!c.dynamical) {
        normal = precessing_normal(s);
    } else {
        const F3 h = m_apply(F3{0.0f, 0.0f, 1.0f}, m_of_q(rot));
        o = d3_cross(to, d3_of(h));
        l2 = d3_lensq(o);
        normal = (l2 <= NORMAL_MIN) ? precessing_normal(s) : d3_mul(o, ddiv(1.0, dsqrt(l2)));
    }
    const D3 radial = d3_unit(d3_cross(normal, to));
    const double speed = d3_len(s.vel);
    const double max_speed = (cruise < speed) ? speed : cruise;
    double angle = ddiv(dmul(ANGLE_SCALE, dsub(r, dist)), max_speed);
    if (angle < -1.0) angle = -1.0;
    if (angle > 1.0) angle = 1.0;
    if (dist < ANGLE_SCALE) dist = ANGLE_SCALE;
    const double sq = dsqrt(dmul(dist, max_thrust));
    const double est_v = (sq < max_speed) ? sq : max_speed;
    const double est_d = dmul(est_v, c.dt);
    D3 gp, gv;
    if (dabs(angle) < ANGLE_ZERO) {                                  // the circle
        const double t = ddiv(est_d, dist);
        const lm::SinCos sc = lm::sincos_v(t);
        const double st = sc.s, ct = sc.c;
        const double cp = dmul(dist, dsub(1.0, ct)), sp = dmul(dist, st), cv = dmul(ct, est_v), sv = dmul(st, est_v);
        gp = D3{dadd(dmul(to.x, cp), dmul(radial.x, sp)), dadd(dmul(to.y, cp), dmul(radial.y, sp)),
                dadd(dmul(to.z, cp), dmul(radial.z, sp))};
        gv = D3{dadd(dmul(radial.x, cv), dmul(to.x, sv)), dadd(dmul(radial.y, cv), dmul(to.y, sv)),
                dadd(dmul(radial.z, cv), dmul(to.z, sv))};
    } else {                                                         // the spiral
        const double factor = ddiv(ddiv(dmul(est_d, angle), dist), dsqrt(dadd(dmul(angle, angle), 1.0)));
        double t;
        if (factor < FACTOR_FLOOR) t = ddiv(lm::log(LOG_FLOOR), angle);
        else if (dabs(factor) > ANGLE_ZERO) t = ddiv(lm::log(dadd(1.0, factor)), angle);
        else t = ddiv(factor, angle);
        const double dexp = dmul(dist, lm::exp(dmul(angle, t)));
        const lm::SinCos sc = lm::sincos_v(t);
        const double st = sc.s, ct = sc.c;
        const double cp = dsub(dist, dmul(dexp, ct)), sp = dmul(dexp, st);
        gp = D3{dadd(dmul(to.x, cp), dmul(radial.x, sp)), dadd(dmul(to.y, cp), dmul(radial.y, sp)),
                dadd(dmul(to.z, cp), dmul(radial.z, sp))};
        const double ca = dadd(dmul(dneg(angle), ct), st), sa = dadd(dmul(angle, st), ct);
        gv = d3_mul(d3_unit(D3{dadd(dmul(to.x, ca), dmul(radial.x, sa)), dadd(dmul(to.y, ca), dmul(radial.y, sa)),
                               dadd(dmul(to.z, ca), dmul(radial.z, sa))}),
                    est_v);
    }
    s.gp = d3_add(s.pos, gp);
    return match_thrust(s, s.gp, d3_add(gv, tvel), c);
}

// ============================================================================================ warp

// IsAlignedForWarp of an aligning ship (modes.py:342): within |1 - cos| < 0.01 above 75 % of maxVel, or past 180
// aligning ticks
__device__ __forceinline__ bool aligned_for_warp(D3 gp, D3 pos, D3 vel, float max_vel, int64_t stamp) {
    const D3 d = d3_unit(d3_sub(gp, pos));
    const D3 u = d3_unit(vel);
    const double mv = tod(max_vel);
    if (dabs(dsub(1.0, d3_dot(u, d))) < ALIGN_COS && d3_lensq(vel) > dmul(dmul(ALIGN_SPEED2, mv), mv)) return true;
    return (stamp < 0 ? -stamp : stamp) > MAX_ALIGN_TICKS;
}

// RealWarp's own part (modes.py:391): the exit point min range short of the goto point, warp proper from now
__device__ __forceinline__ void start_warp(Ship& s) {
    D3 dst = s.gp;
    const D3 back = d3_unit(d3_sub(s.pos, dst));
    const double mr = dfrom((uint64_t)s.follow_id);                  // WarpTo keeps the minimum range's bits
    dst = d3_add(dst, d3_mul(back, mr));
    s.gp = dst;
    s.effect_stamp = s.clock;
    s.last_collision = d3_len(d3_sub(dst, s.pos));
    s.massive = false;
    s.sensor = false;
}

// WarpDistance with SetupWarpConstants (modes.py:606-666): the position and velocity t seconds into warp proper on
// the line to the exit point; true when the ship drops out (slow enough, or past the deceleration)
__device__ __forceinline__ bool warp_path(const Ship& s, D3* pp, D3* vp, double t) {
    const double wf = i2d(s.owner_id);
    const double wd = s.last_collision;
    double speed_max = dmul(dmul(wf, WARP_AU_PER_S), AU);
    const double acc = dmul(wf, WARP_ACC);
    const double d0 = dmul(wf, WARP_DEC);
    const double dec = (2.0 < d0) ? 2.0 : d0;
    const double cap = ddiv(dmul(dmul(dadd(wd, 1.0), acc), dec), dadd(acc, dec));
    const double sv = (cap < speed_max) ? cap : speed_max;
    const double t_a = ddiv(lm::log(ddiv(sv, acc)), acc);
    const double t_c = dadd(dsub(dsub(ddiv(wd, sv), ddiv(1.0, acc)), ddiv(1.0, dec)), ddiv(1.0, sv));
    const double t_d = ddiv(lm::log(ddiv(sv, dec)), dec);
    const double d_a = ddiv(sv, acc), d_c = dmul(sv, t_c), d_d = dsub(ddiv(sv, dec), 1.0);
    const D3 d = d3_unit(d3_sub(s.gp, *pp));
    const double total = dadd(dadd(d_a, d_c), d_d);
    if (t < t_a) {
        const double e = lm::exp(dmul(acc, t));
        double speed = dmul(acc, e);
        const double cur = d3_len(*vp);
        if (cur > speed) speed = cur;
        *vp = d3_mul(d, speed);
        *pp = d3_sub(s.gp, d3_mul(d, dsub(total, e)));
        return false;
    }
    if (dsub(t, t_a) < t_c) {
        *vp = d3_mul(d, sv);
        *pp = d3_sub(s.gp, d3_mul(d, dsub(total, dadd(dmul(sv, dsub(t, t_a)), d_a))));
        return false;
    }
    if (dsub(dsub(t, t_c), t_a) < dadd(t_d, 1.0)) {
        const double e = lm::exp(dmul(dneg(dec), dsub(dsub(t, t_c), t_a)));
        const double speed = dmul(sv, e);
        *vp = d3_mul(d, speed);
        const double sd = ddiv(sv, dec);
        *pp = d3_sub(s.gp, d3_mul(d, dsub(total, dadd(dadd(dsub(sd, dmul(sd, e)), d_a), d_c))));
        const double half = ddiv(tod(s.max_vel), 2.0);
        return speed < ((DROP_SPEED < half) ? DROP_SPEED : half);
    }
    *pp = s.gp;
    *vp = D3{0.0, 0.0, 0.0};
    return true;
}

// ============================================================================================ commands in a tick

// Stop(Ball*)'s follow part (modes.py:206): the follow fields cleared (a follower's set membership is implicit)
__device__ __forceinline__ void clear_follow(Ship& s) {
    s.effect_stamp = 0;
    s.follow_ptr = -1;
    s.follow_id = 0;
    s.owner_id = 0;
    s.follow_range = 0.0f;
}

// StopAllFollowers on one member (modes.py:410): an interactive orbiter flies on by GotoDirection(its velocity)
// (refused, so left as it is, when the velocity or the point is not finite); any other member stops. Returns the
// mode it is left in; applies it when `apply`.
__device__ __forceinline__ int32_t release(Ship& s, bool apply) {
    if (s.interactive && s.mode == ORBIT) {
        if (!d3_finite(s.vel)) return s.mode;
        const D3 p = d3_add(s.pos, d3_mul(d3_unit(s.vel), DIR_DIST));
        if (!d3_finite(p)) return s.mode;
        if (apply) {
            clear_follow(s);
            s.gp = p;
            if (s.sf == 0.0f) s.sf = 1.0f;
            s.mode = GOTO;
        }
        return GOTO;
    }
    if (apply) {
        if (s.mode == FOLLOW || s.mode == ORBIT) clear_follow(s);
        s.mode = STOP;
    }
    return STOP;
}

// ============================================================================================ the integrator

// Ballpark::Integrate over one tick (ref.py:354): the closed form with the cached decay factor, or its Taylor branch
__device__ __forceinline__ void integrate(D3* pp, D3* vp, D3 a, double m, double k, double tf, double t) {
    if (t == 0.0) return;
    const D3 p = *pp, v = *vp;
    const double k2 = dmul(k, k), ook2 = ddiv(1.0, k2), ook = ddiv(1.0, k);
    D3 pn;
    if (k < dmul(dmul(TAYLOR_LIMIT, m), t)) {
        const double inv_m = ddiv(1.0, m);
        const double kt = dmul(dneg(k), t);
        pn.x = dmul(dadd(dmul(m, dadd(dmul(a.x, kt), dmul(k, dadd(dmul(a.x, t), dmul(dmul(dmul(v.x, k), inv_m), t))))),
                         dmul(p.x, k2)), ook2);
        pn.y = dmul(dadd(dmul(m, dadd(dmul(a.y, kt), dmul(k, dadd(dmul(a.y, t), dmul(dmul(dmul(v.y, k), inv_m), t))))),
                         dmul(p.y, k2)), ook2);
        pn.z = dmul(dadd(dmul(m, dadd(dmul(a.z, kt), dmul(k, dadd(dmul(a.z, t), dmul(dmul(dmul(v.z, k), inv_m), t))))),
                         dmul(p.z, k2)), ook2);
    } else {
        const double tf1 = dsub(tf, 1.0);
        pn.x = dmul(dadd(dmul(m, dadd(dmul(dmul(m, a.x), tf1), dmul(k, dsub(dadd(dmul(a.x, t), v.x), dmul(tf, v.x))))),
                         dmul(p.x, k2)), ook2);
        pn.y = dmul(dadd(dmul(m, dadd(dmul(dmul(m, a.y), tf1), dmul(k, dsub(dadd(dmul(a.y, t), v.y), dmul(tf, v.y))))),
                         dmul(p.y, k2)), ook2);
        pn.z = dmul(dadd(dmul(m, dadd(dmul(dmul(m, a.z), tf1), dmul(k, dsub(dadd(dmul(a.z, t), v.z), dmul(tf, v.z))))),
                         dmul(p.z, k2)), ook2);
    }
    vp->x = dmul(dsub(dmul(m, a.x), dmul(dsub(dmul(m, a.x), dmul(v.x, k)), tf)), ook);
    vp->y = dmul(dsub(dmul(m, a.y), dmul(dsub(dmul(m, a.y), dmul(v.y, k)), tf)), ook);
    vp->z = dmul(dsub(dmul(m, a.z), dmul(dsub(dmul(m, a.z), dmul(v.z, k)), tf)), ook);
    *pp = pn;
}

// ============================================================================================ dynamical orientation

// A ship's turning values for one tick (full.py:2115-2124)
struct Turn {
    float max_ang_vel, t_scale, tf, tau_s;     // tf = expf(-dt t_scale); tau_s = 1 / t_scale
    double dt;
    float fdt;
    const float* ndt_tab;                      // float(n dt) for n = 0 .. TORQUE_STEPS - 1 (shared memory)
};

// float(n dt)
__device__ __forceinline__ float ndt(int n, double dt) { return tof(dmul((double)n, dt)); }

// The table float(n dt), n = 0 .. TORQUE_STEPS - 1, that a block's searches read (filled by the block's threads)
__device__ __forceinline__ void fill_ndt(float* tab, double dt) {
    for (int k = threadIdx.x; k < TORQUE_STEPS; k += blockDim.x) tab[k] = ndt(k, dt);
}

// The least float y with fsqrt(y) >= m, for m > 0: then fsqrt(x) < m exactly when x < y (fsqrt is correctly rounded,
// so monotonic; x a sum of squares, never negative). Found from m m by unit steps, at most a few. False (the test
// stays fsqrt(x) < m) if it does not settle within 64 steps.
__device__ __forceinline__ bool sqrt_threshold(float m, float* out) {
    float y = fmul(m, m);
    if (!(y == y)) {                                                  // m NaN: no x passes either way
        *out = y;
        return true;
    }
    if (fsqrt(y) >= m) {
        for (int k = 0; k < 64; ++k) {
            if (y == 0.0f) {
                *out = y;
                return true;
            }
            const float below = ffrom(fbits(y) - 1u);
            if (!(fsqrt(below) >= m)) {
                *out = y;
                return true;
            }
            y = below;
        }
        return false;
    }
    for (int k = 0; k < 64; ++k) {
        y = ffrom(fbits(y) + 1u);
        if (fsqrt(y) >= m) {
            *out = y;
            return true;
        }
    }
    return false;
}

// The ship's last two pow(tf, n2) results (tf is fixed for its tick, so a repeated n2 repeats the result exactly)
struct PowCache {
    int n2[2];
    float kappa2[2];
};
__device__ __forceinline__ void pow_cache_clear(PowCache& c) {
    c.n2[0] = c.n2[1] = INT32_MIN;
    c.kappa2[0] = c.kappa2[1] = 0.0f;
}

// CalculateN2Alpha2's braking ticks (full.py:2128): n2 = ceil(log(factor / (1 + factor)) / (-dt t_scale)) as an int
inline __device__ __noinline__ int braking_ticks(float max_ang_vel, float len_omega, float fdt, float t_scale) {
    const float factor = fdiv(max_ang_vel, len_omega);
    return to_i32(tod(fceil(fdiv(lm::logf(fdiv(factor, fadd(1.0f, factor))), fmul(fneg(fdt), t_scale)))));
}
// kappa2 = tf^n2 (glibc's pow, rounded to float)
inline __device__ __noinline__ float braking_kappa(float tf, int n2) { return tof(lm::pow(tod(tf), (double)n2)); }

// CalculateN2Alpha2 (full.py:2124-2150): the braking ticks n2, kappa2 = tf^n2 (pow), and the braking factor
// t_scale kappa2 / (1 - kappa2) the torque is -omega times (when the turning rate is above 1e-10)
__device__ __forceinline__ bool braking(const Turn& t, float len_omega, int* n2, float* kappa2, float* g,
                                        PowCache& pc) {
    if (tod(len_omega) > 1e-10) {
        *n2 = braking_ticks(t.max_ang_vel, len_omega, t.fdt, t.t_scale);
        if (*n2 == pc.n2[0]) {
            *kappa2 = pc.kappa2[0];
        } else if (*n2 == pc.n2[1]) {
            *kappa2 = pc.kappa2[1];
        } else {
            *kappa2 = braking_kappa(t.tf, *n2);
            pc.n2[1] = pc.n2[0];
            pc.kappa2[1] = pc.kappa2[0];
            pc.n2[0] = *n2;
            pc.kappa2[0] = *kappa2;
        }
        *g = fdiv(fmul(t.t_scale, *kappa2), fsub(1.0f, *kappa2));
        return true;
    }
    *n2 = 0;
    *kappa2 = 1.0f;
    *g = 0.0f;
    return false;
}

// The accelerating-ticks search shared by both torques (full.py:2189-2201, 2264-2276): the terms num(n1) and
// den(n1) of alpha1 = (target - omega0 num) / den; kappa1 = tf^n1 by repeated float products
struct Search {
    float tau, n2dt, kappa2, one_k2;
    int n2;
};
__device__ __forceinline__ void search_terms(const Search& q, float kappa1, float n1dt, float* num, float* den) {
    if (q.n2 == 0) {
        *num = fmul(q.tau, fsub(1.0f, kappa1));
        *den = fmul(q.tau, fsub(n1dt, *num));
    } else {
        *num = fsub(q.tau, fdiv(fmul(fmul(kappa1, q.kappa2), q.n2dt), q.one_k2));
        *den = fmul(q.tau, fsub(n1dt, fdiv(fmul(fmul(q.n2dt, q.kappa2), fsub(1.0f, kappa1)), q.one_k2)));
    }
}

// RotationQuaternion(axis, angle): sinf and cosf of the half angle around the normalised axis
inline __device__ __noinline__ F4 q_axis_angle(F3 axis, float angle) {
    const F3 u = f3_unit(axis);
    const float h = fdiv(angle, 2.0f);
    const float s = lm::sinf(h);
    return F4{fmul(s, u.x), fmul(s, u.y), fmul(s, u.z), lm::cosf(h)};
}

struct Turned {
    F4 rot;
    F3 w;
};

// ApplyTorque over one tick (full.py:2292, fraction 1): heading and roll apart; the rotation and angular velocity
__device__ __forceinline__ Turned apply_torque(F4 rotation, F3 w, F3 torque, float roll, float tau, float fdt) {
    const float tf = lm::expf(fdiv(fneg(fdt), tau));
    const F3 heading = m_apply(F3{0.0f, 0.0f, 1.0f}, m_of_q(rotation));
    const float omega_roll = f3_dot(w, heading);
    const F3 omega_heading = f3_sub(w, f3_mul(heading, omega_roll));
    const float span = fsub(fdt, fmul(tau, fsub(1.0f, tf)));
    const float rot_roll = fmul(tau, fadd(fmul(roll, span), fmul(omega_roll, fsub(1.0f, tf))));
    const F3 rot_heading = f3_mul(f3_add(f3_mul(torque, span), f3_mul(omega_heading, fsub(1.0f, tf))), tau);
    const float angle_heading = f3_len(rot_heading);
    const bool turn = tod(angle_heading) > 1e-10;
    F4 qh = q_identity();
    F3 heading_rotated = heading;
    if (turn) {
        qh = q_axis_angle(rot_heading, angle_heading);
        heading_rotated = m_apply(heading, m_of_q(qh));
    }
    F3 wn = f3_add(f3_mul(torque, fmul(tau, fsub(1.0f, tf))), f3_mul(omega_heading, tf));
    wn = f3_add(wn, f3_mul(heading_rotated, fsub(fmul(tau, roll), fmul(fsub(fmul(tau, roll), omega_roll), tf))));
    if (turn) rotation = q_mul(rotation, qh);
    rotation = q_mul(rotation, q_axis_angle(heading_rotated, rot_roll));
    const float norm = fsqrt(q_lensq(rotation));
    if (norm > 0.0f) rotation = q_scale_inv(rotation, norm);
    return Turned{rotation, wn};
}

// Ball::SnapOrientation (full.py:2092): turned to the velocity and rolled upright (the caller clears the turning)
inline __device__ __noinline__ F4 snap_rotation(D3 vel) {
    const F3 d = f3_of(vel);
    const float len_dir = f3_len(d);
    if (tod(len_dir) < 1e-12) return q_identity();
    const F3 axis = f3_cross(F3{0.0f, 0.0f, 1.0f}, d);
    const float angle = lm::acosf(fmax_(-1.0f, fmin_(1.0f, fdiv(d.z, len_dir))));
    F4 r = q_axis_angle(axis, angle);
    const F3 up = m_apply(F3{0.0f, 1.0f, 0.0f}, m_of_q(q_conj(r)));
    const float up_roll = up.z < tof(0.99) ? lm::atan2f(fneg(up.x), up.y) : 0.0f;
    const F3 heading = m_apply(F3{0.0f, 0.0f, 1.0f}, m_of_q(r));
    return q_mul(r, q_axis_angle(heading, up_roll));
}

}  // namespace flight
}  // namespace ebb
