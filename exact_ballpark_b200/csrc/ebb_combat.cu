// SPDX-License-Identifier: MIT
// The combat park's tick on sm_100a (include/ebb.h's ebb_combat_tick): Destiny's flight modes with the two follow
// modes of combat, MISSILE (EvolveMissile, Ballpark.cpp:972; full.py:2337) and FORMATION (EvolveFormation,
// Ballpark.cpp:1023; full.py:2359), their releases (StopAllFollowers: a missile flies off non-massive), a massive
// normal missile's contact with its target in the gradient method (Potential's recursion, counted: the response is
// not kept for a missile's own target) and its collision events at the commit (DispatchCollisions, with the master's
// self-collision), as the reference's combat kernels compute them (exact_ballpark/vec_combat_cuda.cu:121-650) and its
// tensor tick (exact_ballpark/vec_combat.py:839-1042) states them.
//
// One launch, one thread block a tile of whole worlds (at most `block` rows, one thread a row), four steps with block
// barriers between them, where the reference takes four launches over all rows:
//  1. the records pass into shared memory: what each ball shows the others during phase 1 (its start position and
//     velocity, its vertical velocity after its own turn, whether it starts warp proper at its turn, its id, radius
//     and start rotation: a formation's leader turns the slot offsets by it);
//  2. phase 1 for every ball (the releases, the mode's thrust, dynamical orientation through the warp's cooperative
//     orientation step unless disabled for missiles), its fields stored in place (no ball's phase 1 reads them);
//  3. each massive normal missile's contacts with its target, from both balls' phase-1 state;
//  4. phases 3 and 4 for every ball (the warp path or the integrator, the rotation a tick on, the commit, a disabled
//     missile's snap, the dispatch counts, PetrifyTroll, the clock).
// A ball reads other balls only within its world (its follow target, its leader, a missile's owner), so a tile's
// barriers order every read a tick makes after the write it needs, as the reference's launches do.
#include <cuda_runtime.h>

#include "../../include/ebb.h"
#include "ebb_flight.cuh"
#include "ebb_orient.cuh"
#include "ebb_rows.cuh"

#ifndef EBB_COMBAT_MIN_BLOCKS
#define EBB_COMBAT_MIN_BLOCKS 3
#endif

namespace ebb {
namespace combat {

using namespace ebb::flight;

constexpr int64_t MISSILE_STRAIGHT_MS = 800;          // Ballpark.cpp:974: straight on while (time - launch) x tick <= 800
constexpr double DISPATCH_MIN_MOVE_SQ = 0.1;          // Ballpark.cpp:602: a missile that moved at least sqrt(0.1) m
constexpr double SEPARATING_SPEED2 = 0.0001;          // Potential: |v1 - v2|^2 above it returns early
constexpr double FIXED_MASS = 1.0e34;                 // Potential: a fixed ball's mass
constexpr double SNAP_MIN_SPEED2 = 1e-12;             // SnapOrientation: nothing at |v|^2 <= 1e-12
constexpr uint64_t FORMATION_SLOT_BITS = 16;          // Ball's bitset<16> of reserved slots
constexpr int64_t FLAG_UNDEFINED = 2;                 // a call whose result Destiny leaves undefined (vec_combat.py)

// followModes (Ballpark.cpp:68)
__device__ __forceinline__ bool follow_mode(int32_t m) {
    return m == FOLLOW || m == ORBIT || m == MISSILE || m == FORMATION;
}

// DynamicalOrientationDisabledForBall (Ballpark.cpp:408)
__device__ __forceinline__ bool disabled(const EbbCombatState& c, int32_t mode) {
    return c.do_missiles_off && mode == MISSILE;
}

// The tile's records: one a row
struct Rec {
    double px, py, pz, vx, vy, vz, vy_after;
    int64_t id;
    float radius, rx, ry, rz, rw;
    int32_t act;
};

__host__ __device__ inline size_t records_bytes(int block) { return ((size_t)block * sizeof(Rec) + 15) & ~(size_t)15; }
__host__ __device__ inline size_t smem_bytes(int block) {
    return records_bytes(block) + (size_t)(block / 32) * KTAB_FLOATS * sizeof(float);
}

// StopAllFollowers on this follower (vec_combat_cuda.cu:216; MOV-730): a missile is made non-massive and, like an
// interactive orbiter, flies on by GotoDirection(its velocity) (refused, the mode kept, when the velocity or the point
// is not finite); any other follower stops (Stop(Ball*) clears the follow fields only in a follow mode). Returns the
// mode it is left in; applies it when `apply`.
__device__ __forceinline__ int32_t combat_release(Ship& b, bool apply) {
    const bool missile = b.mode == MISSILE;
    if (missile || (b.interactive && b.mode == ORBIT)) {
        if (missile && apply) b.massive = false;
        if (!d3_finite(b.vel)) return b.mode;
        const D3 p = d3_add(b.pos, d3_mul(d3_unit(b.vel), DIR_DIST));
        if (!d3_finite(p)) return b.mode;
        if (apply) {
            clear_follow(b);
            b.gp = p;
            if (b.sf == 0.0f) b.sf = 1.0f;
            b.mode = GOTO;
        }
        return GOTO;
    }
    if (apply) {
        if (follow_mode(b.mode)) clear_follow(b);
        b.mode = STOP;
    }
    return STOP;
}

// Stop(Ball*) on the master frees a FORMATION follower's slot in its leader (Ballpark.cpp:4629-4633;
// Ball::FreeFormationSlot((size_t) mEffectStamp), Ball.cpp:2324): nothing without a loaded formation or for a slot past
// its end; a negative formation index read or a slot of 16 or more (bitset<16>::reset throws) flagged. The leader's
// bits are cleared with an integer atomic AND: order-free, exact.
__device__ __forceinline__ void free_on_stop(const EbbCombatState& c, const Ship& b, int64_t i) {
    if (!c.master || b.mode != FORMATION) return;
    const int64_t t = b.follow_ptr;
    if (t < 0 || t >= c.flight.n) return;
    const int64_t fid = c.formation_id[t];
    if (fid == -1 || fid > c.n_formations - 1) return;
    if (fid < 0) {
        c.flags[i] |= FLAG_UNDEFINED;
        return;
    }
    const uint64_t len = (uint64_t)c.formation_len[fid];
    const uint64_t slot = (uint64_t)b.effect_stamp;
    if (slot > len - 1) return;
    if (slot >= FORMATION_SLOT_BITS) {
        c.flags[i] |= FLAG_UNDEFINED;
        return;
    }
    atomicAnd((unsigned long long*)&c.formation_slots[t], ~(1ULL << slot));
}

// A release in the tick (a target starting warp proper, before or after the follower's own turn): the master's slot
// free, the release, and where the follow fields were cleared the owner's row too (vec_combat_cuda.cu:255)
__device__ __forceinline__ void release_in_tick(const EbbCombatState& c, Ship& b, int64_t i) {
    free_on_stop(c, b, i);
    combat_release(b, true);
    if (b.follow_ptr < 0) c.owner_ptr[i] = -1;
}

// EvolveMissile (MOV-723; vec_combat_cuda.cu:121): straight on toward mGoto (GotoThrust, tapered) while
// (time - launch) x tick is at most 800 ms; then the lead point (the target's position plus its velocity times
// dist / maxVel, offset along the line from the target by followRange + both radii) at full thrust, never tapered
__device__ __forceinline__ D3 missile_thrust(Ship& b, const Rec& t, const Cfg& cf, int64_t tick_ms) {
    if ((b.clock - b.effect_stamp) * tick_ms <= MISSILE_STRAIGHT_MS) return goto_thrust(b, b.gp, cf);
    const D3 op = D3{t.px, t.py, t.pz};
    D3 ov = D3{t.vx, t.vy, t.vz};
    if (t.id < b.id) ov.y = t.vy_after;                               // the target's turn came first
    const D3 delta = d3_sub(b.pos, op);
    const double dist = d3_len(delta);
    const double ct = ddiv(dist, tod(b.max_vel));
    D3 target = d3_add(op, d3_mul(ov, ct));
    const double r = dadd(dadd(tod(b.follow_range), tod(b.radius)), tod(t.radius));
    if (dist == 0.0) {
        target = D3{dadd(op.x, dmul(1.0, r)), dadd(op.y, dmul(0.0, r)), dadd(op.z, dmul(0.0, r))};
    } else {
        const double inv = ddiv(1.0, dist);
        target = D3{dadd(target.x, dmul(dmul(delta.x, r), inv)), dadd(target.y, dmul(dmul(delta.y, r), inv)),
                    dadd(target.z, dmul(dmul(delta.z, r), inv))};
    }
    b.gp = target;
    const double max_thrust = ddiv(dmul(dmul(cf.friction, tod(b.sf)), tod(b.max_vel)), dmul(b.mass, tod(b.agility)));
    return d3_mul(d3_unit(d3_sub(target, b.pos)), max_thrust);
}

// EvolveFormation (MOV-726; vec_combat_cuda.cu:147): the leader's slot offset scaled to both radii plus its length,
// turned by the leader's rotation at the tick's start as a float vector, added to the leader's start position;
// GotoThrust toward it. Zero thrust (mGoto kept) without a loaded formation or for a slot past its end.
__device__ __forceinline__ D3 formation_thrust(Ship& b, const EbbCombatState& c, int64_t t, const Rec& lr,
                                               const Cfg& cf) {
    const int64_t fid = c.formation_id[t];
    if (fid < 0 || fid > c.n_formations - 1) return D3{0.0, 0.0, 0.0};
    const int64_t slot = (int64_t)(int8_t)(uint8_t)(b.effect_stamp & 0xFF);      // char(mEffectStamp)
    const int64_t len = c.formation_len[fid];
    if (slot > len - 1 || slot < 0) return D3{0.0, 0.0, 0.0};
    const double* o = c.formations + (fid * c.max_slots + slot) * 3;
    const D3 offset = D3{o[0], o[1], o[2]};
    double length = d3_len(offset);
    if (length == 0.0) length = 1.0;
    const double k = dadd(dadd(tod(b.radius), tod(lr.radius)), length);
    const double inv = ddiv(1.0, length);
    const F3 vec = F3{tof(dmul(dmul(offset.x, k), inv)), tof(dmul(dmul(offset.y, k), inv)),
                      tof(dmul(dmul(offset.z, k), inv))};
    const F3 rv = m_apply(vec, m_of_q(F4{lr.rx, lr.ry, lr.rz, lr.rw}));
    const D3 g = D3{dadd(lr.px, tod(rv.x)), dadd(lr.py, tod(rv.y)), dadd(lr.pz, tod(rv.z))};
    b.gp = g;
    return goto_thrust(b, g, cf);
}

// ---- a missile's Potential with its target (Ballpark.cpp:2789; vec_combat_cuda.cu:286-330) ----

struct Pair {
    D3 vel_me, vel_other, g_me, g_other;
    double m1, m2, tf_me, tf_other, cr, k, dt;
    int64_t id_me, id_other;
    bool other_free;
};

// CollideTwoSpheres (Collision.cpp:108; COL-705): 0 if already touching, else the earlier root in [0, 1], else -1
__device__ __forceinline__ double collide_two_spheres(D3 p0, D3 p1, D3 q0, D3 q1, double cr) {
    const D3 p0q0 = d3_sub(p0, q0);
    const double p0q0_2 = d3_lensq(p0q0);
    if (p0q0_2 <= dmul(cr, cr)) return 0.0;
    const D3 dpq = D3{dsub(dsub(p1.x, p0.x), dsub(q1.x, q0.x)), dsub(dsub(p1.y, p0.y), dsub(q1.y, q0.y)),
                      dsub(dsub(p1.z, p0.z), dsub(q1.z, q0.z))};
    const double a = d3_lensq(dpq);
    const double bb = dmul(2.0, dadd(dadd(dmul(p0q0.x, dpq.x), dmul(p0q0.y, dpq.y)), dmul(p0q0.z, dpq.z)));
    const double cc = dsub(p0q0_2, dmul(cr, cr));
    if (a == 0.0 && bb == 0.0) return -1.0;
    double det = dsub(dmul(bb, bb), dmul(dmul(4.0, a), cc));
    if (det < 0.0) return -1.0;
    det = dsqrt(det);
    const double s2 = ddiv(dmul(dsub(dneg(bb), det), 0.5), a);
    if (s2 >= 0.0 && s2 <= 1.0) return s2;
    return -1.0;
}

__device__ __forceinline__ D3 integrate_pos(D3 p, D3 v, D3 a, double m, double k, double tf, double dt) {
    integrate(&p, &v, a, m, k, tf, dt);
    return p;
}

// Potential(missile, target, depth D): how many times the target's id is appended to the missile's collision list.
// s = -1: none; s > 0: one; s = 0 (touching): with a free target below depth 2 both are pushed apart along the
// normal and the recursion goes on, returning early (no append here) when they separate faster than 0.01 m/s;
// otherwise one append at this depth. The recursion unrolled by depth.
template <int D>
__device__ __forceinline__ int64_t contacts(const Pair& q, D3 p, D3 o) {
    const D3 p1 = integrate_pos(p, q.vel_me, q.g_me, q.m1, q.k, q.tf_me, q.dt);
    const D3 q1 = integrate_pos(o, q.vel_other, q.g_other, q.m2, q.k, q.tf_other, q.dt);
    const double s = collide_two_spheres(p, p1, o, q1, q.cr);
    if (s == -1.0) return 0;
    if (s > 0.0) return 1;
    if constexpr (D >= 2) {
        return 1;
    } else {
        if (!q.other_free) return 1;
        const D3 p0q0 = d3_sub(o, p);
        const double p0q0_2 = d3_lensq(p0q0);
        D3 normal;
        if (p0q0_2 == 0.0) normal = q.id_me > q.id_other ? D3{1.0, 0.0, 0.0} : D3{-1.0, 0.0, 0.0};
        else normal = d3_unit(d3_sub(o, p));
        const double dist = dadd(dsub(q.cr, dsqrt(p0q0_2)), 1.0);
        const double d1 = dmul(ddiv(q.m2, dadd(q.m1, q.m2)), dist);
        const double d2 = dmul(ddiv(q.m1, dadd(q.m1, q.m2)), dist);
        const D3 pp = D3{dsub(p.x, dmul(normal.x, d1)), dsub(p.y, dmul(normal.y, d1)), dsub(p.z, dmul(normal.z, d1))};
        const D3 oo = D3{dadd(o.x, dmul(normal.x, d2)), dadd(o.y, dmul(normal.y, d2)), dadd(o.z, dmul(normal.z, d2))};
        const int64_t inner = contacts<D + 1>(q, pp, oo);
        if (d3_lensq(d3_sub(q.vel_me, q.vel_other)) > SEPARATING_SPEED2) return inner;
        return inner + 1;
    }
}

// The gradient for a massive normal missile (after every ball's phase 1): its one candidate is its target in its
// bubble (Partition::GetCollisionCandidates), less Gradient's skips; the count of target ids appended
__device__ __noinline__ int64_t missile_contacts(const EbbCombatState& c, int64_t i) {
    const EbbFlightState& s = c.flight;
    const int64_t n = s.n;
    const int64_t t = s.follow_ptr[i];
    if (!(s.free_[i] && !s.moribund[i] && s.massive[i] && s.mode[i] == MISSILE && s.owner_id[i] >= 0 && t >= 0 &&
          t < n && c.bubble[i] == c.bubble[t]))
        return 0;
    const int32_t mt = s.mode[t];
    const int64_t own = s.owner_id[i];
    const bool skip = s.ids[t] == own || (mt == MINIBALL && s.owner_id[t] == own) ||
                      ((mt == MISSILE || mt == MUSHROOM) && s.ids[i] == s.owner_id[t]) ||
                      (mt == MISSILE && s.ids[i] == s.follow_id[t]);
    if (skip) return 0;
    Pair q;
    q.vel_me = ld3(s.vel, i, n);
    q.vel_other = ld3(s.vel, t, n);
    q.g_me = ld3(s.last_g, i, n);
    q.g_other = ld3(s.last_g, t, n);
    q.m1 = dmul(s.mass[i], tod(s.agility[i]));
    q.other_free = s.free_[t] != 0;
    q.m2 = q.other_free ? dmul(s.mass[t], tod(s.agility[t])) : FIXED_MASS;
    q.tf_me = s.time_factor[i];
    q.tf_other = s.time_factor[t];
    q.cr = dadd(tod(s.radius[i]), tod(s.radius[t]));
    q.k = s.friction;
    q.dt = s.dt;
    q.id_me = s.ids[i];
    q.id_other = s.ids[t];
    return contacts<0>(q, ld3(s.pos, i, n), ld3(s.pos, t, n));
}

// ---- the tick's steps for one row ----

// The records of row i (vec_combat_cuda.cu:381, the prepass): the flight records with the combat release (a missile
// follower flies on, a formation follower stops) for the vertical velocity after the turn, and the start rotation
__device__ __forceinline__ void record(const EbbCombatState& c, int64_t i, Rec& q) {
    const EbbFlightState& s = c.flight;
    const int64_t n = s.n;
    const D3 p = ld3(s.pos, i, n), v = ld3(s.vel, i, n);
    q.act = activates(s, i) ? 1 : 0;
    double vy = v.y;
    if (s.free_[i] && !s.moribund[i] && !s.dynamical) {
        int32_t m = s.mode[i];
        const int64_t t = s.follow_ptr[i];
        if (c.exists[i] && member_of(s, t, s.follow_id[i]) && s.ids[t] < s.ids[i] && activates(s, t)) {
            Ship f;
            f.mode = m;
            f.interactive = s.interactive[i] != 0;
            f.massive = s.massive[i] != 0;
            f.vel = v;
            f.pos = p;
            f.gp = ld3(s.goto_pt, i, n);
            f.sf = s.speed_fraction[i];
            m = combat_release(f, false);
        }
        if (m == STOP) vy = dmul(dsub(vy, dmul(STOP_DECAY, vy)), STOP_DAMP);
    }
    q.px = p.x;
    q.py = p.y;
    q.pz = p.z;
    q.vx = v.x;
    q.vy = v.y;
    q.vz = v.z;
    q.vy_after = vy;
    q.id = s.ids[i];
    q.radius = s.radius[i];
    const F4 r = ldf4(s.rot, i, n);
    q.rx = r.x;
    q.ry = r.y;
    q.rz = r.z;
    q.rw = r.w;
}

// Phase 1 of row i (vec_combat_cuda.cu:417): the release by a target starting warp proper before its turn, the mode's
// thrust, the orientation step's inputs; the release after its turn is returned for after the orientation step
__device__ __forceinline__ void phase1(const EbbCombatState& c, int64_t i, int64_t r0, int64_t r1, const Rec* rec,
                                       DoLane& d, bool* release_after, int32_t* status) {
    const EbbFlightState& s = c.flight;
    const int64_t n = s.n;
    const Cfg cf = cfg_of(s);
    Ship b = load_ship(s, i);
    const bool live = s.free_[i] && !s.moribund[i];
    *release_after = false;
    {
        const int64_t t = b.follow_ptr;
        if (t >= 0 && t < n && (t < r0 || t >= r1)) atomicOr(status, 1);   // a target outside its world's tile
        if (c.exists[i] && t >= r0 && t < r1 && rec[t - r0].id == b.follow_id && rec[t - r0].act) {
            if (rec[t - r0].id < b.id) release_in_tick(c, b, i);
            else *release_after = true;
        }
    }
    D3 a = D3{0.0, 0.0, 0.0};
    d.on = false;
    if (live) {
        const int64_t t = b.follow_ptr;
        const bool tv = t >= r0 && t < r1;
        if (b.mode == WARP) {                                         // EvolveWarp
            if (b.effect_stamp >= 0) {
                a = D3{0.0, 0.0, 0.0};
            } else if (rec[i - r0].act) {
                start_warp(b);
            } else {
                b.effect_stamp -= 1;
                a = goto_thrust(b, b.gp, cf);
            }
        } else if (b.mode == GOTO) {
            a = goto_thrust(b, b.gp, cf);
        } else if (follow_mode(b.mode) && !tv) {
            a = D3{0.0, 0.0, 0.0};
        } else if (b.mode == FOLLOW) {
            const Rec& q = rec[t - r0];
            a = follow_thrust(b, D3{q.px, q.py, q.pz}, q.radius, cf);
        } else if (b.mode == ORBIT) {
            const Rec& q = rec[t - r0];
            const D3 tp = D3{q.px, q.py, q.pz};
            if (cf.new_orbit) {
                D3 tv3 = D3{q.vx, q.vy, q.vz};
                if (q.id < b.id) tv3.y = q.vy_after;
                const F4 rr = s.dynamical ? ldf4(s.rot, i, n) : q_identity();
                a = new_orbit_thrust(b, tp, tv3, q.radius, cf, rr);
            } else {
                a = old_orbit_thrust(b, tp, q.radius, cf);
            }
        } else if (b.mode == MISSILE) {
            a = missile_thrust(b, rec[t - r0], cf, c.tick_ms);
        } else if (b.mode == FORMATION) {
            a = formation_thrust(b, c, t, rec[t - r0], cf);
        } else if (b.mode == STOP) {
            if (!cf.dynamical) b.vel.y = dmul(dsub(b.vel.y, dmul(STOP_DECAY, b.vel.y)), STOP_DAMP);
        }
        if (s.dynamical && !disabled(c, b.mode)) {
            d.on = true;
            d.fmass = tof(b.mass);
            d.agility = b.agility;
            d.sf = b.sf;
            d.max_vel = b.max_vel;
            d.max_ang_vel = s.max_ang_vel[i];
            d.rot_agility = s.rot_agility[i];
            d.warping = b.mode == WARP && b.effect_stamp >= 0;
            d.to_exit = f3_of(d3_sub(b.gp, b.pos));
            d.r0 = ldf4(s.rot, i, n);
            d.w0 = ldf3(s.ang_vel, i, n);
        }
    }
    if (!d.on) {
        d.r0 = q_identity();
        d.w0 = F3{0.0f, 0.0f, 0.0f};
    }
    d.a = a;
    store_phase1(s, i, b);
}

// After the orientation step: mLastG, the torque and roll, the release after the ball's own turn
__device__ __forceinline__ void phase1_end(const EbbCombatState& c, int64_t i, const DoLane& d, bool release_after) {
    const EbbFlightState& s = c.flight;
    const int64_t n = s.n;
    const bool live = s.free_[i] && !s.moribund[i];
    if (live) st3(s.last_g, i, n, d.a);
    if (d.on) {
        stf3(s.torque, i, n, d.torque);
        s.rot_roll[i] = d.roll;
    }
    if (release_after) {
        Ship b = load_ship(s, i);
        release_in_tick(c, b, i);
        store_phase1(s, i, b);
    }
}

// Phases 3 and 4 of row i (vec_combat_cuda.cu:552): the warp path or the integrator, the rotation a tick on (by the
// mode then: ApplyTorque, or a disabled missile's old rotation), the commit, a disabled missile's snap, the dispatch
// counts, PetrifyTroll, the clock
__device__ __forceinline__ void commit(const EbbCombatState& c, int64_t i, const DoLane& d, int64_t hits) {
    const EbbFlightState& s = c.flight;
    const int64_t n = s.n;
    const Cfg cf = cfg_of(s);
    Ship b = load_ship(s, i);
    const bool live = s.free_[i] && !s.moribund[i];
    int64_t ev_n = 0;
    uint8_t ev_self = 0;
    if (live) {
        if (b.massive) b.last_collision = -1.0;                       // the gradient (a missile's response not kept)
        D3 p = b.pos, v = b.vel;
        const D3 a = D3{dadd(b.last_g.x, 0.0), dadd(b.last_g.y, 0.0), dadd(b.last_g.z, 0.0)};   // mLastG + mLastC
        const double m = dmul(b.mass, tod(b.agility));
        if (b.mode == WARP && b.effect_stamp >= 0) {
            if (warp_path(b, &p, &v, dmul(i2d(b.clock - b.effect_stamp), cf.dt))) {
                b.massive = true;                                     // dropped out: massive and sensing again, Stop
                b.sensor = true;
                b.mode = STOP;
                b.pos = p;
                b.vel = v;
                integrate(&p, &v, a, m, cf.friction, b.tf, cf.dt);
            }
        } else {
            integrate(&p, &v, a, m, cf.friction, b.tf, cf.dt);
        }
        F4 r0 = q_identity(), rot1 = r0;
        F3 w0 = F3{0.0f, 0.0f, 0.0f}, w1 = w0;
        if (cf.dynamical) {
            r0 = ldf4(s.rot, i, n);
            w0 = ldf3(s.ang_vel, i, n);
            if (d.on) {
                rot1 = d.rot1;
                w1 = d.w1;
            } else if (!disabled(c, b.mode)) {                        // released after a disabled turn: ApplyTorque
                const float inertia = fmul(fmul(tof(b.mass), b.agility), s.rot_agility[i]);
                const Turned tr = apply_torque(r0, w0, ldf3(s.torque, i, n), s.rot_roll[i],
                                               fdiv(inertia, cf.ffriction), cf.fdt);
                rot1 = tr.rot;
                w1 = tr.w;
            } else {                                                  // phase 3 leaves mOldRot as it was
                rot1 = ldf4(s.old_rot, i, n);
                w1 = ldf3(s.old_ang_vel, i, n);
            }
        }
        const D3 before = b.pos;
        st3(s.old_pos, i, n, b.pos);
        st3(s.old_vel, i, n, b.vel);
        b.pos = p;
        b.vel = v;
        if (cf.dynamical) {                                           // the new values where finite
            const bool rot_ok = ffinite(q_lensq(rot1));
            const bool w_ok = ffinite(f3_dot(w1, w1));
            F4 rn = rot_ok ? rot1 : r0, ro = rot_ok ? r0 : rot1;
            F3 wn = w_ok ? w1 : w0, wo = w_ok ? w0 : w1;
            if (disabled(c, b.mode) && d3_lensq(b.vel) > SNAP_MIN_SPEED2) {   // SnapOrientation (phase 4)
                rn = snap_rotation(b.vel);
                ro = rn;
                wn = F3{0.0f, 0.0f, 0.0f};
                wo = wn;
            }
            stf4(s.rot, i, n, rn);
            stf4(s.old_rot, i, n, ro);
            stf3(s.ang_vel, i, n, wn);
            stf3(s.old_ang_vel, i, n, wo);
        }
        // DispatchCollisions (COL-719): a missile that moved at least sqrt(0.1) m; on the master its owner gone,
        // cloaked or in another bubble is a collision with itself, after its target's
        if (b.mode == MISSILE && !(d3_lensq(d3_sub(b.pos, before)) < DISPATCH_MIN_MOVE_SQ)) {
            ev_n = hits;
            if (c.master) {
                const int64_t o = c.owner_ptr[i];
                const bool gone = o < 0 || o >= n || !c.exists[o];
                ev_self = (gone || (c.bubble[o] != c.bubble[i] && c.bubble[i] != -1) || c.cloaked[o] != 0) ? 1 : 0;
            }
        }
        if (c.exists[i] && b.mode == TROLL && !(b.effect_stamp > b.clock)) {
            // PetrifyTroll (Ballpark.cpp:6327) of a troll due: at rest, mLastG cleared, fixed, non-interactive, RIGID
            b.vel = D3{0.0, 0.0, 0.0};
            st3(s.old_vel, i, n, b.vel);
            b.last_g = D3{0.0, 0.0, 0.0};
            s.free_[i] = 0;
            s.interactive[i] = 0;
            b.mode = RIGID;
        }
    }
    st3(s.pos, i, n, b.pos);
    st3(s.vel, i, n, b.vel);
    st3(s.goto_pt, i, n, b.gp);
    st3(s.last_g, i, n, b.last_g);
    s.last_collision[i] = b.last_collision;
    s.mode[i] = b.mode;
    s.massive[i] = b.massive ? 1 : 0;
    s.sensor[i] = b.sensor ? 1 : 0;
    s.clock[i] = b.clock + 1;
    c.ev_n[i] = ev_n;
    c.ev_self[i] = ev_self;
}

// The tick: one block a tile of whole worlds (rows [tile_rows[b], tile_rows[b + 1]), at most blockDim.x of them)
__global__ void __launch_bounds__(256, EBB_COMBAT_MIN_BLOCKS) tick_kernel(EbbCombatState c,
                                                                          const int64_t* __restrict__ tile_rows,
                                                                          int64_t tiles, int32_t* status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ float ndt_tab[TORQUE_STEPS];
    if (blockIdx.x >= tiles) return;
    const int64_t r0 = tile_rows[blockIdx.x], r1 = tile_rows[blockIdx.x + 1];
    if (r1 - r0 > (int64_t)blockDim.x || r1 < r0) {                  // the host plans tiles no wider than the block
        if (threadIdx.x == 0) atomicOr(status, 2);
        return;
    }
    Rec* rec = (Rec*)smem_raw;
    float* ktab = (float*)(smem_raw + records_bytes(blockDim.x)) + (threadIdx.x >> 5) * KTAB_FLOATS;
    fill_ndt(ndt_tab, c.flight.dt);
    const int m = (int)(r1 - r0);
    const int j = threadIdx.x;
    const bool mine = j < m;
    const int64_t i = r0 + j;
    if (mine) record(c, i, rec[j]);
    __syncthreads();
    DoLane d;
    d.on = false;
    bool release_after = false;
    if (mine) phase1(c, i, r0, r1, rec, d, &release_after, status);
    orient_warp(d, cfg_of(c.flight), ndt_tab, ktab);
    if (mine) phase1_end(c, i, d, release_after);
    __syncthreads();
    int64_t hits = 0;
    if (mine) {
        hits = missile_contacts(c, i);
        c.hits_n[i] = hits;
    }
    __syncthreads();
    if (mine) commit(c, i, d, hits);
}

cudaError_t kernel_attributes(cudaFuncAttributes* fa) { return cudaFuncGetAttributes(fa, tick_kernel); }

}  // namespace combat
}  // namespace ebb

// ==================================================================================================== the C ABI

extern "C" {

int ebb_combat_tick(const EbbCombatState* s, const int64_t* tile_rows, int64_t tiles, int32_t* status, void* stream,
                    int block) {
    if (s == nullptr) return EBB_EINVAL;
    if (s->flight.n <= 0 || tiles <= 0) return 0;
    if (block < 32 || block > 256 || block % 32 != 0 || tile_rows == nullptr || status == nullptr ||
        !s->flight.dynamical || s->exists == nullptr || s->formation_len == nullptr || s->formations == nullptr ||
        tiles > 0x7FFFFFFF)
        return EBB_EINVAL;
    const size_t smem = ebb::combat::smem_bytes(block);
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(ebb::combat::tick_kernel,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
    }
    ebb::combat::tick_kernel<<<(unsigned)tiles, block, smem, (cudaStream_t)stream>>>(*s, tile_rows, tiles, status);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}

}  // extern "C"
