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
//
// The composed park (exact_ballpark/vec_composed.py, vec_composed_cuda.cu) is the same tick with step 3 the gradient
// method's collisions between every massive ball (COLLIDE): each row's warp path first (a drop-out's state, re-filed
// at rest, is what the responders with higher ids meet), then every ball's view of the gradient staged in shared
// memory (position, velocity, mLastG, the depth-0 end of the tick, the filing, the flags the candidate rules read),
// then each live massive ball's Gradient over its world: GetNearbyBalls' candidates (massive or dropping out before
// its turn, uncloaked, in a related box; no missile but for a defender; a normal missile's one candidate its target)
// less Gradient's skips, in the partition's walk order, Potential with its recursion and COL-711's missile exception;
// the commit integrates mLastG + mLastC, re-files the balls that moved and appends the master's self-collision.
#include <cuda_runtime.h>

#include "../../include/ebb.h"
#include "ebb_flight.cuh"
#include "ebb_orient.cuh"
#include "ebb_rows.cuh"

// Resident blocks a multiprocessor is asked to fit (the register budget the compiler gets), per tick: the combat tick
// at 80 registers (3 blocks of 256 threads), the composed tick at 128 with its Gradient and commit out of line (2
// blocks): measured fastest on B200 at 65,536 worlds (1.21 and 1.65 ms a tick, against 1.54 and 2.84 ms with the
// composed tick at 80 registers, everything inlined and 128-thread blocks)
#ifndef EBB_COMBAT_MIN_BLOCKS
#define EBB_COMBAT_MIN_BLOCKS 3
#endif
#ifndef EBB_COMPOSED_MIN_BLOCKS
#define EBB_COMPOSED_MIN_BLOCKS 2
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
constexpr double REST_SQ = 0.1;                       // a drop-out at rest is re-filed there; so is a ball that moved
constexpr double LIGHT_BALL_RATIO = 25.0;             // Potential: a light ball's response is the push's length
constexpr double RESPONSE_SCALE = 0.85;               // mLastC = 0.85 x the response
constexpr int NUM_LEVELS = 8;                         // the partition's levels (space.py:69-75)
constexpr double BIG_BOX = 7864320.0;                 // a top box's width
constexpr int64_t CODE_BASE = 65;                     // a walk key's post-order digit: 64 children, then past the level
constexpr int64_t NOT_A_CANDIDATE = int64_t(1) << 62;

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

// Ballpark::Integrate over t seconds: the cached decay factor tf for a whole tick, else glibc's exp(-k t / m)
__device__ __forceinline__ void integrate_for(D3* p, D3* v, D3 a, double m, double k, double tf, double t, double dt) {
    if (t == 0.0) return;
    if (t != dt) tf = lm::exp(dmul(ddiv(dneg(k), m), t));
    integrate(p, v, a, m, k, tf, t);
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

// ---- the composed park's partition and gradient (vec_composed.py, vec_collide.py's gradient on the view) ----

__device__ __forceinline__ double level_width(int l) { return ddiv(BIG_BOX, i2d(int64_t(1) << (2 * l))); }
__device__ __forceinline__ int64_t level_grid(int l) { return int64_t(1) << (2 * l + 23); }

struct Filing {
    int64_t key[3];
    int32_t level;
    int8_t mod[3];
    bool bad;
};

// Ball::InsertInBoxes' outcome (vec_collide.py:776-807): the level of the radius inflated by a tick's reach at the
// ball's terminal speed, the key of the box holding the centre, the side (-1, 0, +1) on each axis where the inflated
// sphere reaches the next box; `bad`: a key at the grid's edge or a ball wider than a top box (the reference refuses)
__device__ __forceinline__ Filing filing_of(D3 p, D3 v, double radius, bool free_, double mass, double agility,
                                            double sf, double max_vel, double tf, double k, double dt) {
    double infl = radius;
    if (free_) {
        const double m = dmul(mass, agility);
        const double a = ddiv(dmul(dmul(k, sf), max_vel), m);
        const double speed = dsqrt(d3_lensq(v));
        const double ma = dmul(m, a);
        const double mps = ddiv(dsub(ma, dmul(dsub(ma, dmul(speed, k)), tf)), k);
        infl = dadd(radius, dmul(dt, mps));
    }
    int level = -1;
    for (int l = 0; l < NUM_LEVELS; ++l)
        if (!(dmul(3.0, infl) > level_width(l))) ++level;
    if (level < 0) level = 0;
    const double w = level_width(level);
    const int64_t grid = level_grid(level);
    const double half = dmul(dmul(0.5, w), i2d(grid)), center = dmul(dmul(w, i2d(grid)), 0.5), fac = ddiv(1.0, w);
    const double pa[3] = {p.x, p.y, p.z};
    Filing f;
    f.level = level;
    f.bad = level == 0 && dmul(radius, 2.0) > level_width(0);
    for (int q = 0; q < 3; ++q) {
        int64_t kq = to_i64(dmul(dadd(pa[q], half), fac));
        kq = kq < 0 ? 0 : (kq >= grid ? grid - 1 : kq);
        const double lo = dsub(dmul(i2d(kq), w), center), hi = dsub(dmul(i2d(kq + 1), w), center);
        const bool down = dsub(dadd(lo, infl), pa[q]) > 0.0, up = dsub(dsub(hi, infl), pa[q]) < 0.0;
        const int8_t mq = down ? -1 : (up ? 1 : 0);
        f.key[q] = kq;
        f.mod[q] = mq;
        if (kq <= 0 || kq >= grid - 1 || kq + mq < 0 || kq + mq >= grid) f.bad = true;
    }
    return f;
}

// The filing of row i from its state (or the given position, velocity and speed fraction), stored on the row
__device__ __forceinline__ void file_row(const EbbComposedState& x, int64_t i, D3 p, D3 v, float sf) {
    const EbbFlightState& s = x.combat.flight;
    const int64_t n = s.n;
    const Filing f = filing_of(p, v, tod(s.radius[i]), s.free_[i] != 0, s.mass[i], tod(s.agility[i]), tod(sf),
                               tod(s.max_vel[i]), s.time_factor[i], s.friction, s.dt);
    x.level[i] = f.level;
    for (int q = 0; q < 3; ++q) {
        x.key[q * n + i] = f.key[q];
        x.mod[q * n + i] = f.mod[q];
    }
    if (f.bad) x.combat.flags[i] |= EBB_COMPOSED_FLAG_PARTITION;
}

// A ball as the gradient's view of its world holds it (vec_composed.py:_fill_view, _gradient_rows): its position and
// velocity (a drop-out's at its drop-out point), mLastG, the depth-0 end of the tick, the filing (re-made at a drop-out
// at rest) and what the candidate rules read
constexpr uint8_t G_EXISTS = 1, G_MASSIVE = 2, G_CLOAKED = 4, G_FREE = 8, G_DROPPED = 16;
struct GBall {
    D3 pos, vel, g, end;
    double m, mass, tf, radius;
    int64_t id, owner, follow, bubble, world;
    int64_t key[3];
    int32_t level, mode, tslot;
    int8_t mod[3];
    uint8_t flags;
};

// Whether a box of ball n is one of ball b's boxes, an ancestor of one or below one (vec_collide.py:809): per axis,
// some option of the finer ball shifted to the coarser level equals some option of the coarser
__device__ __forceinline__ bool related(const GBall& b, const GBall& o) {
    const int64_t Lb = b.level, Ln = o.level;
    const int64_t sh = 2 * (Lb > Ln ? Lb - Ln : Ln - Lb);
    const bool coarse = Ln <= Lb;
    for (int q = 0; q < 3; ++q) {
        const int64_t kb = b.key[q], mb = b.mod[q], kn = o.key[q], mn = o.mod[q];
        const int64_t lo_b = kb + (mb < 0 ? mb : 0), hi_b = kb + (mb > 0 ? mb : 0);
        const int64_t lo_n = kn + (mn < 0 ? mn : 0), hi_n = kn + (mn > 0 ? mn : 0);
        const int64_t xl = (coarse ? lo_b : lo_n) >> sh, xh = (coarse ? hi_b : hi_n) >> sh;
        const int64_t yl = coarse ? lo_n : lo_b, yh = coarse ? hi_n : hi_b;
        if (!(xl == yl || xl == yh || xh == yl || xh == yh)) return false;
    }
    return true;
}

// The position of ball n's first box in ball b's GetNearbyBalls walk (vec_collide.py:825): the first of b's boxes (by
// key) that n's box relates to, the part (0 an ancestor, 1 below, 2 the box itself) and within it the ancestor's
// distance or the box's post-order code
__device__ __forceinline__ int64_t order_key(const GBall& b, const GBall& o) {
    const int64_t Lb = b.level, Ln = o.level;
    int64_t Kn[3], Mn[3], cb[3], lo_b[3], hi_b[3];
    for (int q = 0; q < 3; ++q) {
        const int64_t kb = b.key[q], mb = b.mod[q];
        Kn[q] = o.key[q];
        Mn[q] = o.mod[q];
        cb[q] = 1 + (mb != 0);
        lo_b[q] = kb + (mb < 0 ? mb : 0);
        hi_b[q] = kb + (mb > 0 ? mb : 0);
    }
    int64_t span = 1;
    for (int l = 0; l < NUM_LEVELS - 1; ++l) span *= CODE_BASE;
    if (Ln <= Lb) {
        const int64_t s_up = 2 * (Lb - Ln);
        int64_t idx[3];
        for (int q = 0; q < 3; ++q) {
            const int64_t v = lo_b[q] >> s_up;
            idx[q] = ((v == Kn[q]) || (Mn[q] != 0 && v == Kn[q] + Mn[q])) ? 0 : 1;
        }
        const int64_t seg = (idx[0] * cb[1] + idx[1]) * cb[2] + idx[2];
        return Ln < Lb ? (seg * 3) * span + (Lb - Ln) : (seg * 3 + 2) * span;
    }
    const int64_t s_dn = 2 * (Ln - Lb);
    int64_t best = NOT_A_CANDIDATE;
    for (int c = 0; c < 8; ++c) {
        const int64_t bit[3] = {(c >> 2) & 1, (c >> 1) & 1, c & 1};
        bool ok = true;
        int64_t box[3], jx[3];
        for (int q = 0; q < 3; ++q) {
            if (bit[q] != 0 && Mn[q] == 0) ok = false;
            box[q] = Kn[q] + Mn[q] * bit[q];
            const int64_t anc = box[q] >> s_dn;
            const bool in0 = anc == lo_b[q], in1 = anc == hi_b[q] && cb[q] == 2;
            if (!(in0 || in1)) ok = false;
            jx[q] = in0 ? 0 : 1;
        }
        if (!ok) continue;
        const int64_t seg = (jx[0] * cb[1] + jx[1]) * cb[2] + jx[2];
        int64_t code = 0, power = span;
        for (int lvl = 1; lvl < NUM_LEVELS; ++lvl) {
            power /= CODE_BASE;
            const int64_t shift = 2 * (Ln - lvl) > 0 ? 2 * (Ln - lvl) : 0;
            int64_t digit = ((box[0] >> shift) & 3) * 16 + ((box[1] >> shift) & 3) * 4 + ((box[2] >> shift) & 3);
            if (lvl > Ln) digit = CODE_BASE - 1;
            if (lvl <= Lb) digit = 0;
            code += digit * power;
        }
        const int64_t key = (seg * 3 + 1) * span + code;
        if (key < best) best = key;
    }
    return best;
}

// A responder's running state through its Gradient
struct Acc {
    D3 last_c;
    double last_collision;
    int64_t hits_n;
};

// Potential (Ballpark.cpp:2789; vec_collide.py's _gradient) of responder b with candidate o at recursion depth D, the
// positions as the recursion pushed them, from the world's view in shared memory; the composed park's end
// (vec_composed.py:_GradientView._update): a missile's response to its own target is not kept (COL-711's exception),
// the candidate's id is appended either way
template <int D>
__device__ __forceinline__ void potential(const EbbComposedState& x, int64_t ib, const GBall& B, const GBall& O,
                                          D3 me_pos, D3 o_pos, bool exempt, Acc& acc) {
    const EbbFlightState& s = x.combat.flight;
    const double k = s.friction, dt = s.dt;
    const double cr = dadd(B.radius, O.radius);
    const double m1 = B.m;
    const bool free2 = (O.flags & G_FREE) != 0;
    const double m2 = O.m;
    D3 p1, q1;
    if (D == 0) {
        p1 = B.end;
        q1 = O.end;
    } else {
        p1 = integrate_pos(me_pos, B.vel, B.g, m1, k, B.tf, dt);
        q1 = integrate_pos(o_pos, O.vel, O.g, m2, k, O.tf, dt);
    }
    const double sv = collide_two_spheres(me_pos, p1, o_pos, q1, cr);
    if (sv == -1.0) return;
    D3 a1;
    if (sv > 0.0) {                                                   // COL-707, COL-708: the impact
        D3 pp = me_pos, vp = B.vel, qq = o_pos, vq = O.vel;
        integrate_for(&pp, &vp, B.g, m1, k, B.tf, dmul(sv, dt), dt);
        integrate_for(&qq, &vq, O.g, m2, k, O.tf, dmul(sv, dt), dt);
        const D3 normal = d3_unit(d3_sub(qq, pp));
        const double u1 = d3_dot(vp, normal), u2 = d3_dot(vq, normal);
        if (!free2) {
            vp = d3_sub(vp, d3_mul(normal, dmul(2.0, u1)));
        } else {
            const double mm1 = B.mass, mm2 = O.mass;
            const double u1p = ddiv(dadd(dsub(dmul(mm1, u1), dmul(mm2, u1)), dmul(dmul(2.0, mm2), u2)), dadd(mm1, mm2));
            vp = d3_add(vp, d3_mul(normal, dsub(u1p, u1)));
        }
        integrate_for(&pp, &vp, B.g, m1, k, B.tf, dmul(dsub(1.0, sv), dt), dt);
        const double inv_m = ddiv(1.0, m1), inv_t = ddiv(1.0, dsub(B.tf, 1.0));
        const double ga[3] = {B.g.x, B.g.y, B.g.z}, va[3] = {B.vel.x, B.vel.y, B.vel.z}, wa[3] = {vp.x, vp.y, vp.z};
        double r[3];
        for (int q = 0; q < 3; ++q) {
            const double xq = dadd(dsub(dadd(dmul(ga[q], dneg(m1)), dmul(ga[q], dmul(B.tf, m1))),
                                        dmul(dmul(va[q], B.tf), k)), dmul(wa[q], k));
            r[q] = dmul(dmul(dneg(xq), inv_m), inv_t);
        }
        a1 = D3{r[0], r[1], r[2]};
    } else {                                                          // COL-709, COL-710: already overlapping
        const D3 p0q0 = d3_sub(o_pos, me_pos);
        const double p0q0_2 = d3_dot(p0q0, p0q0);
        D3 normal;
        if (p0q0_2 == 0.0) normal = (B.id > O.id) ? D3{1.0, 0.0, 0.0} : D3{-1.0, 0.0, 0.0};
        else normal = d3_unit(p0q0);
        const double dist = dadd(dsub(cr, dsqrt(p0q0_2)), 1.0);
        const double msum = dadd(m1, m2);
        const double d1 = dmul(ddiv(m2, msum), dist);
        [[maybe_unused]] const double d2 = dmul(ddiv(m1, msum), dist);
        if constexpr (D < 2) {                                       // COL-710: two free balls pushed apart first
            if (free2) {
                potential<D + 1>(x, ib, B, O, d3_sub(me_pos, d3_mul(normal, d1)), d3_add(o_pos, d3_mul(normal, d2)),
                                 exempt, acc);
                if (ddiv(m2, m1) > LIGHT_BALL_RATIO) acc.last_c = d3_mul(d3_unit(acc.last_c), dist);
                const D3 dv = d3_sub(B.vel, O.vel);
                if (d3_dot(dv, dv) > SEPARATING_SPEED2) return;
            }
        }
        const double normal_comp = d3_dot(B.g, normal);
        const double tmp = ddiv(1.0, dadd(m1, dmul(dt, k)));
        const double c = ddiv(dneg(d1), dmul(dmul(dt, tmp), m1));
        a1 = d3_sub(d3_mul(d3_sub(d3_mul(normal, c), B.vel), ddiv(1.0, dt)), d3_mul(normal, normal_comp));
    }
    if (!exempt && sv >= acc.last_collision) {                       // COL-711: the later impact, the stronger at a tie
        const D3 lc = d3_mul(a1, RESPONSE_SCALE);
        if (sv == acc.last_collision) {
            if (d3_dot(lc, lc) > d3_dot(acc.last_c, acc.last_c)) acc.last_c = lc;
        } else {
            acc.last_c = lc;
            acc.last_collision = sv;
        }
    }
    x.hits[ib * x.hit_cap + (acc.hits_n < x.hit_cap ? acc.hits_n : x.hit_cap - 1)] = O.id;
    ++acc.hits_n;
}

constexpr int MAX_WORLD_ROWS = 64;                  // a world's rows at most in the composed park (its candidate list)

// Gradient (Ballpark.cpp:2745) of responder j (a live massive ball) over its world's rows [w0, w1) of the tile's view:
// the composed candidates (vec_composed.py:_pair_mask) that Potential's depth 0 does not rule out, in the partition's
// walk order (then id; a normal missile's target first), each through Potential
__device__ __noinline__ void gradient(const EbbComposedState& x, int64_t ib, int j, int w0, int w1, const GBall* gv) {
    const GBall& B = gv[j];
    const bool missile_b = (B.flags & G_EXISTS) && B.mode == MISSILE;
    const bool defender = missile_b && B.owner < 0;
    int64_t okey[MAX_WORLD_ROWS];
    uint8_t oslot[MAX_WORLD_ROWS];                                    // tile rows: below the block's 256 threads
    int nact = 0;
    for (int o = w0; o < w1; ++o) {
        if (o == j) continue;
        const GBall& O = gv[o];
        const bool ex = (O.flags & G_EXISTS) != 0;
        const bool seen = (O.flags & G_MASSIVE) || ((O.flags & G_DROPPED) && O.id < B.id);
        const bool missile_o = ex && O.mode == MISSILE;
        bool pair;
        bool first = false;
        if (missile_b && !defender) {                                // a normal missile: its target, unfiltered
            pair = o == B.tslot && ex && O.bubble == B.bubble;
            first = pair;
        } else {
            const bool nearby = ex && seen && !(O.flags & G_CLOAKED) && related(B, O);
            pair = defender ? nearby : (nearby && !missile_o);
        }
        if (!pair) continue;
        const bool skip = (missile_b && (O.id == B.owner || (O.mode == MINIBALL && O.owner == B.owner))) ||
                          ((O.mode == MISSILE || O.mode == MUSHROOM) && B.id == O.owner) ||
                          (O.mode == MISSILE && B.id == O.follow);
        if (skip) continue;
        if (collide_two_spheres(B.pos, B.end, O.pos, O.end, dadd(B.radius, O.radius)) == -1.0) continue;
        const int64_t key = first ? 0 : order_key(B, O), id = O.id;
        if (nact >= MAX_WORLD_ROWS) break;
        int at = nact++;                                              // insertion by (key, id)
        while (at > 0 && (okey[at - 1] > key || (okey[at - 1] == key && gv[oslot[at - 1]].id > id))) {
            okey[at] = okey[at - 1];
            oslot[at] = oslot[at - 1];
            --at;
        }
        okey[at] = key;
        oslot[at] = (uint8_t)o;
    }
    Acc acc{D3{0.0, 0.0, 0.0}, -1.0, 0};
    for (int q = 0; q < nact; ++q) {
        const GBall& O = gv[oslot[q]];
        potential<0>(x, ib, B, O, B.pos, O.pos, missile_b && O.id == B.follow, acc);
    }
    const int64_t n = x.combat.flight.n;
    for (int q = 0; q < 3; ++q) x.last_c[q * n + ib] = (&acc.last_c.x)[q];
    x.combat.flight.last_collision[ib] = acc.last_collision;
    x.combat.hits_n[ib] = acc.hits_n;
}

// Row i's view of the gradient (after every ball's phase 1): its warp path first (a drop-out's state and, at rest,
// its filing there), the depth-0 end of the tick; a massive ball in warp proper flagged
__device__ __forceinline__ void stage(const EbbComposedState& x, int64_t i, int64_t r0, int64_t r1, GBall& g) {
    const EbbCombatState& c = x.combat;
    const EbbFlightState& s = c.flight;
    const int64_t n = s.n;
    const Cfg cf = cfg_of(s);
    const Ship b = load_ship(s, i);
    const bool exists = c.exists[i] && !s.moribund[i];
    const bool live = s.free_[i] && !s.moribund[i];
    D3 p = b.pos, v = b.vel;
    bool dropped = false, rest = false;
    if (live && b.mode == WARP && b.effect_stamp >= 0) {
        if (b.massive) c.flags[i] |= EBB_COMPOSED_FLAG_WARP_MASSIVE;
        D3 wp = p, wv = v;
        dropped = warp_path(b, &wp, &wv, dmul(i2d(b.clock - b.effect_stamp), cf.dt));
        if (dropped && !b.massive) {                                  // the view holds it at its drop-out point
            p = wp;
            v = wv;
        }
        rest = dropped && !(d3_lensq(wv) >= REST_SQ);
    }
    g.pos = p;
    g.vel = v;
    g.g = b.last_g;
    const bool free_ = s.free_[i] != 0;
    g.m = free_ ? dmul(b.mass, tod(b.agility)) : FIXED_MASS;
    g.mass = b.mass;
    g.tf = b.tf;
    g.radius = tod(b.radius);
    g.end = integrate_pos(p, v, b.last_g, g.m, cf.friction, b.tf, cf.dt);
    g.id = b.id;
    g.owner = b.owner_id;
    g.follow = b.follow_id;
    g.bubble = c.bubble[i];
    g.world = x.world[i];
    g.mode = b.mode;
    g.tslot = (b.follow_ptr >= r0 && b.follow_ptr < r1 && x.world[b.follow_ptr] == g.world) ? (int32_t)(b.follow_ptr - r0)
                                                                                            : -1;
    if (rest) {
        const Filing f = filing_of(p, v, g.radius, free_, b.mass, tod(b.agility), tod(b.sf), tod(b.max_vel), b.tf,
                                   cf.friction, cf.dt);
        g.level = f.level;
        for (int q = 0; q < 3; ++q) {
            g.key[q] = f.key[q];
            g.mod[q] = f.mod[q];
        }
    } else {
        g.level = (int32_t)x.level[i];
        for (int q = 0; q < 3; ++q) {
            g.key[q] = x.key[q * n + i];
            g.mod[q] = (int8_t)x.mod[q * n + i];
        }
    }
    uint8_t fl = 0;
    if (exists) fl |= G_EXISTS;
    if (b.massive) fl |= G_MASSIVE;
    if (c.cloaked[i] != 0) fl |= G_CLOAKED;
    if (free_) fl |= G_FREE;
    if (dropped && !b.massive) fl |= G_DROPPED;
    g.flags = fl;
}

// Phases 3 and 4 of row i (vec_combat_cuda.cu:552): the warp path or the integrator, the rotation a tick on (by the
// mode then: ApplyTorque, or a disabled missile's old rotation), the commit, a disabled missile's snap, the dispatch
// counts, PetrifyTroll, the clock. COLLIDE: the composed park's (mLastG + mLastC, mLastCollision the gradient's, a
// drop-out at rest re-filed there and every ball that moved at least sqrt(0.1) m re-filed after the commit, the
// master's self-collision appended to the missile's collision list)
template <bool COLLIDE>
__device__ __forceinline__ void commit(const EbbComposedState& x, int64_t i, const DoLane& d, int64_t hits) {
    const EbbCombatState& c = x.combat;
    const EbbFlightState& s = c.flight;
    const int64_t n = s.n;
    const Cfg cf = cfg_of(s);
    Ship b = load_ship(s, i);
    const bool live = s.free_[i] && !s.moribund[i];
    int64_t ev_n = 0;
    uint8_t ev_self = 0;
    if (live) {
        if (!COLLIDE && b.massive) b.last_collision = -1.0;           // the gradient (a missile's response not kept)
        D3 p = b.pos, v = b.vel;
        D3 a;
        if (COLLIDE) {
            const D3 lc = ld3(x.last_c, i, n);
            a = D3{dadd(b.last_g.x, lc.x), dadd(b.last_g.y, lc.y), dadd(b.last_g.z, lc.z)};
        } else {
            a = D3{dadd(b.last_g.x, 0.0), dadd(b.last_g.y, 0.0), dadd(b.last_g.z, 0.0)};   // mLastG + mLastC
        }
        const double m = dmul(b.mass, tod(b.agility));
        if (b.mode == WARP && b.effect_stamp >= 0) {
            if (warp_path(b, &p, &v, dmul(i2d(b.clock - b.effect_stamp), cf.dt))) {
                b.massive = true;                                     // dropped out: massive and sensing again, Stop
                b.sensor = true;
                b.mode = STOP;
                b.pos = p;
                b.vel = v;
                if (COLLIDE && !(d3_lensq(v) >= REST_SQ)) file_row(x, i, p, v, b.sf);   // re-filed at rest
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
        const bool moved = !(d3_lensq(d3_sub(b.pos, before)) < DISPATCH_MIN_MOVE_SQ);
        if (COLLIDE && moved) file_row(x, i, b.pos, b.vel, b.sf);   // re-filed where it moved (modes.py:723)
        // DispatchCollisions (COL-719): a missile that moved at least sqrt(0.1) m; on the master its owner gone,
        // cloaked or in another bubble is a collision with itself, after its target's
        if (b.mode == MISSILE && moved) {
            ev_n = hits;
            if (c.master) {
                const int64_t o = c.owner_ptr[i];
                const bool gone = o < 0 || o >= n || !c.exists[o];
                ev_self = (gone || (c.bubble[o] != c.bubble[i] && c.bubble[i] != -1) || c.cloaked[o] != 0) ? 1 : 0;
            }
        }
        if (COLLIDE && ev_self) {                                     // appended to the missile's collision list
            x.hits[i * x.hit_cap + (hits < x.hit_cap ? hits : x.hit_cap - 1)] = b.id;
            c.hits_n[i] = hits + 1;
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

// The composed tick's commit, out of line (its own register allocation)
__device__ __noinline__ void commit_composed(const EbbComposedState& x, int64_t i, const DoLane& d, int64_t hits) {
    commit<true>(x, i, d, hits);
}

// The composed park's phase-1 clearing of a live ball's collision response and list (vec_composed.py:_clear_contacts)
__device__ __forceinline__ void clear_contacts(const EbbComposedState& x, int64_t i) {
    const int64_t n = x.combat.flight.n;
    for (int q = 0; q < 3; ++q) x.last_c[q * n + i] = 0.0;
    for (int64_t q = 0; q < x.hit_cap; ++q) x.hits[i * x.hit_cap + q] = -1;
    x.combat.hits_n[i] = 0;
}

__host__ __device__ inline size_t view_bytes(int block) { return (size_t)block * sizeof(GBall); }
__host__ __device__ inline size_t tick_smem_bytes(int block, bool collide) {
    const size_t a = smem_bytes(block), b = view_bytes(block);
    return collide && b > a ? b : a;
}

// The tick: one block a tile of whole worlds (rows [tile_rows[b], tile_rows[b + 1]), at most blockDim.x of them).
// COLLIDE: the composed park's; the gradient's view of the tile reuses the records' and the orientation tables' shared
// memory (both done with at the barrier after phase 1).
template <bool COLLIDE>
__global__ void __launch_bounds__(256, COLLIDE ? EBB_COMPOSED_MIN_BLOCKS : EBB_COMBAT_MIN_BLOCKS) tick_kernel(EbbComposedState x,
                                                                          const int64_t* __restrict__ tile_rows,
                                                                          int64_t tiles, int32_t* status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ float ndt_tab[TORQUE_STEPS];
    const EbbCombatState& c = x.combat;
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
    const int64_t i = r0 + j;
    const bool mine = j < m && (c.active == nullptr || c.active[i] != 0);   // OnTick: a world's rows alike
    if (mine) record(c, i, rec[j]);
    __syncthreads();
    DoLane d;
    d.on = false;
    bool release_after = false;
    if (mine) {
        if (COLLIDE && c.flight.free_[i] && !c.flight.moribund[i]) clear_contacts(x, i);
        phase1(c, i, r0, r1, rec, d, &release_after, status);
    }
    orient_warp(d, cfg_of(c.flight), ndt_tab, ktab);
    if (mine) phase1_end(c, i, d, release_after);
    __syncthreads();
    int64_t hits = 0;
    if (COLLIDE) {
        GBall* gv = (GBall*)smem_raw;
        if (mine) stage(x, i, r0, r1, gv[j]);
        else if (j < m) gv[j].world = INT64_MIN;                      // a world outside OnTick's mask: no view
        __syncthreads();
        if (mine && c.flight.free_[i] && !c.flight.moribund[i] && (gv[j].flags & G_MASSIVE)) {
            int w0 = j, w1 = j + 1;                                   // the world's rows in the tile
            while (w0 > 0 && gv[w0 - 1].world == gv[j].world) --w0;
            while (w1 < m && gv[w1].world == gv[j].world) ++w1;
            if (w1 - w0 > MAX_WORLD_ROWS) atomicOr(status, 4);
            else gradient(x, i, j, w0, w1, gv);
        }
        __syncthreads();
        if (mine) hits = c.hits_n[i];
    } else {
        if (mine) {
            hits = missile_contacts(c, i);
            c.hits_n[i] = hits;
        }
        __syncthreads();
    }
    if (mine) {
        if constexpr (COLLIDE) commit_composed(x, i, d, hits);
        else commit<false>(x, i, d, hits);
    }
}

// The composed park's filing of the rows in a mask (the commands' re-filings), one thread a row
__global__ void file_kernel(EbbComposedState x, const uint8_t* __restrict__ mask, const double* __restrict__ pos,
                            const double* __restrict__ vel, const float* __restrict__ sf) {
    const EbbFlightState& s = x.combat.flight;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.n || !mask[i]) return;
    const D3 p = ld3(pos ? pos : s.pos, i, s.n), v = ld3(vel ? vel : s.vel, i, s.n);
    file_row(x, i, p, v, sf ? sf[i] : s.speed_fraction[i]);
}

cudaError_t kernel_attributes(cudaFuncAttributes* fa) { return cudaFuncGetAttributes(fa, tick_kernel<false>); }
cudaError_t composed_attributes(cudaFuncAttributes* fa) { return cudaFuncGetAttributes(fa, tick_kernel<true>); }

}  // namespace combat
}  // namespace ebb

// ==================================================================================================== the C ABI

namespace {
int launch_tick(const EbbComposedState& x, bool collide, const int64_t* tile_rows, int64_t tiles, int32_t* status,
                void* stream, int block) {
    const EbbCombatState& c = x.combat;
    if (c.flight.n <= 0 || tiles <= 0) return 0;
    if (block < 32 || block > 256 || block % 32 != 0 || tile_rows == nullptr || status == nullptr ||
        !c.flight.dynamical || c.exists == nullptr || c.formation_len == nullptr || c.formations == nullptr ||
        tiles > 0x7FFFFFFF)
        return EBB_EINVAL;
    if (collide && (x.world == nullptr || x.last_c == nullptr || x.level == nullptr || x.key == nullptr ||
                    x.mod == nullptr || x.hits == nullptr || x.hit_cap < 1))
        return EBB_EINVAL;
    const size_t smem = ebb::combat::tick_smem_bytes(block, collide);
    auto kernel = collide ? ebb::combat::tick_kernel<true> : ebb::combat::tick_kernel<false>;
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
    }
    kernel<<<(unsigned)tiles, block, smem, (cudaStream_t)stream>>>(x, tile_rows, tiles, status);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}
}  // namespace

extern "C" {

int ebb_combat_tick(const EbbCombatState* s, const int64_t* tile_rows, int64_t tiles, int32_t* status, void* stream,
                    int block) {
    if (s == nullptr) return EBB_EINVAL;
    EbbComposedState x{};
    x.combat = *s;
    return launch_tick(x, false, tile_rows, tiles, status, stream, block);
}

int ebb_composed_tick(const EbbComposedState* s, const int64_t* tile_rows, int64_t tiles, int32_t* status,
                      void* stream, int block) {
    if (s == nullptr) return EBB_EINVAL;
    return launch_tick(*s, true, tile_rows, tiles, status, stream, block);
}

int ebb_composed_file(const EbbComposedState* s, const uint8_t* mask, const double* pos, const double* vel,
                      const float* sf, void* stream) {
    if (s == nullptr || mask == nullptr) return EBB_EINVAL;
    const int64_t n = s->combat.flight.n;
    if (n <= 0) return 0;
    if (s->level == nullptr || s->key == nullptr || s->mod == nullptr || s->combat.flags == nullptr) return EBB_EINVAL;
    const int block = 128;
    ebb::combat::file_kernel<<<(unsigned)((n + block - 1) / block), block, 0, (cudaStream_t)stream>>>(*s, mask, pos,
                                                                                                   vel, sf);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}

}  // extern "C"

EBB_OP_COUNTER(ebb_count_ops_combat)
