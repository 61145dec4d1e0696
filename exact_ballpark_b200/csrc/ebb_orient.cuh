// SPDX-License-Identifier: MIT
// Dynamical orientation for a warp of 32 ships at once (EvolveBehaviorForBall's orientation branch, full.py:2459;
// GotoTorqueBreaks full.py:2155, GotoRollBreaks full.py:2224, ApplyTorque full.py:2292), warp-cooperative.
//
// Each torque search tries n1 = 1, 2, ... 99 accelerating ticks and keeps the first whose torque is within the
// maximum, in up to five rounds (each round re-derives the braking ticks n2). One thread a ship runs those loops in
// lockstep: a warp pays, round by round, its slowest ship's n1 while the others idle (about 15 % of the lanes busy on
// the flight benchmark's worlds). Here the warp searches one ship at a time with all 32 lanes, lane j evaluating
// candidate n1 = b + j + 1 of the block b = 0, 32, 64, 96, and a ballot takes the first candidate that passes: the
// serial loop's n1, its alpha1 and kappa1 bit for bit, since every candidate is the same computation on the same
// inputs (kappa1 = tf^n1 by the serial loop's own float products: kept in a per-lane table for n1 <= 32, each lane
// carrying the chain further from the block's first kappa beyond). The set-up, the braking rounds (logf, pow) and
// ApplyTorque stay one lane a ship, the warp's ships taking their rounds together.
#pragma once

#include "ebb_flight.cuh"

namespace ebb {
namespace flight {

constexpr unsigned FULL_WARP = 0xffffffffu;
constexpr int KTAB_STRIDE = 33;             // a lane's row kappa_1 .. kappa_32 (padded: the fill is conflict-free)
constexpr int KTAB_FLOATS = 32 * KTAB_STRIDE;

// One lane's ship for the warp's orientation step
struct DoLane {
    bool on;                 // live, and dynamical orientation applies
    D3 a;                    // in: the behaviour's thrust; out: the thrust after orientation
    float fmass, agility, sf, max_vel, max_ang_vel, rot_agility;
    bool warping;            // in warp proper: coasting, it turns toward its exit point
    F3 to_exit;              // (exit point - position) as floats
    F4 r0;
    F3 w0;
    F3 torque;               // out: GotoTorqueBreaks, GotoRollBreaks, ApplyTorque's rotation and angular velocity
    float roll;
    F4 rot1;
    F3 w1;
};

__device__ __forceinline__ float wbc(float v, int src) { return __shfl_sync(FULL_WARP, v, src); }
__device__ __forceinline__ int wbc(int v, int src) { return __shfl_sync(FULL_WARP, v, src); }
__device__ __forceinline__ F3 wbc(F3 v, int src) { return F3{wbc(v.x, src), wbc(v.y, src), wbc(v.z, src)}; }

// kappa1 for candidate b + lane + 1: the table for the first block, else the chain from the block's first kappa
__device__ __forceinline__ float candidate_kappa(const float* krow, int b, int lane, float kbase, float tf) {
    if (b == 0) return krow[lane];
    float k = kbase;
    for (int j = 0; j <= lane; ++j) k = fmul(k, tf);
    return k;
}

// The heading search's round for one ship (the loop of full.py:2189-2201), all lanes: the first n1 in 1 .. 99 whose
// alpha1 = (target - omega0 num) / den is within max_alpha (n1 = 100 with the 99th candidate when none is), and its
// alpha1 and kappa1, returned to every lane
__device__ __forceinline__ void warp_search_v(const float* krow, const float* ndt_tab, F3 target, F3 omega0,
                                           const Search& q, float tf, float max_alpha, float limit2, bool squared,
                                           int lane, int* n1_out, F3* a1_out, float* k1_out) {
    float kbase = 1.0f;
    for (int b = 0;; b += 32) {
        const int cand = b + lane + 1;
        const float k1 = candidate_kappa(krow, b, lane, kbase, tf);
        float num, den;
        search_terms(q, k1, ndt_tab[cand < TORQUE_STEPS ? cand : TORQUE_STEPS - 1], &num, &den);
        const F3 a1 = f3_div(f3_sub(target, f3_mul(omega0, num)), den);
        const bool pass = squared ? (f3_dot(a1, a1) < limit2) : (f3_len(a1) < max_alpha);
        const unsigned hit = __ballot_sync(FULL_WARP, cand < TORQUE_STEPS && pass);
        if (hit) {
            const int first = __ffs(hit) - 1;
            *n1_out = b + first + 1;
            *a1_out = wbc(a1, first);
            *k1_out = wbc(k1, first);
            return;
        }
        if (b + 32 >= TORQUE_STEPS - 1) {                            // none passes: n1 = 100, the 99th's values
            const int last = TORQUE_STEPS - 2 - b;
            *n1_out = TORQUE_STEPS;
            *a1_out = wbc(a1, last);
            *k1_out = wbc(k1, last);
            return;
        }
        kbase = wbc(k1, 31);
    }
}

// The roll search's round for one ship (full.py:2264-2276): a true division, |alpha1| against max_alpha
__device__ __forceinline__ void warp_search_f(const float* krow, const float* ndt_tab, float desired, float omega_roll,
                                           const Search& q, float tf, float max_alpha, int lane, int* n1_out,
                                           float* a1_out, float* k1_out) {
    float kbase = 1.0f;
    for (int b = 0;; b += 32) {
        const int cand = b + lane + 1;
        const float k1 = candidate_kappa(krow, b, lane, kbase, tf);
        float num, den;
        search_terms(q, k1, ndt_tab[cand < TORQUE_STEPS ? cand : TORQUE_STEPS - 1], &num, &den);
        const float a1 = fdiv(fsub(desired, fmul(omega_roll, num)), den);
        const unsigned hit = __ballot_sync(FULL_WARP, cand < TORQUE_STEPS && fabs_(a1) < max_alpha);
        if (hit) {
            const int first = __ffs(hit) - 1;
            *n1_out = b + first + 1;
            *a1_out = wbc(a1, first);
            *k1_out = wbc(k1, first);
            return;
        }
        if (b + 32 >= TORQUE_STEPS - 1) {
            const int last = TORQUE_STEPS - 2 - b;
            *n1_out = TORQUE_STEPS;
            *a1_out = wbc(a1, last);
            *k1_out = wbc(k1, last);
            return;
        }
        kbase = wbc(k1, 31);
    }
}

// The warp's orientation step: every lane calls it together (lanes whose ship is off pass through). `ktab` is the
// warp's KTAB_FLOATS floats of shared memory; `ndt_tab` the block's table float(n dt).
__device__ __forceinline__ void orient_warp(DoLane& d, const Cfg& c, const float* ndt_tab, float* ktab) {
    const int lane = threadIdx.x & 31;
    const F3 zero = F3{0.0f, 0.0f, 0.0f};
    d.torque = zero;
    d.roll = 0.0f;
    d.rot1 = d.r0;
    d.w1 = d.w0;
    PowCache pc;
    pow_cache_clear(pc);
    Turn t;
    float accel = 0.0f, inertia = 1.0f;
    bool thrust = false;
    F3 a32 = zero;
    if (d.on) {                                                       // full.py:2463-2465, 2115-2124
        accel = tof(d3_len(d.a));
        const float fmag = fmul(d.fmass, d.agility);
        const float max_accel = fdiv(fmul(fmul(c.ffriction, d.sf), d.max_vel), fmag);
        thrust = tod(accel) > dmul(DO_THRUST, tod(max_accel));
        t.max_ang_vel = d.max_ang_vel;
        inertia = fmul(fmag, d.rot_agility);
        t.t_scale = fdiv(c.ffriction, inertia);
        t.tf = lm::expf(fmul(fneg(c.fdt), t.t_scale));
        t.tau_s = fdiv(1.0f, t.t_scale);
        t.dt = c.dt;
        t.fdt = c.fdt;
        t.ndt_tab = ndt_tab;
        a32 = f3_of(d.a);
        float k = 1.0f;                                               // kappa_1 .. kappa_32, as the loops form them
        for (int j = 0; j < 32; ++j) {
            k = fmul(k, t.tf);
            ktab[lane * KTAB_STRIDE + j] = k;
        }
    }
    __syncwarp();

    // ---- GotoTorqueBreaks: the heading torque (toward the thrust, or a coasting warper's exit point)
    bool h_active = false;
    F3 h_target = zero, h_omega0 = zero, h_alpha1 = zero, h_alpha2 = zero;
    float h_max = 0.0f, h_limit2 = 0.0f, h_kappa1 = 1.0f, h_kappa2 = 1.0f, h_g = 0.0f;
    int h_n1 = 0, h_n2 = 0;
    bool h_sq = false;
    if (d.on && (thrust || d.warping)) {
        const F3 dir = thrust ? a32 : d.to_exit;
        h_max = fmul(t.max_ang_vel, t.t_scale);
        const float len_dir = f3_len(dir);
        if (!(h_max <= 0.0f) && !(len_dir == 0.0f)) {
            const F3 heading = f3_unit(m_apply(F3{0.0f, 0.0f, 1.0f}, m_of_q(d.r0)));
            F3 target = f3_div(f3_cross(heading, dir), len_dir);
            const float rot_len = f3_len(target);
            const float rot_angle = lm::acosf(fmax_(-1.0f, fmin_(1.0f, fdiv(f3_dot(dir, heading), len_dir))));
            if (tod(rot_len) > 1e-12) target = f3_mul(target, fdiv(rot_angle, rot_len));
            else if (rot_angle > 1.0f) target = F3{fneg(rot_angle), 0.0f, 0.0f};
            const F3 omega0 = f3_sub(d.w0, f3_mul(heading, f3_dot(heading, d.w0)));
            const float len_omega0 = f3_len(omega0);
            if (!(dmul(tod(len_omega0), t.dt) < 1e-4 && tod(rot_angle) < 1e-4)) {
                h_active = true;
                h_target = target;
                h_omega0 = omega0;
                h_sq = sqrt_threshold(h_max, &h_limit2);
                if (braking(t, len_omega0, &h_n2, &h_kappa2, &h_g, pc))
                    h_alpha2 = f3_mul(F3{fneg(omega0.x), fneg(omega0.y), fneg(omega0.z)}, h_g);
            }
        }
    }
    const bool h_ran = h_active;
    for (int round = 0; round < TORQUE_ROUNDS; ++round) {
        Search q;
        q.tau = t.tau_s;
        q.n2 = h_n2;
        q.kappa2 = h_kappa2;
        q.n2dt = 0.0f;
        q.one_k2 = 0.0f;
        if (h_active) {
            q.n2dt = ndt(h_n2, t.dt);
            q.one_k2 = fsub(1.0f, h_kappa2);
            if (h_n2 > 0) {
                const F3 theta2 = f3_add(f3_mul(f3_mul(h_alpha2, q.tau), fsub(q.n2dt, fmul(q.tau, q.one_k2))),
                                         f3_mul(f3_mul(h_omega0, q.tau), q.one_k2));
                if (tod(f3_len(f3_sub(h_target, theta2))) < 1e-3) {    // braking alone gets there
                    h_n1 = 0;
                    h_active = false;
                }
            }
        }
        unsigned want = __ballot_sync(FULL_WARP, h_active);
        if (!want) break;
        while (want) {
            const int k = __ffs(want) - 1;
            want &= want - 1;
            Search qk;
            qk.tau = wbc(q.tau, k);
            qk.n2 = wbc(q.n2, k);
            qk.kappa2 = wbc(q.kappa2, k);
            qk.n2dt = wbc(q.n2dt, k);
            qk.one_k2 = wbc(q.one_k2, k);
            int n1;
            F3 a1;
            float k1;
            warp_search_v(ktab + k * KTAB_STRIDE, ndt_tab, wbc(h_target, k), wbc(h_omega0, k), qk, wbc(t.tf, k),
                          wbc(h_max, k), wbc(h_limit2, k), wbc((int)h_sq, k) != 0, lane, &n1, &a1, &k1);
            if (lane == k) {
                h_n1 = n1;
                h_alpha1 = a1;
                h_kappa1 = k1;
            }
        }
        if (h_active) {
            const F3 omega1 = f3_add(f3_mul(h_alpha1, fmul(t.tau_s, fsub(1.0f, h_kappa1))), f3_mul(h_omega0, h_kappa1));
            const int n2_old = h_n2;
            h_alpha2 = zero;
            if (braking(t, f3_len(omega1), &h_n2, &h_kappa2, &h_g, pc))
                h_alpha2 = f3_mul(F3{fneg(omega1.x), fneg(omega1.y), fneg(omega1.z)}, h_g);
            if (h_n2 == n2_old) h_active = false;
        }
    }
    if (h_ran) {
        if (h_n1 > 0) d.torque = h_n1 > 1 ? f3_mul(f3_unit(h_alpha1), h_max) : h_alpha1;
        else if (h_n2 > 0) d.torque = h_alpha2;
    }

    // ---- GotoRollBreaks: the roll torque, rolling into strong turns, otherwise upright
    bool r_active = false;
    float r_max = 0.0f, r_desired = 0.0f, r_omega = 0.0f, r_alpha1 = 0.0f, r_alpha2 = 0.0f, r_kappa1 = 1.0f;
    float r_kappa2 = 1.0f, r_g = 0.0f;
    int r_n1 = 0, r_n2 = 0;
    if (d.on) {
        r_max = fmul(t.t_scale, t.max_ang_vel);
        if (!(r_max <= 0.0f)) {
            const M3 mat = m_of_q(q_conj(d.r0));
            const F3 ship_omega = m_apply(d.w0, mat);
            r_omega = ship_omega.z;
            const float len_torque = f3_len(d.torque);
            float turn_roll = 0.0f, weight = 0.0f;
            if (tod(len_torque) > dmul(0.05, tod(r_max))) {
                const F3 ship_torque = m_apply(d.torque, mat);
                const F3 flat = F3{ship_omega.x, ship_omega.y, 0.0f};
                if (f3_dot(flat, ship_torque) >= 0.0f || f3_len(flat) < fmul(tof(0.01), t.max_ang_vel)) {
                    turn_roll = lm::atan2f(fneg(ship_torque.y), fneg(ship_torque.x));
                    weight = fdiv(len_torque, t.t_scale);
                    if (weight > 1.0f) weight = 1.0f;
                }
            }
            const F3 up = m_apply(F3{0.0f, 1.0f, 0.0f}, mat);
            const float up_roll = up.z < tof(0.95) ? lm::atan2f(fneg(up.x), up.y) : 0.0f;
            r_desired = weight < tof(0.05) ? up_roll : fmul(weight, turn_roll);
            if (!(tod(fabs_(r_omega)) < 1e-4 && tod(fabs_(r_desired)) < 1e-4)) {
                r_active = true;
                if (braking(t, fabs_(r_omega), &r_n2, &r_kappa2, &r_g, pc)) r_alpha2 = fmul(fneg(r_omega), r_g);
            }
        }
    }
    const bool r_ran = r_active;
    for (int round = 0; round < TORQUE_ROUNDS; ++round) {
        Search q;
        q.tau = t.tau_s;
        q.n2 = r_n2;
        q.kappa2 = r_kappa2;
        q.n2dt = 0.0f;
        q.one_k2 = 0.0f;
        if (r_active) {
            q.n2dt = ndt(r_n2, t.dt);
            q.one_k2 = fsub(1.0f, r_kappa2);
            if (r_n2 > 0) {
                const float theta2 = fadd(fmul(fmul(q.tau, r_alpha2), fsub(q.n2dt, fmul(q.tau, q.one_k2))),
                                          fmul(fmul(q.tau, r_omega), q.one_k2));
                if (tod(fabs_(fsub(r_desired, theta2))) < 1e-3) {
                    r_n1 = 0;
                    r_active = false;
                }
            }
        }
        unsigned want = __ballot_sync(FULL_WARP, r_active);
        if (!want) break;
        while (want) {
            const int k = __ffs(want) - 1;
            want &= want - 1;
            Search qk;
            qk.tau = wbc(q.tau, k);
            qk.n2 = wbc(q.n2, k);
            qk.kappa2 = wbc(q.kappa2, k);
            qk.n2dt = wbc(q.n2dt, k);
            qk.one_k2 = wbc(q.one_k2, k);
            int n1;
            float a1, k1;
            warp_search_f(ktab + k * KTAB_STRIDE, ndt_tab, wbc(r_desired, k), wbc(r_omega, k), qk, wbc(t.tf, k),
                          wbc(r_max, k), lane, &n1, &a1, &k1);
            if (lane == k) {
                r_n1 = n1;
                r_alpha1 = a1;
                r_kappa1 = k1;
            }
        }
        if (r_active) {
            const float omega1 = fadd(fmul(fmul(r_alpha1, t.tau_s), fsub(1.0f, r_kappa1)), fmul(r_omega, r_kappa1));
            const int n2_old = r_n2;
            r_alpha2 = 0.0f;
            if (braking(t, fabs_(omega1), &r_n2, &r_kappa2, &r_g, pc)) r_alpha2 = fmul(fneg(omega1), r_g);
            if (r_n2 == n2_old) r_active = false;
        }
    }
    if (r_ran) {
        if (r_n1 > 0) d.roll = r_n1 > 1 ? fmul(r_alpha1 >= 0.0f ? 1.0f : -1.0f, r_max) : r_alpha1;
        else if (r_n2 > 0) d.roll = r_alpha2;
    }

    // ---- ApplyTorque (the tick's rotation, the commit's too) and the thrust along the heading a tick on
    if (d.on) {
        const float tau = fdiv(inertia, c.ffriction);
        const Turned tr = apply_torque(d.r0, d.w0, d.torque, d.roll, tau, c.fdt);
        d.rot1 = tr.rot;
        d.w1 = tr.w;
        if (thrust) {
            const F3 heading = m_apply(F3{0.0f, 0.0f, 1.0f}, m_of_q(d.rot1));
            const float cosangle = fmin_(1.0f, fdiv(f3_dot(heading, a32), accel));
            d.a = (cosangle <= 0.0f) ? D3{0.0, 0.0, 0.0} : d3_of(f3_mul(heading, fmul(fmul(cosangle, cosangle), accel)));
        }
    }
    __syncwarp();
}

}  // namespace flight
}  // namespace ebb
