// SPDX-License-Identifier: MIT
// A park's rows on the device: the structure-of-arrays access to EbbFlightState's planes, and the per-row facts a
// tick's records pass and its behaviours read (whether a ship starts warp proper at its turn, StopAllFollowers'
// membership test, the records of a row, a ship loaded into its thread and its phase-1 fields stored back). Shared by
// the flight tick (ebb_flight.cu) and the combat tick (ebb_combat.cu).
#pragma once

#include "../../include/ebb.h"
#include "ebb_flight.cuh"

namespace ebb {
namespace flight {

// ---- SoA access ----
__device__ __forceinline__ D3 ld3(const double* p, int64_t i, int64_t n) { return D3{p[i], p[n + i], p[2 * n + i]}; }
__device__ __forceinline__ void st3(double* p, int64_t i, int64_t n, D3 v) {
    p[i] = v.x;
    p[n + i] = v.y;
    p[2 * n + i] = v.z;
}
__device__ __forceinline__ F3 ldf3(const float* p, int64_t i, int64_t n) { return F3{p[i], p[n + i], p[2 * n + i]}; }
__device__ __forceinline__ void stf3(float* p, int64_t i, int64_t n, F3 v) {
    p[i] = v.x;
    p[n + i] = v.y;
    p[2 * n + i] = v.z;
}
__device__ __forceinline__ F4 ldf4(const float* p, int64_t i, int64_t n) {
    return F4{p[i], p[n + i], p[2 * n + i], p[3 * n + i]};
}
__device__ __forceinline__ void stf4(float* p, int64_t i, int64_t n, F4 v) {
    p[i] = v.x;
    p[n + i] = v.y;
    p[2 * n + i] = v.z;
    p[3 * n + i] = v.w;
}

__device__ __forceinline__ Cfg cfg_of(const EbbFlightState& s) {
    return Cfg{s.friction, s.dt, s.ffriction, s.fdt, s.new_orbit, s.dynamical};
}

// Starts warp proper at its own turn this tick: free, live, aligning, aligned (its start state: nothing changes an
// aligning ship's own state before its turn)
__device__ __forceinline__ bool activates(const EbbFlightState& s, int64_t i) {
    if (!s.free_[i] || s.moribund[i] || s.mode[i] != WARP || s.effect_stamp[i] >= 0) return false;
    return aligned_for_warp(ld3(s.goto_pt, i, s.n), ld3(s.pos, i, s.n), ld3(s.vel, i, s.n), s.max_vel[i],
                            s.effect_stamp[i]);
}

// A follower's membership in row t's set (StopAllFollowers' test, Ballpark.cpp:5433-5450): its follow_ptr is t and
// its follow id t's id
__device__ __forceinline__ bool member_of(const EbbFlightState& s, int64_t t, int64_t follow_id) {
    return t >= 0 && t < s.n && s.ids[t] == follow_id;
}

// The records of row i: whether it starts warp proper, and its vertical velocity after its own turn
__device__ __forceinline__ void records_of(const EbbFlightState& s, int64_t i, bool* act, double* vy_after) {
    *act = activates(s, i);
    double vy = s.vel[s.n + i];
    if (s.free_[i] && !s.moribund[i] && !s.dynamical) {
        int32_t m = s.mode[i];
        const int64_t t = s.follow_ptr[i];
        if (member_of(s, t, s.follow_id[i]) && s.ids[t] < s.ids[i] && activates(s, t)) {
            Ship f;                                                   // released before its own turn
            f.mode = m;
            f.interactive = s.interactive[i] != 0;
            f.vel = ld3(s.vel, i, s.n);
            f.pos = ld3(s.pos, i, s.n);
            m = release(f, false);
        }
        if (m == STOP) vy = dmul(dsub(vy, dmul(STOP_DECAY, vy)), STOP_DAMP);
    }
    *vy_after = vy;
}

// What a ship's tick reads of another ship: the records and its id and radius
struct View {
    D3 pos, vel;
    double vy_after;
    int64_t id;
    float radius;
    bool act, valid;
};

__device__ __forceinline__ Ship load_ship(const EbbFlightState& s, int64_t i) {
    const int64_t n = s.n;
    Ship b;
    b.pos = ld3(s.pos, i, n);
    b.vel = ld3(s.vel, i, n);
    b.gp = ld3(s.goto_pt, i, n);
    b.last_g = ld3(s.last_g, i, n);
    b.mass = s.mass[i];
    b.tf = s.time_factor[i];
    b.last_collision = s.last_collision[i];
    b.radius = s.radius[i];
    b.max_vel = s.max_vel[i];
    b.agility = s.agility[i];
    b.sf = s.speed_fraction[i];
    b.follow_range = s.follow_range[i];
    b.id = s.ids[i];
    b.mode = s.mode[i];
    b.effect_stamp = s.effect_stamp[i];
    b.follow_id = s.follow_id[i];
    b.owner_id = s.owner_id[i];
    b.follow_ptr = s.follow_ptr[i];
    b.clock = s.clock[i];
    b.massive = s.massive[i] != 0;
    b.interactive = s.interactive[i] != 0;
    b.sensor = s.sensor[i] != 0;
    return b;
}

// The fields a tick's phase 1 may change (the velocity's STOP damping, a release, a warp's start), stored in place
// between the phases: no other ship reads them this tick (they read the records)
__device__ __forceinline__ void store_phase1(const EbbFlightState& s, int64_t i, const Ship& b) {
    const int64_t n = s.n;
    st3(s.vel, i, n, b.vel);
    st3(s.goto_pt, i, n, b.gp);
    s.last_collision[i] = b.last_collision;
    s.speed_fraction[i] = b.sf;
    s.follow_range[i] = b.follow_range;
    s.mode[i] = b.mode;
    s.effect_stamp[i] = b.effect_stamp;
    s.follow_id[i] = b.follow_id;
    s.owner_id[i] = b.owner_id;
    s.follow_ptr[i] = b.follow_ptr;
    s.massive[i] = b.massive ? 1 : 0;
    s.sensor[i] = b.sensor ? 1 : 0;
}

}  // namespace flight
}  // namespace ebb
