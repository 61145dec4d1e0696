// SPDX-License-Identifier: MIT
// The server layer over the flight park on the device, one thread a world (include/ebb.h: ebb_server_tick). What
// exact_ballpark.vec_server.VecServer's torch path does for a tick's queue (vec_server.py:707-1060) in one launch:
//
//   stamps    each world's stamp for its calls and the next one (the world's park time + 1);
//   queue     the pushes in order: the ball's row (and a FollowBall's or Orbit's target's) found among the world's
//             ids, CloakBall's bubble (0 once the ball's old bubble is its bubble, else -1; a ball not in the park not
//             queued), the duplicate test against the world's last queued call of this tick (same kind, ball,
//             target, floats by value, int argument and local flag: TIME-710), and every queued call but CloakBall
//             applied at once by the park's own command or setter (exact_ballpark.vec_modes' and vec_orient's
//             commands for one row: the guards, Stop(Ball*)'s clearing of a follower's fields, StopAllFollowers for a
//             ball entering warp, the decay factor with glibc's exp, SnapOrientation);
//   bubble    BubbleUpdater once per park time (_bubbleupdater.py:19-54): a user ball not yet settled gets every
//             uncloaked ball of its bubble, then is settled;
//   history   each queued call routed (to the bubble; to the ball's character while it is cloaked or for an uncloak;
//             a local SetBallPosition and a bubble without an interactive ball nowhere), CloakBall applied there, an
//             uncloak's AddBallsToPark recipients marked;
//   flags     after the park's tick: per row, whether its pilot gets the bubble's narrowcast and a character update.
//
// A world's calls are sequential, so its thread walks them in order; worlds never touch each other's rows. Each
// command is stated for one row in the order of operations the torch path's row-parallel version uses, with the
// rounding pinned as in the flight tick (doubles by __dadd_rn and friends, the setters' float arguments rounded to
// float, the rotation in float).

#include "../../include/ebb.h"
#include "ebb_flight.cuh"
#include "ebb_rows.cuh"

namespace ebb {
namespace server {

using namespace flight;

constexpr double MIN_WARP_DISTANCE_SQ = 10000000000.0;   // WarpTo's short hop: within 1e5 m a GotoPoint
constexpr int64_t TROLL_MIN_DELAY = 1;
constexpr double SNAP_MIN_SPEED_SQ = 1e-12;

struct World {
    const EbbServerState& s;
    const EbbFlightState& p;
    int64_t w;
    const int64_t* rows;                                  // the world's rows, -1 padded to s.width
    const int64_t* ids;

    __device__ int64_t lookup(int64_t id) const {        // the first listed ball with this id (a pad's id is 0)
        return lookup(id, s.width);
    }
    // the same over the first `span` positions, past which the world has pads alone (row -1: the same answer)
    __device__ int64_t lookup(int64_t id, int64_t span) const {
        for (int64_t k = 0; k < span; ++k)
            if (ids[k] == id) return rows[k];
        return -1;
    }
    __device__ int64_t listed_span() const {              // one past the world's last listed ball
        int64_t span = 0;
        for (int64_t k = 0; k < s.width; ++k)
            if (rows[k] >= 0) span = k + 1;
        return span;
    }
    __device__ bool any_interactive() const {
        for (int64_t k = 0; k < s.width; ++k) {
            const int64_t r = rows[k];
            if (r >= 0 && p.interactive[r] && s.exists[r]) return true;
        }
        return false;
    }

    // ---- Stop(Ball*) and the commands that move a ball (vec_modes.py:289-420) ----
    __device__ void stop_row(int64_t i) const {
        const int32_t m = p.mode[i];
        if (m == FOLLOW || m == ORBIT) {
            p.effect_stamp[i] = 0;
            p.follow_ptr[i] = -1;
            p.follow_id[i] = 0;
            p.owner_id[i] = 0;
            p.follow_range[i] = 0.0f;
        }
        p.mode[i] = STOP;
    }
    __device__ void goto_point(int64_t i, D3 pt) const {
        if (!d3_finite(pt)) return;
        stop_row(i);
        st3(p.goto_pt, i, p.n, pt);
        if (p.speed_fraction[i] == 0.0f) p.speed_fraction[i] = 1.0f;
        p.mode[i] = GOTO;
    }
    __device__ void goto_direction(int64_t i, D3 d) const {
        if (!d3_finite(d)) return;
        goto_point(i, d3_add(ld3(p.pos, i, p.n), d3_mul(d3_unit(d), DIR_DIST)));
    }
    __device__ void follow(int64_t i, int64_t t, double range, int32_t mode) const {
        const float rng = tof(range);
        if (!ffinite(rng) || t < 0 || t >= p.n || t == i) return;
        if (s.label[t] != s.label[i] || p.moribund[t] || s.bubble[t] != s.bubble[i] || s.cloaked[t] != 0) return;
        stop_row(i);
        p.follow_id[i] = p.ids[t];
        p.follow_ptr[i] = (int32_t)t;
        p.follow_range[i] = rng;
        p.mode[i] = mode;
    }
    // StopAllFollowers of row t: its followers stopped, an interactive orbiter sent along its velocity instead
    __device__ void release_followers(int64_t t) const {
        const int64_t tid = p.ids[t];
        for (int64_t k = 0; k < s.width; ++k) {
            const int64_t r = rows[k];
            if (r < 0 || p.follow_ptr[r] != t || p.follow_id[r] != tid) continue;
            if (p.interactive[r] && p.mode[r] == ORBIT)
                goto_direction(r, ld3(p.vel, r, p.n));
            else
                stop_row(r);
        }
    }
    __device__ void warp_to(int64_t i, D3 pt, double min_range, int64_t factor) const {
        bool ok = d3_finite(pt);
        const double mr = (min_range < 0.0) ? 0.0 : min_range;
        const int64_t wf = (factor <= 0) ? 1 : factor;
        const bool hop = ok && d3_lensq(d3_sub(ld3(p.pos, i, p.n), pt)) < MIN_WARP_DISTANCE_SQ;
        if (hop) goto_point(i, pt);
        if (!ok || hop) return;
        if (p.mode[i] == WARP) {
            const D3 g = ld3(p.goto_pt, i, p.n);
            if (g.x == pt.x && g.y == pt.y && g.z == pt.z) return;     // the same warp again: nothing
        }
        stop_row(i);
        st3(p.goto_pt, i, p.n, pt);
        p.effect_stamp[i] = -1;
        p.follow_range[i] = 0.0f;
        p.follow_id[i] = (int64_t)dbits(mr);
        p.owner_id[i] = wf;
        p.mode[i] = WARP;
    }
    __device__ void snap(int64_t i) const {               // SnapOrientation (a ball moving faster than 1e-6 m/s)
        const D3 v = ld3(p.vel, i, p.n);
        if (!(d3_lensq(v) > SNAP_MIN_SPEED_SQ)) return;
        const F4 r = snap_rotation(v);
        stf4(p.rot, i, p.n, r);
        stf4(p.old_rot, i, p.n, r);
        stf3(p.ang_vel, i, p.n, F3{0.0f, 0.0f, 0.0f});
        stf3(p.old_ang_vel, i, p.n, F3{0.0f, 0.0f, 0.0f});
    }
    __device__ void entity_warp_in(int64_t i, D3 pt, int64_t factor) const {
        warp_to(i, pt, 0.0, factor);
        if (p.mode[i] == GOTO) return;
        release_followers(i);
        const D3 pos = ld3(p.pos, i, p.n), g = ld3(p.goto_pt, i, p.n);
        const D3 delta = d3_unit(d3_sub(pos, g));
        const double mr = dfrom((uint64_t)p.follow_id[i]);
        const D3 dst = d3_add(g, d3_mul(delta, mr));
        st3(p.goto_pt, i, p.n, dst);
        p.massive[i] = 0;
        p.sensor[i] = 0;
        st3(p.vel, i, p.n, d3_mul(d3_unit(pt), AU));
        if (p.dynamical) snap(i);
        const int64_t back5 = p.clock[i] - 5;
        p.effect_stamp[i] = back5 < 0 ? 0 : back5;
        p.last_collision[i] = d3_len(d3_sub(pos, dst));
    }
    __device__ void set_velocity(int64_t i, D3 v) const {
        st3(p.vel, i, p.n, v);
        st3(p.old_vel, i, p.n, v);
        if (p.dynamical) snap(i);
    }
    __device__ void set_free(int64_t i, bool flag) const {
        if ((p.free_[i] != 0) == flag) return;
        p.free_[i] = flag;
        if (flag) return;
        stop_row(i);
        set_velocity(i, D3{0.0, 0.0, 0.0});
        st3(p.last_g, i, p.n, D3{0.0, 0.0, 0.0});
    }
    __device__ void decay(int64_t i) const {              // SetBallTimeFactor
        const double m = dmul(p.mass[i], tod(p.agility[i]));
        p.time_factor[i] = (m <= 0.0) ? 0.0 : lm::exp(ddiv(s.neg_kdt, m));
    }
    __device__ bool warping(int64_t i) const { return p.mode[i] == WARP && p.effect_stamp[i] >= 0; }

    // ---- the cloak's two halves (Ballpark.cpp:5223, 5257) ----
    __device__ void cloak(int64_t i, int64_t n, double range) const {
        const int64_t mode = ((n + 128) & 0xFF) - 128;   // the C char
        if (!s.exists[i] || mode <= 0) return;
        if (s.master && mode == 1) {                      // a normal cloak's proximity sensor (AddProximitySensor)
            const double r32 = tod(tof(range));
            if (!(tof(dadd(tod(p.radius[i]), r32)) < 0.0f)) p.sensor[i] = 1;
        }
        release_followers(i);
        s.cloaked[i] = mode & 0xFF;
        p.massive[i] = 0;
    }
    __device__ void uncloak(int64_t i) const {
        if (!s.exists[i]) return;
        if (s.master && s.cloaked[i] == 1) p.sensor[i] = 0;
        s.cloaked[i] = 0;
        if (!warping(i)) p.massive[i] = 1;
    }

    // ---- one queued call on its row ----
    __device__ void apply(int32_t kind, int64_t i, int64_t trow, const double* f, int64_t n) const {
        const D3 xyz{f[0], f[1], f[2]};
        switch (kind) {
            case EBB_KIND_GOTO_POINT: goto_point(i, xyz); break;
            case EBB_KIND_GOTO_DIRECTION: goto_direction(i, xyz); break;
            case EBB_KIND_STOP:
                if (p.mode[i] != STOP) stop_row(i);
                break;
            case EBB_KIND_FOLLOW_BALL: follow(i, trow, f[0], FOLLOW); break;
            case EBB_KIND_ORBIT: follow(i, trow, f[0], ORBIT); break;
            case EBB_KIND_WARP_TO: warp_to(i, xyz, f[3], n); break;
            case EBB_KIND_ENTITY_WARP_IN: entity_warp_in(i, xyz, n); break;
            case EBB_KIND_SET_SPEED_FRACTION: {
                const float v = tof(f[0]);
                if (ffinite(v)) p.speed_fraction[i] = (v < 0.0f) ? 0.0f : ((v > 1.0f) ? 1.0f : v);
                break;
            }
            case EBB_KIND_SET_MAX_SPEED: {
                const float v = tof(f[0]);
                if (!(v < 0.0f)) {
                    p.max_vel[i] = v;
                    s.refiled[i] += 1;
                }
                break;
            }
            case EBB_KIND_SET_MASS:
                if (!(f[0] <= 0.0)) {
                    p.mass[i] = f[0];
                    decay(i);
                }
                break;
            case EBB_KIND_SET_AGILITY: {
                const float v = tof(f[0]);
                if (!(v <= 0.0f)) {
                    p.agility[i] = v;
                    decay(i);
                }
                break;
            }
            case EBB_KIND_SET_RADIUS: {
                const float v = tof(f[0]);
                if (!(v < 0.0f)) {
                    p.radius[i] = v;
                    s.refiled[i] += 1;
                }
                break;
            }
            case EBB_KIND_SET_VELOCITY: set_velocity(i, xyz); break;
            case EBB_KIND_SET_MASSIVE: p.massive[i] = n != 0; break;
            case EBB_KIND_SET_INTERACTIVE: p.interactive[i] = n != 0; break;
            case EBB_KIND_SET_POSITION:
                st3(p.pos, i, p.n, xyz);
                st3(p.old_pos, i, p.n, xyz);
                break;
            case EBB_KIND_UNCLOAK: uncloak(i); break;
            case EBB_KIND_SET_MAX_ANGULAR_SPEED: {
                const float v = tof(f[0]);
                if (!(v < 0.0f)) p.max_ang_vel[i] = v;
                break;
            }
            case EBB_KIND_SET_ANGULAR_VELOCITY: {
                const F3 v{tof(f[0]), tof(f[1]), tof(f[2])};
                stf3(p.ang_vel, i, p.n, v);
                stf3(p.old_ang_vel, i, p.n, v);
                break;
            }
            case EBB_KIND_SET_ROTATION: {
                const float a = tof(f[0]), b = tof(f[1]), c = tof(f[2]), d = tof(f[3]);
                const float len = fsqrt(fadd(fadd(fadd(fmul(a, a), fmul(b, b)), fmul(c, c)), fmul(d, d)));
                if (!(tod(len) > 1e-20)) break;
                const float inv = fdiv(1.0f, len);
                const F4 q{fmul(a, inv), fmul(b, inv), fmul(c, inv), fmul(d, inv)};
                stf4(p.rot, i, p.n, q);
                stf4(p.old_rot, i, p.n, q);
                stf3(p.ang_vel, i, p.n, F3{0.0f, 0.0f, 0.0f});
                stf3(p.old_ang_vel, i, p.n, F3{0.0f, 0.0f, 0.0f});
                break;
            }
            case EBB_KIND_SET_ANGULAR_AGILITY: {
                const float v = tof(f[0]);
                if (!(v <= 0.0f)) p.rot_agility[i] = v;
                break;
            }
            case EBB_KIND_SET_TROLL: {
                const int64_t d = n < TROLL_MIN_DELAY ? TROLL_MIN_DELAY : n;
                stop_row(i);
                set_free(i, true);
                p.interactive[i] = 1;
                p.effect_stamp[i] = p.clock[i] + d;
                p.mode[i] = TROLL;
                break;
            }
            case EBB_KIND_SET_FREE: set_free(i, n != 0); break;
            default: break;                                // SetMaxAngularVelocity: the park has no such method
        }
    }

    __device__ int8_t route_of(int64_t r) const {
        if (s.cloaked[r] == 0) return EBB_ROUTE_BUBBLE;
        return s.pilot[r] >= 0 ? EBB_ROUTE_CHARACTER : EBB_ROUTE_NONE;
    }
};

// The queue pass: each push's rows, CloakBall's bubble and the duplicate test, nothing written to the park (so the
// loads of later slots need not wait for earlier slots' commands); the world's ids held in registers for the lookups.
constexpr int IDS_IN_REGISTERS = 8;

__device__ void queue(const World& x, const EbbServerQueue& q) {
    const EbbServerState& s = x.s;
    const int64_t W = s.worlds, w = x.w, J = q.slots;
    const int32_t* __restrict__ kinds = q.kinds;
    const uint8_t* __restrict__ mask = q.mask;
    const int64_t* __restrict__ balls = q.ball;
    const int64_t* __restrict__ targets = q.target;
    const int64_t* __restrict__ ns = q.n;
    const int64_t* __restrict__ locs = q.loc_in;
    const double* __restrict__ fs = q.f;
    uint8_t* __restrict__ oks = q.ok;
    int64_t* __restrict__ rows_out = q.row;
    int64_t* __restrict__ trows_out = q.trow;
    int64_t* __restrict__ locs_out = q.loc;
    int64_t ids[IDS_IN_REGISTERS], rows[IDS_IN_REGISTERS];
#pragma unroll
    for (int k = 0; k < IDS_IN_REGISTERS; ++k) {
        ids[k] = k < s.width ? x.ids[k] : 0;
        rows[k] = k < s.width ? x.rows[k] : -1;
    }
    const int64_t span = s.width > IDS_IN_REGISTERS ? x.listed_span() : s.width;
    // a wide world whose listed balls are ids 1, 2, ... in order (each id once, no pad among them): a ball's row is
    // then at its id's position, and an id outside them is no ball's (the pads past them have row -1)
    bool ordered = s.width > IDS_IN_REGISTERS;
    for (int64_t k = 0; ordered && k < span; ++k) ordered = x.ids[k] == k + 1 && x.rows[k] >= 0;
    auto lookup = [&](int64_t id) -> int64_t {
        if (ordered) return id >= 1 && id <= span ? x.rows[id - 1] : -1;
        if (s.width > IDS_IN_REGISTERS) return x.lookup(id, span);
        int64_t found = -1;
#pragma unroll
        for (int k = IDS_IN_REGISTERS - 1; k >= 0; --k)       // the first match wins
            if (k < s.width && ids[k] == id) found = rows[k];
        return found;
    };
    int32_t lk = 0;                                       // the world's last queued call (none yet: all zero)
    int64_t lb = 0, lt = 0, ln = 0, ll = 0;
    double lf0 = 0.0, lf1 = 0.0, lf2 = 0.0, lf3 = 0.0;
#pragma unroll 2
    for (int64_t j = 0; j < J; ++j) {
        const int64_t a = j * W + w;
        const int32_t kind = kinds[j];
        const int64_t ball = balls[a], target = targets[a], n = ns[a];
        const double f0 = fs[a * 4], f1 = fs[a * 4 + 1], f2 = fs[a * 4 + 2], f3 = fs[a * 4 + 3];
        const int64_t row = lookup(ball);
        const int64_t trow = (kind == EBB_KIND_FOLLOW_BALL || kind == EBB_KIND_ORBIT) ? lookup(target) : -1;
        const uint8_t byte = mask[a];
        int64_t loc = locs[a];
        bool ok;
        if (byte & 2) {                                   // tested already by an undo: bit 0 is its queued flag
            ok = (byte & 1) != 0;
        } else {
            bool pushed = (byte & 1) != 0;
            if (kind == EBB_KIND_CLOAK) {                 // the bubble it is queued in (row 0's flag for a miss)
                loc = s.settled[row < 0 ? 0 : row] ? 0 : -1;
                pushed = pushed && row >= 0;
            }
            const bool dup = lk == kind && lb == ball && lt == target && lf0 == f0 && lf1 == f1 && lf2 == f2 &&
                             lf3 == f3 && ln == n && ll == loc;
            ok = pushed && !dup;
        }
        if (ok) {
            lk = kind;
            lb = ball;
            lt = target;
            ln = n;
            ll = loc;
            lf0 = f0;
            lf1 = f1;
            lf2 = f2;
            lf3 = f3;
        }
        oks[a] = ok;
        rows_out[a] = row;
        trows_out[a] = trow;
        locs_out[a] = loc;
    }
}

__device__ void queue_and_apply(const World& x, const EbbServerQueue& q) {
    const EbbServerState& s = x.s;
    const int64_t W = s.worlds, w = x.w;
    const int64_t clock = x.p.clock[x.rows[0]];
    q.clock[w] = clock;
    q.stamp[w] = s.stamp_for_system[w];
    s.stamp_for_system[w] = clock + 1;
    queue(x, q);
    for (int64_t j = 0; j < q.slots; ++j) {               // every queued call but CloakBall, in queue order
        const int64_t a = j * W + w;
        const int32_t kind = q.kinds[j];
        const int64_t row = q.row[a];
        if (!q.ok[a] || row < 0 || kind == EBB_KIND_CLOAK) continue;
        const double f[4] = {q.f[a * 4], q.f[a * 4 + 1], q.f[a * 4 + 2], q.f[a * 4 + 3]};
        x.apply(kind, row, q.trow[a], f, q.n[a]);
    }
    // the bubble update, once per park time
    if (clock == s.bubble_time[w]) return;
    bool any_listed = false;
    for (int64_t k = 0; k < s.width; ++k) {
        const int64_t r = x.rows[k];
        if (r >= 0 && s.exists[r] && s.cloaked[r] == 0) any_listed = true;
    }
    for (int64_t k = 0; k < s.width; ++k) {
        const int64_t r = x.rows[k];
        if (r < 0) continue;
        const bool user = x.p.interactive[r] && s.exists[r];
        s.fresh[r] = user && !s.settled[r] && any_listed;
        s.listed[r] = s.exists[r] && s.cloaked[r] == 0;
        if (user) s.settled[r] = 1;
    }
    s.bubble_time[w] = clock;
}

__device__ void history(const World& x, const EbbServerQueue& q, int64_t j0, int64_t j1) {
    const EbbServerState& s = x.s;
    const int64_t W = s.worlds, w = x.w, R = x.p.n;
    const bool live = x.any_interactive();
    for (int64_t j = j0; j < j1; ++j) {
        const int64_t a = j * W + w;
        const int32_t kind = q.kinds[j];
        const bool ok = q.ok[a] != 0;
        const int64_t row = q.row[a];
        const bool valid = ok && row >= 0;
        int8_t route = EBB_ROUTE_NONE;
        if (kind == EBB_KIND_CLOAK) {
            if (ok && q.loc[a] == 0) route = EBB_ROUTE_BUBBLE;
            if (valid) x.cloak(row, q.n[a], q.f[a * 4]);
        } else if (kind == EBB_KIND_UNCLOAK) {
            if (valid && live && x.p.interactive[row] && s.pilot[row] >= 0) route = EBB_ROUTE_CHARACTER;
            for (int64_t k = 0; k < s.width; ++k) {
                const int64_t r = x.rows[k];
                if (r < 0) continue;
                q.notice[j * R + r] = valid && live && x.p.interactive[r] && s.exists[r] && r != row && s.pilot[r] >= 0;
            }
        } else {
            const bool go = (kind == EBB_KIND_SET_POSITION) ? (valid && q.loc[a] == 0 && live)
                                                             : (valid && live && q.ball[a] > 0);
            if (go) route = x.route_of(row);
        }
        q.route[j * s.worlds + w] = route;
    }
}

__device__ void flags(const World& x, const EbbServerQueue& q) {
    const EbbServerState& s = x.s;
    const int64_t W = s.worlds, w = x.w, R = x.p.n, J = q.slots;
    bool bubble = false;
    uint64_t character[2] = {0, 0};                       // the world's rows (by position) routed to their character
    bool uncloaks = false;
    for (int64_t j = 0; j < J; ++j) {
        const int8_t route = q.route[j * W + w];
        bubble = bubble || route == EBB_ROUTE_BUBBLE;
        uncloaks = uncloaks || q.kinds[j] == EBB_KIND_UNCLOAK;
        if (route != EBB_ROUTE_CHARACTER) continue;
        const int64_t a = j * W + w;
        if (!q.ok[a]) continue;
        const int64_t row = q.row[a];
        for (int64_t k = 0; k < s.width && k < 128; ++k)
            if (x.rows[k] == row) character[k >> 6] |= uint64_t(1) << (k & 63);
    }
    for (int64_t k = 0; k < s.width; ++k) {
        const int64_t r = x.rows[k];
        if (r < 0) continue;
        bool has = s.fresh[r] != 0;
        if (k < 128) {
            has = has || ((character[k >> 6] >> (k & 63)) & 1u);
        } else {                                          // a world wider than the mask: the slots again
            for (int64_t j = 0; j < J && !has; ++j) {
                const int64_t a = j * W + w;
                has = q.ok[a] && q.row[a] == r && q.route[j * W + w] == EBB_ROUTE_CHARACTER;
            }
        }
        for (int64_t j = 0; j < J && uncloaks && !has; ++j)
            has = q.kinds[j] == EBB_KIND_UNCLOAK && q.notice[j * R + r];
        const bool pilot = s.pilot[r] >= 0;
        q.has_character[r] = has && pilot;
        q.gets_bubble[r] = bubble && x.p.interactive[r] && s.exists[r] && pilot;
    }
}

__global__ void __launch_bounds__(128) server_kernel(EbbServerState s, EbbServerQueue q, int phase, int64_t j0,
                                                      int64_t j1) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= s.worlds) return;
    const World x{s, s.flight, w, s.world_rows + w * s.width, s.world_ids + w * s.width};
    switch (phase) {
        case 0:
            queue_and_apply(x, q);
            history(x, q, 0, q.slots);
            break;
        case 1: queue_and_apply(x, q); break;
        case 2: history(x, q, j0, j1); break;
        case 3: flags(x, q); break;
        case 4:
            if (!x.any_interactive()) s.dead[w] = 1;
            break;
        case 5:                                           // phase 0, then the park's tick's dead-bubble test
            queue_and_apply(x, q);
            history(x, q, 0, q.slots);
            if (!x.any_interactive()) s.dead[w] = 1;
            break;
        case 6: queue(x, q); break;                       // the queue's test alone: flags, rows, CloakBall's bubble
        default: break;
    }
}

cudaError_t attributes(cudaFuncAttributes* fa) { return cudaFuncGetAttributes(fa, server_kernel); }

}  // namespace server
}  // namespace ebb

extern "C" {

int ebb_server_tick(const EbbServerState* s, const EbbServerQueue* q, int phase, int64_t j0, int64_t j1, void* stream,
                    int block) {
    if (s == nullptr || q == nullptr || phase < 0 || phase > 6) return EBB_EINVAL;
    if (q->slots < 0 || q->slots > EBB_SERVER_MAX_SLOTS || block <= 0 || block > 128 || block % 32 != 0)
        return EBB_EINVAL;
    if (phase == 2 && (j0 < 0 || j1 < j0 || j1 > q->slots)) return EBB_EINVAL;
    if (s->worlds <= 0) return 0;
    if (s->width <= 0 || s->world_rows == nullptr || s->world_ids == nullptr || s->pilot == nullptr ||
        s->exists == nullptr || s->label == nullptr || s->cloaked == nullptr || s->bubble == nullptr ||
        s->refiled == nullptr || s->stamp_for_system == nullptr || s->bubble_time == nullptr || s->dead == nullptr ||
        s->settled == nullptr || s->fresh == nullptr || s->listed == nullptr)
        return EBB_EINVAL;
    if (phase != 4 && (q->stamp == nullptr || q->clock == nullptr || q->has_character == nullptr ||
                       q->gets_bubble == nullptr))
        return EBB_EINVAL;
    if (phase != 4 && q->slots > 0 &&
        (q->kinds == nullptr || q->mask == nullptr || q->ball == nullptr || q->target == nullptr || q->n == nullptr ||
         q->loc_in == nullptr || q->f == nullptr || q->ok == nullptr || q->row == nullptr || q->trow == nullptr ||
         q->loc == nullptr || q->route == nullptr || q->notice == nullptr))
        return EBB_EINVAL;
    const unsigned grid = (unsigned)((s->worlds + block - 1) / block);
    ebb::server::server_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(*s, *q, phase, j0, j1);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}

}  // extern "C"

EBB_OP_COUNTER(ebb_count_ops_server)
