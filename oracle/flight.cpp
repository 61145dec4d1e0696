// TEST INFRASTRUCTURE, NOT THE PRODUCT. The CPU oracle of the flight-mode tick: a scalar restatement of the
// reference's sequential algorithm, used by tests/ (and smoke(), bench.py's cpu_baseline) as the checker of the CUDA
// kernels. Nothing in exact_ballpark_b200 links or calls it.
//
// One tick of every world, as exact_ballpark/modes.py's ModeBallpark.evolve (modes.py:702-745) and, with dynamical
// orientation, exact_ballpark/full.py's FullBallpark.evolve (full.py:2487-2588) run it: the worlds one after another,
// each world's live balls in ascending id, phase 1 (the behaviours, modes.py:359-377 / full.py:2416-2446) reading the
// other balls as they stand at that moment; phase 3 (the warp path or the integrator, and the rotation a tick on);
// phase 4 (the commit, full.py:2532-2560); PetrifyTroll (full.py:1800); every row's clock. The layout is the
// reference park's (exact_ballpark/vec_modes.py: vectors as [n, 3] or [n, 4] doubles, floats held in doubles,
// integers int64, flags bytes). The follower set of a ball is the rows whose follow_ptr is its row and whose follow
// id is its id (vec_modes.py:37-47).
//
// With the combat park's state (exact_ballpark/vec_combat.py, full.py's missiles and formations) the same tick also
// runs MISSILE (EvolveMissile, full.py:2337) and FORMATION (EvolveFormation, full.py:2359), the release of a missile
// (non-massive, GotoDirection along its velocity) or a formation member (Stop, its slot freed on the master), each
// massive normal missile's Potential with its target after every behaviour (counted: its response is not kept),
// dynamical orientation disabled for missiles when asked (the old rotation kept, snapped to the velocity at the
// commit), and the commit's dispatch counts (DoCollision with the target, the master's self-collision).
//
// Arithmetic: plain C++ double and float operations (built with -ffp-contract=off: each one IEEE-rounded, nothing
// fused), glibc 2.34 aarch64's libm through ebb_libm.cuh's host build (pinned separately to the reference's
// transcriptions by tests/test_libm_oracle.py).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "../exact_ballpark_b200/csrc/ebb_libm.cuh"

#include "flight_state.h"

namespace {

namespace lm = ebb::lm;

// Destiny's modes (IDstConstants.h; modes.py:65-67)
constexpr int64_t GOTO = 0, FOLLOW = 1, STOP = 2, WARP = 3, ORBIT = 4, MISSILE = 5, MUSHROOM = 6, TROLL = 8;
constexpr int64_t MINIBALL = 9, RIGID = 11, FORMATION = 12;
constexpr double STOP_DAMP = 0.9345794392523364485981308411215;   // ref.py:48
constexpr double AU = .1495978707e12;                              // modes.py:72
constexpr double ORBITAL_PRECESSION = 0.001;                       // modes.py:73
constexpr double WARP_AU_PER_S = 0.001, WARP_ACC = 1.0 / 1000, WARP_DEC = 1.0 / 3000;   // modes.py:74-76
constexpr int64_t MAX_ALIGN_TICKS = 180;                           // modes.py:77

// The combat park's state beside the flight fields (vec_combat.py:151-170): which rows hold a ball, a leader's
// formation and slot bits, a missile's owner row, the tick's counts, the bubbles and cloaks, the formation table
struct Combat {
    uint8_t* exists;
    int64_t *formation_id, *formation_slots, *owner_ptr, *hits_n, *ev_n;
    uint8_t* ev_self;
    int64_t *bubble, *cloaked, *flags;
    const double* formations;
    const int64_t* formation_len;
    int64_t n_formations, max_slots, tick_ms;
    int32_t do_missiles_off, master;
};

// The composed park's state beside the combat state (vec_composed.py:189-205): each row's collision acceleration
// mLastC [n][3], its filing in the partition (level [n], key and side [n][3]) and its collision list [n][hit_cap]
struct Composed {
    double* last_c;
    int64_t *level, *key, *mod, *hits;
    int64_t hit_cap;
};

struct Park {
    Combat* c = nullptr;
    Composed* x = nullptr;
    const OracleTickHooks* h = nullptr;
    int64_t n;
    double friction, dt;
    float ffriction, fdt;
    int new_orbit, dynamical;
    double *pos, *vel, *old_pos, *old_vel, *goto_, *last_g;
    double *mass, *time_factor, *last_collision;
    double *radius, *max_vel, *agility, *speed_fraction, *follow_range, *max_ang_vel, *rot_agility, *rot_roll;
    double *rot, *old_rot, *ang_vel, *old_ang_vel, *torque;
    int64_t *ids, *world, *mode, *effect_stamp, *follow_id, *owner_id, *follow_ptr, *clock;
    uint8_t *free_, *moribund, *massive, *interactive, *sensor;
};

struct V { double x, y, z; };
V ld(const double* p, int64_t i) { return V{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
void st(double* p, int64_t i, V v) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }
V sub(V a, V b) { return V{a.x - b.x, a.y - b.y, a.z - b.z}; }
V add(V a, V b) { return V{a.x + b.x, a.y + b.y, a.z + b.z}; }
V scl(V a, double c) { return V{a.x * c, a.y * c, a.z * c}; }
double lensq(V v) { return v.x * v.x + v.y * v.y + v.z * v.z; }                     // modes.py:81
double length(V v) { return std::sqrt(lensq(v)); }
V normalized(V v) {                                                                    // ref.py:58
    const double n = length(v);
    if (n == 0.0) return v;
    return scl(v, 1.0 / n);
}
V cross(V u, V v) { return V{u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x}; }   // modes.py:89
bool finite3(V v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }
int64_t to_i64(double x) { return ebb::to_i64(x); }
double trunc7(double x) { return (double)to_i64(x * 10000000) / 10000000; }          // modes.py:94

// ---- C++ float vectors (full.py:140-300) ----
struct F3 { float x, y, z; };
struct F4 { float x, y, z, w; };
F3 f3mul(F3 a, float f) { return F3{a.x * f, a.y * f, a.z * f}; }
F3 f3add(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
F3 f3sub(F3 a, F3 b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }
F3 f3div(F3 a, float f) { return f3mul(a, 1.0f / f); }
float f3dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
float f3len(F3 a) { return std::sqrt(f3dot(a, a)); }
F3 f3cross(F3 a, F3 b) { return F3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
float fmaxs(float a, float b) { return (a < b) ? b : a; }
float fmins(float a, float b) { return (b < a) ? b : a; }
F3 f3normalize(F3 v) {                     // Vector3::Normalize: by the largest magnitude, then by the length
    const float mx = fmaxs(fmaxs(std::fabs(v.x), std::fabs(v.y)), std::fabs(v.z));
    const F3 m = f3div(v, mx != 0.0f ? mx : 1.0f);
    const float l = f3len(m);
    return f3mul(m, l != 0.0f ? 1.0f / l : l);
}
F4 qmul(F4 q, F4 o) {
    return F4{o.w * q.x + o.x * q.w + o.y * q.z - o.z * q.y, o.w * q.y - o.x * q.z + o.y * q.w + o.z * q.x,
              o.w * q.z + o.x * q.y - o.y * q.x + o.z * q.w, o.w * q.w - o.x * q.x - o.y * q.y - o.z * q.z};
}
float qlensq(F4 q) { return q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w; }
F4 qdiv(F4 q, float f) {
    const float d = 1.0f / f;
    return F4{q.x * d, q.y * d, q.z * d, q.w * d};
}
F4 qconj(F4 q) { return F4{-q.x, -q.y, -q.z, q.w}; }
F4 qrot(F3 axis, float angle) {            // RotationQuaternion(axis, angle)
    const F3 t = f3normalize(axis);
    const float h = angle / 2.0f;
    const float s = lm::sinf(h);
    return F4{s * t.x, s * t.y, s * t.z, lm::cosf(h)};
}
struct M3 { float m[3][3]; };
M3 mrot(F4 q) {                             // RotationMatrix(Quaternion), the 3x3 part
    const float x = q.x, y = q.y, z = q.z, w = q.w;
    M3 r;
    r.m[0][0] = 1.0f - 2.0f * (y * y + z * z);
    r.m[0][1] = 2.0f * (x * y + z * w);
    r.m[0][2] = 2.0f * (x * z - y * w);
    r.m[1][0] = 2.0f * (x * y - z * w);
    r.m[1][1] = 1.0f - 2.0f * (x * x + z * z);
    r.m[1][2] = 2.0f * (y * z + x * w);
    r.m[2][0] = 2.0f * (x * z + y * w);
    r.m[2][1] = 2.0f * (y * z - x * w);
    r.m[2][2] = 1.0f - 2.0f * (x * x + y * y);
    return r;
}
F3 tcoord(F3 v, const M3& m) {              // TransformCoord: the row vector times the matrix, over the w norm
    const float norm = 0.0f * v.x + 0.0f * v.y + 0.0f * v.z + 1.0f;
    if (!(norm != 0.0f)) return F3{0.0f, 0.0f, 0.0f};
    return F3{(v.x * m.m[0][0] + v.y * m.m[1][0] + v.z * m.m[2][0] + 0.0f) / norm,
              (v.x * m.m[0][1] + v.y * m.m[1][1] + v.z * m.m[2][1] + 0.0f) / norm,
              (v.x * m.m[0][2] + v.y * m.m[1][2] + v.z * m.m[2][2] + 0.0f) / norm};
}
float f(double x) { return (float)x; }

// ---- dynamical orientation (full.py:2124-2320) ----
struct Turn {
    float max_ang_vel, t_scale;
    double dt;
    float fdt;
};

void n2_alpha2_v(const Turn& t, F3 omega0, float len_omega0, float tf, int* n2, float* kappa2, F3* alpha2) {
    if (len_omega0 > 1e-10) {
        const float factor = t.max_ang_vel / len_omega0;
        *n2 = ebb::to_i32(std::ceil(lm::logf(factor / (1.0f + factor)) / (-t.fdt * t.t_scale)));
        *kappa2 = f(lm::pow(tf, (double)*n2));
        *alpha2 = f3mul(F3{-omega0.x, -omega0.y, -omega0.z}, (t.t_scale * *kappa2) / (1.0f - *kappa2));
    } else {
        *n2 = 0;
        *kappa2 = 1.0f;
        *alpha2 = F3{0, 0, 0};
    }
}
void n2_alpha2_f(const Turn& t, float omega0, float tf, int* n2, float* kappa2, float* alpha2) {
    if (std::fabs(omega0) > 1e-10) {
        const float factor = t.max_ang_vel / std::fabs(omega0);
        *n2 = ebb::to_i32(std::ceil(lm::logf(factor / (1.0f + factor)) / (-t.fdt * t.t_scale)));
        *kappa2 = f(lm::pow(tf, (double)*n2));
        *alpha2 = -omega0 * ((t.t_scale * *kappa2) / (1.0f - *kappa2));
    } else {
        *n2 = 0;
        *kappa2 = 1.0f;
        *alpha2 = 0.0f;
    }
}

F3 goto_torque_breaks(const Turn& t, F4 rot, F3 w, F3 direction) {     // full.py:2155
    const float max_alpha = t.max_ang_vel * t.t_scale;
    if (max_alpha <= 0.0f) return F3{0, 0, 0};
    const float len_dir = f3len(direction);
    if (len_dir == 0.0f) return F3{0, 0, 0};
    const F3 heading = f3normalize(tcoord(F3{0, 0, 1}, mrot(rot)));
    F3 r = f3div(f3cross(heading, direction), len_dir);
    const float rot_len = f3len(r);
    const float rot_angle = lm::acosf(fmaxs(-1.0f, fmins(1.0f, f3dot(direction, heading) / len_dir)));
    if (rot_len > 1e-12) r = f3mul(r, rot_angle / rot_len);
    else if (rot_angle > 1) r = F3{-rot_angle, 0, 0};
    const F3 omega0 = f3sub(w, f3mul(heading, f3dot(heading, w)));
    const float len_omega0 = f3len(omega0);
    const double dt = t.dt;
    if (len_omega0 * dt < 1e-4 && rot_angle < 1e-4) return F3{0, 0, 0};
    const float fdt = t.fdt;
    const float tf = lm::expf(-fdt * t.t_scale);
    const float tau = 1.0f / t.t_scale;
    int n1 = 0;
    F3 alpha1{0, 0, 0};
    float kappa1 = 1.0f;
    int n2;
    float kappa2;
    F3 alpha2;
    n2_alpha2_v(t, omega0, len_omega0, tf, &n2, &kappa2, &alpha2);
    for (int round = 0; round < 5; ++round) {
        if (n2 > 0) {
            const F3 theta2 = f3add(f3mul(f3mul(alpha2, tau), f(n2 * dt) - tau * (1.0f - kappa2)),
                                    f3mul(f3mul(omega0, tau), 1 - kappa2));
            if (f3len(f3sub(r, theta2)) < 1e-3) {
                n1 = 0;
                break;
            }
        }
        kappa1 = 1.0f;
        n1 = 1;
        while (n1 < 100) {
            kappa1 = kappa1 * tf;
            if (n2 == 0) {
                alpha1 = f3div(f3sub(r, f3mul(omega0, tau * (1.0f - kappa1))), tau * (f(n1 * dt) - tau * (1.0f - kappa1)));
            } else {
                const float num = tau - (kappa1 * kappa2 * f(n2 * dt)) / (1 - kappa2);
                const float den = tau * (f(n1 * dt) - (f(n2 * dt) * kappa2 * (1 - kappa1)) / (1 - kappa2));
                alpha1 = f3div(f3sub(r, f3mul(omega0, num)), den);
            }
            if (f3len(alpha1) < max_alpha) break;
            ++n1;
        }
        const int n2_old = n2;
        const F3 omega1 = f3add(f3mul(alpha1, tau * (1 - kappa1)), f3mul(omega0, kappa1));
        n2_alpha2_v(t, omega1, f3len(omega1), tf, &n2, &kappa2, &alpha2);
        if (n2_old == n2) break;
    }
    if (n1 > 0) return n1 > 1 ? f3mul(f3normalize(alpha1), max_alpha) : alpha1;
    if (n2 > 0) return alpha2;
    return F3{0, 0, 0};
}

float goto_roll_breaks(const Turn& t, F4 rot, F3 w, F3 heading_torque) {   // full.py:2224
    const float max_alpha = t.t_scale * t.max_ang_vel;
    if (max_alpha <= 0) return 0.0f;
    const M3 mat = mrot(qconj(rot));
    F3 ship_omega = tcoord(w, mat);
    const float omega_roll = ship_omega.z;
    const float len_torque = f3len(heading_torque);
    float turn_roll = 0.0f, weight = 0.0f;
    if (len_torque > 0.05 * max_alpha) {
        const F3 ship_torque = tcoord(heading_torque, mat);
        ship_omega = F3{ship_omega.x, ship_omega.y, 0.0f};
        if (f3dot(ship_omega, ship_torque) >= 0 || f3len(ship_omega) < f(0.01) * t.max_ang_vel) {
            turn_roll = lm::atan2f(-ship_torque.y, -ship_torque.x);
            weight = len_torque / t.t_scale;
            if (weight > 1.0f) weight = 1.0f;
        }
    }
    const F3 up = tcoord(F3{0, 1, 0}, mat);
    const float up_roll = up.z < f(0.95) ? lm::atan2f(-up.x, up.y) : 0.0f;
    const float desired = weight < f(0.05) ? up_roll : weight * turn_roll;
    if (std::fabs(omega_roll) < 1e-4 && std::fabs(desired) < 1e-4) return 0.0f;
    const double dt = t.dt;
    const float tf = lm::expf(-t.fdt * t.t_scale);
    const float tau = 1.0f / t.t_scale;
    int n1 = 0;
    float alpha1 = 0.0f, kappa1 = 1.0f;
    int n2;
    float kappa2, alpha2;
    n2_alpha2_f(t, omega_roll, tf, &n2, &kappa2, &alpha2);
    for (int round = 0; round < 5; ++round) {
        if (n2 > 0) {
            const float theta2 = tau * alpha2 * (f(n2 * dt) - tau * (1.0f - kappa2)) + tau * omega_roll * (1 - kappa2);
            if (std::fabs(desired - theta2) < 1e-3) {
                n1 = 0;
                break;
            }
        }
        kappa1 = 1.0f;
        n1 = 1;
        while (n1 < 100) {
            kappa1 = kappa1 * tf;
            if (n2 == 0) {
                alpha1 = (desired - omega_roll * (tau * (1.0f - kappa1))) / (tau * (f(n1 * dt) - tau * (1.0f - kappa1)));
            } else {
                const float num = tau - (kappa1 * kappa2 * f(n2 * dt)) / (1 - kappa2);
                const float den = tau * (f(n1 * dt) - (f(n2 * dt) * kappa2 * (1 - kappa1)) / (1 - kappa2));
                alpha1 = (desired - omega_roll * num) / den;
            }
            if (std::fabs(alpha1) < max_alpha) break;
            ++n1;
        }
        const int n2_old = n2;
        const float omega1 = alpha1 * tau * (1 - kappa1) + omega_roll * kappa1;
        n2_alpha2_f(t, omega1, tf, &n2, &kappa2, &alpha2);
        if (n2_old == n2) break;
    }
    if (n1 > 0) return n1 > 1 ? (alpha1 >= 0.0f ? 1.0f : -1.0f) * max_alpha : alpha1;
    if (n2 > 0) return alpha2;
    return 0.0f;
}

void apply_torque(F4 rotation, F3 angvel, F3 torque, float roll, float tau, float fdt, F4* rot_out, F3* w_out) {
    // full.py:2292, fraction 1
    const float tf = lm::expf((-fdt * 1.0f) / tau);
    const F3 heading = tcoord(F3{0, 0, 1}, mrot(rotation));
    const float omega_roll = f3dot(angvel, heading);
    const F3 omega_heading = f3sub(angvel, f3mul(heading, omega_roll));
    const float span = 1.0f * fdt - tau * (1.0f - tf);
    const float rot_roll = tau * (roll * span + omega_roll * (1.0f - tf));
    const F3 rot_heading = f3mul(f3add(f3mul(torque, span), f3mul(omega_heading, 1.0f - tf)), tau);
    const float angle_heading = f3len(rot_heading);
    const bool apply = angle_heading > 1e-10;
    const F4 quat_heading = apply ? qrot(rot_heading, f3len(rot_heading)) : F4{0, 0, 0, 1};
    const F3 heading_rotated = apply ? tcoord(heading, mrot(quat_heading)) : heading;
    F3 w = f3add(f3mul(torque, tau * (1.0f - tf)), f3mul(omega_heading, tf));
    w = f3add(w, f3mul(heading_rotated, tau * roll - (tau * roll - omega_roll) * tf));
    if (apply) rotation = qmul(rotation, quat_heading);
    rotation = qmul(rotation, qrot(heading_rotated, rot_roll));
    const float norm = std::sqrt(qlensq(rotation));
    if (norm > 0) rotation = qdiv(rotation, norm);
    *rot_out = rotation;
    *w_out = w;
}

void snap_one(const double* v, double* rot, double* old_rot, double* w, double* old_w);

// ============================================================================================= the tick

struct Tick {
    Park& p;
    explicit Tick(Park& park) : p(park) {}

    bool live(int64_t i) const { return p.free_[i] && !p.moribund[i]; }
    float ff(const double* a, int64_t i) const { return (float)a[i]; }
    F4 rot_of(int64_t i) const {
        return F4{ff(p.rot, 4 * i), ff(p.rot, 4 * i + 1), ff(p.rot, 4 * i + 2), ff(p.rot, 4 * i + 3)};
    }
    F3 w_of(int64_t i) const { return F3{ff(p.ang_vel, 3 * i), ff(p.ang_vel, 3 * i + 1), ff(p.ang_vel, 3 * i + 2)}; }
    float t_scale(int64_t i) const {        // full.py:2120
        return p.ffriction / ((float)p.mass[i] * ff(p.agility, i) * ff(p.rot_agility, i));
    }
    float tau(int64_t i) const { return ((float)p.mass[i] * ff(p.agility, i) * ff(p.rot_agility, i)) / p.ffriction; }

    bool warping(int64_t i) const { return p.mode[i] == WARP && !(p.effect_stamp[i] < 0); }

    V goto_thrust(int64_t i, V target) {     // ref.py:343 (GotoThrust), C's division
        const V a = sub(target, ld(p.pos, i));
        const double length2 = lensq(a);
        const double sf = p.speed_fraction[i], mv = p.max_vel[i];
        const double dist = sf * mv * p.dt;
        const double max_thrust = p.friction * sf * mv / (p.mass[i] * p.agility[i]);
        const V unit = normalized(a);
        if (length2 < dist * dist) {
            const double coff = length2 / (dist * dist);
            return scl(unit, max_thrust * coff * coff);
        }
        return scl(unit, max_thrust);
    }

    // Stop(Ball*) (modes.py:206)
    void stop_ball(int64_t i) {
        const int64_t m = p.mode[i];
        if (p.c && p.c->master && m == FORMATION) free_slot(i);
        if (m == FOLLOW || m == ORBIT || m == MISSILE || m == FORMATION) {
            p.effect_stamp[i] = 0;
            p.follow_ptr[i] = -1;
            p.follow_id[i] = 0;
            p.owner_id[i] = 0;
            p.follow_range[i] = 0.0;
            if (p.c) p.c->owner_ptr[i] = -1;
        }
        p.mode[i] = STOP;
    }
    // On the master, Stop(Ball*) of a FORMATION member frees its slot in the leader (Ballpark.cpp:4629-4633;
    // Ball::FreeFormationSlot((size_t) mEffectStamp), Ball.cpp:2324): nothing without a loaded formation or past its
    // end; a negative formation index or a slot of 16 or more flagged
    void free_slot(int64_t i) {
        const int64_t t = p.follow_ptr[i];
        if (t < 0 || t >= p.n) return;
        const int64_t fid = p.c->formation_id[t];
        if (fid == -1 || fid > p.c->n_formations - 1) return;
        if (fid < 0) {
            p.c->flags[i] |= 2;
            return;
        }
        const uint64_t len = (uint64_t)p.c->formation_len[fid], slot = (uint64_t)p.effect_stamp[i];
        if (slot > len - 1) return;
        if (slot >= 16) {
            p.c->flags[i] |= 2;
            return;
        }
        p.c->formation_slots[t] &= ~(int64_t)(1ULL << slot);
    }
    bool disabled(int64_t i) const { return p.c && p.c->do_missiles_off && p.mode[i] == MISSILE; }
    // GotoDirection(Ball*) (modes.py:252) with GotoPoint(Ball*) (modes.py:238)
    void goto_direction(int64_t i, V d) {
        if (!finite3(d)) return;
        d = normalized(d);
        const V pos = ld(p.pos, i);
        const V pt = V{pos.x + d.x * 1.0e17, pos.y + d.y * 1.0e17, pos.z + d.z * 1.0e17};
        if (!finite3(pt)) return;
        stop_ball(i);
        st(p.goto_, i, pt);
        if (p.speed_fraction[i] == 0.0) p.speed_fraction[i] = 1.0;
        p.mode[i] = GOTO;
    }
    // StopAllFollowers (modes.py:410): the members of row w's set (the world's rows only)
    void stop_all_followers(int64_t w, const std::vector<int64_t>& rows) {
        for (int64_t f : rows) {
            if (p.follow_ptr[f] != w || p.follow_id[f] != p.ids[w]) continue;
            if (p.c && !p.c->exists[f]) continue;
            if (p.mode[f] == MISSILE || (p.interactive[f] && p.mode[f] == ORBIT)) {
                if (p.mode[f] == MISSILE) p.massive[f] = 0;
                goto_direction(f, ld(p.vel, f));
            } else {
                stop_ball(f);
            }
        }
    }
    // IsAlignedForWarp (modes.py:342)
    bool aligned(int64_t i) {
        if (!(p.mode[i] == WARP && p.effect_stamp[i] < 0)) return false;
        const V d = normalized(sub(ld(p.goto_, i), ld(p.pos, i)));
        const V u = normalized(ld(p.vel, i));
        const double mv = p.max_vel[i];
        if (std::fabs(1.0 - (u.x * d.x + u.y * d.y + u.z * d.z)) < 0.01 && lensq(ld(p.vel, i)) > 0.5625 * mv * mv)
            return true;
        const int64_t es = p.effect_stamp[i];
        return (es < 0 ? -es : es) > MAX_ALIGN_TICKS;
    }
    // RealWarp (modes.py:391)
    void real_warp(int64_t i, const std::vector<int64_t>& rows) {
        stop_all_followers(i, rows);
        V dst = ld(p.goto_, i);
        const V delta = normalized(sub(ld(p.pos, i), dst));
        const double mr = ebb::dfrom((uint64_t)p.follow_id[i]);
        dst = V{dst.x + delta.x * mr, dst.y + delta.y * mr, dst.z + delta.z * mr};
        st(p.goto_, i, dst);
        p.effect_stamp[i] = p.clock[i];
        p.last_collision[i] = length(sub(dst, ld(p.pos, i)));
        p.massive[i] = 0;
        p.sensor[i] = 0;
    }
    V evolve_follow(int64_t i, int64_t o) {   // modes.py:428
        const V op = ld(p.pos, o);
        const V delta = sub(ld(p.pos, i), op);
        const double dist = length(delta);
        const double r = p.follow_range[i] + p.radius[i] + p.radius[o];
        V target;
        if (dist == 0.0) {
            target = V{op.x + 1.0 * r, op.y + 0.0 * r, op.z + 0.0 * r};
        } else {
            const double inv = 1.0 / dist;
            target = V{op.x + delta.x * r * inv, op.y + delta.y * r * inv, op.z + delta.z * r * inv};
        }
        st(p.goto_, i, target);
        return goto_thrust(i, target);
    }
    V precessing(int64_t i) {                 // modes.py:480
        const double t = (double)p.clock[i];
        const double phi1 = t * ORBITAL_PRECESSION;
        const double phi2 = (double)(p.ids[i] & 0x000000000000FFFFLL) + t * ORBITAL_PRECESSION;
        double s1, c1, s2, c2;
        lm::sincos(phi1, &s1, &c1);
        lm::sincos(phi2, &s2, &c2);
        return V{trunc7(c1 * c2), trunc7(s2), trunc7(s1 * c2)};
    }
    V evolve_old_orbit(int64_t i, int64_t o) {   // modes.py:444
        const double cruise = p.speed_fraction[i] * p.max_vel[i];
        const double max_thrust = p.friction * cruise / (p.mass[i] * p.agility[i]);
        const V pos = ld(p.pos, i);
        const V op = ld(p.pos, o);
        const double r = p.follow_range[i] + p.radius[i] + p.radius[o];
        V to = sub(op, pos);
        const double dist = length(to);
        to = normalized(to);
        const V w = normalized(cross(precessing(i), to));
        const double to_comp = dist * dist - r * r;
        if (to_comp >= 0.0) {
            const double rad_comp = r * std::sqrt(to_comp) / dist;
            const double s = to_comp / dist;
            to = normalized(V{to.x * s + w.x * rad_comp, to.y * s + w.y * rad_comp, to.z * s + w.z * rad_comp});
        }
        const double rf = trunc7(lm::exp(-(r - dist) * (r - dist) / 40000.0));
        const double phi1 = (-to.x) * w.x + (-to.y) * w.y + (-to.z) * w.z;
        double tf = 1.0 + rf * rf * (phi1 * phi1 - 1.0);
        if (tf > 0.0) tf = rf * phi1 + std::sqrt(tf);
        else tf = rf * phi1;
        tf *= (dist - r >= 0.0) ? 1.0 : -1.0;
        const V a = V{(w.x * rf + to.x * tf) * max_thrust, (w.y * rf + to.y * tf) * max_thrust,
                      (w.z * rf + to.z * tf) * max_thrust};
        st(p.goto_, i, V{pos.x + a.x * (10.0 * AU), pos.y + a.y * (10.0 * AU), pos.z + a.z * (10.0 * AU)});
        return a;
    }
    V orbit_thrust(int64_t i, V target) {     // modes.py:586
        const double fom = p.friction / (p.mass[i] * p.agility[i]);
        const double max_accel = fom * p.speed_fraction[i] * p.max_vel[i];
        if (max_accel <= 0) return V{0, 0, 0};
        const V pos = ld(p.pos, i), vel = ld(p.vel, i);
        V a = V{(target.x - pos.x) * fom - vel.x, (target.y - pos.y) * fom - vel.y, (target.z - pos.z) * fom - vel.z};
        const double tacc = length(a) / max_accel;
        if (tacc > 1) a = scl(a, 1.0 / tacc);
        if (tacc < 0.1) return V{0, 0, 0};
        return a;
    }
    V goto_thrust_follow(int64_t i, V target, V tv) {   // modes.py:557, weight 1
        const double speed = length(tv);
        const double mv = p.max_vel[i], sf = p.speed_fraction[i];
        if (speed < 5e-2 * mv * sf) {
            if (p.new_orbit && p.mode[i] == ORBIT) return orbit_thrust(i, target);
            return goto_thrust(i, ld(p.goto_, i));
        }
        const double fom = p.friction / (p.mass[i] * p.agility[i]);
        const double max_accel = fom * sf * mv;
        if (max_accel <= 0) return V{0, 0, 0};
        const double tfac = p.time_factor[i];
        const double one_minus = 1 - tfac;
        const V pos = ld(p.pos, i), vel = ld(p.vel, i);
        double inv = 1.0 / (p.dt * fom - one_minus);
        V a = V{((target.x - pos.x) * fom - vel.x * one_minus) * fom * inv,
                ((target.y - pos.y) * fom - vel.y * one_minus) * fom * inv,
                ((target.z - pos.z) * fom - vel.z * one_minus) * fom * inv};
        inv = 1.0 / (1.0 - tfac);
        const V avel = V{(tv.x - vel.x * tfac) * fom * inv, (tv.y - vel.y * tfac) * fom * inv,
                         (tv.z - vel.z * tfac) * fom * inv};
        const double weight = 1.0;
        inv = 1.0 / (1.0 + weight);
        a = V{(a.x + avel.x * weight) * inv, (a.y + avel.y * weight) * inv, (a.z + avel.z * weight) * inv};
        const double accel = lensq(a);
        if (accel > max_accel * max_accel) a = scl(a, max_accel / std::sqrt(accel));
        return a;
    }
    V evolve_new_orbit(int64_t i, int64_t o) {   // modes.py:509 with full.py:2385's normal
        const double cruise = p.speed_fraction[i] * p.max_vel[i];
        const double tau_ = (p.mass[i] * p.agility[i]) / p.friction;
        const double max_thrust = cruise / tau_;
        const double r = p.follow_range[i] + p.radius[i] + p.radius[o];
        const V pos = ld(p.pos, i), vel = ld(p.vel, i);
        const V opos = ld(p.pos, o), ovel = ld(p.vel, o);
        V to = sub(opos, pos);
        to = V{to.x + ovel.x * p.dt, to.y + ovel.y * p.dt, to.z + ovel.z * p.dt};
        double dist = length(to);
        if (dist > 0) {
            const double inv = 1.0 / dist;
            to = scl(to, inv);
        } else {
            to = V{0.0, 0.0, 1.0};
        }
        V normal;
        V ocr = cross(to, vel);
        double length2 = lensq(ocr);
        if (length2 > 1e-12) {
            normal = scl(ocr, 1.0 / std::sqrt(length2));
        } else if (!p.dynamical) {
            normal = precessing(i);
        } else {
            const F3 h = tcoord(F3{0, 0, 1}, mrot(rot_of(i)));
            ocr = cross(to, V{(double)h.x, (double)h.y, (double)h.z});
            length2 = lensq(ocr);
            normal = length2 <= 1e-12 ? precessing(i) : scl(ocr, 1.0 / std::sqrt(length2));
        }
        const V radial = normalized(cross(normal, to));
        const double spd = length(vel);
        const double max_speed = (cruise < spd) ? spd : cruise;
        double angle = (0.1 * (r - dist)) / max_speed;
        if (angle < -1) angle = -1.0;
        if (angle > 1) angle = 1.0;
        if (dist < 0.1) dist = 0.1;
        const double sq = std::sqrt(dist * max_thrust);
        const double est_v = (sq < max_speed) ? sq : max_speed;
        const double est_d = est_v * p.dt;
        V gp, gv;
        if (std::fabs(angle) < 1e-10) {
            const double t = est_d / dist;
            double st_, ct;
            lm::sincos(t, &st_, &ct);
            gp = V{to.x * (dist * (1.0 - ct)) + radial.x * (dist * st_), to.y * (dist * (1.0 - ct)) + radial.y * (dist * st_),
                   to.z * (dist * (1.0 - ct)) + radial.z * (dist * st_)};
            gv = V{radial.x * (ct * est_v) + to.x * (st_ * est_v), radial.y * (ct * est_v) + to.y * (st_ * est_v),
                   radial.z * (ct * est_v) + to.z * (st_ * est_v)};
        } else {
            const double factor = est_d * angle / dist / std::sqrt(angle * angle + 1);
            double t;
            if (factor < -0.999) t = lm::log(0.001) / angle;
            else if (std::fabs(factor) > 1e-10) t = lm::log(1 + factor) / angle;
            else t = factor / angle;
            const double dexp = dist * lm::exp(angle * t);
            double st_, ct;
            lm::sincos(t, &st_, &ct);
            gp = V{to.x * (dist - dexp * ct) + radial.x * (dexp * st_), to.y * (dist - dexp * ct) + radial.y * (dexp * st_),
                   to.z * (dist - dexp * ct) + radial.z * (dexp * st_)};
            gv = normalized(V{to.x * (-angle * ct + st_) + radial.x * (angle * st_ + ct),
                              to.y * (-angle * ct + st_) + radial.y * (angle * st_ + ct),
                              to.z * (-angle * ct + st_) + radial.z * (angle * st_ + ct)});
            gv = scl(gv, est_v);
        }
        const V g = add(pos, gp);
        st(p.goto_, i, g);
        gv = add(gv, ovel);
        return goto_thrust_follow(i, g, gv);
    }
    V orient(int64_t i, V a) {               // full.py:2459
        Turn t;
        t.max_ang_vel = ff(p.max_ang_vel, i);
        t.t_scale = t_scale(i);
        t.dt = p.dt;
        t.fdt = p.fdt;
        const F4 r0 = rot_of(i);
        const F3 w0 = w_of(i);
        const float accel = (float)length(a);
        const float max_accel = (p.ffriction * ff(p.speed_fraction, i) * ff(p.max_vel, i)) /
                                ((float)p.mass[i] * ff(p.agility, i));
        const F3 a32 = F3{(float)a.x, (float)a.y, (float)a.z};
        F3 torque{0, 0, 0};
        const bool thrust = accel > 1e-2 * max_accel;
        if (thrust) torque = goto_torque_breaks(t, r0, w0, a32);
        else if (warping(i)) {
            const V g = sub(ld(p.goto_, i), ld(p.pos, i));
            torque = goto_torque_breaks(t, r0, w0, F3{(float)g.x, (float)g.y, (float)g.z});
        }
        const float roll = goto_roll_breaks(t, r0, w0, torque);
        p.torque[3 * i] = torque.x;
        p.torque[3 * i + 1] = torque.y;
        p.torque[3 * i + 2] = torque.z;
        p.rot_roll[i] = roll;
        if (!thrust) return a;
        F4 rotation;
        F3 wdum;
        apply_torque(r0, w0, torque, roll, tau(i), p.fdt, &rotation, &wdum);
        const F3 heading = tcoord(F3{0, 0, 1}, mrot(rotation));
        const float cosangle = fmins(1.0f, f3dot(heading, a32) / accel);
        if (cosangle <= 0.0f) return V{0, 0, 0};
        const F3 h = f3mul(heading, cosangle * cosangle * accel);
        return V{h.x, h.y, h.z};
    }
    // EvolveMissile (full.py:2337; Ballpark.cpp:972): straight on toward mGoto while (time - launch) x tick is at most
    // 800 ms, then the lead point (the target's position plus its velocity times dist / maxVel, offset along the line
    // from it by followRange + both radii) at full thrust, never tapered
    V evolve_missile(int64_t i, int64_t o) {
        if ((p.clock[i] - p.effect_stamp[i]) * p.c->tick_ms <= 800) return goto_thrust(i, ld(p.goto_, i));
        const V op = ld(p.pos, o), ov = ld(p.vel, o);
        const V delta = sub(ld(p.pos, i), op);
        const double dist = length(delta);
        const double ct = dist / p.max_vel[i];
        V target = V{op.x + ov.x * ct, op.y + ov.y * ct, op.z + ov.z * ct};
        const double r = p.follow_range[i] + p.radius[i] + p.radius[o];
        if (dist == 0.0) {
            target = V{op.x + 1.0 * r, op.y + 0.0 * r, op.z + 0.0 * r};
        } else {
            const double inv = 1.0 / dist;
            target = V{target.x + delta.x * r * inv, target.y + delta.y * r * inv, target.z + delta.z * r * inv};
        }
        st(p.goto_, i, target);
        const double max_thrust = p.friction * p.speed_fraction[i] * p.max_vel[i] / (p.mass[i] * p.agility[i]);
        return scl(normalized(sub(target, ld(p.pos, i))), max_thrust);
    }
    // EvolveFormation (full.py:2359; Ballpark.cpp:1023): the leader's slot offset scaled to both radii plus its
    // length, turned by the leader's rotation as floats, at the leader's position; GotoThrust toward it
    V evolve_formation(int64_t i, int64_t o) {
        const int64_t fid = p.c->formation_id[o];
        if (fid < 0 || fid > p.c->n_formations - 1) return V{0, 0, 0};
        const int64_t slot = (int64_t)(int8_t)(uint8_t)(p.effect_stamp[i] & 0xFF);
        if (slot > p.c->formation_len[fid] - 1 || slot < 0) return V{0, 0, 0};
        const double* f = p.c->formations + (fid * p.c->max_slots + slot) * 3;
        const V offset = V{f[0], f[1], f[2]};
        double len = length(offset);
        if (len == 0.0) len = 1.0;
        const double k = p.radius[i] + p.radius[o] + len;
        const double inv = 1.0 / len;
        const F3 vec = F3{(float)(offset.x * k * inv), (float)(offset.y * k * inv), (float)(offset.z * k * inv)};
        const F3 rv = tcoord(vec, mrot(rot_of(o)));
        const V op = ld(p.pos, o);
        const V g = V{op.x + (double)rv.x, op.y + (double)rv.y, op.z + (double)rv.z};
        st(p.goto_, i, g);
        return goto_thrust(i, g);
    }
    // CollideTwoSpheres (Collision.cpp:108): 0 if touching, the earlier root in [0, 1], else -1
    static double spheres(V p0, V p1, V q0, V q1, double cr) {
        const V d = sub(p0, q0);
        const double d2 = lensq(d);
        if (d2 <= cr * cr) return 0.0;
        const V e = V{(p1.x - p0.x) - (q1.x - q0.x), (p1.y - p0.y) - (q1.y - q0.y), (p1.z - p0.z) - (q1.z - q0.z)};
        const double a = lensq(e);
        const double b = 2.0 * (d.x * e.x + d.y * e.y + d.z * e.z);
        const double c = d2 - cr * cr;
        if (a == 0.0 && b == 0.0) return -1.0;
        double det = b * b - 4.0 * a * c;
        if (det < 0.0) return -1.0;
        det = std::sqrt(det);
        const double s2 = ((-b - det) * 0.5) / a;
        return (s2 >= 0.0 && s2 <= 1.0) ? s2 : -1.0;
    }
    // Potential(missile, target, depth) (Ballpark.cpp:2789; space.py's _potential): the target ids appended
    int64_t potential(int64_t i, int64_t t, V pi, V pt, int depth) {
        const double m1 = p.mass[i] * p.agility[i];
        const bool other_free = p.free_[t] != 0;
        const double m2 = other_free ? p.mass[t] * p.agility[t] : 1.0e34;
        V p1 = pi, v1 = ld(p.vel, i), q1 = pt, w1 = ld(p.vel, t);
        integrate(&p1, &v1, ld(p.last_g, i), m1, p.time_factor[i]);
        integrate(&q1, &w1, ld(p.last_g, t), m2, p.time_factor[t]);
        const double cr = p.radius[i] + p.radius[t];
        const double s = spheres(pi, p1, pt, q1, cr);
        if (s == -1.0) return 0;
        if (s > 0.0) return 1;
        if (!other_free || depth >= 2) return 1;
        const V d = sub(pt, pi);
        const double d2 = lensq(d);
        const V normal = d2 == 0.0 ? V{p.ids[i] > p.ids[t] ? 1.0 : -1.0, 0.0, 0.0} : normalized(d);
        const double dist = (cr - std::sqrt(d2)) + 1.0;
        const double d1 = m2 / (m1 + m2) * dist, dd2 = m1 / (m1 + m2) * dist;
        const V pp = V{pi.x - normal.x * d1, pi.y - normal.y * d1, pi.z - normal.z * d1};
        const V qq = V{pt.x + normal.x * dd2, pt.y + normal.y * dd2, pt.z + normal.z * dd2};
        const int64_t inner = potential(i, t, pp, qq, depth + 1);
        const V rel = sub(ld(p.vel, i), ld(p.vel, t));
        if (lensq(rel) > 0.0001) return inner;
        return inner + 1;
    }
    // The gradient of a massive normal missile: its one candidate is its target in its bubble, less Gradient's skips
    int64_t missile_contacts(int64_t i) {
        const int64_t t = p.follow_ptr[i];
        if (!(live(i) && p.massive[i] && p.mode[i] == MISSILE && p.owner_id[i] >= 0 && t >= 0 && t < p.n &&
              p.c->bubble[i] == p.c->bubble[t]))
            return 0;
        const int64_t mt = p.mode[t], own = p.owner_id[i];
        if (p.ids[t] == own || (mt == MINIBALL && p.owner_id[t] == own) ||
            ((mt == MISSILE || mt == MUSHROOM) && p.ids[i] == p.owner_id[t]) ||
            (mt == MISSILE && p.ids[i] == p.follow_id[t]))
            return 0;
        return potential(i, t, ld(p.pos, i), ld(p.pos, t), 0);
    }
    // ---- the composed park: the partition's filing and the gradient (vec_composed.py; space.py:1631-1760) ----
    static constexpr int NUM_LEVELS = 8;
    static double level_width(int l) { return 7864320.0 / (double)(int64_t(1) << (2 * l)); }
    static int64_t level_grid(int l) { return int64_t(1) << (2 * l + 23); }
    // Ball::InsertInBoxes' level, key and side for row i at (pos, vel) with speed fraction sf (vec_collide.py:767-807);
    // a filing the reference refuses flags the row (FLAG_PARTITION)
    void file(int64_t i, V pos, V vel, double sf) {
        const double k = p.friction;
        double infl = p.radius[i];
        if (p.free_[i]) {
            const double m = p.mass[i] * p.agility[i];
            const double a = k * sf * p.max_vel[i] / m;
            const double speed = std::sqrt(lensq(vel));
            const double ma = m * a;
            infl = p.radius[i] + p.dt * ((ma - (ma - speed * k) * p.time_factor[i]) / k);
        }
        int level = -1;
        for (int l = 0; l < NUM_LEVELS; ++l)
            if (!(3.0 * infl > level_width(l))) ++level;
        if (level < 0) level = 0;
        const double w = level_width(level);
        const int64_t grid = level_grid(level);
        const double half = 0.5 * w * (double)grid, center = w * (double)grid * 0.5, fac = 1.0 / w;
        const double pa[3] = {pos.x, pos.y, pos.z};
        bool bad = level == 0 && p.radius[i] * 2.0 > level_width(0);
        p.x->level[i] = level;
        for (int q = 0; q < 3; ++q) {
            int64_t kq = to_i64((pa[q] + half) * fac);
            kq = kq < 0 ? 0 : (kq >= grid ? grid - 1 : kq);
            const double lo = (double)kq * w - center, hi = (double)(kq + 1) * w - center;
            const int64_t mq = (lo + infl) - pa[q] > 0.0 ? -1 : ((hi - infl) - pa[q] < 0.0 ? 1 : 0);
            p.x->key[3 * i + q] = kq;
            p.x->mod[3 * i + q] = mq;
            if (kq <= 0 || kq >= grid - 1 || kq + mq < 0 || kq + mq >= grid) bad = true;
        }
        if (bad) p.c->flags[i] |= 128;
    }
    // Whether a box of ball n is one of ball b's boxes, an ancestor of one or below one (vec_collide.py:809)
    bool related(int64_t b, int64_t n) const {
        const int64_t Lb = p.x->level[b], Ln = p.x->level[n];
        const int64_t sh = 2 * (Lb > Ln ? Lb - Ln : Ln - Lb);
        for (int q = 0; q < 3; ++q) {
            const int64_t kb = p.x->key[3 * b + q], mb = p.x->mod[3 * b + q];
            const int64_t kn = p.x->key[3 * n + q], mn = p.x->mod[3 * n + q];
            const int64_t bo[2] = {kb + std::min<int64_t>(mb, 0), kb + std::max<int64_t>(mb, 0)};
            const int64_t no[2] = {kn + std::min<int64_t>(mn, 0), kn + std::max<int64_t>(mn, 0)};
            const int64_t* fine = Ln <= Lb ? bo : no;
            const int64_t* coarse = Ln <= Lb ? no : bo;
            bool any = false;
            for (int u = 0; u < 2; ++u)
                for (int w = 0; w < 2; ++w) any = any || (fine[u] >> sh) == coarse[w];
            if (!any) return false;
        }
        return true;
    }
    // Ball n's first box's place in ball b's GetNearbyBalls walk (vec_collide.py:825): b's box (by key order) that
    // n's box relates to first, the part (an ancestor, below, the box itself) and the ancestor's distance or the box's
    // post-order code below b's level
    int64_t walk_key(int64_t b, int64_t n) const {
        const int64_t Lb = p.x->level[b], Ln = p.x->level[n];
        constexpr int64_t BASE = 65;
        int64_t span = 1;
        for (int l = 0; l < NUM_LEVELS - 1; ++l) span *= BASE;
        int64_t lo_b[3], hi_b[3], cb[3], Kn[3], Mn[3];
        for (int q = 0; q < 3; ++q) {
            const int64_t kb = p.x->key[3 * b + q], mb = p.x->mod[3 * b + q];
            lo_b[q] = kb + std::min<int64_t>(mb, 0);
            hi_b[q] = kb + std::max<int64_t>(mb, 0);
            cb[q] = mb != 0 ? 2 : 1;
            Kn[q] = p.x->key[3 * n + q];
            Mn[q] = p.x->mod[3 * n + q];
        }
        if (Ln <= Lb) {
            const int64_t up = 2 * (Lb - Ln);
            int64_t seg = 0;
            for (int q = 0; q < 3; ++q) {
                const int64_t v = lo_b[q] >> up;
                const int64_t idx = (v == Kn[q] || (Mn[q] != 0 && v == Kn[q] + Mn[q])) ? 0 : 1;
                seg = q == 0 ? idx : seg * cb[q] + idx;
            }
            return Ln < Lb ? seg * 3 * span + (Lb - Ln) : (seg * 3 + 2) * span;
        }
        const int64_t dn = 2 * (Ln - Lb);
        int64_t best = int64_t(1) << 62;
        for (int c = 0; c < 8; ++c) {
            int64_t box[3], jx[3];
            bool ok = true;
            for (int q = 0; q < 3; ++q) {
                const int64_t bit = (c >> (2 - q)) & 1;
                if (bit && Mn[q] == 0) ok = false;
                box[q] = Kn[q] + Mn[q] * bit;
                const int64_t anc = box[q] >> dn;
                const bool in0 = anc == lo_b[q], in1 = cb[q] == 2 && anc == hi_b[q];
                if (!in0 && !in1) ok = false;
                jx[q] = in0 ? 0 : 1;
            }
            if (!ok) continue;
            const int64_t seg = (jx[0] * cb[1] + jx[1]) * cb[2] + jx[2];
            int64_t code = 0, power = span;
            for (int lvl = 1; lvl < NUM_LEVELS; ++lvl) {
                power /= BASE;
                const int64_t sh = std::max<int64_t>(2 * (Ln - lvl), 0);
                int64_t digit = ((box[0] >> sh) & 3) * 16 + ((box[1] >> sh) & 3) * 4 + ((box[2] >> sh) & 3);
                if (lvl > Ln) digit = BASE - 1;
                if (lvl <= Lb) digit = 0;
                code += digit * power;
            }
            best = std::min(best, (seg * 3 + 1) * span + code);
        }
        return best;
    }
    struct Acc {
        V last_c;
        double last_collision;
        int64_t hits_n;
    };
    double gmass(int64_t i) const { return p.free_[i] ? p.mass[i] * p.agility[i] : 1.0e34; }
    // Potential(b, o, depth) (space.py:1663; Ballpark.cpp:2789) at the positions the recursion pushed, with the
    // composed park's end: a missile's response to its own target not kept (COL-711), the id appended either way
    void potential_c(int64_t b, int64_t o, V pb, V po, int depth, bool exempt, Acc& acc) {
        const double k = p.friction, dt = p.dt;
        const double cr = p.radius[b] + p.radius[o];
        const double m1 = gmass(b), m2 = gmass(o);
        const bool free2 = p.free_[o] != 0;
        const V v1 = ld(p.vel, b), v2 = ld(p.vel, o), g1 = ld(p.last_g, b), g2 = ld(p.last_g, o);
        const double tf1 = p.time_factor[b], tf2 = p.time_factor[o];
        V p1 = pb, w1 = v1, q1 = po, w2 = v2;
        integrate_for(&p1, &w1, g1, m1, tf1, dt);
        integrate_for(&q1, &w2, g2, m2, tf2, dt);
        const double sv = spheres(pb, p1, po, q1, cr);
        if (sv == -1.0) return;
        V a1;
        if (sv > 0.0) {                         // the impact: both to the time of impact, the reflection, the rest
            V pp = pb, vp = v1, qq = po, vq = v2;
            integrate_for(&pp, &vp, g1, m1, tf1, sv * dt);
            integrate_for(&qq, &vq, g2, m2, tf2, sv * dt);
            const V normal = normalized(sub(qq, pp));
            const double u1 = vp.x * normal.x + vp.y * normal.y + vp.z * normal.z;
            const double u2 = vq.x * normal.x + vq.y * normal.y + vq.z * normal.z;
            if (!free2) {
                vp = sub(vp, scl(normal, 2.0 * u1));
            } else {
                const double mm1 = p.mass[b], mm2 = p.mass[o];
                const double u1p = (mm1 * u1 - mm2 * u1 + 2.0 * mm2 * u2) / (mm1 + mm2);
                vp = add(vp, scl(normal, u1p - u1));
            }
            integrate_for(&pp, &vp, g1, m1, tf1, (1.0 - sv) * dt);
            const double inv_m = 1.0 / m1, inv_t = 1.0 / (tf1 - 1.0);
            const double ga[3] = {g1.x, g1.y, g1.z}, va[3] = {v1.x, v1.y, v1.z}, wa[3] = {vp.x, vp.y, vp.z};
            double r[3];
            for (int q = 0; q < 3; ++q) r[q] = -(ga[q] * -m1 + ga[q] * (tf1 * m1) - va[q] * tf1 * k + wa[q] * k) * inv_m * inv_t;
            a1 = V{r[0], r[1], r[2]};
        } else {                                // already overlapping: pushed apart, the recursion, the response
            const V d = sub(po, pb);
            const double d2 = lensq(d);
            const V normal = d2 == 0.0 ? V{p.ids[b] > p.ids[o] ? 1.0 : -1.0, 0.0, 0.0} : normalized(d);
            const double dist = (cr - std::sqrt(d2)) + 1.0;
            const double d1 = m2 / (m1 + m2) * dist, dd2 = m1 / (m1 + m2) * dist;
            if (depth < 2 && free2) {
                potential_c(b, o, sub(pb, scl(normal, d1)), add(po, scl(normal, dd2)), depth + 1, exempt, acc);
                if (m2 / m1 > 25.0) acc.last_c = scl(normalized(acc.last_c), dist);
                if (lensq(sub(v1, v2)) > 0.0001) return;
            }
            const double normal_comp = g1.x * normal.x + g1.y * normal.y + g1.z * normal.z;
            const double tmp = 1.0 / (m1 + dt * k);
            const double c = -d1 / (dt * tmp * m1);
            a1 = sub(scl(sub(scl(normal, c), v1), 1.0 / dt), scl(normal, normal_comp));
        }
        if (!exempt && sv >= acc.last_collision) {
            const V lc = scl(a1, 0.85);
            if (sv == acc.last_collision) {
                if (lensq(lc) > lensq(acc.last_c)) acc.last_c = lc;
            } else {
                acc.last_c = lc;
                acc.last_collision = sv;
            }
        }
        p.x->hits[b * p.x->hit_cap + std::min(acc.hits_n, p.x->hit_cap - 1)] = p.ids[o];
        ++acc.hits_n;
    }
    // Gradient of responder b at its turn (Ballpark.cpp:2745): the others as they stand now (a warper that dropped out
    // at an earlier turn is massive again, at its drop-out point), GetNearbyBalls' candidates less Gradient's skips,
    // those Potential's depth 0 does not rule out, in the walk's order then id (a normal missile: its target only)
    void gradient(int64_t b, const std::vector<int64_t>& rows) {
        const bool ex_b = p.c->exists[b] && !p.moribund[b];
        const bool missile_b = ex_b && p.mode[b] == MISSILE, defender = missile_b && p.owner_id[b] < 0;
        const double k = p.friction;
        V eb = ld(p.pos, b), wb = ld(p.vel, b);
        integrate_for(&eb, &wb, ld(p.last_g, b), gmass(b), p.time_factor[b], p.dt);
        std::vector<std::pair<std::pair<int64_t, int64_t>, int64_t>> cand;
        for (int64_t o : rows) {
            if (o == b) continue;
            const bool ex = p.c->exists[o] && !p.moribund[o];
            const bool missile_o = ex && p.mode[o] == MISSILE;
            bool pair, first = false;
            if (missile_b && !defender) {
                pair = o == p.follow_ptr[b] && ex && p.c->bubble[o] == p.c->bubble[b];
                first = pair;
            } else {
                const bool nearby = ex && p.massive[o] && p.c->cloaked[o] == 0 && related(b, o);
                pair = defender ? nearby : nearby && !missile_o;
            }
            if (!pair) continue;
            const int64_t mo = p.mode[o];
            if ((missile_b && (p.ids[o] == p.owner_id[b] || (mo == MINIBALL && p.owner_id[o] == p.owner_id[b]))) ||
                ((mo == MISSILE || mo == MUSHROOM) && p.ids[b] == p.owner_id[o]) ||
                (mo == MISSILE && p.ids[b] == p.follow_id[o]))
                continue;
            V eo = ld(p.pos, o), wo = ld(p.vel, o);
            integrate_for(&eo, &wo, ld(p.last_g, o), gmass(o), p.time_factor[o], p.dt);
            if (spheres(ld(p.pos, b), eb, ld(p.pos, o), eo, p.radius[b] + p.radius[o]) == -1.0) continue;
            cand.push_back({{first ? 0 : walk_key(b, o), p.ids[o]}, o});
        }
        std::sort(cand.begin(), cand.end());
        Acc acc{V{0, 0, 0}, -1.0, 0};
        for (const auto& c : cand) {
            const int64_t o = c.second;
            potential_c(b, o, ld(p.pos, b), ld(p.pos, o), 0, missile_b && p.ids[o] == p.follow_id[b], acc);
        }
        (void)k;
        st(p.x->last_c, b, acc.last_c);
        p.last_collision[b] = acc.last_collision;
        p.c->hits_n[b] = acc.hits_n;
    }
    // EvolveBehaviorForBall (modes.py:359, full.py:2416)
    void behaviour(int64_t i, const std::vector<int64_t>& rows) {
        st(p.last_g, i, V{0, 0, 0});
        V a{0, 0, 0};
        const int64_t m = p.mode[i];
        const int64_t o = p.follow_ptr[i];
        const bool has_target = o >= 0 && o < p.n;
        if (m == WARP) {
            if (warping(i)) {
                a = V{0, 0, 0};
            } else if (aligned(i)) {
                real_warp(i, rows);
            } else {
                p.effect_stamp[i] -= 1;
                a = goto_thrust(i, ld(p.goto_, i));
            }
        } else if (m == GOTO) {
            a = goto_thrust(i, ld(p.goto_, i));
        } else if ((m == FOLLOW || m == ORBIT || m == MISSILE || m == FORMATION) && !has_target) {
            a = V{0, 0, 0};
        } else if (m == FOLLOW) {
            a = evolve_follow(i, o);
        } else if (m == ORBIT) {
            a = p.new_orbit ? evolve_new_orbit(i, o) : evolve_old_orbit(i, o);
        } else if (m == MISSILE) {
            a = evolve_missile(i, o);
        } else if (m == FORMATION) {
            a = evolve_formation(i, o);
        } else if (m == STOP) {
            if (!p.dynamical) p.vel[3 * i + 1] = (p.vel[3 * i + 1] - 0.07 * p.vel[3 * i + 1]) * STOP_DAMP;
        }
        if (p.dynamical && !disabled(i)) a = orient(i, a);
        st(p.last_g, i, a);
    }
    // Ballpark::Integrate over one tick (ref.py:354)
    void integrate(V* pp, V* vp, V a, double m, double tfac) { integrate_for(pp, vp, a, m, tfac, p.dt); }
    // Ballpark::Integrate over t seconds: the cached decay factor for a whole tick, else glibc's exp(-k t / m)
    void integrate_for(V* pp, V* vp, V a, double m, double tfac, double t) {
        const double k = p.friction;
        if (t == 0.0) return;
        if (t != p.dt) tfac = lm::exp(-k / m * t);
        const double k2 = k * k, ook2 = 1.0 / k2, ook = 1.0 / k;
        const V pv = *pp, v = *vp;
        V pn;
        if (k < 1e-10 * m * t) {
            const double inv_m = 1.0 / m;
            pn = V{(m * (a.x * (-k * t) + k * (a.x * t + v.x * k * inv_m * t)) + pv.x * k2) * ook2,
                   (m * (a.y * (-k * t) + k * (a.y * t + v.y * k * inv_m * t)) + pv.y * k2) * ook2,
                   (m * (a.z * (-k * t) + k * (a.z * t + v.z * k * inv_m * t)) + pv.z * k2) * ook2};
        } else {
            pn = V{(m * (m * a.x * (tfac - 1.0) + k * (a.x * t + v.x - tfac * v.x)) + pv.x * k2) * ook2,
                   (m * (m * a.y * (tfac - 1.0) + k * (a.y * t + v.y - tfac * v.y)) + pv.y * k2) * ook2,
                   (m * (m * a.z * (tfac - 1.0) + k * (a.z * t + v.z - tfac * v.z)) + pv.z * k2) * ook2};
        }
        *vp = V{(m * a.x - (m * a.x - v.x * k) * tfac) * ook, (m * a.y - (m * a.y - v.y * k) * tfac) * ook,
                (m * a.z - (m * a.z - v.z * k) * tfac) * ook};
        *pp = pn;
    }
    // WarpDistance (modes.py:618): the new position and velocity; true when the ball drops out
    bool warp_distance(int64_t i, V* pp, V* vp, double t) {
        const double wf = (double)p.owner_id[i];
        const double wd = p.last_collision[i];
        double s = wf * WARP_AU_PER_S * AU;
        const double acc = wf * WARP_ACC;
        const double d0 = wf * WARP_DEC;
        const double dec = (2.0 < d0) ? 2.0 : d0;
        const double cap = (wd + 1) * acc * dec / (acc + dec);
        s = (cap < s) ? cap : s;
        const double t_a = lm::log(s / acc) / acc;
        const double t_c = (wd / s) - (1.0 / acc) - (1.0 / dec) + (1.0 / s);
        const double t_d = lm::log(s / dec) / dec;
        const double d_a = s / acc, d_c = s * t_c, d_d = s / dec - 1;
        const V g = ld(p.goto_, i);
        const V d = normalized(sub(g, *pp));
        if (t < t_a) {
            double speed = acc * lm::exp(acc * t);
            const double cur = length(*vp);
            if (cur > speed) speed = cur;
            *vp = scl(d, speed);
            const double x = lm::exp(acc * t);
            const double rest = d_a + d_c + d_d - x;
            *pp = sub(g, scl(d, rest));
            return false;
        }
        if ((t - t_a) < t_c) {
            *vp = scl(d, s);
            const double x = s * (t - t_a) + d_a;
            *pp = sub(g, scl(d, d_a + d_c + d_d - x));
            return false;
        }
        if ((t - t_c - t_a) < (t_d + 1)) {
            const double e = lm::exp(-dec * (t - t_c - t_a));
            const double speed = s * e;
            *vp = scl(d, speed);
            const double x = s / dec - (s / dec) * e + d_a + d_c;
            *pp = sub(g, scl(d, d_a + d_c + d_d - x));
            const double half = p.max_vel[i] / 2.0;
            return speed < ((100.0 < half) ? 100.0 : half);
        }
        *pp = g;
        *vp = V{0, 0, 0};
        return true;
    }

    void world(const std::vector<int64_t>& rows) {
        // (1) behaviours, ascending id
        if (p.x)                                // the composed park: the live balls' responses and lists cleared
            for (int64_t i : rows)
                if (live(i)) {
                    st(p.x->last_c, i, V{0, 0, 0});
                    for (int64_t q = 0; q < p.x->hit_cap; ++q) p.x->hits[i * p.x->hit_cap + q] = -1;
                    p.c->hits_n[i] = 0;
                }
        for (int64_t i : rows)
            if (live(i)) behaviour(i, rows);
        if (p.c && !p.x)                        // the missiles' contacts with their targets, after every behaviour
            for (int64_t i : rows) p.c->hits_n[i] = missile_contacts(i);
        // (3) end-of-tick states into temporaries, and the rotation a tick on
        const size_t k = rows.size();
        std::vector<V> np(k), nv(k);
        std::vector<F4> nrot(k);
        std::vector<F3> nw(k);
        for (size_t j = 0; j < k; ++j) {
            const int64_t i = rows[j];
            if (!live(i)) continue;
            if (p.x) {                          // the gradient at its turn (a massive ball), then its end state
                if (p.massive[i]) gradient(i, rows);
            } else if (p.massive[i]) {
                p.last_collision[i] = -1.0;
                if (p.h && p.h->gradient) p.h->gradient(p.h->world, i);
            }
            V pv = ld(p.pos, i), vv = ld(p.vel, i);
            const V lg = ld(p.last_g, i);
            const V lc = p.x ? ld(p.x->last_c, i) : (p.h && p.h->last_c) ? ld(p.h->last_c, i) : V{0.0, 0.0, 0.0};
            const V a = V{lg.x + lc.x, lg.y + lc.y, lg.z + lc.z};
            if (warping(i)) {
                const bool drop = warp_distance(i, &pv, &vv, (double)(p.clock[i] - p.effect_stamp[i]) * p.dt);
                if (drop) {                     // massive and sensing again, Stop (a warper follows nothing)
                    p.massive[i] = 1;
                    p.sensor[i] = 1;
                    stop_ball(i);
                    st(p.pos, i, pv);           // TRV-714: the drop-out point becomes the old state
                    st(p.vel, i, vv);
                    if (p.x && !(lensq(vv) >= 0.1)) file(i, pv, vv, p.speed_fraction[i]);   // re-filed at rest
                    if (p.h && p.h->drop_out && !(lensq(vv) >= 0.1)) p.h->drop_out(p.h->world, i);
                    integrate(&pv, &vv, a, p.mass[i] * p.agility[i], p.time_factor[i]);
                }
            } else {
                integrate(&pv, &vv, a, p.mass[i] * p.agility[i], p.time_factor[i]);
            }
            np[j] = pv;
            nv[j] = vv;
            if (p.dynamical && disabled(i)) {  // phase 3 leaves a disabled missile's mOldRot as it was
                nrot[j] = F4{ff(p.old_rot, 4 * i), ff(p.old_rot, 4 * i + 1), ff(p.old_rot, 4 * i + 2),
                             ff(p.old_rot, 4 * i + 3)};
                nw[j] = F3{ff(p.old_ang_vel, 3 * i), ff(p.old_ang_vel, 3 * i + 1), ff(p.old_ang_vel, 3 * i + 2)};
            } else if (p.dynamical) {
                const F3 tq = F3{ff(p.torque, 3 * i), ff(p.torque, 3 * i + 1), ff(p.torque, 3 * i + 2)};
                apply_torque(rot_of(i), w_of(i), tq, ff(p.rot_roll, i), tau(i), p.fdt, &nrot[j], &nw[j]);
            }
        }
        // (4) the commit; PetrifyTroll of the trolls due; the clock
        for (size_t j = 0; j < k; ++j) {
            const int64_t i = rows[j];
            if (p.c) {
                p.c->ev_n[i] = 0;
                p.c->ev_self[i] = 0;
            }
            if (live(i)) {
                const V before = ld(p.pos, i);
                st(p.old_pos, i, ld(p.pos, i));
                st(p.old_vel, i, ld(p.vel, i));
                st(p.pos, i, np[j]);
                st(p.vel, i, nv[j]);
                if (p.dynamical) {
                    const F4 r0 = rot_of(i);
                    const F3 w0 = w_of(i);
                    const F4 r1 = nrot[j];
                    const F3 w1 = nw[j];
                    const bool rot_ok = std::isfinite(qlensq(r1));
                    const bool w_ok = std::isfinite(f3dot(w1, w1));
                    const F4 rn = rot_ok ? r1 : r0, ro = rot_ok ? r0 : r1;
                    const F3 wn = w_ok ? w1 : w0, wo = w_ok ? w0 : w1;
                    const float rr[4] = {rn.x, rn.y, rn.z, rn.w}, orr[4] = {ro.x, ro.y, ro.z, ro.w};
                    for (int c = 0; c < 4; ++c) {
                        p.rot[4 * i + c] = rr[c];
                        p.old_rot[4 * i + c] = orr[c];
                    }
                    const float ww[3] = {wn.x, wn.y, wn.z}, ow[3] = {wo.x, wo.y, wo.z};
                    for (int c = 0; c < 3; ++c) {
                        p.ang_vel[3 * i + c] = ww[c];
                        p.old_ang_vel[3 * i + c] = ow[c];
                    }
                    if (disabled(i))            // SnapOrientation of a disabled missile (phase 4)
                        snap_one(p.vel + 3 * i, p.rot + 4 * i, p.old_rot + 4 * i, p.ang_vel + 3 * i,
                                 p.old_ang_vel + 3 * i);
                }
                const bool moved = !(lensq(sub(ld(p.pos, i), before)) < 0.1);
                if (p.x && moved) file(i, ld(p.pos, i), ld(p.vel, i), p.speed_fraction[i]);   // re-filed
                if (p.c && p.mode[i] == MISSILE && moved) {
                    // DispatchCollisions (Ballpark.cpp:600-639): the target ids, then on the master a collision with
                    // itself when its owner is gone, cloaked or in another bubble
                    p.c->ev_n[i] = p.c->hits_n[i];
                    if (p.c->master) {
                        const int64_t o = p.c->owner_ptr[i];
                        const bool gone = o < 0 || o >= p.n || !p.c->exists[o];
                        p.c->ev_self[i] = (gone || (p.c->bubble[o] != p.c->bubble[i] && p.c->bubble[i] != -1) ||
                                           p.c->cloaked[o] != 0) ? 1 : 0;
                    }
                    if (p.x && p.c->ev_self[i]) {   // the master's self-collision joins the missile's list
                        p.x->hits[i * p.x->hit_cap + std::min(p.c->hits_n[i], p.x->hit_cap - 1)] = p.ids[i];
                        p.c->hits_n[i] += 1;
                    }
                }
                if (p.mode[i] == TROLL && !(p.effect_stamp[i] > p.clock[i])) {   // TrollReady, PetrifyTroll
                    st(p.vel, i, V{0, 0, 0});
                    st(p.old_vel, i, V{0, 0, 0});
                    st(p.last_g, i, V{0, 0, 0});
                    p.free_[i] = 0;
                    p.interactive[i] = 0;
                    p.mode[i] = RIGID;
                }
            }
        }
        for (int64_t i : rows) p.clock[i] += 1;
    }

    // The worlds in world order, each its rows in ascending id; `threads` workers take disjoint worlds (a world's
    // tick reads and writes its own rows only).
    void run(int threads) {
        std::vector<int64_t> order((size_t)p.n);
        for (int64_t i = 0; i < p.n; ++i) order[(size_t)i] = i;
        std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
            return p.world[a] != p.world[b] ? p.world[a] < p.world[b] : p.ids[a] < p.ids[b];
        });
        std::vector<size_t> starts;
        size_t s = 0;
        while (s < order.size()) {
            starts.push_back(s);
            size_t e = s + 1;
            while (e < order.size() && p.world[order[e]] == p.world[order[s]]) ++e;
            s = e;
        }
        starts.push_back(order.size());
        const size_t worlds = starts.size() - 1;
        auto work = [&](size_t w0, size_t w1) {
            for (size_t w = w0; w < w1; ++w)
                world(std::vector<int64_t>(order.begin() + starts[w], order.begin() + starts[w + 1]));
        };
        if (threads <= 1 || worlds < 2) {
            work(0, worlds);
            return;
        }
        const size_t t = std::min((size_t)threads, worlds);
        std::vector<std::thread> pool;
        for (size_t k = 0; k < t; ++k) pool.emplace_back(work, worlds * k / t, worlds * (k + 1) / t);
        for (auto& th : pool) th.join();
    }
};

}  // namespace

extern "C" {

// The oracle's park: oracle/flight_state.h.

// One tick of every world in place, the worlds shared among `threads` host threads. Returns 0.
// The combat park's extra state (the Combat structure above, field for field).
struct OracleCombat {
    uint8_t* exists;
    int64_t *formation_id, *formation_slots, *owner_ptr, *hits_n, *ev_n;
    uint8_t* ev_self;
    int64_t *bubble, *cloaked, *flags;
    const double* formations;
    const int64_t* formation_len;
    int64_t n_formations, max_slots, tick_ms;
    int32_t do_missiles_off, master;
};

// One tick of every world of a combat park in place (dynamical orientation on), `threads` host threads. Returns 0.
int oracle_combat_tick_mt(const OracleFlight* s, const OracleCombat* c, int threads);

// The composed park's extra state (the Composed structure above, field for field).
struct OracleComposed {
    double* last_c;
    int64_t *level, *key, *mod, *hits;
    int64_t hit_cap;
};

// One tick of every world of a composed park in place (dynamical orientation on), `threads` host threads. Returns 0.
int oracle_composed_tick_mt(const OracleFlight* s, const OracleCombat* c, const OracleComposed* x, int threads);

// The filing of the rows with mask[i] != 0 from their state or the given pos, vel ([n][3]) and sf ([n]) (null for the
// row's own). Returns 0.
int oracle_composed_file(const OracleFlight* s, const OracleCombat* c, const OracleComposed* x, const uint8_t* mask,
                         const double* pos, const double* vel, const double* sf);

static Park park_of(const OracleFlight* s);

int oracle_flight_tick_mt(const OracleFlight* s, int threads) {
    Park p = park_of(s);
    Tick(p).run(threads);
    return 0;
}

int oracle_flight_tick_hooked(const OracleFlight* s, const OracleTickHooks* h) {
    Park p = park_of(s);
    p.h = h;
    Tick(p).run(1);
    return 0;
}

static Combat combat_of(const OracleCombat* c);

int oracle_combat_tick_mt(const OracleFlight* s, const OracleCombat* c, int threads) {
    Park p = park_of(s);
    Combat cx = combat_of(c);
    p.c = &cx;
    Tick(p).run(threads);
    return 0;
}

int oracle_composed_tick_mt(const OracleFlight* s, const OracleCombat* c, const OracleComposed* x, int threads) {
    Park p = park_of(s);
    Combat cx = combat_of(c);
    Composed xx{x->last_c, x->level, x->key, x->mod, x->hits, x->hit_cap};
    p.c = &cx;
    p.x = &xx;
    Tick(p).run(threads);
    return 0;
}

int oracle_composed_file(const OracleFlight* s, const OracleCombat* c, const OracleComposed* x, const uint8_t* mask,
                         const double* pos, const double* vel, const double* sf) {
    Park p = park_of(s);
    Combat cx = combat_of(c);
    Composed xx{x->last_c, x->level, x->key, x->mod, x->hits, x->hit_cap};
    p.c = &cx;
    p.x = &xx;
    Tick t(p);
    for (int64_t i = 0; i < p.n; ++i) {
        if (!mask[i]) continue;
        const V pv = ld(pos ? pos : p.pos, i), vv = ld(vel ? vel : p.vel, i);
        t.file(i, pv, vv, sf ? sf[i] : p.speed_fraction[i]);
    }
    return 0;
}

static Combat combat_of(const OracleCombat* c) {
    Combat cx;
    cx.exists = c->exists; cx.formation_id = c->formation_id; cx.formation_slots = c->formation_slots;
    cx.owner_ptr = c->owner_ptr; cx.hits_n = c->hits_n; cx.ev_n = c->ev_n; cx.ev_self = c->ev_self;
    cx.bubble = c->bubble; cx.cloaked = c->cloaked; cx.flags = c->flags; cx.formations = c->formations;
    cx.formation_len = c->formation_len; cx.n_formations = c->n_formations; cx.max_slots = c->max_slots;
    cx.tick_ms = c->tick_ms; cx.do_missiles_off = c->do_missiles_off; cx.master = c->master;
    return cx;
}

static Park park_of(const OracleFlight* s) {
    Park p;
    p.n = s->n;
    p.friction = s->friction;
    p.dt = s->dt;
    p.ffriction = s->ffriction;
    p.fdt = s->fdt;
    p.new_orbit = s->new_orbit;
    p.dynamical = s->dynamical;
    p.pos = s->pos; p.vel = s->vel; p.old_pos = s->old_pos; p.old_vel = s->old_vel; p.goto_ = s->goto_;
    p.last_g = s->last_g; p.mass = s->mass; p.time_factor = s->time_factor; p.last_collision = s->last_collision;
    p.radius = s->radius; p.max_vel = s->max_vel; p.agility = s->agility; p.speed_fraction = s->speed_fraction;
    p.follow_range = s->follow_range; p.max_ang_vel = s->max_ang_vel; p.rot_agility = s->rot_agility;
    p.rot_roll = s->rot_roll; p.rot = s->rot; p.old_rot = s->old_rot; p.ang_vel = s->ang_vel;
    p.old_ang_vel = s->old_ang_vel; p.torque = s->torque; p.ids = s->ids; p.world = s->world; p.mode = s->mode;
    p.effect_stamp = s->effect_stamp; p.follow_id = s->follow_id; p.owner_id = s->owner_id;
    p.follow_ptr = s->follow_ptr; p.clock = s->clock; p.free_ = s->free_; p.moribund = s->moribund;
    p.massive = s->massive; p.interactive = s->interactive; p.sensor = s->sensor;
    return p;
}

// One tick of every world in place, on the calling thread. Returns 0.
int oracle_flight_tick(const OracleFlight* s) { return oracle_flight_tick_mt(s, 1); }


}  // extern "C"

namespace {
// Ball::SnapOrientation (full.py:2092; vec_orient.py:556): turned to the velocity and rolled upright, the rotation
// stopped; at a speed of 1e-6 m/s or less nothing changes.
void snap_one(const double* v, double* rot, double* old_rot, double* w, double* old_w) {
    const double l2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (!(l2 > 1e-12)) return;
    const F3 d = F3{(float)v[0], (float)v[1], (float)v[2]};
    const float len_dir = f3len(d);
    F4 r;
    if (len_dir < 1e-12) {
        r = F4{0, 0, 0, 1};
    } else {
        const F3 vec = f3cross(F3{0, 0, 1}, d);
        const float angle = lm::acosf(fmaxs(-1.0f, fmins(1.0f, d.z / len_dir)));
        r = qrot(vec, angle);
        const F3 up = tcoord(F3{0, 1, 0}, mrot(qconj(r)));
        const float up_roll = up.z < (float)0.99 ? lm::atan2f(-up.x, up.y) : 0.0f;
        const F3 heading = tcoord(F3{0, 0, 1}, mrot(r));
        r = qmul(r, qrot(heading, up_roll));
    }
    const float rr[4] = {r.x, r.y, r.z, r.w};
    for (int c = 0; c < 4; ++c) rot[c] = old_rot[c] = rr[c];
    for (int c = 0; c < 3; ++c) w[c] = old_w[c] = 0.0;
}

// RotationQuaternion(axis, angle) and its product, for a new ball's mOldRot (vec_modes.py:261-263)
void q_rot_mul(const double* rot, const double* axis, double angle, double* out) {
    const F4 q = F4{(float)rot[0], (float)rot[1], (float)rot[2], (float)rot[3]};
    const F4 b = qrot(F3{(float)axis[0], (float)axis[1], (float)axis[2]}, (float)angle);
    const F4 m = qmul(q, b);
    out[0] = m.x;
    out[1] = m.y;
    out[2] = m.z;
    out[3] = m.w;
}
}  // namespace

extern "C" {

// SnapOrientation of the rows in mask ([n] bytes), in place.
int oracle_snap(int64_t n, const uint8_t* mask, const double* vel, double* rot, double* old_rot, double* ang_vel,
                double* old_ang_vel) {
    for (int64_t i = 0; i < n; ++i)
        if (mask[i]) snap_one(vel + 3 * i, rot + 4 * i, old_rot + 4 * i, ang_vel + 3 * i, old_ang_vel + 3 * i);
    return 0;
}

// out[i] = rot[i] x RotationQuaternion(axis[i], angle[i]) for n rows ([n, 4], [n, 3], [n])
int oracle_q_rot_mul(int64_t n, const double* rot, const double* axis, const double* angle, double* out) {
    for (int64_t i = 0; i < n; ++i) q_rot_mul(rot + 4 * i, axis + 3 * i, angle[i], out + 4 * i);
    return 0;
}

}  // extern "C"
