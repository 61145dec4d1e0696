// SPDX-License-Identifier: MIT
// The collision park's tick on sm_100a: the gradient method on spheres, behind include/ebb.h's ebb_collide_* entry
// points.
//
// A tick of Destiny's Evolve with collisions (TIME-706/707; exact_ballpark/vec_collide.py, evolve :990): every free
// ball's behaviour (GOTO's thrust or STOP's damping; mLastC and the collision list cleared), then for every free
// massive ball Gradient (space.py:1650): Potential (space.py:1663) with each collision candidate in the order
// Partition::GetNearbyBalls walks them, recursing on overlaps; then the commit of every free ball (integrated with
// mLastG + mLastC) and the re-filing in the partition of the balls that moved at least sqrt(0.1) m.
//
// One fused kernel: a thread block holds whole worlds (128 / N of them, one thread a slot), so the phases meet at
// block barriers: behaviours, each ball's end-of-tick prediction into shared memory (depth 0 of every Potential
// reads it), the gradient (one thread a responder: its candidates, their walk-order keys, the active ones sorted, then
// Potential on each in turn with the recursion unrolled by depth), then the commit and filing. A ball's gradient reads
// the others' start-of-tick state only, as Destiny's does (the end states are committed after every Gradient).
//
// Exactness: every double operation a single correctly rounded IEEE operation in the reference's order (ebb_arith),
// glibc's exp (ebb_libm) for integrations over part of a tick, aarch64's int64 conversion for the partition keys.
#include <cuda_runtime.h>

#include "../../include/ebb.h"
#include "ebb_arith.cuh"
#include "ebb_libm.cuh"

namespace ebb {
namespace collide {

constexpr int NUM_LEVELS = 8;
constexpr double BIG_BOX = 7864320.0;                 // (1 << 2 NUM_LEVELS) x 480 m x 0.25 (space.py:71)
constexpr int64_t CODE_BASE = 65;                      // a post-order digit: 0..63 a child box, 64 past the box's level
constexpr int64_t NOT_A_CANDIDATE = int64_t(1) << 62;
constexpr double LIGHT_BALL_RATIO = 25.0;
constexpr double RESPONSE_SCALE = 0.85;
constexpr double STOP_DAMP = 0.9345794392523364485981308411215;
constexpr double FIXED_MASS = 1.0e34;
constexpr int64_t GOTO = 0, STOP = 2;

struct V {
    double x, y, z;
};
__device__ __forceinline__ V vsub(V a, V b) { return V{dsub(a.x, b.x), dsub(a.y, b.y), dsub(a.z, b.z)}; }
__device__ __forceinline__ V vadd(V a, V b) { return V{dadd(a.x, b.x), dadd(a.y, b.y), dadd(a.z, b.z)}; }
__device__ __forceinline__ V vmul(V a, double c) { return V{dmul(a.x, c), dmul(a.y, c), dmul(a.z, c)}; }
__device__ __forceinline__ double vdot(V a, V b) { return dadd(dadd(dmul(a.x, b.x), dmul(a.y, b.y)), dmul(a.z, b.z)); }
// Vector3d::Normalize: times the reciprocal of the length; a zero vector as it is
__device__ __forceinline__ V vnorm(V v) {
    const double n = dsqrt(vdot(v, v));
    if (n == 0.0) return v;
    return vmul(v, ddiv(1.0, n));
}
__device__ __forceinline__ V ldv(const double* p, int64_t i) { return V{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ __forceinline__ void stv(double* p, int64_t i, V v) {
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}

// The partition's level widths (exact: BIG_BOX / 4^level) and grid sizes (1 << (2 level + 23))
__device__ __forceinline__ double level_width(int l) { return ddiv(BIG_BOX, i2d(int64_t(1) << (2 * l))); }
__device__ __forceinline__ int64_t level_grid(int l) { return int64_t(1) << (2 * l + 23); }

// Ballpark::Integrate (space.py:1609; vec_collide.py:903-932): nothing for t = 0, the cached factor for t = dt, else
// glibc's exp of (-k / m) t; the Taylor form when k < 1e-10 m t
__device__ __forceinline__ void integrate(V& p, V& v, V a, double m, double k, double tf, double t, double dt) {
    if (t == 0.0) return;
    if (t != dt) tf = lm::exp(dmul(ddiv(dneg(k), m), t));
    const double k2 = dmul(k, k), ook2 = ddiv(1.0, k2), ook = ddiv(1.0, k);
    const double pa[3] = {p.x, p.y, p.z}, va[3] = {v.x, v.y, v.z}, aa[3] = {a.x, a.y, a.z};
    double pn[3], vn[3];
    if (k < dmul(dmul(1e-10, m), t)) {
        const double inv_m = ddiv(1.0, m), kt = dmul(dneg(k), t);
        for (int q = 0; q < 3; ++q) {
            const double in = dadd(dmul(aa[q], t), dmul(dmul(dmul(va[q], k), inv_m), t));
            pn[q] = dmul(dadd(dmul(m, dadd(dmul(aa[q], kt), dmul(k, in))), dmul(pa[q], k2)), ook2);
        }
    } else {
        const double tf1 = dsub(tf, 1.0);
        for (int q = 0; q < 3; ++q) {
            const double in = dsub(dadd(dmul(aa[q], t), va[q]), dmul(tf, va[q]));
            pn[q] = dmul(dadd(dmul(m, dadd(dmul(dmul(m, aa[q]), tf1), dmul(k, in))), dmul(pa[q], k2)), ook2);
        }
    }
    for (int q = 0; q < 3; ++q) {
        const double ma = dmul(m, aa[q]);
        vn[q] = dmul(dsub(ma, dmul(dsub(ma, dmul(va[q], k)), tf)), ook);
    }
    p = V{pn[0], pn[1], pn[2]};
    v = V{vn[0], vn[1], vn[2]};
}

// CollideTwoSpheres (Collision.cpp:108; space.py:1631): 0 if already touching, the earlier root in [0, 1], else -1
__device__ __forceinline__ double collide_two_spheres(V p0, V p1, V q0, V q1, double cr) {
    const V p0q0 = vsub(p0, q0);
    const double p0q0_2 = vdot(p0q0, p0q0), cr2 = dmul(cr, cr);
    if (p0q0_2 <= cr2) return 0.0;
    const V dpq = vsub(vsub(p1, p0), vsub(q1, q0));
    const double a = vdot(dpq, dpq), b = dmul(2.0, vdot(p0q0, dpq)), c = dsub(p0q0_2, cr2);
    if (a == 0.0 && b == 0.0) return -1.0;
    const double det = dsub(dmul(b, b), dmul(dmul(4.0, a), c));
    if (det < 0.0) return -1.0;
    const double s2 = ddiv(dmul(dsub(dneg(b), dsqrt(det)), 0.5), a);
    return (s2 >= 0.0 && s2 <= 1.0) ? s2 : -1.0;
}

// A responder's running state through its Gradient: mLastC, mLastCollision, the collision list and the impact record
struct Acc {
    V last_c;
    double last_collision;
    int64_t hits_n, imp_n;
};

struct World {
    const EbbCollideState* s;
    int64_t base;                 // the world's first slot
    const V* ends;                // each slot's end-of-tick prediction (shared memory)
};

// Potential (Ballpark.cpp:2789; space.py:1663) of responder slot b with slot o at recursion depth D, the positions
// as the recursion has pushed them; its updates of mLastC, mLastCollision, the collision list and the impact record
template <int D>
__device__ __forceinline__ void potential(const World& W, int b, int o, V me_pos, V o_pos, Acc& acc) {
    const EbbCollideState& s = *W.s;
    const int64_t ib = W.base + b, io = W.base + o;
    const double k = s.friction, dt = s.dt;
    const double cr = dadd(s.radius[ib], s.radius[io]);
    const double m1 = dmul(s.mass[ib], s.agility[ib]);                     // the responder is free
    const bool free2 = s.free_[io] != 0;
    const double m2 = free2 ? dmul(s.mass[io], s.agility[io]) : FIXED_MASS;
    const V v1 = ldv(s.vel, ib), v2 = ldv(s.vel, io), g1 = ldv(s.last_g, ib), g2 = ldv(s.last_g, io);
    const double tf1 = s.time_factor[ib], tf2 = s.time_factor[io];
    V p1, q1;
    if (D == 0) {
        p1 = W.ends[b];
        q1 = W.ends[o];
    } else {
        V t1 = v1, t2 = v2;
        p1 = me_pos;
        q1 = o_pos;
        integrate(p1, t1, g1, m1, k, tf1, dt, dt);
        integrate(q1, t2, g2, m2, k, tf2, dt, dt);
    }
    const double sv = collide_two_spheres(me_pos, p1, o_pos, q1, cr);
    if (sv == -1.0) return;
    V a1;
    if (sv > 0.0) {                                                   // COL-707, COL-708: the impact
        V pp = me_pos, vp = v1, qq = o_pos, vq = v2;
        integrate(pp, vp, g1, m1, k, tf1, dmul(sv, dt), dt);
        integrate(qq, vq, g2, m2, k, tf2, dmul(sv, dt), dt);
        const V normal = vnorm(vsub(qq, pp));
        const double u1 = vdot(vp, normal), u2 = vdot(vq, normal);
        if (!free2) {
            vp = vsub(vp, vmul(normal, dmul(2.0, u1)));
        } else {
            const double mm1 = s.mass[ib], mm2 = s.mass[io];
            const double u1p = ddiv(dadd(dsub(dmul(mm1, u1), dmul(mm2, u1)), dmul(dmul(2.0, mm2), u2)), dadd(mm1, mm2));
            vp = vadd(vp, vmul(normal, dsub(u1p, u1)));
        }
        integrate(pp, vp, g1, m1, k, tf1, dmul(dsub(1.0, sv), dt), dt);
        const double inv_m = ddiv(1.0, m1), inv_t = ddiv(1.0, dsub(tf1, 1.0));
        const double ga[3] = {g1.x, g1.y, g1.z}, va[3] = {v1.x, v1.y, v1.z}, wa[3] = {vp.x, vp.y, vp.z};
        double r[3];
        for (int q = 0; q < 3; ++q) {
            const double x = dadd(dsub(dadd(dmul(ga[q], dneg(m1)), dmul(ga[q], dmul(tf1, m1))), dmul(dmul(va[q], tf1), k)),
                                  dmul(wa[q], k));
            r[q] = dmul(dmul(dneg(x), inv_m), inv_t);
        }
        a1 = V{r[0], r[1], r[2]};
        if (D == 0) {                                                 // the impact record, in candidate order
            const int64_t at = ib * s.impact_cap + (acc.imp_n < s.impact_cap ? acc.imp_n : s.impact_cap - 1);
            s.imp_slot[at] = o;
            s.imp_s[at] = sv;
            s.imp_closing[at] = dsub(u1, u2);
            ++acc.imp_n;
        }
    } else {                                                          // COL-709, COL-710: already overlapping
        const V p0q0 = vsub(o_pos, me_pos);
        const double p0q0_2 = vdot(p0q0, p0q0);
        V normal;
        if (p0q0_2 == 0.0) normal = (s.id[ib] > s.id[io]) ? V{1.0, 0.0, 0.0} : V{-1.0, 0.0, 0.0};
        else normal = vnorm(p0q0);
        const double dist = dadd(dsub(cr, dsqrt(p0q0_2)), 1.0);
        const double msum = dadd(m1, m2);
        const double d1 = dmul(ddiv(m2, msum), dist);
        [[maybe_unused]] const double d2 = dmul(ddiv(m1, msum), dist);
        if constexpr (D < 2) {                                       // COL-710: two free balls pushed apart first
            if (free2) {
                potential<D + 1>(W, b, o, vsub(me_pos, vmul(normal, d1)), vadd(o_pos, vmul(normal, d2)), acc);
                if (ddiv(m2, m1) > LIGHT_BALL_RATIO) acc.last_c = vmul(vnorm(acc.last_c), dist);
                const V dv = vsub(v1, v2);
                if (vdot(dv, dv) > 0.0001) return;
            }
        }
        const double normal_comp = vdot(g1, normal);
        const double tmp = ddiv(1.0, dadd(m1, dmul(dt, k)));
        const double c = ddiv(dneg(d1), dmul(dmul(dt, tmp), m1));
        a1 = vsub(vmul(vsub(vmul(normal, c), v1), ddiv(1.0, dt)), vmul(normal, normal_comp));
    }
    if (sv >= acc.last_collision) {                                  // COL-711: the later impact, the stronger at a tie
        const V lc = vmul(a1, RESPONSE_SCALE);
        if (sv == acc.last_collision) {
            if (vdot(lc, lc) > vdot(acc.last_c, acc.last_c)) acc.last_c = lc;
        } else {
            acc.last_c = lc;
            acc.last_collision = sv;
        }
    }
    s.hits[ib * s.hit_cap + (acc.hits_n < s.hit_cap ? acc.hits_n : s.hit_cap - 1)] = s.id[io];
    ++acc.hits_n;
}

// A slot's filing as the candidate tests read it: the level, the key of the box holding the centre and the side
// (-1, 0, +1) an axis; the tick stages every slot's in shared memory, the static walk reads the park's
struct Filing {
    int64_t level, key[3], mod[3];
};
__device__ __forceinline__ Filing filing_of(const EbbCollideState& s, int64_t i) {
    return Filing{s.level[i], {s.key[3 * i], s.key[3 * i + 1], s.key[3 * i + 2]},
                  {s.mod[3 * i], s.mod[3 * i + 1], s.mod[3 * i + 2]}};
}

// Whether a box of ball n is one of ball b's boxes, an ancestor of one or below one (vec_collide.py:809): per axis,
// some option of the finer ball shifted to the coarser level equals some option of the coarser
__device__ __forceinline__ bool related(const Filing& fb, const Filing& fn) {
    const int64_t Lb = fb.level, Ln = fn.level;
    const int64_t sh = 2 * (Lb > Ln ? Lb - Ln : Ln - Lb);
    const bool coarse = Ln <= Lb;
    for (int q = 0; q < 3; ++q) {
        const int64_t kb = fb.key[q], mb = fb.mod[q], kn = fn.key[q], mn = fn.mod[q];
        const int64_t lo_b = kb + (mb < 0 ? mb : 0), hi_b = kb + (mb > 0 ? mb : 0);
        const int64_t lo_n = kn + (mn < 0 ? mn : 0), hi_n = kn + (mn > 0 ? mn : 0);
        const int64_t xl = (coarse ? lo_b : lo_n) >> sh, xh = (coarse ? hi_b : hi_n) >> sh;
        const int64_t yl = coarse ? lo_n : lo_b, yh = coarse ? hi_n : hi_b;
        if (!(xl == yl || xl == yh || xh == yl || xh == yh)) return false;
    }
    return true;
}

// The position of ball n's first box in ball b's GetNearbyBalls walk, as a sort key (vec_collide.py:825): the index of
// the first of b's boxes (by key) that n's box relates to, the part (0 an ancestor, 1 below, 2 the box itself) and
// within it the ancestor's distance or the box's post-order code (path digits from b's level; 64 past n's level)
__device__ __forceinline__ int64_t order_key(const Filing& fb, const Filing& fn) {
    const int64_t Lb = fb.level, Ln = fn.level;
    int64_t Kn[3], Mn[3], cb[3], lo_b[3], hi_b[3];
    for (int q = 0; q < 3; ++q) {
        const int64_t kb = fb.key[q], mb = fb.mod[q];
        Kn[q] = fn.key[q];
        Mn[q] = fn.mod[q];
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

// Ball::InsertInBoxes' outcome (vec_collide.py:767-798): the level of the inflated radius, the key of the box holding
// the centre, the side (-1, 0, +1) an axis where the inflated sphere reaches the next box. Returns whether the
// reference's park would refuse the filing (a key at the grid's edge, or a ball wider than a top box).
__device__ __forceinline__ bool file_slot(const EbbCollideState& s, int64_t i) {
    const V p = ldv(s.pos, i), v = ldv(s.vel, i);
    const double k = s.friction;
    double infl = s.radius[i];
    if (s.free_[i]) {
        const double m = dmul(s.mass[i], s.agility[i]);
        const double a = ddiv(dmul(dmul(k, s.speed_fraction[i]), s.max_vel[i]), m);
        const double speed = dsqrt(vdot(v, v));
        const double ma = dmul(m, a);
        const double mps = ddiv(dsub(ma, dmul(dsub(ma, dmul(speed, k)), s.time_factor[i])), k);
        infl = dadd(s.radius[i], dmul(s.dt, mps));
    }
    int level = -1;
    for (int l = 0; l < NUM_LEVELS; ++l)
        if (!(dmul(3.0, infl) > level_width(l))) ++level;
    if (level < 0) level = 0;
    const double w = level_width(level);
    const int64_t grid = level_grid(level);
    const double half = dmul(dmul(0.5, w), i2d(grid)), center = dmul(dmul(w, i2d(grid)), 0.5), fac = ddiv(1.0, w);
    const double pa[3] = {p.x, p.y, p.z};
    bool bad = level == 0 && dmul(s.radius[i], 2.0) > level_width(0);
    s.level[i] = level;
    for (int q = 0; q < 3; ++q) {
        int64_t kq = to_i64(dmul(dadd(pa[q], half), fac));
        kq = kq < 0 ? 0 : (kq >= grid ? grid - 1 : kq);
        const double lo = dsub(dmul(i2d(kq), w), center), hi = dsub(dmul(i2d(kq + 1), w), center);
        const bool down = dsub(dadd(lo, infl), pa[q]) > 0.0, up = dsub(dsub(hi, infl), pa[q]) < 0.0;
        const int64_t mq = down ? -1 : (up ? 1 : 0);
        s.key[3 * i + q] = kq;
        s.mod[3 * i + q] = mq;
        if (kq <= 0 || kq >= grid - 1 || kq + mq < 0 || kq + mq >= grid) bad = true;
    }
    return bad;
}


// ================================================================== static collidables (COL-712)
// Capsule::CollideWithBall / OrientedBox::CollideWithBall and ReactToCollision (Capsule.cpp, OrientedBox.cpp,
// BoxShape.cpp; vec_collide.py:1435-1737): a responder against a capsule or an oriented box from the tick's start, its
// straight path predicted with mLastG. A record is 175 doubles laid out as the reference's park keeps it.
constexpr int G_A = 0, G_B = 3, G_AB = 6, G_RAD = 9, G_CENTER = 10, G_LO = 13, G_HI = 16, G_AXES = 19, G_UNIT = 28;
constexpr int G_HALF = 37, G_LENSQ = 40, G_CORNERS = 43, G_RECT = 67, G_RNORM = 139, G_TNORM = 157, G_SIZE = 175;
constexpr int I_KIND = 0, I_ID = 1, I_PARENT = 2, I_LEVEL = 3, I_NBOX = 4, I_SIZE = 5;
constexpr double DBL_MAX_ = 1.7976931348623157e308, STATIC_TINY = 1e-10, STATIC_FLOOR = 1e-5, EJECT_MARGIN = 1.0;
__constant__ int CONNECTED_SIDES[8][3] = {{1, 2, 5}, {1, 3, 5}, {1, 2, 4}, {0, 2, 5}, {1, 3, 4}, {0, 2, 4},
                                          {0, 3, 5}, {0, 3, 4}};    // BoxShape.cpp:189, a corner's three sides
__constant__ int SIDE_MAPPING[3][2] = {{2, 3}, {5, 4}, {1, 0}};     // BoxShape.cpp:137, an axis's two sides

__device__ __forceinline__ V gv(const double* g, int at) { return V{g[at], g[at + 1], g[at + 2]}; }
__device__ __forceinline__ V vcross(V u, V v) {
    return V{dsub(dmul(u.y, v.z), dmul(u.z, v.y)), dsub(dmul(u.z, v.x), dmul(u.x, v.z)),
             dsub(dmul(u.x, v.y), dmul(u.y, v.x))};
}

// Capsule::HandleCollisionNonIteratively: the time of impact (-1: none), the normal before normalising, and whether
// the end velocity is parallel to the axis (the caps alone, the reaction from the tick's end)
__device__ __forceinline__ double capsule_contact(V p0, V p1, V vp1, double brad, const double* g, V* nrm,
                                                  bool* parallel) {
    const V ca = gv(g, G_A), cb = gv(g, G_B), ab = gv(g, G_AB);
    const double rad = dadd(brad, g[G_RAD]);
    const V ao = vsub(p0, ca);
    const double abab = vdot(ab, ab);
    const double m = ddiv(vdot(ab, vp1), abab), n = ddiv(vdot(ab, ao), abab);
    const V q = vsub(vp1, vmul(ab, m)), r = vsub(ao, vmul(ab, n));
    const double a = vdot(q, q), bq = dmul(2.0, vdot(q, r)), rad_sq = dmul(rad, rad);
    const double cq = dsub(vdot(r, r), rad_sq);
    const double sa = collide_two_spheres(p0, p1, ca, ca, rad), sb = collide_two_spheres(p0, p1, cb, cb, rad);
    const V na = vsub(p0, ca), nb = vsub(p0, cb), zero = V{0.0, 0.0, 0.0};
    if (a == 0.0) {
        *parallel = true;
        const bool take_a = sa != -1.0;
        double toi = take_a ? sa : -1.0;
        const bool take_b = sb != -1.0 && (toi == -1.0 || sb < toi);
        if (take_b) toi = sb;
        *nrm = take_b ? nb : (take_a ? na : zero);
        return toi;
    }
    *parallel = false;
    const double det = dsub(dmul(bq, bq), dmul(dmul(4.0, a), cq));
    if (det < 0.0) {
        *nrm = zero;
        return -1.0;
    }
    const double root = dsqrt(det), nbq = dneg(bq);
    const double s1 = ddiv(dmul(dadd(nbq, root), 0.5), a), s2 = ddiv(dmul(dsub(nbq, root), 0.5), a);
    double sv = (s1 >= 0.0 && s1 <= 1.0) ? s1 : -1.0;
    const bool second = s2 >= 0.0 && s2 <= 1.0 && s2 < s1;
    if (second) sv = s2;
    const double t = ddiv(vdot(ao, ab), abab);
    const V dist = vsub(p0, vadd(ca, vmul(ab, t)));
    if (!second && sv == -1.0 && t >= 0.0 && t <= 1.0 && vdot(dist, dist) < rad_sq) {
        *nrm = dist;
        return 0.0;
    }
    const V mid_n = vsub(ao, vmul(ab, t));
    const double mid_t = vdot(mid_n, mid_n) < rad_sq ? 0.0 : sv;
    double toi = -1.0;
    V out = zero;
    const double tk[2] = {dadd(dmul(s1, m), n), dadd(dmul(s2, m), n)};
    const V far[2] = {p0, p1};
    for (int k = 0; k < 2; ++k) {
        const bool low = tk[k] < 0.0, high = tk[k] > 1.0;
        if (low && sa != -1.0 && (toi == -1.0 || sa < toi)) {
            toi = sa;
            out = na;
        } else if (!low && high && sb != -1.0 && (toi == -1.0 || sb < toi)) {
            toi = sb;
            out = vsub(far[k], cb);
        } else if (!low && !high && sv != -1.0 && (toi == -1.0 || sv < toi)) {
            toi = mid_t;
            out = mid_n;
        }
    }
    *nrm = out;
    return toi;
}

// Triangle::ClosestPoint, its regions in order
__device__ __forceinline__ V triangle_closest(V A, V B, V C, V P) {
    const V ab = vsub(B, A), ac = vsub(C, A), ap = vsub(P, A);
    const double d1 = vdot(ab, ap), d2 = vdot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) return A;
    const V bp = vsub(P, B);
    const double d3 = vdot(ab, bp), d4 = vdot(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) return B;
    const double vc = dsub(dmul(d1, d4), dmul(d3, d2));
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) return vadd(A, vmul(ab, ddiv(d1, dsub(d1, d3))));
    const V cp = vsub(P, C);
    const double d5 = vdot(ab, cp), d6 = vdot(ac, cp);
    if (d6 > 0.0 && d5 <= d6) return C;
    const double vb = dsub(dmul(d5, d2), dmul(d1, d6));
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return vadd(A, vmul(ac, ddiv(d2, dsub(d2, d6))));
    const double va = dsub(dmul(d3, d6), dmul(d5, d4));
    const double e43 = dsub(d4, d3), e56 = dsub(d5, d6);
    if (va <= 0.0 && e43 >= 0.0 && e56 >= 0.0) return vadd(B, vmul(vsub(C, B), ddiv(e43, dadd(e43, e56))));
    const double denom = ddiv(1.0, dadd(dadd(va, vb), vc));
    return vadd(vadd(A, vmul(ab, dmul(vb, denom))), vmul(ac, dmul(vc, denom)));
}

// RectangleShape::CollideWithSphere on one side: whether it is struck, the normal, the time
__device__ __forceinline__ bool rect_contact(V p, double radius, V vel, int side, const double* g, V* nrm, double* tt) {
    const double* rc = g + G_RECT + 12 * side;
    const V a = gv(rc, 0), b = gv(rc, 3), c = gv(rc, 6), d = gv(rc, 9);
    const V m = vcross(vsub(c, p), vsub(a, p));
    const bool abc = vdot(vel, m) <= 0.0;
    const V TA = a, TB = abc ? b : c, TC = abc ? c : d;
    const V n = abc ? gv(g, G_RNORM + 3 * side) : gv(g, G_TNORM + 3 * side);
    const V p0 = vsub(p, vmul(n, radius));
    const V p0p1 = vsub(vadd(p0, vel), p0);
    const double ndab = vdot(n, p0p1);
    const double t = ddiv(dsub(vdot(TA, n), vdot(n, p0)), ndab);
    const bool plane = ndab != 0.0 && t >= 0.0 && t <= 1.0;
    const V point = vadd(p0, vmul(p0p1, t));
    const V v0 = vsub(TC, TA), v1 = vsub(TB, TA), v2 = vsub(point, TA);
    const double dot00 = vdot(v0, v0), dot01 = vdot(v0, v1), dot02 = vdot(v0, v2), dot11 = vdot(v1, v1),
                 dot12 = vdot(v1, v2);
    const double inv = ddiv(1.0, dsub(dmul(dot00, dot11), dmul(dot01, dot01)));
    const double u = dmul(dsub(dmul(dot11, dot02), dmul(dot01, dot12)), inv);
    const double v = dmul(dsub(dmul(dot00, dot12), dmul(dot01, dot02)), inv);
    const bool within = u >= 0.0 && v >= 0.0 && dadd(u, v) < 1.0;
    const V q0 = triangle_closest(TA, TB, TC, point);
    const V direction = vsub(vsub(q0, vel), q0);
    const V nd = vnorm(direction);
    const V mm = vsub(q0, p);
    const double bb = vdot(mm, nd), cc = dsub(vdot(mm, mm), dmul(radius, radius));
    const double disc = dsub(dmul(bb, bb), cc);
    const double tq = dsub(dneg(bb), dsqrt(disc < 0.0 ? 0.0 : disc));
    const double ts = tq < 0.0 ? 0.0 : ddiv(tq, dsqrt(vdot(direction, direction)));
    const bool swept = !(cc > 0.0 && bb > 0.0) && !(disc < 0.0) && !(ts > 1.0);
    *nrm = within ? n : vnorm(vsub(p, vadd(q0, vmul(direction, ts))));
    *tt = within ? t : ts;
    return plane && (within || swept);
}

__device__ __forceinline__ double fmax5(double x) { return x < STATIC_FLOOR ? STATIC_FLOOR : x; }

// OrientedBox::CollideWithBall with BoxShape::CollideWithSphere: the time of impact (-1: none) and the normal
__device__ __forceinline__ double box_contact(V p0, V p1, double brad, const double* g, V* nrm) {
    const double r = brad;
    const double p0a[3] = {p0.x, p0.y, p0.z}, p1a[3] = {p1.x, p1.y, p1.z};
    bool excl = false;                                                // AABB::CanExclude
    for (int q = 0; q < 3; ++q) {
        const double lo = g[G_LO + q], hi = g[G_HI + q];
        excl = excl || (dsub(p0a[q], r) > hi && dsub(p1a[q], r) > hi) || (dadd(p0a[q], r) < lo && dadd(p1a[q], r) < lo);
    }
    if (excl) {                                                       // the AABB excludes the move: no contact,
        *nrm = V{0.0, 0.0, 0.0};                                      // whatever the tests below would find
        return -1.0;
    }
    const V vel = vsub(p1, p0), p = p0;
    const double radius = brad;
    V dd = vsub(gv(g, G_CORNERS), p);                                 // ClosestCorner: the first nearest
    double min_d = vdot(dd, dd);
    int closest = 0;
    for (int i = 1; i < 8; ++i) {
        dd = vsub(gv(g, G_CORNERS + 3 * i), p);
        const double di = vdot(dd, dd);
        if (di < min_d) {
            min_d = di;
            closest = i;
        }
    }
    bool alive = true;
    double shortest = -1.0;
    int half = 0;
    for (int i = 0; i < 3; ++i) {
        const int side = CONNECTED_SIDES[closest][i];
        const V n_s = gv(g, G_RNORM + 3 * side);
        const V point = vsub(p, vmul(n_s, radius));
        const double hs = vdot(n_s, vsub(gv(g, G_RECT + 12 * side), point));
        const bool ok = hs >= 0.0;
        if (alive && ok && (hs < shortest || shortest == -1.0)) {
            shortest = hs;
            half = side;
        }
        alive = alive && ok;
    }
    V q = gv(g, G_CENTER);                                            // BoxShape::ClosestPoint
    const V d = vsub(p, q);
    for (int i = 0; i < 3; ++i) {
        const V u = gv(g, G_UNIT + 3 * i);
        const double hl = g[G_HALF + i];
        double dist = vdot(d, u);
        dist = dist > hl ? hl : (dist < dneg(hl) ? dneg(hl) : dist);
        q = vadd(q, vmul(u, dist));
    }
    const V normal = vsub(p, q);
    const double n_len = dsqrt(vdot(normal, normal)), speed = dsqrt(vdot(vel, vel));
    const bool inside = alive && n_len < radius;
    V n_in = V{0.0, 0.0, 0.0};
    if (inside) {
        if (n_len < STATIC_TINY) {
            const V n_half = gv(g, G_RNORM + 3 * half);
            if (speed < STATIC_TINY) {
                n_in = vmul(n_half, fmax5(shortest));
            } else {
                const V o = vsub(p, gv(g, G_CENTER));                 // BoxShape::RayIntersect, the slabs
                double tmin[3], tmax[3];
                int rev[3];
                for (int i = 0; i < 3; ++i) {
                    const V arm = gv(g, G_AXES + 3 * i);
                    const double als = g[G_LENSQ + i], a_o = vdot(arm, o), a_r = vdot(arm, vel);
                    const bool neg = a_r < 0.0, pos = a_r > 0.0;
                    tmin[i] = neg ? ddiv(dsub(dmul(0.5, als), a_o), a_r)
                                  : (pos ? ddiv(dsub(dmul(-0.5, als), a_o), a_r) : dneg(DBL_MAX_));
                    tmax[i] = neg ? ddiv(dsub(dmul(-0.5, als), a_o), a_r)
                                  : (pos ? ddiv(dsub(dmul(0.5, als), a_o), a_r) : DBL_MAX_);
                    rev[i] = neg ? 1 : 0;
                }
                int i_min = 0;
                double v_min = tmin[0], v_max = tmax[0];
                for (int i = 1; i < 3; ++i) {
                    if (v_min < tmin[i]) {
                        i_min = i;
                        v_min = tmin[i];
                    }
                    if (tmax[i] < v_max) v_max = tmax[i];
                }
                if (v_min < v_max) {
                    const int rv = rev[i_min];
                    n_in = dabs(v_min) < dabs(v_max)
                               ? vmul(gv(g, G_RNORM + 3 * SIDE_MAPPING[i_min][rv]), fmax5(dmul(dabs(v_min), speed)))
                               : vmul(gv(g, G_RNORM + 3 * SIDE_MAPPING[i_min][1 - rv]), fmax5(dmul(dabs(v_max), speed)));
                } else {
                    n_in = vmul(n_half, shortest);
                }
            }
        } else {
            n_in = vmul(vnorm(normal), dabs(dsub(radius, n_len)));
        }
    }
    bool hit = false;
    V out = V{0.0, 0.0, 0.0};
    double time = 0.0;
    for (int i = 0; i < 3; ++i) {                                     // else the sides' triangles, the first struck
        V n_i;
        double t_i;
        const bool h = rect_contact(p, radius, vel, CONNECTED_SIDES[closest][i], g, &n_i, &t_i);
        if (!hit && h) {
            out = n_i;
            time = t_i;
        }
        hit = hit || h;
    }
    hit = inside || hit;
    if (inside) {
        out = n_in;
        time = 0.0;
    }
    *nrm = out;
    return hit ? time : -1.0;
}

// The position of a static collidable's first box in responder ib's walk (its boxes all at its one level), as the
// balls' key: the ball's box (by key) it relates to first, the part (ancestor, below, the box itself) and the
// ancestor's distance or the box's post-order code
__device__ __forceinline__ int64_t static_order_key(const EbbCollideState& s, int64_t ib, const int64_t* ints,
                                                    const int64_t* keys) {
    const int64_t Lb = s.level[ib], Ln = ints[I_LEVEL];
    int64_t cb[3], lo_b[3], hi_b[3];
    for (int q = 0; q < 3; ++q) {
        const int64_t kb = s.key[3 * ib + q], mb = s.mod[3 * ib + q];
        cb[q] = 1 + (mb != 0);
        lo_b[q] = kb + (mb < 0 ? mb : 0);
        hi_b[q] = kb + (mb > 0 ? mb : 0);
    }
    int64_t span = 1;
    for (int l = 0; l < NUM_LEVELS - 1; ++l) span *= CODE_BASE;
    const int64_t s_up = Lb > Ln ? 2 * (Lb - Ln) : 0, s_dn = Ln > Lb ? 2 * (Ln - Lb) : 0;
    int64_t best = NOT_A_CANDIDATE;
    for (int64_t bx = 0; bx < ints[I_NBOX]; ++bx) {
        const int64_t* Kn = keys + 3 * bx;
        int64_t code = 0, power = span;
        for (int lvl = 1; lvl < NUM_LEVELS; ++lvl) {
            power /= CODE_BASE;
            const int64_t shift = 2 * (Ln - lvl) > 0 ? 2 * (Ln - lvl) : 0;
            int64_t digit = ((Kn[0] >> shift) & 3) * 16 + ((Kn[1] >> shift) & 3) * 4 + ((Kn[2] >> shift) & 3);
            if (Ln < lvl) digit = CODE_BASE - 1;
            if (Lb >= lvl) digit = 0;
            code += digit * power;
        }
        for (int c = 0; c < 8; ++c) {
            const int64_t bit[3] = {(c >> 2) & 1, (c >> 1) & 1, c & 1};
            bool valid = true, up = true, same = true, down = true;
            for (int q = 0; q < 3; ++q) {
                if (bit[q] != 0 && cb[q] != 2) valid = false;
                const int64_t box = bit[q] ? hi_b[q] : lo_b[q];
                if ((box >> s_up) != Kn[q]) up = false;
                if (box != Kn[q]) same = false;
                if (box != (Kn[q] >> s_dn)) down = false;
            }
            if (!valid) continue;
            const int64_t seg = (bit[0] * cb[1] + bit[1]) * cb[2] + bit[2];
            int64_t k = NOT_A_CANDIDATE;
            if (Ln < Lb) {
                if (up) k = (seg * 3) * span + (Lb - Ln);
            } else if (Ln == Lb) {
                if (same) k = (seg * 3 + 2) * span;
            } else if (down) {
                k = (seg * 3 + 1) * span + code;
            }
            if (k < best) best = k;
        }
    }
    return best;
}

// CollideWithBall then ReactToCollision (Capsule.cpp:365-437, OrientedBox.cpp:44-106) of responder ib with one static
// collidable: whether the reaction is called (not for no contact, nor for a capsule when mLastG points out of it at an
// impact within the tick), its time and 0.85 of its acceleration (the reflection off it, or the ejection by the
// overlap plus a metre)
__device__ __forceinline__ bool static_values(const EbbCollideState& s, int64_t ib, V pe, V ve, const double* g,
                                              int64_t kind, double* toi_out, V* lc) {
    const double k = s.friction, dt = s.dt;
    const double m1 = dmul(s.mass[ib], s.agility[ib]), tf = s.time_factor[ib], brad = s.radius[ib];
    const V p0 = ldv(s.pos, ib), v0 = ldv(s.vel, ib), gg = ldv(s.last_g, ib);
    const bool cap = kind == 0;
    V normal;
    bool parallel = false;
    const double toi = cap ? capsule_contact(p0, pe, ve, brad, g, &normal, &parallel) : box_contact(p0, pe, brad, g, &normal);
    if (toi == -1.0) return false;
    const double cl = dsqrt(vdot(normal, normal));
    const V nn = vnorm(normal);
    const double nc = vdot(gg, nn);
    if (cap && toi > 0.0 && nc > 0.0) return false;
    V a;
    if (toi > 0.0) {
        const bool end = cap && parallel;
        V pos = end ? pe : p0, vel = end ? ve : v0;
        integrate(pos, vel, gg, m1, k, tf, dmul(toi, dt), dt);
        V vb = vsub(vel, vmul(nn, dmul(2.0, vdot(vel, nn))));
        integrate(pos, vb, gg, m1, k, tf, dmul(dsub(1.0, toi), dt), dt);
        const double ga[3] = {gg.x, gg.y, gg.z}, va[3] = {v0.x, v0.y, v0.z}, wa[3] = {vb.x, vb.y, vb.z};
        const double inv_m = ddiv(1.0, m1), inv_t = ddiv(1.0, dsub(tf, 1.0));
        double rr[3];
        for (int q = 0; q < 3; ++q) {
            const double x = dadd(dsub(dadd(dmul(ga[q], dneg(m1)), dmul(ga[q], dmul(tf, m1))), dmul(dmul(va[q], tf), k)),
                                  dmul(wa[q], k));
            rr[q] = dmul(dmul(dneg(x), inv_m), inv_t);
        }
        a = V{rr[0], rr[1], rr[2]};
    } else {
        const double dist = cap ? dadd(dsub(dadd(g[G_RAD], brad), cl), EJECT_MARGIN) : dadd(cl, EJECT_MARGIN);
        const double tmp = ddiv(1.0, dadd(m1, dmul(dt, k)));
        const double c = ddiv(dist, dmul(dmul(dt, tmp), m1));
        a = vsub(vmul(vsub(vmul(nn, c), v0), ddiv(1.0, dt)), vmul(nn, nc));
    }
    *toi_out = toi;
    *lc = vmul(a, RESPONSE_SCALE);
    return true;
}

// A block's neighbourhoods in shared memory (T threads, whole worlds of N slots; built by the tick's second phase):
// each slot's depth-0 end of the tick (position and velocity), start position (x, y, z planes), radius, id, filing and
// flags, then two candidate tables, the balls' (N rows) and the static collidables' (S rows, S = the park's static
// slots): column o of responder t's row at key[o * (T + 1) + t] (the walk key, or NO_CANDIDATE), so that a
// responder's scan reads consecutive words across its warp and the candidates' writes fall in distinct banks; the
// responder sorts its row in place, the slots beside it in slot[o * (T + 1) + t]
constexpr int64_t NO_CANDIDATE = INT64_MAX;          // (above every walk key, NOT_A_CANDIDATE included)
constexpr uint8_t F_EXISTS = 1, F_MASSIVE = 2, F_CLOAKED = 4, F_JUNK = 8, F_RESPONDER = 16;

struct Hood {
    V *ends, *vend;
    double *px, *py, *pz, *rad;
    int64_t *id, *level, *kx, *ky, *kz, *key, *skey;
    int8_t* mod;                                       // [3][T]
    uint8_t *flags, *slot, *sslot;
    int T, P;                                          // threads, and the candidate tables' column pitch (T + 1)

    __device__ __forceinline__ Hood(unsigned char* raw, int T_, int N, int S) : T(T_), P(T_ + 1) {
        ends = (V*)raw;
        vend = ends + T;
        double* d = (double*)(vend + T);
        px = d;
        py = d + T;
        pz = d + 2 * T;
        rad = d + 3 * T;
        int64_t* q = (int64_t*)(d + 4 * T);
        id = q;
        level = q + T;
        kx = q + 2 * T;
        ky = q + 3 * T;
        kz = q + 4 * T;
        key = q + 5 * T;
        skey = key + (size_t)P * N;
        mod = (int8_t*)(skey + (size_t)P * S);
        flags = (uint8_t*)(mod + 3 * T);
        slot = flags + T;
        sslot = slot + (size_t)P * N;
    }
    __device__ __forceinline__ V pos(int t) const { return V{px[t], py[t], pz[t]}; }
    __device__ __forceinline__ Filing filing(int t) const {
        return Filing{level[t], {kx[t], ky[t], kz[t]}, {mod[t], mod[T + t], mod[2 * T + t]}};
    }
};

__host__ __forceinline__ size_t hood_bytes(int T, int N, int S) {
    const size_t P = (size_t)T + 1;
    return (size_t)T * (2 * sizeof(V) + 9 * 8) + P * (N + S) * 8 + (size_t)T * 4 + P * (N + S);
}

// Threads a block (whole worlds of N slots each) and resident blocks a multiprocessor is asked to fit (the register
// budget the compiler gets). 128 threads and 6 blocks (80 registers, 24 warps a multiprocessor) measured fastest on
// B200 at 65,536 worlds of 16 slots: 0.37 ms a tick, against 0.77 ms for 256 threads at the compiler's own 228
// registers (8 warps); the tick is latency-bound, so occupancy pays for the spills.
#ifndef EBB_COLLIDE_THREADS
#define EBB_COLLIDE_THREADS 128
#endif
#ifndef EBB_COLLIDE_MIN_BLOCKS
#define EBB_COLLIDE_MIN_BLOCKS 6
#endif

// STATICS: the park has static collidables (the balls-only tick is compiled without their steps)
template <bool STATICS>
__global__ void __launch_bounds__(EBB_COLLIDE_THREADS, EBB_COLLIDE_MIN_BLOCKS) tick_kernel(EbbCollideState s, const uint8_t* __restrict__ active,
                                                   int32_t* status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N = (int)s.slots, wpb = blockDim.x / N;
    const int S = STATICS ? (int)s.statics : 0;                      // (at most EBB_COLLIDE_MAX_STATICS)
    const Hood H(smem_raw, (int)blockDim.x, N, S);
    V* ends = H.ends;
    const int lw = threadIdx.x / N, j = threadIdx.x - lw * N, t = threadIdx.x, w0 = lw * N;
    const int64_t w = (int64_t)blockIdx.x * wpb + lw;
    const bool mine = lw < wpb && w < s.worlds && (active == nullptr || active[w] != 0);
    const int64_t base = w * N, i = base + j;
    const bool live = mine && s.exists[i] && s.free_[i];
    const double k = s.friction, dt = s.dt;
    // (1) the behaviours: mLastG, STOP's damping, mLastC and the collision list cleared
    if (live) {
        V g = V{0.0, 0.0, 0.0};
        if (s.mode[i] == GOTO) {
            const V a = vsub(ldv(s.goto_pt, i), ldv(s.pos, i));
            const double length2 = vdot(a, a);
            const double sf = s.speed_fraction[i], mv = s.max_vel[i];
            const double dist = dmul(dmul(sf, mv), dt);
            const double max_thrust = ddiv(dmul(dmul(k, sf), mv), dmul(s.mass[i], s.agility[i]));
            const V unit = vnorm(a);
            const double dd = dmul(dist, dist);
            double scale = max_thrust;
            if (length2 < dd) {
                const double coff = ddiv(length2, dd);
                scale = dmul(dmul(max_thrust, coff), coff);
            }
            g = vmul(unit, scale);
        }
        stv(s.last_g, i, g);
        if (s.mode[i] == STOP) {
            const double vy = s.vel[3 * i + 1];
            s.vel[3 * i + 1] = dmul(dsub(vy, dmul(0.07, vy)), STOP_DAMP);
        }
        stv(s.last_c, i, V{0.0, 0.0, 0.0});
        s.hits_n[i] = 0;
        s.imp_n[i] = 0;
    }
    {   // the live balls' collision lists and impact slots cleared by their warp, a run of consecutive live slots
        // (contiguous rows) at a time: consecutive lanes write consecutive entries (a thread clearing its own row
        // strides the warp's stores a row apart)
        const int warp0 = t & ~31, lane = t & 31, nl = min(32, (int)blockDim.x - warp0);
        const unsigned lanes = nl == 32 ? 0xffffffffu : (1u << nl) - 1u;
        unsigned todo = __ballot_sync(lanes, live);
        const int64_t first = (int64_t)blockIdx.x * blockDim.x + warp0;      // the warp's first slot in the park
        const int hc = (int)s.hit_cap, ic = (int)s.impact_cap;
        while (todo != 0) {
            const int b = __ffs(todo) - 1;
            const unsigned gaps = ~(todo >> b);                          // the run's end: the first clear bit from b
            const int len = gaps == 0u ? 32 - b : __ffs(gaps) - 1;
            todo &= ~((len == 32 ? 0xffffffffu : (1u << len) - 1u) << b);
            int64_t* h = s.hits + (first + b) * hc;
            for (int q = lane; q < len * hc; q += nl) h[q] = -1;
            int64_t* m = s.imp_slot + (first + b) * ic;
            for (int q = lane; q < len * ic; q += nl) m[q] = -1;
        }
    }
    __syncthreads();
    // (2) every ball's end of the tick as depth 0 of Potential predicts it (a fixed ball with mass 1e34), and the
    // slot's neighbourhood fields staged for the world's candidate tests
    if (mine) {
        uint8_t f = 0;
        if (s.exists[i]) {
            V p = ldv(s.pos, i), v = ldv(s.vel, i);
            const V p0 = p;
            const double m = s.free_[i] ? dmul(s.mass[i], s.agility[i]) : FIXED_MASS;
            integrate(p, v, ldv(s.last_g, i), m, k, s.time_factor[i], dt, dt);
            ends[t] = p;
            H.vend[t] = v;
            H.px[t] = p0.x;
            H.py[t] = p0.y;
            H.pz[t] = p0.z;
            H.rad[t] = s.radius[i];
            H.id[t] = s.id[i];
            const Filing fi = filing_of(s, i);
            H.level[t] = fi.level;
            H.kx[t] = fi.key[0];
            H.ky[t] = fi.key[1];
            H.kz[t] = fi.key[2];
            for (int q = 0; q < 3; ++q) H.mod[q * H.T + t] = (int8_t)fi.mod[q];
            const bool massive = s.massive[i] != 0;
            f = F_EXISTS | (massive ? F_MASSIVE : 0) | (s.cloaked[i] ? F_CLOAKED : 0) | (s.junk[i] ? F_JUNK : 0) |
                (live && massive ? F_RESPONDER : 0);
        }
        H.flags[t] = f;
    }
    __syncthreads();
    // (3a) the candidate tests spread over the world's threads: this slot as a candidate of each responder b (a free
    // massive ball), its walk key written into b's row
    if (mine) {
        const uint8_t fo = H.flags[t];
        const bool can = (fo & (F_EXISTS | F_MASSIVE | F_CLOAKED)) == (F_EXISTS | F_MASSIVE);
        const V po = H.pos(t), eo = ends[t];
        const Filing fo_ = H.filing(t);
        const double ro = H.rad[t];
        for (int b = 0; b < N; ++b) {
            const int tb = w0 + b;
            const uint8_t fb = H.flags[tb];
            if (!(fb & F_RESPONDER)) continue;
            int64_t key = NO_CANDIDATE;
            if (can && b != j && !((fo & F_JUNK) && !(fb & F_JUNK))) {
                const Filing fb_ = H.filing(tb);
                if (related(fb_, fo_) &&
                    collide_two_spheres(H.pos(tb), ends[tb], po, eo, dadd(H.rad[tb], ro)) != -1.0)
                    key = order_key(fb_, fo_);
            }
            H.key[(size_t)j * H.P + tb] = key;
        }
        // and the world's static collidables, static q by thread q mod N: each one's walk key (its first box) for
        // every responder it reacts with (CollideWithBall from the responder's depth-0 end of the tick)
        for (int q = j; STATICS && q < S; q += N) {
            const int64_t at = w * S + q;
            const bool ex = s.s_exists[at] != 0;
            const int64_t* ints = s.s_int + at * I_SIZE;
            for (int b = 0; b < N; ++b) {
                const int tb = w0 + b;
                if (!(H.flags[tb] & F_RESPONDER)) continue;
                int64_t key = NO_CANDIDATE;
                if (ex) {
                    const int64_t kq = static_order_key(s, base + b, ints, s.s_keys + at * s.boxes * 3);
                    double toi;
                    V lc;
                    if (kq < NOT_A_CANDIDATE &&
                        static_values(s, base + b, ends[tb], H.vend[tb], s.s_geo + at * G_SIZE, ints[I_KIND], &toi, &lc))
                        key = kq;
                }
                H.skey[(size_t)q * H.P + tb] = key;
            }
        }
    }
    __syncthreads();
    // (3b) the gradient: each free massive ball against its candidates in GetNearbyBalls' order (its row sorted in
    // place by walk key, then id, as the candidates arrive in slot order)
    if (live && (H.flags[t] & F_RESPONDER)) {
        const World W{&s, base, ends + w0};
        const V pb = H.pos(t);
        int nact = 0;
        for (int o = 0; o < N; ++o) {
            const int64_t key = H.key[(size_t)o * H.P + t];
            if (key == NO_CANDIDATE) continue;
            const int64_t id = H.id[w0 + o];
            int at = nact++;                                          // insertion by (key, id)
            while (at > 0) {
                const int64_t kp = H.key[(size_t)(at - 1) * H.P + t];
                const int sp = H.slot[(size_t)(at - 1) * H.P + t];
                if (!(kp > key || (kp == key && H.id[w0 + sp] > id))) break;
                H.key[(size_t)at * H.P + t] = kp;
                H.slot[(size_t)at * H.P + t] = (uint8_t)sp;
                --at;
            }
            H.key[(size_t)at * H.P + t] = key;
            H.slot[(size_t)at * H.P + t] = (uint8_t)o;
        }
        Acc acc{V{0.0, 0.0, 0.0}, -1.0, 0, 0};
        for (int q = 0; q < nact; ++q) {
            const int o = H.slot[(size_t)q * H.P + t];
            potential<0>(W, j, o, pb, H.pos(w0 + o), acc);
        }
        if (STATICS) {                                                // then the static collidables (COL-712)
            V pe = pb, ve = ldv(s.vel, i);
            integrate(pe, ve, ldv(s.last_g, i), dmul(s.mass[i], s.agility[i]), k, s.time_factor[i], dt, dt);
            int64_t* okey = H.skey + t;                                   // the row, a stride P apart
            uint8_t* oslot = H.sslot + t;
            int nst = 0;                                                  // the reacting ones in the walk's order:
            for (int q = 0; q < S; ++q) {                                 // first box, parent id, id, slot
                const int64_t key = okey[(size_t)q * H.P];
                if (key == NO_CANDIDATE) continue;
                const int64_t* ints = s.s_int + (w * S + q) * I_SIZE;
                int pos = nst++;
                while (pos > 0) {
                    const int64_t kp = okey[(size_t)(pos - 1) * H.P];
                    const int sp = oslot[(size_t)(pos - 1) * H.P];
                    const int64_t* pi = s.s_int + (w * S + sp) * I_SIZE;
                    const bool after = kp > key ||
                                       (kp == key && (pi[I_PARENT] > ints[I_PARENT] ||
                                                                 (pi[I_PARENT] == ints[I_PARENT] && pi[I_ID] > ints[I_ID])));
                    if (!after) break;
                    okey[(size_t)pos * H.P] = kp;
                    oslot[(size_t)pos * H.P] = (uint8_t)sp;
                    --pos;
                }
                okey[(size_t)pos * H.P] = key;
                oslot[(size_t)pos * H.P] = (uint8_t)q;
            }
            for (int q = 0; q < nst; ++q) {
                const int64_t at = w * s.statics + oslot[(size_t)q * H.P];
                const int64_t* ints = s.s_int + at * I_SIZE;
                double toi;
                V lc;
                static_values(s, i, pe, ve, s.s_geo + at * G_SIZE, ints[I_KIND], &toi, &lc);
                const bool eq = toi == acc.last_collision;              // the stronger at a tie, no later-impact test
                if (!eq || vdot(lc, lc) > vdot(acc.last_c, acc.last_c)) acc.last_c = lc;
                if (!eq) acc.last_collision = toi;
                s.hits[i * s.hit_cap + (acc.hits_n < s.hit_cap ? acc.hits_n : s.hit_cap - 1)] = ints[I_ID];
                ++acc.hits_n;
            }
        }
        stv(s.last_c, i, acc.last_c);
        s.last_collision[i] = acc.last_collision;
        s.hits_n[i] = acc.hits_n;
        s.imp_n[i] = acc.imp_n;
    }
    __syncthreads();
    // (4) the commit, then the re-filing of the balls that moved at least sqrt(0.1) m
    if (live) {
        V p = ldv(s.pos, i), v = ldv(s.vel, i);
        const V old = p, oldv = v;
        integrate(p, v, vadd(ldv(s.last_g, i), ldv(s.last_c, i)), dmul(s.mass[i], s.agility[i]), k, s.time_factor[i],
                  dt, dt);
        stv(s.old_pos, i, old);
        stv(s.old_vel, i, oldv);
        stv(s.pos, i, p);
        stv(s.vel, i, v);
        const V d = vsub(p, old);
        if (!(vdot(d, d) < 0.1) && file_slot(s, i)) atomicOr(status, 2);
    }
}

// The load's last steps for every existing slot: the decay factor (exp(-k dt / m), 0 for m <= 0) and the first filing
__global__ void load_kernel(EbbCollideState s, int32_t* status) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.worlds * s.slots || !s.exists[i]) return;
    const double m = dmul(s.mass[i], s.agility[i]);
    s.time_factor[i] = m > 0.0 ? lm::exp(ddiv(dmul(dneg(s.friction), s.dt), m)) : 0.0;
    if (file_slot(s, i)) atomicOr(status, 1);
}

}  // namespace collide
}  // namespace ebb

namespace {
int launched() {
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}
bool shape_ok(const EbbCollideState* s) {
    return s != nullptr && s->worlds >= 0 && s->slots >= 1 && s->slots <= EBB_COLLIDE_MAX_SLOTS && s->statics >= 0 &&
           s->statics <= EBB_COLLIDE_MAX_STATICS && s->boxes >= 1 &&
           s->hit_cap == (s->slots > 1 ? 3 * (s->slots - 1) : 1) + s->statics &&
           s->impact_cap == (s->slots > 1 ? s->slots - 1 : 1) &&
           (s->statics == 0 || (s->s_exists && s->s_geo && s->s_int && s->s_keys));
}
}  // namespace

extern "C" {

int ebb_collide_tick(const EbbCollideState* s, const uint8_t* active, int32_t* status, void* stream) {
    if (!shape_ok(s) || status == nullptr) return EBB_EINVAL;
    if (s->worlds == 0) return 0;
    const int N = (int)s->slots, wpb = EBB_COLLIDE_THREADS / N > 0 ? EBB_COLLIDE_THREADS / N : 1, threads = wpb * N;
    const unsigned grid = (unsigned)((s->worlds + wpb - 1) / wpb);
    const size_t smem = ebb::collide::hood_bytes(threads, N, (int)s->statics);   // 34 KB at 16 slots, 164 KB at most
    const bool st = s->statics > 0;
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(st ? ebb::collide::tick_kernel<true> : ebb::collide::tick_kernel<false>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
    }
    if (st)
        ebb::collide::tick_kernel<true><<<grid, threads, smem, (cudaStream_t)stream>>>(*s, active, status);
    else
        ebb::collide::tick_kernel<false><<<grid, threads, smem, (cudaStream_t)stream>>>(*s, active, status);
    return launched();
}

int ebb_collide_load(const EbbCollideState* s, int32_t* status, void* stream) {
    if (!shape_ok(s) || status == nullptr) return EBB_EINVAL;
    const int64_t n = s->worlds * s->slots;
    if (n == 0) return 0;
    ebb::collide::load_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(*s, status);
    return launched();
}

}  // extern "C"

EBB_OP_COUNTER(ebb_count_ops_collide)
