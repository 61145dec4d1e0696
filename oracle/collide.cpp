// SPDX-License-Identifier: MIT
// TEST INFRASTRUCTURE, NOT THE PRODUCT. The CPU oracle of the collision park's tick: a scalar, sequential restatement
// of the reference's gradient method on spheres (exact_ballpark/space.py: SpaceBallpark._gradient :1650,
// _potential :1663, collide_two_spheres :1631, integrate :1609) with the batched park's load, behaviours, commit and
// partition filing (exact_ballpark/vec_collide.py: load :550, _behaviour :953, _goto_thrust :975, evolve :990,
// _inflated_radius :767, _filing :776) and GetNearbyBalls' candidate order as the batched park states it per pair
// (_related :809, _order_keys :825). Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it.
//
// One world at a time, slot by slot: every free ball's behaviour, then for each free massive ball (a responder) its
// candidates sorted into the walk's order and Potential called on each in turn, recursing on overlaps with the
// positions pushed apart (as the scalar code mutates and restores them), then the commit and the re-filing.
// Exactness: plain IEEE double operations in the reference's order (compiled with -ffp-contract=off), glibc's exp from
// the oracle's libm (oracle_libm.cpp).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>
#include <algorithm>

extern "C" int oracle_libm(int func, int64_t n, const double* x, const double* y, double* out);

namespace {

constexpr int NUM_LEVELS = 8;
constexpr double GRID_UNIT = 480.0;
constexpr int64_t CODE_BASE = 65;
constexpr int64_t NOT_A_CANDIDATE = int64_t(1) << 62;
constexpr double LIGHT_BALL_RATIO = 25.0;
constexpr double RESPONSE_SCALE = 0.85;
constexpr double STOP_DAMP = 0.9345794392523364485981308411215;
constexpr int64_t GOTO = 0, STOP = 2;

double level_width(int i) { return ((double)(int64_t(1) << (2 * NUM_LEVELS)) * GRID_UNIT * 0.25) / (double)(int64_t(1) << (2 * i)); }
int64_t level_grid(int i) { return int64_t(1) << (2 * i - 2 * NUM_LEVELS + 39); }

double glibc_exp(double x) {
    double y = 0.0, out = 0.0;
    oracle_libm(3, 1, &x, &y, &out);
    return out;
}

struct V3 {
    double x, y, z;
};
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 mul(V3 a, double c) { return {a.x * c, a.y * c, a.z * c}; }
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 normalized(V3 v) {
    const double n = std::sqrt(dot(v, v));
    if (n == 0.0) return v;
    const double inv = 1.0 / n;
    return mul(v, inv);
}

// int64_t(x) as aarch64's fcvtzs: toward zero, saturating, NaN to 0
int64_t to_int64(double x) {
    if (x != x) return 0;
    if (x >= 9223372036854775808.0) return INT64_MAX;
    if (x < -9223372036854775808.0) return INT64_MIN;
    return (int64_t)x;
}

}  // namespace

extern "C" {

// The park's state, [W][N] slots, vectors [W][N][3] (the reference's [W, N] tensors, row-major)
struct OracleCollide {
    int64_t W, N, C, I;               // worlds, slots, collision-list and impact-record capacities
    double k, dt;
    double *pos, *vel, *old_pos, *old_vel, *goto_pt, *last_g, *last_c;
    double *mass, *radius, *max_vel, *agility, *sf, *tf, *last_collision;
    int64_t *id, *mode, *level, *key, *mod;
    uint8_t *exists, *free_, *massive, *junk, *cloaked;
    int64_t *hits, *hits_n, *imp_slot, *imp_n;
    double *imp_s, *imp_closing;
};

}  // extern "C"

namespace {

struct Park {
    const OracleCollide& s;
    int64_t w;
    int64_t at(int64_t j) const { return w * s.N + j; }
    V3 ld(const double* p, int64_t j) const {
        const int64_t q = 3 * at(j);
        return {p[q], p[q + 1], p[q + 2]};
    }
    void st(double* p, int64_t j, V3 v) const {
        const int64_t q = 3 * at(j);
        p[q] = v.x;
        p[q + 1] = v.y;
        p[q + 2] = v.z;
    }
    int64_t ki(const int64_t* p, int64_t j, int q) const { return p[3 * at(j) + q]; }
};

// Ballpark::Integrate (space.py:1609): nothing for t = 0, the cached factor for t = dt, else glibc's exp
void integrate(V3& p, V3& v, V3 a, double m, double k, double tf, double t, double dt) {
    if (t == 0.0) return;
    if (t != dt) tf = glibc_exp((-k / m) * t);
    const double k2 = k * k, ook2 = 1.0 / k2, ook = 1.0 / k;
    double pa[3] = {p.x, p.y, p.z}, va[3] = {v.x, v.y, v.z}, aa[3] = {a.x, a.y, a.z}, pn[3], vn[3];
    if (k < 1e-10 * m * t) {
        const double inv_m = 1.0 / m;
        for (int i = 0; i < 3; ++i)
            pn[i] = (m * (aa[i] * (-k * t) + k * (aa[i] * t + va[i] * k * inv_m * t)) + pa[i] * k2) * ook2;
    } else {
        for (int i = 0; i < 3; ++i)
            pn[i] = (m * (m * aa[i] * (tf - 1.0) + k * (aa[i] * t + va[i] - tf * va[i])) + pa[i] * k2) * ook2;
    }
    for (int i = 0; i < 3; ++i) vn[i] = (m * aa[i] - (m * aa[i] - va[i] * k) * tf) * ook;
    p = {pn[0], pn[1], pn[2]};
    v = {vn[0], vn[1], vn[2]};
}

// CollideTwoSpheres (space.py:1631)
double collide_two_spheres(V3 p0, V3 p1, V3 q0, V3 q1, double cr) {
    const V3 p0q0 = sub(p0, q0);
    const double p0q0_2 = dot(p0q0, p0q0);
    if (p0q0_2 <= cr * cr) return 0.0;
    const V3 dpq = sub(sub(p1, p0), sub(q1, q0));
    const double a = dot(dpq, dpq), b = 2.0 * dot(p0q0, dpq), c = p0q0_2 - cr * cr;
    if (a == 0.0 && b == 0.0) return -1.0;
    double det = b * b - 4.0 * a * c;
    if (det < 0.0) return -1.0;
    det = std::sqrt(det);
    const double s2 = ((-b - det) * 0.5) / a;
    if (s2 >= 0.0 && s2 <= 1.0) return s2;
    return -1.0;
}

// The mutable part of a responder during its Gradient, and the positions Potential's recursion pushes
struct Me {
    V3 last_c;
    double last_collision;
    std::vector<int64_t> hits;
    std::vector<int64_t> imp_slot;
    std::vector<double> imp_s, imp_closing;
};

struct Ctx {
    const Park& P;
    int64_t b;        // the responder's slot
    Me& me;
};

void potential(Ctx& c, int64_t o, V3 me_pos, V3 o_pos, int depth) {
    const OracleCollide& s = c.P.s;
    const Park& P = c.P;
    const int64_t ib = P.at(c.b), io = P.at(o);
    const double k = s.k, dt = s.dt;
    const double cr = s.radius[ib] + s.radius[io];
    const double m1 = s.free_[ib] ? s.mass[ib] * s.agility[ib] : 1.0e34;
    const double m2 = s.free_[io] ? s.mass[io] * s.agility[io] : 1.0e34;
    const V3 me_vel = P.ld(s.vel, c.b), o_vel = P.ld(s.vel, o);
    const V3 g1 = P.ld(s.last_g, c.b), g2 = P.ld(s.last_g, o);
    const double tf1 = s.tf[ib], tf2 = s.tf[io];
    const V3 p0 = me_pos, q0 = o_pos;
    V3 p1 = me_pos, vtmp = me_vel, q1 = o_pos, wtmp = o_vel;
    integrate(p1, vtmp, g1, m1, k, tf1, dt, dt);
    integrate(q1, wtmp, g2, m2, k, tf2, dt, dt);
    const double sv = collide_two_spheres(p0, p1, q0, q1, cr);
    if (sv == -1.0) return;
    p1 = me_pos;
    V3 vp1 = me_vel;
    q1 = o_pos;
    V3 vq1 = o_vel;
    V3 a1;
    if (sv > 0.0) {
        integrate(p1, vp1, g1, m1, k, tf1, sv * dt, dt);
        integrate(q1, vq1, g2, m2, k, tf2, sv * dt, dt);
        const V3 normal = normalized(sub(q1, p1));
        const double v1 = dot(vp1, normal), v2 = dot(vq1, normal);
        if (!s.free_[io]) {
            const double cc = 2.0 * v1;
            vp1 = sub(vp1, mul(normal, cc));
        } else {
            const double mm1 = s.mass[ib], mm2 = s.mass[io];
            const double v1p = (mm1 * v1 - mm2 * v1 + 2.0 * mm2 * v2) / (mm1 + mm2);
            vp1 = add(vp1, mul(normal, v1p - v1));
        }
        integrate(p1, vp1, g1, m1, k, tf1, (1.0 - sv) * dt, dt);
        const double inv_m = 1.0 / m1, inv_t = 1.0 / (tf1 - 1.0);
        const double ga[3] = {g1.x, g1.y, g1.z}, va[3] = {me_vel.x, me_vel.y, me_vel.z}, wa[3] = {vp1.x, vp1.y, vp1.z};
        double r[3];
        for (int i = 0; i < 3; ++i) r[i] = -((((ga[i] * -m1) + ga[i] * (tf1 * m1)) - (va[i] * tf1) * k) + wa[i] * k) * inv_m * inv_t;
        a1 = {r[0], r[1], r[2]};
        if (depth == 0) {                                             // the impact record (vec_collide.py:1282)
            c.me.imp_slot.push_back(o);
            c.me.imp_s.push_back(sv);
            c.me.imp_closing.push_back(v1 - v2);
        }
    } else {
        const V3 p0q0 = sub(q0, p0);
        const double p0q0_2 = dot(p0q0, p0q0);
        V3 normal;
        if (p0q0_2 == 0.0) normal = (s.id[ib] > s.id[io]) ? V3{1.0, 0.0, 0.0} : V3{-1.0, 0.0, 0.0};
        else normal = normalized(sub(q1, p1));
        const double dist = cr - std::sqrt(p0q0_2) + 1;
        const double d1 = m2 / (m1 + m2) * dist;
        const double d2 = m1 / (m1 + m2) * dist;
        if (s.free_[ib] && s.free_[io]) {
            if (depth < 2) {
                potential(c, o, sub(me_pos, mul(normal, d1)), add(o_pos, mul(normal, d2)), depth + 1);
                if (m2 / m1 > LIGHT_BALL_RATIO) c.me.last_c = mul(normalized(c.me.last_c), dist);
                const V3 dv = sub(me_vel, o_vel);
                if (dot(dv, dv) > 0.0001) return;
            }
        }
        const double normal_comp = dot(g1, normal);
        const double tmp = 1.0 / (m1 + dt * k);
        const double cc = -d1 / (dt * tmp * m1);
        const double inv_dt = 1.0 / dt;
        a1 = sub(mul(sub(mul(normal, cc), me_vel), inv_dt), mul(normal, normal_comp));
    }
    if (sv >= c.me.last_collision) {                                 // COL-711 (no missiles here)
        const V3 lc = mul(a1, RESPONSE_SCALE);
        if (sv == c.me.last_collision) {
            if (dot(lc, lc) > dot(c.me.last_c, c.me.last_c)) c.me.last_c = lc;
        } else {
            c.me.last_c = lc;
            c.me.last_collision = sv;
        }
    }
    c.me.hits.push_back(s.id[io]);
}

// The partition relation and the walk's sort key of the other ball (slot n) for the ball (slot b)
bool related(const Park& P, int64_t b, int64_t n) {
    const OracleCollide& s = P.s;
    const int64_t Lb = s.level[P.at(b)], Ln = s.level[P.at(n)];
    const int64_t sh = 2 * (Lb > Ln ? Lb - Ln : Ln - Lb);
    const bool coarse = Ln <= Lb;
    for (int q = 0; q < 3; ++q) {
        const int64_t kb = P.ki(s.key, b, q), mb = P.ki(s.mod, b, q), kn = P.ki(s.key, n, q), mn = P.ki(s.mod, n, q);
        const int64_t lo_b = kb + std::min<int64_t>(mb, 0), hi_b = kb + std::max<int64_t>(mb, 0);
        const int64_t lo_n = kn + std::min<int64_t>(mn, 0), hi_n = kn + std::max<int64_t>(mn, 0);
        const int64_t xl = (coarse ? lo_b : lo_n) >> sh, xh = (coarse ? hi_b : hi_n) >> sh;
        const int64_t yl = coarse ? lo_n : lo_b, yh = coarse ? hi_n : hi_b;
        if (!(xl == yl || xl == yh || xh == yl || xh == yh)) return false;
    }
    return true;
}

int64_t order_key(const Park& P, int64_t b, int64_t n) {
    const OracleCollide& s = P.s;
    const int64_t Lb = s.level[P.at(b)], Ln = s.level[P.at(n)];
    int64_t Kb[3], Mb[3], Kn[3], Mn[3], cb[3], lo_b[3], hi_b[3], cn[3];
    for (int q = 0; q < 3; ++q) {
        Kb[q] = P.ki(s.key, b, q);
        Mb[q] = P.ki(s.mod, b, q);
        Kn[q] = P.ki(s.key, n, q);
        Mn[q] = P.ki(s.mod, n, q);
        cb[q] = 1 + (Mb[q] != 0);
        cn[q] = 1 + (Mn[q] != 0);
        lo_b[q] = Kb[q] + std::min<int64_t>(Mb[q], 0);
        hi_b[q] = Kb[q] + std::max<int64_t>(Mb[q], 0);
    }
    int64_t span = 1;
    for (int i = 0; i < NUM_LEVELS - 1; ++i) span *= CODE_BASE;
    if (Ln <= Lb) {
        const int64_t s_up = 2 * (Lb - Ln);
        int64_t idx[3];
        for (int q = 0; q < 3; ++q) {
            const int64_t v = lo_b[q] >> s_up;
            const bool holds = (v == Kn[q]) || (Mn[q] != 0 && v == Kn[q] + Mn[q]);
            idx[q] = holds ? 0 : 1;
        }
        const int64_t seg = (idx[0] * cb[1] + idx[1]) * cb[2] + idx[2];
        if (Ln < Lb) return (seg * 3) * span + (Lb - Ln);
        return (seg * 3 + 2) * span;
    }
    const int64_t s_dn = 2 * (Ln - Lb);
    int64_t best = NOT_A_CANDIDATE;
    for (int c = 0; c < 8; ++c) {
        const int64_t bit[3] = {(c >> 2) & 1, (c >> 1) & 1, c & 1};
        bool valid = true, own = true;
        int64_t box[3], j[3];
        for (int q = 0; q < 3; ++q) {
            if (!(bit[q] == 0 || cn[q] == 2)) valid = false;
            box[q] = Kn[q] + Mn[q] * bit[q];
            const int64_t anc = box[q] >> s_dn;
            const bool in0 = anc == lo_b[q], in1 = anc == hi_b[q] && cb[q] == 2;
            if (!(in0 || in1)) own = false;
            j[q] = in0 ? 0 : 1;
        }
        if (!(own && valid)) continue;
        const int64_t seg = (j[0] * cb[1] + j[1]) * cb[2] + j[2];
        int64_t code = 0, power = span;
        for (int lvl = 1; lvl < NUM_LEVELS; ++lvl) {
            power /= CODE_BASE;
            const int64_t shift = std::max<int64_t>(2 * (Ln - lvl), 0);
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

// Ball::InsertInBoxes' level, key and side for one ball (vec_collide.py:767-798)
void file_ball(const Park& P, int64_t j) {
    const OracleCollide& s = P.s;
    const int64_t i = P.at(j);
    const V3 p = P.ld(s.pos, j), v = P.ld(s.vel, j);
    double infl = s.radius[i];
    if (s.free_[i]) {
        const double m = s.mass[i] * s.agility[i];
        const double a = (s.k * s.sf[i]) * s.max_vel[i] / m;
        const double speed = std::sqrt(dot(v, v));
        const double ma = m * a;
        const double mps = (ma - (ma - speed * s.k) * s.tf[i]) / s.k;
        infl = s.radius[i] + s.dt * mps;
    }
    int level = -1;
    for (int q = 0; q < NUM_LEVELS; ++q)
        if (!(3.0 * infl > level_width(q))) ++level;
    if (level < 0) level = 0;
    const double width = level_width(level);
    const int64_t grid = level_grid(level);
    const double half = 0.5 * width * (double)grid, center = width * (double)grid * 0.5, fac = 1.0 / width;
    const double pa[3] = {p.x, p.y, p.z};
    s.level[i] = level;
    for (int q = 0; q < 3; ++q) {
        int64_t kq = to_int64((pa[q] + half) * fac);
        if (kq < 0) kq = 0;
        if (kq >= grid) kq = grid - 1;
        const double lo = (double)kq * width - center, hi = (double)(kq + 1) * width - center;
        const bool down = (lo + infl) - pa[q] > 0.0, up = (hi - infl) - pa[q] < 0.0;
        s.key[3 * i + q] = kq;
        s.mod[3 * i + q] = down ? -1 : (up ? 1 : 0);
    }
}

void tick_world(const OracleCollide& s, int64_t w) {
    const Park P{s, w};
    const int64_t N = s.N;
    const double k = s.k, dt = s.dt;
    std::vector<uint8_t> live((size_t)N);
    for (int64_t j = 0; j < N; ++j) live[(size_t)j] = s.exists[P.at(j)] && s.free_[P.at(j)];
    // (1) behaviours
    for (int64_t j = 0; j < N; ++j) {
        if (!live[(size_t)j]) continue;
        const int64_t i = P.at(j);
        V3 g = {0.0, 0.0, 0.0};
        if (s.mode[i] == GOTO) {
            const V3 a = sub(P.ld(s.goto_pt, j), P.ld(s.pos, j));
            const double length2 = a.x * a.x + a.y * a.y + a.z * a.z;
            const double dist = s.sf[i] * s.max_vel[i] * dt;
            const double max_thrust = k * s.sf[i] * s.max_vel[i] / (s.mass[i] * s.agility[i]);
            const V3 unit = normalized(a);
            const double dd = dist * dist;
            double scale = max_thrust;
            if (length2 < dd) {
                const double coff = length2 / dd;
                scale = max_thrust * coff * coff;
            }
            g = mul(unit, scale);
        }
        P.st(s.last_g, j, g);
        if (s.mode[i] == STOP) {
            const double vy = s.vel[3 * i + 1];
            s.vel[3 * i + 1] = (vy - 0.07 * vy) * STOP_DAMP;
        }
        P.st(s.last_c, j, V3{0.0, 0.0, 0.0});
        for (int64_t q = 0; q < s.C; ++q) s.hits[i * s.C + q] = -1;
        s.hits_n[i] = 0;
        for (int64_t q = 0; q < s.I; ++q) s.imp_slot[i * s.I + q] = -1;
        s.imp_n[i] = 0;
    }
    // (3) the gradient: each free massive ball against its candidates in GetNearbyBalls' order
    for (int64_t b = 0; b < N; ++b) {
        const int64_t ib = P.at(b);
        if (!(live[(size_t)b] && s.massive[ib])) continue;
        s.last_collision[ib] = -1.0;
        std::vector<std::pair<int64_t, int64_t>> cand;               // (order key, id) -> slot below
        std::vector<int64_t> slot_of;
        for (int64_t n = 0; n < N; ++n) {
            const int64_t in = P.at(n);
            if (n == b || !s.exists[in] || !s.massive[in] || s.cloaked[in]) continue;
            if (s.junk[in] && !s.junk[ib]) continue;
            if (!related(P, b, n)) continue;
            cand.push_back({order_key(P, b, n), s.id[in]});
            slot_of.push_back(n);
        }
        std::vector<size_t> idx(cand.size());
        for (size_t q = 0; q < idx.size(); ++q) idx[q] = q;
        std::stable_sort(idx.begin(), idx.end(), [&](size_t x, size_t y) { return cand[x] < cand[y]; });
        Me me{P.ld(s.last_c, b), s.last_collision[ib], {}, {}, {}, {}};
        Ctx c{P, b, me};
        for (size_t q : idx) potential(c, slot_of[q], P.ld(s.pos, b), P.ld(s.pos, slot_of[q]), 0);
        P.st(s.last_c, b, me.last_c);
        s.last_collision[ib] = me.last_collision;
        s.hits_n[ib] = (int64_t)me.hits.size();
        for (size_t q = 0; q < me.hits.size(); ++q) s.hits[ib * s.C + std::min<int64_t>((int64_t)q, s.C - 1)] = me.hits[q];
        s.imp_n[ib] = (int64_t)me.imp_slot.size();
        for (size_t q = 0; q < me.imp_slot.size(); ++q) {
            const int64_t at = ib * s.I + std::min<int64_t>((int64_t)q, s.I - 1);
            s.imp_slot[at] = me.imp_slot[q];
            s.imp_s[at] = me.imp_s[q];
            s.imp_closing[at] = me.imp_closing[q];
        }
    }
    // (4) the commit, then the re-filing of the balls that moved at least sqrt(0.1) m
    for (int64_t j = 0; j < N; ++j) {
        if (!live[(size_t)j]) continue;
        const int64_t i = P.at(j);
        V3 p = P.ld(s.pos, j), v = P.ld(s.vel, j);
        const V3 old = p, oldv = v;
        const V3 a = add(P.ld(s.last_g, j), P.ld(s.last_c, j));
        integrate(p, v, a, s.mass[i] * s.agility[i], k, s.tf[i], dt, dt);
        P.st(s.old_pos, j, old);
        P.st(s.old_vel, j, oldv);
        P.st(s.pos, j, p);
        P.st(s.vel, j, v);
        const V3 d = sub(p, old);
        if (!(dot(d, d) < 0.1)) file_ball(P, j);
    }
}

}  // namespace

extern "C" {

// One tick of every world (active[w] != 0 when given), with `threads` host threads over disjoint worlds
int oracle_collide_tick(const OracleCollide* s, const uint8_t* active, int threads) {
    if (threads < 1) threads = 1;
    auto run = [&](int t) {
        for (int64_t w = t; w < s->W; w += threads)
            if (!active || active[w]) tick_world(*s, w);
    };
    if (threads == 1) {
        run(0);
        return 0;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(run, t);
    for (auto& th : pool) th.join();
    return 0;
}

// The filing of the slots with which[w * N + j] != 0 (the load's first filing)
int oracle_collide_filing(const OracleCollide* s, const uint8_t* which) {
    for (int64_t w = 0; w < s->W; ++w) {
        const Park P{*s, w};
        for (int64_t j = 0; j < s->N; ++j)
            if (which[P.at(j)]) file_ball(P, j);
    }
    return 0;
}

}  // extern "C"
