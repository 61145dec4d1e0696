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
    int64_t S, B;                     // static collidable slots a world, boxes a static collidable (at most)
    uint8_t* s_exists;                // [W][S]
    double* s_geo;                    // [W][S][175]
    int64_t *s_int, *s_keys;          // [W][S][5], [W][S][B][3]
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


// ---- static collidables (vec_collide.py:1362-1737; full.py's Capsule, OrientedBox, BoxShape, RectangleShape) ----
constexpr int G_A = 0, G_B = 3, G_AB = 6, G_RAD = 9, G_CENTER = 10, G_LO = 13, G_HI = 16, G_AXES = 19, G_UNIT = 28;
constexpr int G_HALF = 37, G_LENSQ = 40, G_CORNERS = 43, G_RECT = 67, G_RNORM = 139, G_TNORM = 157, G_SIZE = 175;
constexpr int I_KIND = 0, I_ID = 1, I_PARENT = 2, I_LEVEL = 3, I_NBOX = 4, I_SIZE = 5;
constexpr double DBL_MAX_ = 1.7976931348623157e308, STATIC_TINY = 1e-10, STATIC_FLOOR = 1e-5, EJECT_MARGIN = 1.0;
constexpr int CONNECTED_SIDES[8][3] = {{1, 2, 5}, {1, 3, 5}, {1, 2, 4}, {0, 2, 5}, {1, 3, 4}, {0, 2, 4}, {0, 3, 5},
                                       {0, 3, 4}};
constexpr int SIDE_MAPPING[3][2] = {{2, 3}, {5, 4}, {1, 0}};

V3 gv(const double* g, int at) { return {g[at], g[at + 1], g[at + 2]}; }
V3 cross(V3 u, V3 v) { return {u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x}; }

// Capsule::HandleCollisionNonIteratively: (toi, the normal before normalising, whether the end velocity is parallel)
void capsule_contact(V3 p0, V3 p1, V3 vp1, double brad, const double* g, double* toi_out, V3* nrm_out, bool* par_out) {
    const V3 ca = gv(g, G_A), cb = gv(g, G_B), ab = gv(g, G_AB);
    const double rad = brad + g[G_RAD];
    const V3 ao = sub(p0, ca);
    const double abab = dot(ab, ab);
    const double m = dot(ab, vp1) / abab, n = dot(ab, ao) / abab;
    const V3 q = sub(vp1, mul(ab, m)), r = sub(ao, mul(ab, n));
    const double a = dot(q, q), bq = 2.0 * dot(q, r), cq = dot(r, r) - rad * rad, rad_sq = rad * rad;
    const double sa = collide_two_spheres(p0, p1, ca, ca, rad), sb = collide_two_spheres(p0, p1, cb, cb, rad);
    const V3 na = sub(p0, ca), nb = sub(p0, cb), zero{0.0, 0.0, 0.0};
    if (a == 0.0) {                                                   // parallel: the caps alone
        const bool take_a = sa != -1.0;
        double toi_p = take_a ? sa : -1.0;
        const bool take_b = sb != -1.0 && (toi_p == -1.0 || sb < toi_p);
        if (take_b) toi_p = sb;
        *toi_out = toi_p;
        *nrm_out = take_b ? nb : (take_a ? na : zero);
        *par_out = true;
        return;
    }
    *par_out = false;
    const double det = bq * bq - 4.0 * a * cq;
    if (det < 0.0) {
        *toi_out = -1.0;
        *nrm_out = zero;
        return;
    }
    const double root = std::sqrt(det);
    const double s1 = ((-bq + root) * 0.5) / a, s2 = ((-bq - root) * 0.5) / a;
    double sv = (s1 >= 0.0 && s1 <= 1.0) ? s1 : -1.0;
    const bool second = s2 >= 0.0 && s2 <= 1.0 && s2 < s1;
    if (second) sv = s2;
    const double t = dot(ao, ab) / abab;
    const V3 dist = sub(p0, add(ca, mul(ab, t)));
    const bool inside = !second && sv == -1.0 && t >= 0.0 && t <= 1.0 && dot(dist, dist) < rad_sq;
    if (inside) {
        *toi_out = 0.0;
        *nrm_out = dist;
        return;
    }
    const V3 mid_n = sub(ao, mul(ab, t));
    const double mid_t = dot(mid_n, mid_n) < rad_sq ? 0.0 : sv;
    double toi = -1.0;
    V3 nrm = zero;
    const double tks[2] = {(s1 * m) + n, (s2 * m) + n};
    const V3 fars[2] = {p0, p1};
    for (int k = 0; k < 2; ++k) {
        const bool low = tks[k] < 0.0, high = tks[k] > 1.0;
        const bool ta = low && sa != -1.0 && (toi == -1.0 || sa < toi);
        const bool tb = !low && high && sb != -1.0 && (toi == -1.0 || sb < toi);
        const bool tm = !low && !high && sv != -1.0 && (toi == -1.0 || sv < toi);
        if (ta) {
            toi = sa;
            nrm = na;
        } else if (tb) {
            toi = sb;
            nrm = sub(fars[k], cb);
        } else if (tm) {
            toi = mid_t;
            nrm = mid_n;
        }
    }
    *toi_out = toi;
    *nrm_out = nrm;
}

// Triangle::ClosestPoint, its regions in order
V3 triangle_closest(V3 A, V3 B, V3 C, V3 P) {
    const V3 ab = sub(B, A), ac = sub(C, A), ap = sub(P, A);
    const double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) return A;
    const V3 bp = sub(P, B);
    const double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) return B;
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) return add(A, mul(ab, d1 / (d1 - d3)));
    const V3 cp = sub(P, C);
    const double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 > 0.0 && d5 <= d6) return C;
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return add(A, mul(ac, d2 / (d2 - d6)));
    const double va = d3 * d6 - d5 * d4;
    const double e43 = d4 - d3, e56 = d5 - d6;
    if (va <= 0.0 && e43 >= 0.0 && e56 >= 0.0) return add(B, mul(sub(C, B), e43 / (e43 + e56)));
    const double denom = 1.0 / (va + vb + vc);
    return add(add(A, mul(ab, vb * denom)), mul(ac, vc * denom));
}

// RectangleShape::CollideWithSphere on one side: (hit, normal, time)
bool rect_contact(V3 p, double radius, V3 vel, int side, const double* g, V3* nrm_out, double* t_out) {
    const V3 a = gv(g, G_RECT + 12 * side), b = gv(g, G_RECT + 12 * side + 3), c = gv(g, G_RECT + 12 * side + 6),
            d = gv(g, G_RECT + 12 * side + 9);
    const V3 m = cross(sub(c, p), sub(a, p));
    const bool abc = dot(vel, m) <= 0.0;
    const V3 TA = a, TB = abc ? b : c, TC = abc ? c : d;
    const V3 n = abc ? gv(g, G_RNORM + 3 * side) : gv(g, G_TNORM + 3 * side);
    const V3 p0 = sub(p, mul(n, radius));
    const V3 p0p1 = sub(add(p0, vel), p0);
    const double ndab = dot(n, p0p1);
    const double t = (dot(TA, n) - dot(n, p0)) / ndab;
    const bool plane = ndab != 0.0 && t >= 0.0 && t <= 1.0;
    const V3 point = add(p0, mul(p0p1, t));
    const V3 v0 = sub(TC, TA), v1 = sub(TB, TA), v2 = sub(point, TA);
    const double dot00 = dot(v0, v0), dot01 = dot(v0, v1), dot02 = dot(v0, v2), dot11 = dot(v1, v1),
                 dot12 = dot(v1, v2);
    const double inv = 1.0 / (dot00 * dot11 - dot01 * dot01);
    const double u = (dot11 * dot02 - dot01 * dot12) * inv, v = (dot00 * dot12 - dot01 * dot02) * inv;
    const bool within = u >= 0 && v >= 0 && u + v < 1;
    const V3 q0 = triangle_closest(TA, TB, TC, point);
    const V3 direction = sub(sub(q0, vel), q0);
    const V3 nd = normalized(direction);
    const V3 mm = sub(q0, p);
    const double bb = dot(mm, nd), cc = dot(mm, mm) - radius * radius;
    const double disc = bb * bb - cc;
    const double tt = -bb - std::sqrt(disc < 0.0 ? 0.0 : disc);
    const double ts = tt < 0.0 ? 0.0 : tt / std::sqrt(dot(direction, direction));
    const bool swept = !(cc > 0.0 && bb > 0.0) && !(disc < 0.0) && !(ts > 1.0);
    const V3 impact = add(q0, mul(direction, ts));
    *nrm_out = within ? n : normalized(sub(p, impact));
    *t_out = within ? t : ts;
    return plane && (within || swept);
}

// OrientedBox::CollideWithBall + BoxShape::CollideWithSphere: (toi or -1, the normal before normalising)
void box_contact(V3 p0, V3 p1, double brad, const double* g, double* toi_out, V3* nrm_out) {
    const V3 lo = gv(g, G_LO), hi = gv(g, G_HI);
    const double r = brad;
    const double p0a[3] = {p0.x, p0.y, p0.z}, p1a[3] = {p1.x, p1.y, p1.z}, loa[3] = {lo.x, lo.y, lo.z},
                 hia[3] = {hi.x, hi.y, hi.z};
    bool excl = false;
    for (int q = 0; q < 3; ++q)
        excl = excl || ((p0a[q] - r) > hia[q] && (p1a[q] - r) > hia[q]) || ((p0a[q] + r) < loa[q] && (p1a[q] + r) < loa[q]);
    const V3 vel = sub(p1, p0), p = p0;
    const double radius = brad;
    V3 dd = sub(gv(g, G_CORNERS), p);
    double min_d = dot(dd, dd);
    int closest = 0;
    for (int i = 1; i < 8; ++i) {
        dd = sub(gv(g, G_CORNERS + 3 * i), p);
        const double di = dot(dd, dd);
        if (di < min_d) {
            min_d = di;
            closest = i;
        }
    }
    const int* sides = CONNECTED_SIDES[closest];
    bool alive = true;
    double shortest = -1.0;
    int half = 0;
    for (int i = 0; i < 3; ++i) {
        const int side = sides[i];
        const V3 n_s = gv(g, G_RNORM + 3 * side);
        const V3 point = sub(p, mul(n_s, radius));
        const double hs = dot(n_s, sub(gv(g, G_RECT + 12 * side), point));
        const bool ok = hs >= 0.0;
        if (alive && ok && (hs < shortest || shortest == -1.0)) {
            shortest = hs;
            half = side;
        }
        alive = alive && ok;
    }
    V3 q = gv(g, G_CENTER);
    const V3 d = sub(p, q);
    for (int i = 0; i < 3; ++i) {
        const V3 u = gv(g, G_UNIT + 3 * i);
        const double hl = g[G_HALF + i];
        double dist = dot(d, u);
        dist = dist > hl ? hl : (dist < -hl ? -hl : dist);
        q = add(q, mul(u, dist));
    }
    const V3 normal = sub(p, q);
    const double n_len = std::sqrt(dot(normal, normal)), speed = std::sqrt(dot(vel, vel));
    const V3 o = sub(p, gv(g, G_CENTER));
    double tmin[3], tmax[3];
    int rev[3];
    for (int i = 0; i < 3; ++i) {
        const V3 arm = gv(g, G_AXES + 3 * i);
        const double als = g[G_LENSQ + i], a_o = dot(arm, o), a_r = dot(arm, vel);
        const bool neg = a_r < 0, pos = a_r > 0;
        tmin[i] = neg ? (0.5 * als - a_o) / a_r : (pos ? (-0.5 * als - a_o) / a_r : -DBL_MAX_);
        tmax[i] = neg ? (-0.5 * als - a_o) / a_r : (pos ? (0.5 * als - a_o) / a_r : DBL_MAX_);
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
    const int rv = rev[i_min];
    const int side1 = SIDE_MAPPING[i_min][rv], side2 = SIDE_MAPPING[i_min][1 - rv];
    const bool found = v_min < v_max;
    auto fmax5 = [](double x) { return x < STATIC_FLOOR ? STATIC_FLOOR : x; };
    const V3 n_half = gv(g, G_RNORM + 3 * half);
    V3 n_in;
    if (n_len < STATIC_TINY) {
        if (speed < STATIC_TINY) n_in = mul(n_half, fmax5(shortest));
        else if (found)
            n_in = std::fabs(v_min) < std::fabs(v_max) ? mul(gv(g, G_RNORM + 3 * side1), fmax5(std::fabs(v_min) * speed))
                                                      : mul(gv(g, G_RNORM + 3 * side2), fmax5(std::fabs(v_max) * speed));
        else n_in = mul(n_half, shortest);
    } else {
        n_in = mul(normalized(normal), std::fabs(radius - n_len));
    }
    const bool inside = alive && n_len < radius;
    bool hit = false;
    V3 nrm{0.0, 0.0, 0.0};
    double time = 0.0;
    for (int i = 0; i < 3; ++i) {
        V3 n_i;
        double t_i;
        const bool h = rect_contact(p, radius, vel, sides[i], g, &n_i, &t_i);
        if (!hit && h) {
            nrm = n_i;
            time = t_i;
        }
        hit = hit || h;
    }
    hit = !excl && (inside || hit);
    if (inside) {
        nrm = n_in;
        time = 0.0;
    }
    *toi_out = hit ? time : -1.0;
    *nrm_out = nrm;
}

// The position of a static collidable's first box in the responder's walk (its boxes all at one level)
int64_t static_order_key(const Park& P, int64_t b, const int64_t* ints, const int64_t* keys) {
    const OracleCollide& s = P.s;
    const int64_t Lb = s.level[P.at(b)], Ln = ints[I_LEVEL];
    int64_t Kb[3], Mb[3], cb[3], lo_b[3], hi_b[3];
    for (int q = 0; q < 3; ++q) {
        Kb[q] = P.ki(s.key, b, q);
        Mb[q] = P.ki(s.mod, b, q);
        cb[q] = 1 + (Mb[q] != 0);
        lo_b[q] = Kb[q] + std::min<int64_t>(Mb[q], 0);
        hi_b[q] = Kb[q] + std::max<int64_t>(Mb[q], 0);
    }
    int64_t span = 1;
    for (int i = 0; i < NUM_LEVELS - 1; ++i) span *= CODE_BASE;
    const int64_t s_up = std::max<int64_t>(2 * (Lb - Ln), 0), s_dn = std::max<int64_t>(2 * (Ln - Lb), 0);
    int64_t best_all = NOT_A_CANDIDATE;
    for (int64_t bx = 0; bx < ints[I_NBOX]; ++bx) {
        const int64_t* Kn = keys + 3 * bx;
        int64_t code = 0, power = span;
        for (int lvl = 1; lvl < NUM_LEVELS; ++lvl) {
            power /= CODE_BASE;
            const int64_t shift = std::max<int64_t>(2 * (Ln - lvl), 0);
            int64_t digit = ((Kn[0] >> shift) & 3) * 16 + ((Kn[1] >> shift) & 3) * 4 + ((Kn[2] >> shift) & 3);
            if (Ln < lvl) digit = CODE_BASE - 1;
            if (Lb >= lvl) digit = 0;
            code += digit * power;
        }
        for (int c = 0; c < 8; ++c) {
            const int64_t bit[3] = {(c >> 2) & 1, (c >> 1) & 1, c & 1};
            bool valid = true, up = true, same = true, down = true;
            int64_t box[3];
            for (int q = 0; q < 3; ++q) {
                if (!(bit[q] == 0 || cb[q] == 2)) valid = false;
                box[q] = bit[q] ? hi_b[q] : lo_b[q];
                if ((box[q] >> s_up) != Kn[q]) up = false;
                if (box[q] != Kn[q]) same = false;
                if (box[q] != (Kn[q] >> s_dn)) down = false;
            }
            if (!valid) continue;
            const int64_t seg = (bit[0] * cb[1] + bit[1]) * cb[2] + bit[2];
            int64_t k = NOT_A_CANDIDATE;
            if (Ln < Lb) k = up ? (seg * 3) * span + (Lb - Ln) : NOT_A_CANDIDATE;
            else if (Ln == Lb) k = same ? (seg * 3 + 2) * span : NOT_A_CANDIDATE;
            else k = down ? (seg * 3 + 1) * span + code : NOT_A_CANDIDATE;
            if (k < best_all) best_all = k;
        }
    }
    return best_all;
}

// CollideWithBall then ReactToCollision of one (responder, static collidable): whether it is called, toi, 0.85 a
bool static_values(const Park& P, int64_t b, const double* g, const int64_t* ints, double* toi_out, V3* lc_out) {
    const OracleCollide& s = P.s;
    const int64_t ib = P.at(b);
    const double k = s.k, dt = s.dt;
    const double m1 = s.mass[ib] * s.agility[ib], tf = s.tf[ib], brad = s.radius[ib];
    const V3 p0 = P.ld(s.pos, b), v0 = P.ld(s.vel, b), gg = P.ld(s.last_g, b);
    V3 p1 = p0, vp1 = v0;
    integrate(p1, vp1, gg, m1, k, tf, dt, dt);
    const bool cap = ints[I_KIND] == 0;
    double toi;
    V3 normal;
    bool parallel = false;
    if (cap) capsule_contact(p0, p1, vp1, brad, g, &toi, &normal, &parallel);
    else box_contact(p0, p1, brad, g, &toi, &normal);
    const bool end = cap && parallel;
    V3 pos = end ? p1 : p0, vel = end ? vp1 : v0;
    const double cl = std::sqrt(dot(normal, normal));
    const V3 nn = normalized(normal);
    const double nc = dot(gg, nn);
    if (toi == -1.0 || (cap && toi > 0.0 && nc > 0.0)) return false;
    V3 a;
    if (toi > 0.0) {
        integrate(pos, vel, gg, m1, k, tf, toi * dt, dt);
        V3 vb = sub(vel, mul(nn, 2.0 * dot(vel, nn)));
        integrate(pos, vb, gg, m1, k, tf, (1.0 - toi) * dt, dt);
        const double ga[3] = {gg.x, gg.y, gg.z}, va[3] = {v0.x, v0.y, v0.z}, wa[3] = {vb.x, vb.y, vb.z};
        double r[3];
        for (int i = 0; i < 3; ++i) r[i] = (-((((ga[i] * -m1) + ga[i] * (tf * m1)) - (va[i] * tf) * k) + wa[i] * k)) * (1.0 / m1) * (1.0 / (tf - 1.0));
        a = {r[0], r[1], r[2]};
    } else {
        const double dist = cap ? ((g[G_RAD] + brad) - cl) + EJECT_MARGIN : cl + EJECT_MARGIN;
        const double tmp = 1.0 / (m1 + dt * k);
        const double c = dist / ((dt * tmp) * m1);
        a = sub(mul(sub(mul(nn, c), v0), 1.0 / dt), mul(nn, nc));
    }
    *toi_out = toi;
    *lc_out = mul(a, RESPONSE_SCALE);
    return true;
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
        // then its static collidables, in the walk's order (first box, parent id, id)
        struct SC {
            int64_t order, parent, id, slot;
            double toi;
            V3 lc;
        };
        std::vector<SC> sc;
        for (int64_t j = 0; j < s.S; ++j) {
            const int64_t at = w * s.S + j;
            if (!s.s_exists[at]) continue;
            const int64_t* ints = s.s_int + at * I_SIZE;
            const int64_t ord = static_order_key(P, b, ints, s.s_keys + at * s.B * 3);
            if (ord >= NOT_A_CANDIDATE) continue;
            double toi;
            V3 lc;
            if (!static_values(P, b, s.s_geo + at * G_SIZE, ints, &toi, &lc)) continue;
            sc.push_back({ord, ints[I_PARENT], ints[I_ID], j, toi, lc});
        }
        std::stable_sort(sc.begin(), sc.end(), [](const SC& x, const SC& y) {
            if (x.order != y.order) return x.order < y.order;
            if (x.parent != y.parent) return x.parent < y.parent;
            if (x.id != y.id) return x.id < y.id;
            return x.slot < y.slot;
        });
        for (const SC& e : sc) {                                      // no later-impact test; the stronger at a tie
            const bool eq = e.toi == me.last_collision;
            if (!eq || dot(e.lc, e.lc) > dot(me.last_c, me.last_c)) me.last_c = e.lc;
            if (!eq) me.last_collision = e.toi;
            me.hits.push_back(e.id);
        }
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
