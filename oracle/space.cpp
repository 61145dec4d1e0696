// TEST INFRASTRUCTURE, NOT THE PRODUCT. The master's partition and bubble partition of one world, restated as a plain
// sequential C++ program from the reference's scalar transcription (exact_ballpark/space.py: Partition's GetBox,
// CheckBox and the BoxAllocator, space.py:596-676; Ball::InsertInBoxes and DeleteFromBoxes, :683-818; NearbyBubbles,
// Traverse, AddToBubble, InitializeBubbles, CopyBubbles, InDeadBubble, :896-1056; AddBall, the re-filing setters and
// RemoveBall, :1097-1319). A world is driven by a list of operations and its state is printed after each one, as a text
// the tests compare with the reference's own state on the same operations (tests/golden/space_trace.py).
//
// Boxes are made on demand with their parents and released when empty; a released box's memory is kept (up to 256
// boxes, BoxAllocator's free list) or deleted, and Destiny reads a released box in one path (a ball that was its
// box's only occupant): every box ever made is kept here, so that read sees the stale values, and a read of a deleted
// box sets `undefined` (Destiny's result is undefined there). Balls, bubbles and the bubble dictionaries keep the
// reference's insertion orders; the queries (GetNearbyBalls' walk, CheckVisibility, GetBallIdsInRange,
// GetBubbleAtCoordinates) read them; the proximity sensors (AddProximitySensor, HandleProximities: the candidates of
// GetNearbyBalls with the inflated radius, the ball re-filed twice, enter and leave in the unordered maps' order).
// Notification ranges (of a goto point or a followed ball), target tracking and a shuffled sensor's first period (glibc's rand) too. The follow
// modes (FOLLOW, ORBIT, WARP, with the targets' follower sets and StopAllFollowers) and the tick are too: the flight
// oracle's tick of every ball (a dead bubble's balls marked so that it skips them and others still read them), a warp's
// drop-out re-filed at its drop-out point and each massive ball's Gradient (Potential with GetNearbyBalls' candidates,
// space.py:1609-1735) at their turns in phase 3, through the flight oracle's hooks, then the re-filings of the balls
// that moved, HandleProximities. The iterative collision method is not in this slice.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <utility>
#include <vector>

#include "../exact_ballpark_b200/csrc/ebb_libm.cuh"
#include "flight_state.h"

namespace space_oracle {

constexpr int NUM_LEVELS = 8;
constexpr double GRID_UNIT = 480.0;
constexpr int BOX_KEEP = 256;                              // BoxAllocator's kept boxes

double level_width(int i) { return double(int64_t(1) << (2 * NUM_LEVELS)) * GRID_UNIT * 0.25 / double(int64_t(1) << (2 * i)); }
int64_t level_grid(int i) { return int64_t(1) << (2 * i - 2 * NUM_LEVELS + 39); }

using Key = std::array<int64_t, 3>;

int64_t to_int64(double x) {                               // int64_t(x) as aarch64 converts: NaN 0, saturating
    if (x != x) return 0;
    if (x >= 9223372036854775808.0) return INT64_MAX;
    if (x < -9223372036854775808.0) return INT64_MIN;
    return (int64_t)x;
}

Key clamp(int64_t ix, int64_t iy, int64_t iz, int64_t n) {
    auto c = [n](int64_t i) { return i < 0 ? int64_t(0) : (i >= n ? n - 1 : i); };
    return Key{c(ix), c(iy), c(iz)};
}

// an insertion-ordered map (the reference's dicts)
template <class V>
struct Ordered {
    std::vector<std::pair<int64_t, V>> items;
    V* find(int64_t k) {
        for (auto& kv : items)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
    V& add(int64_t k, V v) {
        items.emplace_back(k, std::move(v));
        return items.back().second;
    }
    void erase(int64_t k) {
        for (size_t i = 0; i < items.size(); ++i)
            if (items[i].first == k) {
                items.erase(items.begin() + i);
                return;
            }
    }
};

// std::unordered_map<int64_t, ...>'s iteration order under libstdc++'s prime rehash policy (space.py:193-322, the
// reference's clean-room statement of it; max load factor 1): a fresh map has one bucket and its first insertion asks
// for room for 11 keys, which gives 13 buckets; a key past the bucket count grows the table to the first bucket count
// of the library's prime list at or above twice the old count (the policy's want: the larger of the keys plus one and
// twice the buckets), and the keys are re-linked one at a time in their old order. Up to 257 buckets that list holds
// every prime (its first gaps come after 257), so the counts a map of up to 257 keys reaches, 13, 29, 59, 127 and 257,
// are found here by trial division; a 258th key is outside this oracle (`overflow`). A key is linked just before the
// first key of the order in its bucket (the key modulo the bucket count, as an unsigned 64-bit value), else at the
// front; erasures and clear() keep the other keys' order and the bucket count.
struct HashOrder {
    std::vector<int64_t> order;
    uint64_t buckets = 1;
    bool overflow = false;
    static bool prime(uint64_t n) {
        if (n < 2) return false;
        for (uint64_t d = 2; d * d <= n; ++d)
            if (n % d == 0) return false;
        return true;
    }
    bool contains(int64_t k) const { return std::find(order.begin(), order.end(), k) != order.end(); }
    void link(int64_t k) {
        const uint64_t b = (uint64_t)k % buckets;
        for (size_t i = 0; i < order.size(); ++i)
            if ((uint64_t)order[i] % buckets == b) {
                order.insert(order.begin() + i, k);
                return;
            }
        order.insert(order.begin(), k);
    }
    void insert(int64_t k) {
        if (contains(k)) return;
        if (buckets == 1) {
            buckets = 13;
        } else if (order.size() + 1 > buckets) {
            if (buckets >= 257) overflow = true;
            uint64_t n = 2 * buckets;
            while (!prime(n)) ++n;
            buckets = n;
            const std::vector<int64_t> old = order;
            order.clear();
            for (int64_t x : old) link(x);
        }
        link(k);
    }
    void erase(int64_t k) {
        auto it = std::find(order.begin(), order.end(), k);
        if (it != order.end()) order.erase(it);
    }
};

// glibc's rand() after srand(seed) (random_r's TYPE_3: degree 31, separation 3; glibc's published algorithm): a
// shuffled sensor's first period (floatrand, Ball.cpp:19)
struct GlibcRand {
    int32_t t[31];
    int f = 3, r = 0;
    explicit GlibcRand(uint32_t seed) {
        int32_t word = (int32_t)(seed == 0 ? 1u : seed);
        t[0] = word;
        for (int i = 1; i < 31; ++i) {
            const int32_t hi = word / 127773, lo = word % 127773;
            word = 16807 * lo - 2836 * hi;
            if (word < 0) word += 2147483647;
            t[i] = word;
        }
        for (int i = 0; i < 310; ++i) next();
    }
    int32_t next() {
        const uint32_t val = (uint32_t)t[f] + (uint32_t)t[r];
        t[f] = (int32_t)val;
        if (++f >= 31) {
            f = 0;
            ++r;
        } else if (++r >= 31) {
            r = 0;
        }
        return (int32_t)(val >> 1);
    }
};

struct Ball;

struct Box {
    int level;
    Key key;
    double lo[3], hi[3];
    Box* parent = nullptr;
    std::map<Key, Box*> children;
    std::map<int64_t, Ball*> balls;
    int64_t bubble = -1;
    bool released = false, deleted = false, handled = false;
};

struct Ball {
    int64_t id;
    double mass = 0.0, radius = 0.0, max_vel = 0.0, agility = 1.0, speed_fraction = 1.0, time_factor = 1.0;
    double pos[3] = {1e10, 1e10, 1e10}, vel[3] = {0.0, 0.0, 0.0};
    bool free = false, interactive = false, massive = false, handled = false;
    int64_t cloaked = 0;
    bool sensor_active = false, sensor_only_interactives = false, has_proximity = false;
    float sensor_range = 0.0f;
    double sensor_period = 2.0, sensor_elapsed = 0.0;
    HashOrder sensor_balls;
    int mode = 2;                                          // GOTO 0, FOLLOW 1, STOP 2, WARP 3, ORBIT 4
    double old_pos[3] = {0.0, 0.0, 0.0}, old_vel[3] = {0.0, 0.0, 0.0}, last_g[3] = {0.0, 0.0, 0.0};
    int64_t follow_ptr = 0, follow_id = 0, owner_id = 0, effect_stamp = 0;   // follow_ptr: the target's id, 0 none
    float follow_range = 10.0f;
    double last_collision = -1.0, last_c[3] = {0.0, 0.0, 0.0};
    HashOrder followers;
    double goto_pt[3] = {0.0, 0.0, 0.0};
    double notification_range = 0.0, tracking_range = 0.0;
    bool within_range = false, within_tracking = false;
    Ball* tracking = nullptr;                              // mTrackingPtr: the ball itself, which may outlive removal
    int64_t bubble = -1, old_bubble = -1;
    std::map<Key, Box*> boxes;
    Box* my_box = nullptr;
    int mod[3] = {-2, -2, -2};
    bool active[27] = {};
};

float f32(double x) { return (float)x; }

struct World {
    double friction, dt;
    std::map<Key, Box*> levels[NUM_LEVELS];                // the live boxes
    std::vector<std::unique_ptr<Box>> made;                // every box ever made (stale reads)
    int free_boxes = 0;
    Ordered<std::unique_ptr<Ball>> balls;                  // mBalls, in the order of their first filing
    Ordered<Ordered<int>> bubbles;                         // bubble -> {ball: +1, 0, -1}
    std::map<int64_t, std::set<int64_t>> interactives, keep_alives;
    std::set<int64_t> keep_alive_balls;
    int64_t bubble_id = 0;
    bool undefined = false;
    HashOrder proximity;                                   // mProximityBalls
    std::vector<std::unique_ptr<Ball>> removed;            // removed balls a tracking pointer may still read
    GlibcRand rng{1};
    int64_t current_time = 0;

    Ball* ball(int64_t id) {
        auto* p = balls.find(id);
        return p ? p->get() : nullptr;
    }

    // ---- the partition ----
    Box* get_box(int64_t ix, int64_t iy, int64_t iz, int level) {
        if (level < 0 || level >= NUM_LEVELS) return nullptr;
        const Key k = clamp(ix, iy, iz, level_grid(level));
        auto it = levels[level].find(k);
        if (it != levels[level].end()) return it->second;
        if (free_boxes > 0) --free_boxes;
        made.emplace_back(new Box());
        Box* b = made.back().get();
        b->level = level;
        b->key = k;
        const double w = level_width(level), n = (double)level_grid(level), center = w * n * 0.5;
        for (int i = 0; i < 3; ++i) {
            b->lo[i] = (double)k[i] * w - center;
            b->hi[i] = (double)(k[i] + 1) * w - center;
        }
        if (level != 0) {
            b->parent = get_box(k[0] >> 2, k[1] >> 2, k[2] >> 2, level - 1);
            b->parent->children[k] = b;
        }
        levels[level][k] = b;
        return b;
    }
    Box* check_box(int64_t ix, int64_t iy, int64_t iz, int level) {
        if (level < 0 || level >= NUM_LEVELS) return nullptr;
        auto it = levels[level].find(clamp(ix, iy, iz, level_grid(level)));
        return it == levels[level].end() ? nullptr : it->second;
    }
    static int level_for(double radius) {
        int level = 0;
        for (int i = 0; i < NUM_LEVELS; ++i) {
            if (3.0 * radius > level_width(i)) break;
            level = i;
        }
        return level;
    }
    static Key key_for(int level, const double* pos) {
        const double w = level_width(level), fac = 1.0 / w, half = 0.5 * w * (double)level_grid(level);
        return Key{to_int64((pos[0] + half) * fac), to_int64((pos[1] + half) * fac), to_int64((pos[2] + half) * fac)};
    }
    Box* get_box_r(double radius, const double* pos) {
        const int level = level_for(radius);
        const Key k = key_for(level, pos);
        return get_box(k[0], k[1], k[2], level);
    }
    static Box* topmost(Box* b) {
        while (b && b->parent) b = b->parent;
        return b;
    }
    void release(Box* box) {
        const bool keep = free_boxes < BOX_KEEP;
        if (box->parent) {
            Box* p = box->parent;
            p->children.erase(box->key);
            if (p->children.empty() && p->balls.empty()) release(p);
        }
        levels[box->level].erase(box->key);
        box->released = true;
        if (keep)
            ++free_boxes;
        else
            box->deleted = true;
    }
    Box* stale(Box* b) {
        if (b->deleted) undefined = true;
        return b;
    }
    void box_remove_ball(Box* box, Ball* b) {
        box->balls.erase(b->id);
        if (box->children.empty() && box->balls.empty()) release(box);
    }
    static void clear_boxes(Ball* b) {
        b->boxes.clear();
        b->my_box = nullptr;
        std::fill(b->active, b->active + 27, false);
        b->mod[0] = b->mod[1] = b->mod[2] = -2;
    }
    void delete_from_boxes(Ball* b) {
        std::vector<Box*> order;
        for (auto& kv : b->boxes) order.push_back(kv.second);    // in key order
        for (Box* box : order) box_remove_ball(box, b);
        clear_boxes(b);
    }
    static void insert_in_box(Ball* b, Box* box) {
        if (!box) return;
        box->balls[b->id] = b;
        b->boxes[box->key] = box;
    }
    double inflated_radius(const Ball* b) const {         // a free ball's radius plus a tick at full thrust
        if (!b->free) return b->radius;
        const double m = b->mass * b->agility;
        const double a = friction * b->speed_fraction * b->max_vel / m;
        const double v = std::sqrt(b->vel[0] * b->vel[0] + b->vel[1] * b->vel[1] + b->vel[2] * b->vel[2]);
        const double k = friction;
        const double max_speed = (m * a - (m * a - v * k) * b->time_factor) / k;
        return b->radius + dt * max_speed;
    }

    // ---- bubbles ----
    int64_t nearby_bubbles(Box* box) {
        for (int i = -1; i <= 1; ++i)
            for (int j = -1; j <= 1; ++j)
                for (int k = -1; k <= 1; ++k) {
                    if (i == 0 && j == 0 && k == 0) continue;
                    Box* o = check_box(box->key[0] + i, box->key[1] + j, box->key[2] + k, box->level);
                    if (o && o->bubble != -1) return o->bubble;
                }
        return -1;
    }
    void traverse(Box* box, int64_t seed) {
        if (box->bubble != -1) return;
        box->bubble = seed;
        for (int i = -1; i <= 1; ++i)
            for (int j = -1; j <= 1; ++j)
                for (int k = -1; k <= 1; ++k) {
                    if (i == 0 && j == 0 && k == 0) continue;
                    Box* o = check_box(box->key[0] + i, box->key[1] + j, box->key[2] + k, box->level);
                    if (o) traverse(o, seed);
                }
    }
    void add_to_bubble(Ball* b) {
        if (b->bubble != -1) {
            Ordered<int>* nb = bubbles.find(b->bubble);
            if (!nb) nb = &bubbles.add(b->bubble, Ordered<int>());
            int* v = nb->find(b->id);
            if (!v)
                nb->add(b->id, 1);
            else if (*v == -1)
                *v = 0;
        }
        if (b->old_bubble != -1) {
            Ordered<int>* ob = bubbles.find(b->old_bubble);
            if (ob) {
                int* v = ob->find(b->id);
                if (v) {
                    if (*v == 0)
                        *v = -1;
                    else if (*v == 1)
                        ob->erase(b->id);
                }
            }
        }
        if (b->interactive) {
            increase_interactive(b, b->bubble);
            decrease_interactive(b, b->old_bubble);
        }
        if (keep_alive_balls.count(b->id)) {
            if (b->bubble != -1) keep_alives[b->bubble].insert(b->id);
            if (b->old_bubble != -1) {
                auto it = keep_alives.find(b->old_bubble);
                if (it != keep_alives.end()) {
                    it->second.erase(b->id);
                    if (it->second.empty()) keep_alives.erase(it);
                }
            }
        }
    }
    void increase_interactive(const Ball* b, int64_t bubble) {
        if (b->interactive && bubble != -1) interactives[bubble].insert(b->id);
    }
    void decrease_interactive(const Ball* b, int64_t bubble) {
        if (!b->interactive || bubble == -1) return;
        auto it = interactives.find(bubble);
        if (it == interactives.end()) return;
        it->second.erase(b->id);
        if (it->second.empty()) interactives.erase(it);
    }
    bool in_dead_bubble(const Ball* b) const {
        if (b->mode == 3) return false;                    // a warping (or aligning) ball never is
        auto i = interactives.find(b->bubble);
        if (i != interactives.end() && !i->second.empty()) return false;
        auto k = keep_alives.find(b->bubble);
        if (k != keep_alives.end() && !k->second.empty()) return false;
        return true;
    }

    // ---- filing ----
    void ball_insert_in_boxes(Ball* b, Box* box1, int64_t new_bubble) {
        const double inflated = inflated_radius(b);
        if (box1->released) stale(box1);
        int mod[3] = {0, 0, 0};
        for (int q = 0; q < 3; ++q) {
            if (box1->lo[q] + inflated - b->pos[q] > 0.0)
                mod[q] = -1;
            else if (box1->hi[q] - inflated - b->pos[q] < 0.0)
                mod[q] = 1;
        }
        if (b->my_box && box1->level == b->my_box->level && box1->key == b->my_box->key && mod[0] == b->mod[0] &&
            mod[1] == b->mod[1] && mod[2] == b->mod[2])
            return;
        delete_from_boxes(b);
        for (int q = 0; q < 3; ++q) b->mod[q] = mod[q];
        box1 = get_box_r(inflated, b->pos);
        const int64_t ix = box1->key[0], iy = box1->key[1], iz = box1->key[2];
        const int level = box1->level;
        insert_in_box(b, box1);
        topmost(box1)->bubble = new_bubble;                 // (the master)
        b->active[13] = true;
        b->my_box = box1;
        if (level == 0 && (double)(f32(b->radius) * 2.0f) > level_width(0)) {   // a huge ball: every neighbour
            for (int x = -1; x <= 1; ++x)
                for (int y = -1; y <= 1; ++y)
                    for (int z = -1; z <= 1; ++z) {
                        if (x == 0 && y == 0 && z == 0) continue;
                        insert_in_box(b, get_box(ix + x, iy + y, iz + z, 0));
                        b->active[13 + x + 3 * y + 9 * z] = true;
                    }
            return;
        }
        const int mx = mod[0], my = mod[1], mz = mod[2];
        auto side = [&](int x, int y, int z) {
            insert_in_box(b, get_box(ix + x, iy + y, iz + z, level));
            b->active[13 + x + 3 * y + 9 * z] = true;
        };
        if (mx) side(mx, 0, 0);
        if (my) side(0, my, 0);
        if (mz) side(0, 0, mz);
        if (mx && my) side(mx, my, 0);
        if (mx && mz) side(mx, 0, mz);
        if (my && mz) side(0, my, mz);
        if (mx && my && mz) side(mx, my, mz);
    }
    void insert_in_boxes(Ball* b) {                        // Ballpark::InsertInBoxes on the master
        const double inflated = inflated_radius(b);
        Box* box1 = get_box_r(inflated, b->pos);
        Box* top = topmost(box1);
        int64_t new_bubble = top->bubble;
        if (new_bubble == -1) {
            delete_from_boxes(b);                           // may release box1 and top: both still read
            b->my_box = nullptr;
            new_bubble = nearby_bubbles(stale(top));
            if (new_bubble == -1) new_bubble = bubble_id++;
            stale(top)->bubble = new_bubble;
        }
        if (b->bubble != new_bubble) {
            b->old_bubble = b->bubble;
            b->bubble = new_bubble;
            add_to_bubble(b);
        }
        ball_insert_in_boxes(b, box1, new_bubble);
    }
    void refresh_time_factor(Ball* b) {
        const double m = b->mass * b->agility;
        b->time_factor = (m <= 0.0) ? 0.0 : std::exp(-friction * dt / m);
    }

    // ---- the operations ----
    void add_ball(int64_t id, double mass, double radius, double max_vel, bool free, bool interactive, const double* p,
                  const double* v, double agility, double sf, bool massive) {
        const float r = f32(radius), mv = f32(max_vel), ag = f32(agility), s = f32(sf);
        Ball* b = ball(id);
        const bool created = b == nullptr;
        if (created) {
            std::unique_ptr<Ball> nb(new Ball());
            nb->id = id;
            b = nb.get();
            balls.add(id, std::move(nb));
        } else {
            delete_from_boxes(b);
        }
        for (int i = 0; i < 3; ++i) {
            b->pos[i] = p[i];
            b->vel[i] = v[i];
        }
        if (created) {
            for (int i = 0; i < 3; ++i) {
                b->old_pos[i] = b->pos[i] - b->vel[i] * dt;
                b->old_vel[i] = b->vel[i];
            }
        } else {                                           // a re-added ball keeps its target pointer and set entry
            b->effect_stamp = 0;
            b->owner_id = 0;
            b->follow_id = 0;
            b->follow_range = 10.0f;
        }
        b->mode = 2;
        b->radius = r < 0.0f ? 0.0 : (double)r;
        b->mass = mass < 0.0 ? 0.0 : mass;
        b->free = free;
        b->interactive = interactive;
        b->massive = massive;
        b->max_vel = mv < 0.0f ? 0.0 : (double)mv;
        b->agility = ag <= 0.0f ? 1.0 : (double)ag;
        b->speed_fraction = s < 0.0f ? 0.0 : (double)s;
        refresh_time_factor(b);
        if (!created) {                                    // its own set loses the entries that no longer follow it
            const std::vector<int64_t> ids = b->followers.order;
            for (int64_t fid : ids) {
                const Ball* f = ball(fid);
                if (!f || f->follow_ptr != b->id) b->followers.erase(fid);
            }
        }
        insert_in_boxes(b);
    }
    void set_position(int64_t id, const double* p) {
        Ball* b = ball(id);
        if (!b) return;
        for (int i = 0; i < 3; ++i) b->pos[i] = b->old_pos[i] = p[i];
        insert_in_boxes(b);
    }
    void set_radius(int64_t id, double radius) {
        Ball* b = ball(id);
        const float r = f32(radius);
        if (!b || r < 0.0f) return;
        b->radius = r;
        insert_in_boxes(b);
    }
    void set_max_velocity(int64_t id, double v) {
        const float mv = f32(v);
        Ball* b = ball(id);
        if (mv < 0.0f || !b) return;
        b->max_vel = mv;
        insert_in_boxes(b);
    }
    void remove_ball(int64_t id) {
        Ball* b = ball(id);
        if (!b) return;
        stop_ball(b);
        stop_all_followers(b);
        delete_from_boxes(b);
        b->old_bubble = b->bubble;
        b->bubble = -1;
        add_to_bubble(b);
        if (b->has_proximity) proximity.erase(id);
        for (auto& kv : balls.items)
            if (kv.first == id) removed.push_back(std::move(kv.second));
        balls.erase(id);
    }
    void set_interactive(int64_t id, bool flag) {
        Ball* b = ball(id);
        if (!b) return;
        if (flag && !b->interactive) {
            b->interactive = true;
            increase_interactive(b, b->bubble);
        } else if (!flag && b->interactive) {
            decrease_interactive(b, b->bubble);
            b->interactive = false;
        }
    }
    void initialize_bubbles() {
        for (auto& kv : levels[0]) kv.second->bubble = -1;
        bubble_id = 0;
        bubbles.items.clear();
        interactives.clear();
        keep_alives.clear();
        keep_alive_balls.clear();
        std::vector<Ball*> order;
        for (auto& kv : balls.items) order.push_back(kv.second.get());
        for (Ball* b : order) {
            if (!b->my_box) {
                b->old_bubble = b->bubble;
                b->bubble = -1;
                continue;
            }
            Box* top = topmost(b->my_box);
            if (top->bubble != -1) {
                b->old_bubble = b->bubble;
                b->bubble = top->bubble;
                add_to_bubble(b);
                continue;
            }
            traverse(top, bubble_id);
            b->old_bubble = b->bubble;
            b->bubble = bubble_id;
            add_to_bubble(b);
            ++bubble_id;
        }
    }
    void copy_bubbles() {
        std::vector<int64_t> dead;
        for (auto& kv : bubbles.items) {
            std::vector<int64_t> gone;
            for (auto& e : kv.second.items) {
                if (e.second == 1)
                    e.second = 0;
                else if (e.second == -1)
                    gone.push_back(e.first);
            }
            for (int64_t g : gone) kv.second.erase(g);
            if (kv.second.items.empty()) dead.push_back(kv.first);
        }
        for (int64_t d : dead) bubbles.erase(d);
    }

    // ---- the queries (space.py:819-895, 1057-1061, 1524-1611) ----
    static double lensq(const double* v) { return v[0] * v[0] + v[1] * v[1] + v[2] * v[2]; }
    static double dot(const double* u, const double* v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; }

    void explode_children(Box* box, std::vector<Box*>& out) {
        for (auto& kv : box->children) {
            explode_children(kv.second, out);
            if (!kv.second->balls.empty()) out.push_back(kv.second);
        }
    }
    // GetNearbyBalls: the ball's boxes, their ancestors holding balls and their descendants, then the balls in them that
    // pass the filter, each once, in box order and then id order (no missiles, fields or global balls in this slice)
    std::vector<Ball*> nearby_balls(Ball* b, bool exclude_fixed, bool exclude_inert, bool exclude_cloaked) {
        std::vector<Ball*> uni;
        if (exclude_inert) {
            auto it = interactives.find(b->bubble);
            if (it == interactives.end() || it->second.empty()) return uni;
        }
        std::vector<Box*> s_boxes;
        for (auto& kv : b->boxes) {
            Box* box = kv.second;
            if (box->handled) continue;
            Box* p = box;
            while (p->parent) {
                p = p->parent;
                if (p->handled) break;
                if (!p->balls.empty()) {
                    s_boxes.push_back(p);
                    p->handled = true;
                }
            }
            explode_children(box, s_boxes);
            if (box->balls.size() > 1) {
                s_boxes.push_back(box);
                box->handled = true;
            }
        }
        for (Box* box : s_boxes) {
            box->handled = false;
            for (auto& kv : box->balls) {
                Ball* o = kv.second;
                if (o->handled || o == b) continue;
                if (exclude_cloaked && (o->cloaked || !o->massive)) continue;
                if (exclude_inert) {
                    if (!o->interactive) continue;
                } else {
                    if (o->bubble != b->bubble) continue;
                    if (exclude_fixed && !o->free) continue;
                }
                o->handled = true;
                uni.push_back(o);
            }
        }
        for (Ball* o : uni) o->handled = false;
        return uni;
    }
    int64_t check_visibility(int64_t src_id, int64_t dst_id) {
        Ball *src = ball(src_id), *dst = ball(dst_id);
        if (!src || !dst || src->bubble != dst->bubble) return -2;
        double ray[3] = {dst->pos[0] - src->pos[0], dst->pos[1] - src->pos[1], dst->pos[2] - src->pos[2]};
        const double distance = std::sqrt(lensq(ray));
        const double norm = std::sqrt(ray[0] * ray[0] + ray[1] * ray[1] + ray[2] * ray[2]);
        if (norm != 0.0) {
            const double inv = 1.0 / norm;
            for (double& x : ray) x = x * inv;
        }
        for (auto& kv : balls.items) {
            Ball* o = kv.second.get();
            if (o->bubble != src->bubble || o == src || o == dst || !o->massive || o->cloaked) continue;
            const double to_center[3] = {o->pos[0] - src->pos[0], o->pos[1] - src->pos[1], o->pos[2] - src->pos[2]};
            const double v = dot(ray, to_center), r = o->radius;
            const double dsq = r * r - (dot(to_center, to_center) - v * v);
            if (dsq < 0.0) continue;
            const double d = std::sqrt(dsq);
            if (v - d > 0.0 && v - d < distance) return o->id;
        }
        return 0;
    }
    int64_t top_bubble_at(const double* p) {               // the existing top box's bubble, or -2 for none
        const Key k = key_for(level_for(10000000.0), p);
        Box* top = check_box(k[0], k[1], k[2], level_for(10000000.0));
        return top ? top->bubble : -2;
    }
    // GetBallIdsInRange (and with distances): the balls listed in the bubble's dictionary, in its order
    std::string in_range(Ball* ref, const double* center, int64_t bubble_id, double range, bool cloaked, bool dist) {
        std::string out;
        char buf[96];
        if (bubble_id == -1) return out;
        Ordered<int>* dict = bubbles.find(bubble_id);
        if (!dict) return out;
        std::vector<int64_t> ids;
        for (auto& e : dict->items) ids.push_back(e.first);
        for (int64_t id : ids) {
            Ball* o = ball(id);
            if (!o || o == ref) continue;
            if (o->cloaked && !cloaked) continue;
            const double d[3] = {o->pos[0] - center[0], o->pos[1] - center[1], o->pos[2] - center[2]};
            const double d2 = lensq(d), lim = range + o->radius;
            if (d2 <= lim * lim) {
                if (dist) {
                    uint64_t bits;
                    std::memcpy(&bits, &d2, 8);
                    snprintf(buf, sizeof buf, " %016llx:%lld", (unsigned long long)bits, (long long)o->id);
                } else {
                    snprintf(buf, sizeof buf, " %lld", (long long)o->id);
                }
                out += buf;
            }
        }
        return out;
    }

    // ---- proximity sensors (space.py:1345-1523; SEN-701, SEN-702; no notification range or tracking here) ----
    void update_proximity_status(Ball* b) {
        b->has_proximity = b->tracking_range != 0.0 || b->notification_range != 0.0 || b->sensor_active;
        if (b->has_proximity)
            proximity.insert(b->id);
        else
            proximity.erase(b->id);
    }
    void add_sensor(int64_t id, double range, double period, bool only_interactives, bool shuffle) {
        Ball* b = ball(id);
        if (!b) return;
        const float r = f32(range);
        if (f32((double)f32(b->radius) + (double)r) < 0.0f) return;
        b->sensor_balls.order.clear();
        b->sensor_range = r;
        b->sensor_period = period;
        b->sensor_active = true;
        b->sensor_only_interactives = only_interactives;
        if (shuffle) b->sensor_elapsed = 0.0 + (double)rng.next() / 2147483647.0 * (b->sensor_period - 0.0);
        update_proximity_status(b);
    }
    void set_notification_range(int64_t id, double n) {
        Ball* b = ball(id);
        if (!b || n < 0.0) return;
        b->notification_range = n;
        update_proximity_status(b);
        b->within_range = false;
    }
    void set_target_tracking(int64_t id, int64_t target, double range) {
        Ball* b = ball(id);
        if (!b) return;
        if (range <= 0.0 || target == 0) {
            b->tracking = nullptr;
            b->tracking_range = 0.0;
            return;
        }
        Ball* t = ball(target);
        if (!t) return;
        b->tracking = t;
        b->tracking_range = range;
        update_proximity_status(b);
        b->within_tracking = false;
    }
    // ---- collisions inside the tick: Gradient and Potential (space.py:1609-1735) ----
    // Ballpark::Integrate over t seconds: nothing for t = 0, the ball's cached factor for a whole tick, else glibc's
    // exp(-k t / m)
    void integrate(double* p, double* v, const double* a, double m, double tf, double t) const {
        if (t == 0.0) return;
        const double k = friction;
        if (t != dt) tf = ebb::lm::exp((-k / m) * t);
        const double k2 = k * k, ook2 = 1.0 / k2, ook = 1.0 / k;
        double pn[3], vn[3];
        if (k < 1e-10 * m * t) {
            const double inv_m = 1.0 / m;
            for (int i = 0; i < 3; ++i)
                pn[i] = (m * (a[i] * (-k * t) + k * (a[i] * t + v[i] * k * inv_m * t)) + p[i] * k2) * ook2;
        } else {
            for (int i = 0; i < 3; ++i)
                pn[i] = (m * (m * a[i] * (tf - 1.0) + k * (a[i] * t + v[i] - tf * v[i])) + p[i] * k2) * ook2;
        }
        for (int i = 0; i < 3; ++i) vn[i] = (m * a[i] - (m * a[i] - v[i] * k) * tf) * ook;
        for (int i = 0; i < 3; ++i) {
            p[i] = pn[i];
            v[i] = vn[i];
        }
    }
    // CollideTwoSpheres: 0 when already touching, else the earlier root of the closing quadratic in [0, 1], or -1
    static double collide_two_spheres(const double* p0, const double* p1, const double* q0, const double* q1,
                                      double cr) {
        const double p0q0[3] = {p0[0] - q0[0], p0[1] - q0[1], p0[2] - q0[2]};
        const double p0q0_2 = dot(p0q0, p0q0);
        if (p0q0_2 <= cr * cr) return 0.0;
        double dpq[3];
        for (int i = 0; i < 3; ++i) dpq[i] = (p1[i] - p0[i]) - (q1[i] - q0[i]);
        const double a = dot(dpq, dpq), b = 2.0 * dot(p0q0, dpq), c = p0q0_2 - cr * cr;
        if (a == 0.0 && b == 0.0) return -1.0;
        double det = b * b - 4.0 * a * c;
        if (det < 0.0) return -1.0;
        det = std::sqrt(det);
        const double s2 = ((-b - det) * 0.5) / a;
        return (s2 >= 0.0 && s2 <= 1.0) ? s2 : -1.0;
    }
    static void normalize(double* v) {
        const double n = std::sqrt(lensq(v));
        if (n == 0.0) return;
        const double inv = 1.0 / n;
        for (int i = 0; i < 3; ++i) v[i] = v[i] * inv;
    }
    // Potential of `me` with `other`: the response to their first contact within the tick, or to an overlap (the pair
    // pushed apart by mass and Potential called again on the pushed positions, twice at most); the latest contact's
    // response kept, the larger of two at the same time
    void potential(Ball* me, Ball* other, int depth) {
        const double cr = me->radius + other->radius;
        const double m1 = me->free ? me->mass * me->agility : 1.0e34;
        const double m2 = other->free ? other->mass * other->agility : 1.0e34;
        const double k = friction;
        double p0[3], q0[3], p1[3], q1[3], vp1[3], vq1[3];
        std::memcpy(p0, me->pos, 24);
        std::memcpy(q0, other->pos, 24);
        std::memcpy(p1, me->pos, 24);
        std::memcpy(vp1, me->vel, 24);
        std::memcpy(q1, other->pos, 24);
        std::memcpy(vq1, other->vel, 24);
        integrate(p1, vp1, me->last_g, m1, me->time_factor, dt);
        integrate(q1, vq1, other->last_g, m2, other->time_factor, dt);
        const double sv = collide_two_spheres(p0, p1, q0, q1, cr);
        if (sv == -1.0) return;
        std::memcpy(p1, me->pos, 24);
        std::memcpy(vp1, me->vel, 24);
        std::memcpy(q1, other->pos, 24);
        std::memcpy(vq1, other->vel, 24);
        const double tf = me->time_factor;
        double a1[3];
        if (sv > 0.0) {                                    // a contact within the tick: bounce, then fly on
            integrate(p1, vp1, me->last_g, m1, tf, sv * dt);
            integrate(q1, vq1, other->last_g, m2, other->time_factor, sv * dt);
            double normal[3] = {q1[0] - p1[0], q1[1] - p1[1], q1[2] - p1[2]};
            normalize(normal);
            const double v1 = dot(vp1, normal), v2 = dot(vq1, normal);
            if (!other->free) {                            // a fixed ball reflects
                const double c = 2.0 * v1;
                for (int i = 0; i < 3; ++i) vp1[i] = vp1[i] - normal[i] * c;
            } else {                                       // two free balls exchange momentum along the normal
                const double mm1 = me->mass, mm2 = other->mass;
                const double v1p = (mm1 * v1 - mm2 * v1 + 2.0 * mm2 * v2) / (mm1 + mm2);
                for (int i = 0; i < 3; ++i) vp1[i] = vp1[i] + normal[i] * (v1p - v1);
            }
            integrate(p1, vp1, me->last_g, m1, tf, (1.0 - sv) * dt);
            const double inv_m = 1.0 / m1, inv_t = 1.0 / (tf - 1.0);
            const double* g = me->last_g;
            const double* v0 = me->vel;
            for (int i = 0; i < 3; ++i)
                a1[i] = -((((g[i] * -m1) + g[i] * (tf * m1)) - (v0[i] * tf) * k) + vp1[i] * k) * inv_m * inv_t;
        } else {                                           // already overlapping
            const double p0q0[3] = {q0[0] - p0[0], q0[1] - p0[1], q0[2] - p0[2]};
            const double p0q0_2 = dot(p0q0, p0q0);
            double normal[3];
            if (p0q0_2 == 0.0) {
                normal[0] = me->id > other->id ? 1.0 : -1.0;
                normal[1] = normal[2] = 0.0;
            } else {
                for (int i = 0; i < 3; ++i) normal[i] = q1[i] - p1[i];
                normalize(normal);
            }
            const double dist = cr - std::sqrt(p0q0_2) + 1;
            const double d1 = m2 / (m1 + m2) * dist;
            const double d2 = m1 / (m1 + m2) * dist;
            if (me->free && other->free && depth < 2) {
                double keep_me[3], keep_other[3];
                std::memcpy(keep_me, me->pos, 24);
                std::memcpy(keep_other, other->pos, 24);
                for (int i = 0; i < 3; ++i) {
                    me->pos[i] = me->pos[i] - normal[i] * d1;
                    other->pos[i] = other->pos[i] + normal[i] * d2;
                }
                potential(me, other, depth + 1);
                std::memcpy(me->pos, keep_me, 24);
                std::memcpy(other->pos, keep_other, 24);
                if (m2 / m1 > 25.0) {                      // a light ball: the response scaled to the overlap
                    normalize(me->last_c);
                    for (int i = 0; i < 3; ++i) me->last_c[i] = me->last_c[i] * dist;
                }
                const double dv[3] = {me->vel[0] - other->vel[0], me->vel[1] - other->vel[1], me->vel[2] - other->vel[2]};
                if (lensq(dv) > 0.0001) return;
            }
            const double normal_comp = dot(me->last_g, normal);
            const double tmp = 1.0 / (m1 + dt * k);
            const double c = -d1 / (dt * tmp * m1);
            const double inv_dt = 1.0 / dt;
            for (int i = 0; i < 3; ++i) a1[i] = (normal[i] * c - me->vel[i]) * inv_dt - normal[i] * normal_comp;
        }
        if (sv >= me->last_collision) {                    // no missiles here
            double lc[3];
            for (int i = 0; i < 3; ++i) lc[i] = a1[i] * 0.85;
            if (sv == me->last_collision) {
                if (lensq(lc) > lensq(me->last_c)) std::memcpy(me->last_c, lc, 24);
            } else {
                std::memcpy(me->last_c, lc, 24);
                me->last_collision = sv;
            }
        }
    }
    // Gradient: Potential with each of GetNearbyBalls' candidates (massive, uncloaked, in the ball's bubble), in the
    // walk's order
    void gradient(Ball* b) {
        for (Ball* o : nearby_balls(b, false, false, true)) potential(b, o, 0);
    }

    // ---- the modes' commands (modes.py:206-330, 391-426): Stop, GotoPoint, GotoDirection, FollowBall, Orbit, WarpTo,
    // StopAllFollowers, with the targets' follower sets ----
    void stop_ball(Ball* b) {                              // Stop(Ball*)
        if (b->mode == 1 || b->mode == 4) {
            if (Ball* t = ball(b->follow_ptr)) t->followers.erase(b->id);
            b->effect_stamp = 0;
            b->follow_ptr = 0;
            b->follow_id = 0;
            b->owner_id = 0;
            b->follow_range = 0.0f;
        }
        b->mode = 2;
    }
    void stop(int64_t id) {
        Ball* b = ball(id);
        if (b && b->mode != 2) stop_ball(b);
    }
    void goto_ball(Ball* b, const double* p) {
        if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) return;
        stop_ball(b);
        for (int i = 0; i < 3; ++i) b->goto_pt[i] = p[i];
        if (b->speed_fraction == 0.0) b->speed_fraction = 1.0;
        b->mode = 0;
    }
    void goto_point(int64_t id, const double* p) {
        if (Ball* b = ball(id)) goto_ball(b, p);
    }
    void goto_direction(Ball* b, const double* d) {
        if (!std::isfinite(d[0]) || !std::isfinite(d[1]) || !std::isfinite(d[2])) return;
        double u[3] = {d[0], d[1], d[2]};
        const double norm = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        if (norm != 0.0) {
            const double inv = 1.0 / norm;
            for (double& x : u) x = x * inv;
        }
        const double p[3] = {b->pos[0] + u[0] * 1.0e17, b->pos[1] + u[1] * 1.0e17, b->pos[2] + u[2] * 1.0e17};
        goto_ball(b, p);
    }
    void follow(int64_t src, int64_t dst, double range, int mode) {
        const float rng = f32(range);
        if (!std::isfinite(rng)) return;
        Ball* b = ball(src);
        if (!b || src == dst) return;
        Ball* t = ball(dst);
        if (!t || b->bubble != t->bubble || t->cloaked) return;
        stop_ball(b);
        b->follow_id = dst;
        b->follow_ptr = dst;
        b->follow_range = rng;
        b->mode = mode;
        t->followers.insert(b->id);
    }
    void warp_to(int64_t id, const double* p, double min_range, int64_t factor) {
        if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) return;
        if (min_range < 0.0) min_range = 0.0;
        if (factor <= 0) factor = 1;
        Ball* b = ball(id);
        if (!b) return;
        const double d[3] = {b->pos[0] - p[0], b->pos[1] - p[1], b->pos[2] - p[2]};
        if (lensq(d) < 10000000000.0) {                    // within 1e5 m: a GotoPoint
            goto_ball(b, p);
            return;
        }
        if (b->mode == 3 && b->goto_pt[0] == p[0] && b->goto_pt[1] == p[1] && b->goto_pt[2] == p[2]) return;
        stop_ball(b);
        for (int i = 0; i < 3; ++i) b->goto_pt[i] = p[i];
        b->effect_stamp = -1;
        b->follow_range = 0.0f;
        std::memcpy(&b->follow_id, &min_range, 8);
        b->owner_id = factor;
        b->mode = 3;
    }
    void stop_all_followers(Ball* b) {                     // missiles (none here) and interactive orbiters fly on
        if (b->followers.order.empty()) return;
        const std::vector<int64_t> ids = b->followers.order;
        for (int64_t fid : ids) {
            Ball* f = ball(fid);
            if (!f || f->follow_id != b->id || f->follow_ptr != b->id) {
                b->followers.erase(fid);
                continue;
            }
            if (f->interactive && f->mode == 4) {
                const double v[3] = {f->vel[0], f->vel[1], f->vel[2]};
                goto_direction(f, v);
            } else {
                stop_ball(f);
            }
        }
    }
    void check_notification_range(Ball* b, std::string& events) {
        char buf[64];
        bool send = false, inside = false;
        if (b->notification_range != 0.0) {
            const double n = b->notification_range;
            if (b->mode == 0) {                            // GOTO: within the range of the goto point
                const double lim = n + b->radius;
                const double d[3] = {b->pos[0] - b->goto_pt[0], b->pos[1] - b->goto_pt[1], b->pos[2] - b->goto_pt[2]};
                inside = lensq(d) < lim * lim;
            } else if (b->mode == 1 || b->mode == 4) {     // FOLLOW, ORBIT: within a shell of the range's width
                const Ball* o = ball(b->follow_ptr);
                const double d[3] = {b->pos[0] - o->pos[0], b->pos[1] - o->pos[1], b->pos[2] - o->pos[2]};
                const double len2 = lensq(d);
                const double hi = o->radius + (double)b->follow_range + n + b->radius;
                double lo = hi - 2.0 * n;
                if (lo < 0.0) lo = 0.0;
                inside = len2 < hi * hi && len2 > lo * lo;
            }
            if (inside) {
                if (!b->within_range) send = b->within_range = true;
            } else if (b->within_range) {
                send = true;
                b->within_range = false;
            }
        }
        if (send) {
            snprintf(buf, sizeof buf, " R%lld:%d", (long long)b->id, b->within_range ? 1 : 0);
            events += buf;
        }
    }
    void check_target_tracking(Ball* b, std::string& events) {
        char buf[64];
        bool send = false;
        if (b->tracking_range >= 0.00001 && b->tracking) {
            const double d[3] = {b->pos[0] - b->tracking->pos[0], b->pos[1] - b->tracking->pos[1],
                                 b->pos[2] - b->tracking->pos[2]};
            const double lim = b->tracking_range + b->radius;
            if (lensq(d) < lim * lim) {
                if (!b->within_tracking) send = b->within_tracking = true;
            } else if (b->within_tracking) {
                send = true;
                b->within_tracking = false;
            }
        }
        if (send) {
            snprintf(buf, sizeof buf, " T%lld:%d", (long long)b->id, b->within_tracking ? 1 : 0);
            events += buf;
        }
    }
    void check_for_proximity(Ball* b, std::string& events) {
        check_notification_range(b, events);
        check_target_tracking(b, events);
        if (b->sensor_active) check_sensor(b, events);
    }
    void remove_sensor(int64_t id) {
        Ball* b = ball(id);
        if (!b) return;
        b->sensor_active = false;
        update_proximity_status(b);
    }
    void set_ball_radius(Ball* b, float r) {
        if (r < 0.0f) return;
        b->radius = r;
        insert_in_boxes(b);
    }
    void check_sensor(Ball* b, std::string& events) {
        char buf[96];
        b->sensor_elapsed += dt;
        if (b->sensor_elapsed < b->sensor_period) return;
        b->sensor_elapsed = 0.0;
        const double radius = b->radius;
        const double vel[3] = {b->vel[0], b->vel[1], b->vel[2]};
        b->vel[0] = b->vel[1] = b->vel[2] = 0.0;
        set_ball_radius(b, f32((double)f32(b->radius) + (double)b->sensor_range));   // float + float
        const bool exclude_fixed = b->cloaked == 0;
        std::vector<Ball*> uni = nearby_balls(b, exclude_fixed, b->sensor_only_interactives, false);
        for (int i = 0; i < 3; ++i) b->vel[i] = vel[i];
        set_ball_radius(b, (float)radius);
        if (!b->sensor_balls.order.empty()) {
            std::set<int64_t> near;
            for (Ball* o : uni) near.insert(o->id);
            const std::vector<int64_t> keys = b->sensor_balls.order;
            for (int64_t k : keys) {
                if (k == b->id || near.count(k)) continue;
                b->sensor_balls.erase(k);
                snprintf(buf, sizeof buf, " %lld:%lld:0", (long long)b->id, (long long)k);
                events += buf;
                if (!b->sensor_active) break;
            }
        }
        for (Ball* o : uni) {
            if (o->id == b->id) continue;
            const bool inside = b->sensor_balls.contains(o->id);
            const double d[3] = {b->pos[0] - o->pos[0], b->pos[1] - o->pos[1], b->pos[2] - o->pos[2]};
            const double d2 = lensq(d);
            const double ck = (double)f32((double)f32((double)b->sensor_range + (double)f32(o->radius)) +
                                          (double)f32(b->radius));
            if (d2 > ck * ck) {
                if (inside) {
                    b->sensor_balls.erase(o->id);
                    snprintf(buf, sizeof buf, " %lld:%lld:0", (long long)b->id, (long long)o->id);
                    events += buf;
                }
            } else if (!inside) {
                b->sensor_balls.insert(o->id);
                snprintf(buf, sizeof buf, " %lld:%lld:1", (long long)b->id, (long long)o->id);
                events += buf;
            }
            if (!b->sensor_active) break;
        }
    }
    std::string handle_proximities() {
        std::string events;
        const std::vector<int64_t> keys = proximity.order;
        for (int64_t id : keys) {
            Ball* b = ball(id);
            if (!b) continue;
            if (in_dead_bubble(b)) {
                if (!b->sensor_balls.order.empty()) {
                    b->sensor_elapsed = b->sensor_period;
                    check_for_proximity(b, events);
                }
                b->sensor_balls.order.clear();
                continue;
            }
            if (!b->has_proximity) continue;
            check_for_proximity(b, events);
        }
        return events;
    }

    // ---- the tick (space.py's ModeBallpark.evolve with SpaceBallpark's hooks, modes.py:702-745) ----
    // The free balls outside a dead bubble (TIME-714: a dead bubble's balls skip the whole tick) run one flight tick
    // through the flight oracle (GOTO and STOP here, no collisions: the slice's balls are not massive); each that moved
    // at least sqrt(0.1) m is re-filed, in ascending id; then HandleProximities.
    // The flight tick's view of this world: at a hook the balls' flight state is read back from the tick's arrays
    // (the others as they stand at that turn: before their commit, a drop-out of a lower id at its drop-out point), then
    // the ball's Gradient runs on the partition, or its drop-out is re-filed
    struct TickView {
        World* w;
        const std::vector<Ball*>* order;
        const OracleFlight* s;
        void pull() const {
            for (size_t i = 0; i < order->size(); ++i) {
                Ball* b = (*order)[i];
                for (int c = 0; c < 3; ++c) {
                    b->pos[c] = s->pos[3 * i + c];
                    b->vel[c] = s->vel[3 * i + c];
                    b->last_g[c] = s->last_g[3 * i + c];
                }
                b->mode = (int)s->mode[i];
                b->massive = s->massive[i] != 0;
            }
        }
        static void gradient_at(void* ctx, int64_t row) {
            TickView* v = static_cast<TickView*>(ctx);
            v->pull();
            Ball* b = (*v->order)[(size_t)row];
            b->last_collision = -1.0;
            b->last_c[0] = b->last_c[1] = b->last_c[2] = 0.0;
            v->w->gradient(b);
            v->s->last_collision[row] = b->last_collision;
            OracleTickHooks* h = v->hooks;
            for (int c = 0; c < 3; ++c) h->last_c[3 * row + c] = b->last_c[c];
        }
        static void drop_out_at(void* ctx, int64_t row) {
            TickView* v = static_cast<TickView*>(ctx);
            v->pull();
            v->w->insert_in_boxes((*v->order)[(size_t)row]);
        }
        OracleTickHooks* hooks = nullptr;
    };

    std::string tick() {
        std::vector<Ball*> order;
        for (auto& kv : balls.items) order.push_back(kv.second.get());
        std::sort(order.begin(), order.end(), [](const Ball* a, const Ball* b) { return a->id < b->id; });
        const size_t n = order.size();
        std::vector<bool> dead(n, false);
        std::map<int64_t, int64_t> row_of;
        for (size_t i = 0; i < n; ++i) {
            row_of[order[i]->id] = (int64_t)i;
            dead[i] = order[i]->free && in_dead_bubble(order[i]);    // a dead bubble's balls skip the whole tick
        }
        std::vector<int> mode_before(n), warping_before(n);
        std::vector<int64_t> target_before(n);
        for (size_t i = 0; i < n; ++i) {
            mode_before[i] = order[i]->mode;
            warping_before[i] = order[i]->mode == 3 && order[i]->effect_stamp >= 0;
            target_before[i] = order[i]->follow_ptr;
        }
        if (n) {
            std::vector<double> v3[9], v1[12], q4[2];
            for (auto& v : v3) v.assign(3 * n, 0.0);
            for (auto& v : v1) v.assign(n, 0.0);
            for (auto& v : q4) v.assign(4 * n, 0.0);
            std::vector<int64_t> i64[8];
            for (auto& v : i64) v.assign(n, 0);
            std::vector<uint8_t> u8[5];
            for (auto& v : u8) v.assign(n, 0);
            enum { POS, VEL, OPOS, OVEL, GOTO_, LASTG, ANG, OANG, TORQUE };
            enum { MASS, TF, LASTC, RAD, MAXV, AGI, SF, FRANGE, MAXW, ROTAG, ROLL };
            enum { IDS, WORLD, MODE, STAMP, FID, OWNER, FPTR, CLOCK };
            enum { FREE, MORIBUND, MASSIVE, INTERACTIVE, SENSOR };
            for (size_t i = 0; i < n; ++i) {
                const Ball* b = order[i];
                for (int c = 0; c < 3; ++c) {
                    v3[POS][3 * i + c] = b->pos[c];
                    v3[VEL][3 * i + c] = b->vel[c];
                    v3[OPOS][3 * i + c] = b->old_pos[c];
                    v3[OVEL][3 * i + c] = b->old_vel[c];
                    v3[GOTO_][3 * i + c] = b->goto_pt[c];
                    v3[LASTG][3 * i + c] = b->last_g[c];
                }
                q4[0][4 * i + 3] = q4[1][4 * i + 3] = 1.0;
                v1[MASS][i] = b->mass;
                v1[TF][i] = b->time_factor;
                v1[LASTC][i] = b->last_collision;
                v1[RAD][i] = b->radius;
                v1[MAXV][i] = b->max_vel;
                v1[AGI][i] = b->agility;
                v1[SF][i] = b->speed_fraction;
                v1[FRANGE][i] = b->follow_range;
                v1[MAXW][i] = 1.0;
                v1[ROTAG][i] = 0.9;
                i64[IDS][i] = b->id;
                i64[MODE][i] = b->mode;
                i64[STAMP][i] = b->effect_stamp;
                i64[FID][i] = b->follow_id;
                i64[OWNER][i] = b->owner_id;
                auto t = row_of.find(b->follow_ptr);
                i64[FPTR][i] = (b->follow_ptr != 0 && t != row_of.end()) ? t->second : -1;
                i64[CLOCK][i] = current_time;
                u8[FREE][i] = b->free;
                u8[MORIBUND][i] = dead[i];
                u8[MASSIVE][i] = b->massive;
                u8[INTERACTIVE][i] = b->interactive;
                u8[SENSOR][i] = b->sensor_active;
            }
            OracleFlight s{};
            s.n = (int64_t)n;
            s.friction = friction;
            s.dt = dt;
            s.ffriction = (float)friction;
            s.fdt = (float)dt;
            s.pos = v3[POS].data(); s.vel = v3[VEL].data(); s.old_pos = v3[OPOS].data(); s.old_vel = v3[OVEL].data();
            s.goto_ = v3[GOTO_].data(); s.last_g = v3[LASTG].data();
            s.mass = v1[MASS].data(); s.time_factor = v1[TF].data(); s.last_collision = v1[LASTC].data();
            s.radius = v1[RAD].data(); s.max_vel = v1[MAXV].data(); s.agility = v1[AGI].data();
            s.speed_fraction = v1[SF].data(); s.follow_range = v1[FRANGE].data(); s.max_ang_vel = v1[MAXW].data();
            s.rot_agility = v1[ROTAG].data(); s.rot_roll = v1[ROLL].data();
            s.rot = q4[0].data(); s.old_rot = q4[1].data();
            s.ang_vel = v3[ANG].data(); s.old_ang_vel = v3[OANG].data(); s.torque = v3[TORQUE].data();
            s.ids = i64[IDS].data(); s.world = i64[WORLD].data(); s.mode = i64[MODE].data();
            s.effect_stamp = i64[STAMP].data(); s.follow_id = i64[FID].data(); s.owner_id = i64[OWNER].data();
            s.follow_ptr = i64[FPTR].data(); s.clock = i64[CLOCK].data();
            s.free_ = u8[FREE].data(); s.moribund = u8[MORIBUND].data(); s.massive = u8[MASSIVE].data();
            s.interactive = u8[INTERACTIVE].data(); s.sensor = u8[SENSOR].data();
            std::vector<double> last_c(3 * n, 0.0);      // phase 1 clears every ticked ball's mLastC
            TickView view{this, &order, &s};
            OracleTickHooks hooks{last_c.data(), &view, &TickView::gradient_at, &TickView::drop_out_at};
            view.hooks = &hooks;
            oracle_flight_tick_hooked(&s, &hooks);
            for (size_t i = 0; i < n; ++i) {
                Ball* b = order[i];
                for (int c = 0; c < 3; ++c) {
                    b->pos[c] = v3[POS][3 * i + c];
                    b->vel[c] = v3[VEL][3 * i + c];
                    b->old_pos[c] = v3[OPOS][3 * i + c];
                    b->old_vel[c] = v3[OVEL][3 * i + c];
                    b->goto_pt[c] = v3[GOTO_][3 * i + c];
                    b->last_g[c] = v3[LASTG][3 * i + c];
                }
                b->mode = (int)i64[MODE][i];
                b->effect_stamp = i64[STAMP][i];
                b->follow_id = i64[FID][i];
                b->owner_id = i64[OWNER][i];
                b->follow_range = (float)v1[FRANGE][i];
                b->last_collision = v1[LASTC][i];
                b->speed_fraction = v1[SF][i];
                b->massive = u8[MASSIVE][i] != 0;
                b->sensor_active = u8[SENSOR][i] != 0;
                if (i64[FPTR][i] >= 0)                     // a pointer to a removed ball stays as it was
                    b->follow_ptr = order[(size_t)i64[FPTR][i]]->id;
                else if (ball(target_before[i]))
                    b->follow_ptr = 0;
            }
            // a ball that began warp proper released its followers (stale entries too); a follower released in the
            // tick leaves its target's follower set
            for (size_t i = 0; i < n; ++i)
                if (mode_before[i] == 3 && !warping_before[i] && order[i]->mode == 3 && order[i]->effect_stamp >= 0)
                    order[i]->followers.order.clear();
            for (size_t i = 0; i < n; ++i) {
                Ball* b = order[i];
                const bool was = mode_before[i] == 1 || mode_before[i] == 4;
                const bool is = (b->mode == 1 || b->mode == 4) && b->follow_ptr == target_before[i];
                if (was && !is)
                    if (Ball* t = ball(target_before[i])) t->followers.erase(b->id);
            }
        }
        // every ball that moved re-filed (a warp's drop-out was re-filed at its turn, by the hook)
        for (size_t i = 0; i < n; ++i) {
            Ball* b = order[i];
            if (dead[i] || !b->free) continue;
            const double d[3] = {b->pos[0] - b->old_pos[0], b->pos[1] - b->old_pos[1], b->pos[2] - b->old_pos[2]};
            if (!(lensq(d) < 0.1)) insert_in_boxes(b);
        }
        std::string events = handle_proximities();
        ++current_time;
        return events;
    }

    // ---- the state, as text ----
    std::string state() const {
        std::string out;
        char buf[256];
        std::vector<const Ball*> order;
        for (auto& kv : balls.items) order.push_back(kv.second.get());
        std::sort(order.begin(), order.end(), [](const Ball* a, const Ball* b) { return a->id < b->id; });
        for (const Ball* b : order) {
            int active = 0;
            for (int i = 0; i < 27; ++i) active |= (b->active[i] ? 1 : 0) << i;
            if (b->my_box)
                snprintf(buf, sizeof buf, "B %lld %lld %lld %d %lld %lld %lld %d %d %d %d %d", (long long)b->id,
                         (long long)b->bubble, (long long)b->old_bubble, b->my_box->level, (long long)b->my_box->key[0],
                         (long long)b->my_box->key[1], (long long)b->my_box->key[2], b->mod[0], b->mod[1], b->mod[2],
                         active, in_dead_bubble(b) ? 1 : 0);
            else
                snprintf(buf, sizeof buf, "B %lld %lld %lld - %d %d %d %d %d", (long long)b->id, (long long)b->bubble,
                         (long long)b->old_bubble, b->mod[0], b->mod[1], b->mod[2], active, in_dead_bubble(b) ? 1 : 0);
            out += buf;
            for (auto& kv : b->boxes) {
                snprintf(buf, sizeof buf, " %lld,%lld,%lld", (long long)kv.first[0], (long long)kv.first[1],
                         (long long)kv.first[2]);
                out += buf;
            }
            out += "\n";
        }
        out += "L";
        for (int i = 0; i < NUM_LEVELS; ++i) {
            snprintf(buf, sizeof buf, " %zu", levels[i].size());
            out += buf;
        }
        bool overflow = proximity.overflow;
        for (const Ball* b : order) overflow = overflow || b->sensor_balls.overflow;
        snprintf(buf, sizeof buf, "\nF %d %lld %d\n", free_boxes, (long long)bubble_id, (undefined || overflow) ? 1 : 0);
        out += buf;
        if (!proximity.order.empty()) {
            out += "P";
            for (int64_t id : proximity.order) {
                snprintf(buf, sizeof buf, " %lld", (long long)id);
                out += buf;
            }
            out += "\n";
        }
        for (const Ball* b : order) {
            if (!b->sensor_active && b->sensor_balls.order.empty() && !b->has_proximity) continue;
            uint64_t bits;
            std::memcpy(&bits, &b->sensor_elapsed, 8);
            snprintf(buf, sizeof buf, "S %lld %d %016llx %d %d %d %lld", (long long)b->id, b->sensor_active ? 1 : 0,
                     (unsigned long long)bits, b->has_proximity ? 1 : 0, b->within_range ? 1 : 0,
                     b->within_tracking ? 1 : 0, (long long)(b->tracking ? b->tracking->id : 0));
            out += buf;
            for (int64_t id : b->sensor_balls.order) {
                snprintf(buf, sizeof buf, " %lld", (long long)id);
                out += buf;
            }
            out += "\n";
        }
        std::vector<std::pair<int64_t, const Ordered<int>*>> bs;
        for (auto& kv : bubbles.items) bs.emplace_back(kv.first, &kv.second);
        std::sort(bs.begin(), bs.end(), [](auto& a, auto& b) { return a.first < b.first; });
        for (auto& kv : bs) {
            snprintf(buf, sizeof buf, "U %lld", (long long)kv.first);
            out += buf;
            for (auto& e : kv.second->items) {
                snprintf(buf, sizeof buf, " %lld:%d", (long long)e.first, e.second);
                out += buf;
            }
            out += "\n";
        }
        for (auto* m : {&interactives, &keep_alives}) {
            for (auto& kv : *m) {
                snprintf(buf, sizeof buf, "%s %lld", m == &interactives ? "I" : "K", (long long)kv.first);
                out += buf;
                for (int64_t id : kv.second) {
                    snprintf(buf, sizeof buf, " %lld", (long long)id);
                    out += buf;
                }
                out += "\n";
            }
        }
        for (const Ball* b : order) {                      // each ball's mode and flight state, its followers in order
            uint64_t bits[6];
            std::memcpy(bits, b->pos, 24);
            std::memcpy(bits + 3, b->vel, 24);
            snprintf(buf, sizeof buf, "M %lld %d %d %lld", (long long)b->id, b->mode, b->massive ? 1 : 0,
                     (long long)b->follow_ptr);
            out += buf;
            for (uint64_t x : bits) {
                snprintf(buf, sizeof buf, " %016llx", (unsigned long long)x);
                out += buf;
            }
            out += " :";
            for (int64_t id : b->followers.order) {
                snprintf(buf, sizeof buf, " %lld", (long long)id);
                out += buf;
            }
            out += "\n";
        }
        return out;
    }
};

}  // namespace space_oracle

extern "C" {

// Runs n operations of `stride` doubles each on a fresh master world and writes each state after an operation,
// separated by 0x1e, into out[cap]; returns the bytes needed (the text is whole when that is at most cap). An
// operation: its code, then its arguments: 1 AddBall (id, mass, radius, max velocity, free, interactive, x, y, z, vx,
// vy, vz, agility, speed fraction), 2 SetBallPosition (id, x, y, z), 3 SetBallRadius (id, r), 4 SetMaxSpeed (id, v),
// 5 RemoveBall (id), 6 InitializeBubbles, 7 CopyBubbles, 8 SetBallInteractive (id, flag), 9 a keep-alive ball (id),
// 10 the cloak attribute (id, value); the queries, their answer after the state: 11 CheckVisibility (src, dst),
// 12 GetBallIdsInRange from a ball (id, range, include cloaked, with distances), 13 the same from a point (x, y, z,
// range, include cloaked, with distances), 14 GetBubbleAtCoordinates (x, y, z), 15 GetNearbyBalls (id, exclude fixed,
// exclude inert, exclude cloaked); 16 AddProximitySensor (id, range, period, only interactives, shuffle), 17
// RemoveProximitySensor (id), 18 HandleProximities (the answer: each DoProximity event ball:other:entered, DoRange
// R<ball>:<inside>, DoTargetTracking T<ball>:<inside>), 19 SetNotificationRange (id, range), 20 SetTargetTracking (id,
// target, range), 21 GotoPoint (id, x, y, z), 22 Stop (id), 23 a tick (its answer HandleProximities' events), 24
// FollowBall (id, target, range), 25 Orbit (id, target, range), 26 WarpTo (id, x, y, z, min range, warp factor).
// AddBall's sixteenth value is its massive flag. `seed` is the world's srand seed. A negative `cap` runs the operations
// without writing any text (the CPU baseline's timed runs).
int64_t oracle_space_run(const double* ops, int64_t n, int64_t stride, double friction, double dt, int64_t seed,
                         char* out, int64_t cap) {
    space_oracle::World w;
    w.friction = friction;
    w.dt = dt;
    w.rng = space_oracle::GlibcRand((uint32_t)seed);
    std::string all;
    char buf[64];
    for (int64_t i = 0; i < n; ++i) {
        const double* o = ops + i * stride;
        const int code = (int)o[0];
        const int64_t id = (int64_t)o[1];
        std::string answer;
        switch (code) {
            case 1:
                w.add_ball(id, o[2], o[3], o[4], o[5] != 0.0, o[6] != 0.0, o + 7, o + 10, o[13], o[14], o[15] != 0.0);
                break;
            case 10:
                if (space_oracle::Ball* b = w.ball(id)) b->cloaked = (int64_t)o[2] & 0xFF;
                break;
            case 11:
                snprintf(buf, sizeof buf, "Q %lld\n", (long long)w.check_visibility(id, (int64_t)o[2]));
                answer = buf;
                break;
            case 12: {
                space_oracle::Ball* ref = w.ball(id);
                answer = ref ? "Q" + w.in_range(ref, ref->pos, ref->bubble, o[2], o[3] != 0.0, o[4] != 0.0) + "\n"
                             : "Q None\n";
                break;
            }
            case 13: {
                const int64_t top = w.top_bubble_at(o + 2);
                answer = "Q" + w.in_range(nullptr, o + 2, top == -2 ? -1 : top, o[5], o[6] != 0.0, o[7] != 0.0) + "\n";
                break;
            }
            case 14: {
                const int64_t top = w.top_bubble_at(o + 2);
                if (top == -2)
                    answer = "Q None\n";
                else {
                    snprintf(buf, sizeof buf, "Q %lld\n", (long long)top);
                    answer = buf;
                }
                break;
            }
            case 16: w.add_sensor(id, o[2], o[3], o[4] != 0.0, o[5] != 0.0); break;
            case 19: w.set_notification_range(id, o[2]); break;
            case 20: w.set_target_tracking(id, (int64_t)o[2], o[3]); break;
            case 21: w.goto_point(id, o + 2); break;
            case 22: w.stop(id); break;
            case 23: answer = "Q" + w.tick() + "\n"; break;
            case 24: w.follow(id, (int64_t)o[2], o[3], 1); break;
            case 25: w.follow(id, (int64_t)o[2], o[3], 4); break;
            case 26: w.warp_to(id, o + 2, o[5], (int64_t)o[6]); break;
            case 17: w.remove_sensor(id); break;
            case 18: answer = "Q" + w.handle_proximities() + "\n"; break;
            case 15: {
                space_oracle::Ball* b = w.ball(id);
                answer = "Q";
                if (b)
                    for (space_oracle::Ball* x : w.nearby_balls(b, o[2] != 0.0, o[3] != 0.0, o[4] != 0.0)) {
                        snprintf(buf, sizeof buf, " %lld", (long long)x->id);
                        answer += buf;
                    }
                answer += "\n";
                break;
            }
            case 2: w.set_position(id, o + 2); break;
            case 3: w.set_radius(id, o[2]); break;
            case 4: w.set_max_velocity(id, o[2]); break;
            case 5: w.remove_ball(id); break;
            case 6: w.initialize_bubbles(); break;
            case 7: w.copy_bubbles(); break;
            case 8: w.set_interactive(id, o[2] != 0.0); break;
            case 9: w.keep_alive_balls.insert(id); break;
            default: break;
        }
        if (cap < 0) continue;                             // timed runs: the operations alone, no texts
        all += w.state();
        all += answer;
        all += '\x1e';
    }
    const int64_t need = (int64_t)all.size();
    if (need <= cap && out) std::memcpy(out, all.data(), all.size());
    return need;
}

}  // extern "C"
