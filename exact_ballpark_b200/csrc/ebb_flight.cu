// SPDX-License-Identifier: MIT
// The flight-mode tick on sm_100a: the kernels behind include/ebb.h's ebb_flight_* entry points.
//
// A tick of Destiny's Ballpark::Evolve (modes.py:702-745) runs every world's live ships in ascending id: phase 1 (the
// behaviours) reads other ships of the world as they stand at that moment, then phase 3 (the end-of-tick states) and
// phase 4 (the commit). A ship's behaviour reads another ship only through three facts: its start-of-tick position,
// its velocity after its own turn (STOP's vertical damping, once a release before its turn is known), and whether it
// starts warp proper at its turn (then its followers are released: before their own turn when its id is lower, after
// it otherwise). So a tick is two passes: the records pass writes those facts for every ship, then every ship runs
// its whole tick independently, reading other ships only through the records, bit for bit the sequential order.
//
// Two schedules of the same per-ship code (ebb_flight.cuh):
// - plain: the records pass and the tick as two launches over all rows, the records in caller scratch (global);
// - tiled: worlds packed into tiles of whole worlds, one thread block a tile, a persistent grid; the records live in
//   shared memory and both passes run in one launch (one __syncthreads between them), so a tick reads and writes
//   each ship's state once and never touches scratch.
#include <cuda_runtime.h>

#include <atomic>

#include "../../include/ebb.h"
#include "ebb_flight.cuh"
#include "ebb_orient.cuh"
#include "ebb_rows.cuh"

// Resident blocks a multiprocessor is asked to fit (the register budget the compiler gets), per schedule
// (3: 80 registers a thread, 24 warps a multiprocessor; measured fastest for both schedules on B200)
#ifndef EBB_TICK_MIN_BLOCKS
#define EBB_TICK_MIN_BLOCKS 3
#endif
#ifndef EBB_TILED_MIN_BLOCKS
#define EBB_TILED_MIN_BLOCKS 3
#endif

namespace ebb {
namespace flight {

// A ship's tick, first part: the release when its target starts warp proper before its own turn, and the behaviour
// (modes.py:359-377): the thrust, into the orientation step's lane (with dynamical orientation) or as it stands
__device__ __forceinline__ void tick_begin(const EbbFlightState& s, int64_t i, const View& tgt, bool act_self,
                                           DoLane& d, bool* release_after) {
    const int64_t n = s.n;
    const Cfg c = cfg_of(s);
    Ship b = load_ship(s, i);
    const bool live = s.free_[i] && !s.moribund[i];
    *release_after = false;
    if (tgt.valid && tgt.id == b.follow_id && tgt.act) {
        if (tgt.id < b.id) release(b, true);
        else *release_after = true;
    }
    D3 a = D3{0.0, 0.0, 0.0};
    F4 r0 = q_identity();
    if (live) {
        if (s.dynamical) r0 = ldf4(s.rot, i, n);
        if (b.mode == WARP) {                                         // EvolveWarp (modes.py:379)
            if (b.effect_stamp >= 0) {
                a = D3{0.0, 0.0, 0.0};
            } else if (act_self) {
                start_warp(b);
            } else {
                b.effect_stamp -= 1;
                a = goto_thrust(b, b.gp, c);
            }
        } else if (b.mode == GOTO) {
            a = goto_thrust(b, b.gp, c);
        } else if ((b.mode == FOLLOW || b.mode == ORBIT) && !tgt.valid) {
            a = D3{0.0, 0.0, 0.0};                                    // no target row: the park never leaves one so
        } else if (b.mode == FOLLOW) {
            a = follow_thrust(b, tgt.pos, tgt.radius, c);
        } else if (b.mode == ORBIT) {
            if (c.new_orbit) {
                D3 tv = tgt.vel;
                if (tgt.id < b.id) tv.y = tgt.vy_after;               // the target's turn came first
                a = new_orbit_thrust(b, tgt.pos, tv, tgt.radius, c, r0);
            } else {
                a = old_orbit_thrust(b, tgt.pos, tgt.radius, c);
            }
        } else if (b.mode == STOP) {
            if (!c.dynamical) b.vel.y = dmul(dsub(b.vel.y, dmul(STOP_DECAY, b.vel.y)), STOP_DAMP);
        }                                                             // BOID, MINIBALL, FIELD, RIGID, TROLL: none
    }
    store_phase1(s, i, b);
    d.on = live && s.dynamical;
    d.a = a;
    if (d.on) {
        d.fmass = tof(b.mass);
        d.agility = b.agility;
        d.sf = b.sf;
        d.max_vel = b.max_vel;
        d.max_ang_vel = s.max_ang_vel[i];
        d.rot_agility = s.rot_agility[i];
        d.warping = b.mode == WARP && b.effect_stamp >= 0;
        d.to_exit = f3_of(d3_sub(b.gp, b.pos));
        d.r0 = r0;
        d.w0 = ldf3(s.ang_vel, i, n);
    } else {
        d.r0 = q_identity();
        d.w0 = F3{0.0f, 0.0f, 0.0f};
    }
}

// A ship's tick, last part: the thrust (mLastG), the release after its own turn, phase 3 (the warp path or the
// integrator), phase 4 (the commit, the rotation where finite), PetrifyTroll, its world's clock
__device__ __forceinline__ void tick_end(const EbbFlightState& s, int64_t i, const DoLane& d, bool release_after) {
    const int64_t n = s.n;
    const Cfg c = cfg_of(s);
    Ship b = load_ship(s, i);
    const bool live = s.free_[i] && !s.moribund[i];
    if (live) b.last_g = d.a;
    if (release_after) release(b, true);
    if (live) {
        if (b.massive) b.last_collision = -1.0;                       // the gradient without neighbours
        D3 p = b.pos, v = b.vel;
        const D3 a = D3{dadd(b.last_g.x, 0.0), dadd(b.last_g.y, 0.0), dadd(b.last_g.z, 0.0)};   // mLastG + mLastC
        const double m = dmul(b.mass, tod(b.agility));
        if (b.mode == WARP && b.effect_stamp >= 0) {
            if (warp_path(b, &p, &v, dmul(i2d(b.clock - b.effect_stamp), c.dt))) {
                b.massive = true;                                     // dropped out: massive and sensing again, Stop
                b.sensor = true;
                b.mode = STOP;
                b.pos = p;                                            // TRV-714: the drop-out point is the old state
                b.vel = v;
                integrate(&p, &v, a, m, c.friction, b.tf, c.dt);
            }
        } else {
            integrate(&p, &v, a, m, c.friction, b.tf, c.dt);
        }
        st3(s.old_pos, i, n, b.pos);
        st3(s.old_vel, i, n, b.vel);
        b.pos = p;
        b.vel = v;
        if (c.dynamical) {                                            // the commit: the new values where finite
            const bool rot_ok = ffinite(q_lensq(d.rot1));
            const bool w_ok = ffinite(f3_dot(d.w1, d.w1));
            stf4(s.rot, i, n, rot_ok ? d.rot1 : d.r0);
            stf4(s.old_rot, i, n, rot_ok ? d.r0 : d.rot1);
            stf3(s.ang_vel, i, n, w_ok ? d.w1 : d.w0);
            stf3(s.old_ang_vel, i, n, w_ok ? d.w0 : d.w1);
            stf3(s.torque, i, n, d.torque);
            s.rot_roll[i] = d.roll;
        }
        if (b.mode == TROLL && !(b.effect_stamp > b.clock)) {
            // PetrifyTroll (full.py:1800) of a troll due: fixed, at rest (velocity and old velocity), mLastG cleared,
            // non-interactive, RIGID; only this ship's fields, which no other ship reads this tick
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
    s.speed_fraction[i] = b.sf;
    s.follow_range[i] = b.follow_range;
    s.mode[i] = b.mode;
    s.effect_stamp[i] = b.effect_stamp;
    s.follow_id[i] = b.follow_id;
    s.owner_id[i] = b.owner_id;
    s.follow_ptr[i] = b.follow_ptr;
    s.clock[i] = b.clock + 1;
    s.massive[i] = b.massive ? 1 : 0;
    s.sensor[i] = b.sensor ? 1 : 0;
}

// ================================================================================================ plain schedule

struct Records {
    double *pos, *vel, *vy;                                           // [3][n], [3][n], [n]
    uint8_t* act;                                                     // [n]
};

__host__ __device__ constexpr int64_t align256(int64_t b) { return (b + 255) & ~(int64_t)255; }

__host__ __device__ inline Records records_in(void* scratch, int64_t n) {
    char* p = (char*)scratch;
    Records r;
    r.pos = (double*)p;
    p += align256(3 * n * 8);
    r.vel = (double*)p;
    p += align256(3 * n * 8);
    r.vy = (double*)p;
    p += align256(n * 8);
    r.act = (uint8_t*)p;
    return r;
}

__host__ __device__ constexpr int64_t records_bytes(int64_t n) {
    return align256(3 * n * 8) * 2 + align256(n * 8) + align256(n);
}

// The records of ebb_flight_tick_noalloc, for callers that cannot allocate device memory: a fixed array in the
// library's own device memory, sized for EBB_NOALLOC_MAX_ROWS rows (records_bytes of that count, about 14.4 MB).
// Every device that loads the library holds it until the process exits, and every call on a device shares it.
__device__ __align__(256) static unsigned char noalloc_records[records_bytes(EBB_NOALLOC_MAX_ROWS)];

__global__ void __launch_bounds__(256) records_kernel(EbbFlightState s, Records r) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.n) return;
    bool act;
    double vy;
    records_of(s, i, &act, &vy);
    r.act[i] = act ? 1 : 0;
    r.vy[i] = vy;
    st3(r.pos, i, s.n, ld3(s.pos, i, s.n));
    st3(r.vel, i, s.n, ld3(s.vel, i, s.n));
}

// The plain tick: one thread a row, every warp's 32 rows through the warp's orientation step together (rows past n
// pass through it)
__global__ void __launch_bounds__(256, EBB_TICK_MIN_BLOCKS) tick_kernel(EbbFlightState s, Records r) {
    __shared__ float ndt_tab[TORQUE_STEPS];
    __shared__ float ktab[(256 / 32) * KTAB_FLOATS];
    fill_ndt(ndt_tab, s.dt);
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool mine = i < s.n;
    DoLane d;
    d.on = false;
    bool release_after = false;
    if (mine) {
        View tgt;
        const int64_t t = s.follow_ptr[i];
        tgt.valid = t >= 0 && t < s.n;
        if (tgt.valid) {
            tgt.pos = ld3(r.pos, t, s.n);
            tgt.vel = ld3(r.vel, t, s.n);
            tgt.vy_after = r.vy[t];
            tgt.id = s.ids[t];
            tgt.radius = s.radius[t];
            tgt.act = r.act[t] != 0;
        } else {
            tgt.act = false;
            tgt.id = 0;
        }
        tick_begin(s, i, tgt, r.act[i] != 0, d, &release_after);
    }
    orient_warp(d, cfg_of(s), ndt_tab, ktab + (threadIdx.x >> 5) * KTAB_FLOATS);
    if (mine) tick_end(s, i, d, release_after);
}

// ================================================================================================ tiled schedule

// The tiled tick's shared records: one slot a row of the tile
struct SlotRec {
    double px, py, pz, vx, vy, vz, vy_after;
    int64_t id;
    float radius;
    int32_t act;
};

__host__ __device__ inline size_t tiled_records_bytes(int cap) {
    return ((size_t)cap * sizeof(SlotRec) + 15) & ~(size_t)15;
}

// One tile (a run of whole worlds, rows [r0, r1)): the records pass into shared memory, then the tile's ships' ticks,
// each warp taking 32 ships at a time through the warp's orientation step. ONE_ROUND: the tile has at most as many
// rows as the block has threads, so each thread ticks at most one ship.
template <bool ONE_ROUND>
__device__ __forceinline__ void tiled_tile(const EbbFlightState& s, int64_t r0, int64_t r1, SlotRec* rec,
                                           const float* ndt_tab, float* ktab, int32_t* status) {
    const int m = (int)(r1 - r0);
    for (int j = threadIdx.x; j < m; j += blockDim.x) {               // the records pass, into shared memory
        const int64_t i = r0 + j;
        bool act;
        double vy_after;
        records_of(s, i, &act, &vy_after);
        SlotRec& q = rec[j];
        const D3 p = ld3(s.pos, i, s.n), v = ld3(s.vel, i, s.n);
        q.px = p.x;
        q.py = p.y;
        q.pz = p.z;
        q.vx = v.x;
        q.vy = v.y;
        q.vz = v.z;
        q.vy_after = vy_after;
        q.id = s.ids[i];
        q.radius = s.radius[i];
        q.act = act ? 1 : 0;
    }
    __syncthreads();
    for (int base = threadIdx.x & ~31; base < m; base += blockDim.x) {   // warp-uniform: each warp's 32 ships
        const int j = base + (threadIdx.x & 31);
        const bool mine = j < m;
        DoLane d;
        d.on = false;
        bool release_after = false;
        const int64_t i = r0 + j;
        if (mine) {
            View tgt;
            const int64_t t = s.follow_ptr[i];
            tgt.valid = t >= r0 && t < r1;
            if (!tgt.valid && t >= 0 && t < s.n) atomicOr(status, 1);    // a target outside its world's tile
            if (tgt.valid) {
                const SlotRec& q = rec[t - r0];
                tgt.pos = D3{q.px, q.py, q.pz};
                tgt.vel = D3{q.vx, q.vy, q.vz};
                tgt.vy_after = q.vy_after;
                tgt.id = q.id;
                tgt.radius = q.radius;
                tgt.act = q.act != 0;
            } else {
                tgt.act = false;
                tgt.id = 0;
            }
            tick_begin(s, i, tgt, rec[j].act != 0, d, &release_after);
        }
        orient_warp(d, cfg_of(s), ndt_tab, ktab);
        if (mine) tick_end(s, i, d, release_after);
        if (ONE_ROUND) break;
    }
}

// The tiled tick. SINGLE: one tile a block (grid >= tiles), each of at most `block` rows, so a thread ticks one ship
// and exits: no state lives across tiles or rounds, which halves the register spills of the general form. Otherwise a
// persistent grid takes the tiles in turn, syncing before it reuses the records.
template <bool SINGLE>
__global__ void __launch_bounds__(256, EBB_TILED_MIN_BLOCKS) tiled_kernel(EbbFlightState s, const int64_t* __restrict__ tile_rows,
                                                    int64_t tiles, int cap, int32_t* status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ float ndt_tab[TORQUE_STEPS];
    SlotRec* rec = (SlotRec*)smem_raw;
    float* ktab = (float*)(smem_raw + tiled_records_bytes(cap)) + (threadIdx.x >> 5) * KTAB_FLOATS;
    fill_ndt(ndt_tab, s.dt);
    if (SINGLE) {
        if (blockIdx.x < tiles)
            tiled_tile<true>(s, tile_rows[blockIdx.x], tile_rows[blockIdx.x + 1], rec, ndt_tab, ktab, status);
        return;
    }
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        __syncthreads();                                              // the table, and the previous tile's records
        tiled_tile<false>(s, tile_rows[tile], tile_rows[tile + 1], rec, ndt_tab, ktab, status);
    }
}

__host__ __device__ inline size_t tiled_smem_bytes(int cap, int block) {
    return tiled_records_bytes(cap) + (size_t)(block / 32) * KTAB_FLOATS * sizeof(float);
}

// ================================================================================================ listed worlds

// The listed-worlds tick's shared records: one slot a row of the tile, with the slot's world (its index in the tile)
struct ListRec {
    double px, py, pz, vx, vy, vz, vy_after;
    int64_t id;
    float radius;
    int32_t act;
    int32_t world;
    int32_t pad;
};

__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

// Shared memory of a listed-worlds tile of `cap` rows and at most `cap` worlds: the records, each world's first row
// (int64) and first slot (int32, plus the end), then the warps' kappa tables
__host__ __device__ inline size_t listed_tables_bytes(int cap) {
    return align16((size_t)cap * sizeof(ListRec)) + align16((size_t)cap * 8) + align16((size_t)(cap + 1) * 4);
}
__host__ __device__ inline size_t listed_smem_bytes(int cap, int block) {
    return listed_tables_bytes(cap) + (size_t)(block / 32) * KTAB_FLOATS * sizeof(float);
}

// One tile of a list of worlds: world w is rows [worlds[2w], worlds[2w + 1]), the tile the worlds [w0, w0 + nw),
// gathered into shared-memory slots world after world (warp 0 scans their row counts into slot offsets), then the
// records pass and the ships' ticks as in the tiled tick. Rows with active[i] == 0 (when `active` is given) are not
// ticked, though their records are made for the rest of their world. A malformed tile is skipped (status bit 2).
template <bool ONE_ROUND>
__device__ __forceinline__ void listed_tile(const EbbFlightState& s, const int64_t* __restrict__ worlds, int64_t w0,
                                            int64_t nw64, int cap, const uint8_t* __restrict__ active,
                                            int32_t* status, ListRec* rec, int64_t* wrow, int32_t* wslot,
                                            int* tile_rows, const float* ndt_tab, float* ktab) {
    const int lane = threadIdx.x & 31;
    if (nw64 <= 0 || nw64 > cap) {                                    // block-uniform
        if (nw64 != 0 && threadIdx.x == 0) atomicOr(status, 2);
        return;
    }
    const int nw = (int)nw64;
    if (threadIdx.x < 32) {                                           // warp 0: the worlds' slot offsets (a scan)
        int carry = 0;
        bool bad = false;
        for (int k0 = 0; k0 < nw; k0 += 32) {
            const int k = k0 + lane;
            int64_t b = 0, len = 0;
            if (k < nw) {
                b = worlds[2 * (w0 + k)];
                len = worlds[2 * (w0 + k) + 1] - b;
                if (b < 0 || len < 0 || len > cap || b + len > s.n) {
                    bad = true;
                    len = 0;
                }
            }
            int c = (int)len;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, c, o);
                if (lane >= o) c += y;
            }
            if (k < nw) {
                wrow[k] = b;
                wslot[k] = carry + c - (int)len;
            }
            carry += __shfl_sync(0xffffffffu, c, 31);
            if (carry > cap) bad = true;
        }
        bad = __any_sync(0xffffffffu, bad);
        if (lane == 0) {
            wslot[nw] = carry;
            *tile_rows = bad ? -1 : carry;
        }
    }
    __syncthreads();
    const int m = *tile_rows;
    if (m < 0) {                                                      // block-uniform
        if (threadIdx.x == 0) atomicOr(status, 2);
        return;
    }
    for (int j = threadIdx.x; j < m; j += blockDim.x) {               // the records pass, into shared memory
        int lo = 0, hi = nw - 1;                                      // the slot's world: the last k with wslot[k] <= j
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (wslot[mid] <= j) lo = mid;
            else hi = mid - 1;
        }
        const int64_t i = wrow[lo] + (j - wslot[lo]);
        bool act;
        double vy_after;
        records_of(s, i, &act, &vy_after);
        ListRec& q = rec[j];
        const D3 p = ld3(s.pos, i, s.n), v = ld3(s.vel, i, s.n);
        q.px = p.x;
        q.py = p.y;
        q.pz = p.z;
        q.vx = v.x;
        q.vy = v.y;
        q.vz = v.z;
        q.vy_after = vy_after;
        q.id = s.ids[i];
        q.radius = s.radius[i];
        q.act = act ? 1 : 0;
        q.world = lo;
    }
    __syncthreads();
    for (int base = threadIdx.x & ~31; base < m; base += blockDim.x) {   // warp-uniform: each warp's 32 slots
        const int j = base + lane;
        bool mine = j < m;
        int64_t i = 0;
        int e = 0;
        if (mine) {
            e = rec[j].world;
            i = wrow[e] + (j - wslot[e]);
            if (active != nullptr && active[i] == 0) mine = false;
        }
        DoLane d;
        d.on = false;
        bool release_after = false;
        if (mine) {
            View tgt;
            const int64_t t = s.follow_ptr[i];
            const int64_t b = wrow[e], len = wslot[e + 1] - wslot[e];
            tgt.valid = t >= b && t < b + len;
            if (!tgt.valid && t >= 0 && t < s.n) atomicOr(status, 1);    // a target outside its world
            if (tgt.valid) {
                const ListRec& q = rec[wslot[e] + (int)(t - b)];
                tgt.pos = D3{q.px, q.py, q.pz};
                tgt.vel = D3{q.vx, q.vy, q.vz};
                tgt.vy_after = q.vy_after;
                tgt.id = q.id;
                tgt.radius = q.radius;
                tgt.act = q.act != 0;
            } else {
                tgt.act = false;
                tgt.id = 0;
            }
            tick_begin(s, i, tgt, rec[j].act != 0, d, &release_after);
        }
        orient_warp(d, cfg_of(s), ndt_tab, ktab);
        if (mine) tick_end(s, i, d, release_after);
        if (ONE_ROUND) break;
    }
}

// One tick of a list of worlds anywhere in the park: a tile is the worlds [tile_worlds[t], tile_worlds[t + 1]) (at
// most cap rows). Rows in no listed world are not read or written; rows with active[i] == 0 keep their state (OnTick's
// per-world mask, in the kernel). status: bit 1 a follow pointer leaving its world (the ship ticks without its
// target), bit 2 a malformed tile (rows outside the park, more than cap rows or worlds: skipped). SINGLE: one tile a
// block of at most `block` rows (no state across tiles or rounds), else a persistent grid.
template <bool SINGLE>
__global__ void __launch_bounds__(256, EBB_TILED_MIN_BLOCKS)
    worlds_kernel(EbbFlightState s, const int64_t* __restrict__ worlds, const int64_t* __restrict__ tile_worlds,
                  int64_t tiles, int cap, const uint8_t* __restrict__ active, int32_t* status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ float ndt_tab[TORQUE_STEPS];
    __shared__ int tile_rows;
    ListRec* rec = (ListRec*)smem_raw;
    int64_t* wrow = (int64_t*)(smem_raw + align16((size_t)cap * sizeof(ListRec)));
    int32_t* wslot = (int32_t*)(smem_raw + align16((size_t)cap * sizeof(ListRec)) + align16((size_t)cap * 8));
    float* ktab = (float*)(smem_raw + listed_tables_bytes(cap)) + (threadIdx.x >> 5) * KTAB_FLOATS;
    fill_ndt(ndt_tab, s.dt);
    if (SINGLE) {
        if (blockIdx.x < tiles) {
            const int64_t w0 = tile_worlds[blockIdx.x];
            listed_tile<true>(s, worlds, w0, tile_worlds[blockIdx.x + 1] - w0, cap, active, status, rec, wrow, wslot,
                              &tile_rows, ndt_tab, ktab);
        }
        return;
    }
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        __syncthreads();                                              // the previous tile's tables are done with
        const int64_t w0 = tile_worlds[tile];
        listed_tile<false>(s, worlds, w0, tile_worlds[tile + 1] - w0, cap, active, status, rec, wrow, wslot,
                           &tile_rows, ndt_tab, ktab);
    }
}

// ================================================================================================ moving worlds

// Rows copied from one park to another (a world admitted into a resident park, or taken out of it): every field of
// src row src_rows[k] into dst row dst_rows[k]. A follow pointer moves with its row (a world moves as one run, so its
// target moves by the same number of rows); one that would leave dst becomes -1 (status bit 4), as do rows outside
// either park (skipped).
__global__ void move_kernel(EbbFlightState dst, EbbFlightState src, const int64_t* __restrict__ src_rows,
                            const int64_t* __restrict__ dst_rows, int64_t m, int32_t* status) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const int64_t a = src_rows[k], b = dst_rows[k];
    if (a < 0 || a >= src.n || b < 0 || b >= dst.n) {
        atomicOr(status, 4);
        return;
    }
    const int64_t sn = src.n, dn = dst.n;
#define EBB_MOVE(f, planes)                                                                                      \
    for (int p = 0; p < (planes); ++p) dst.f[p * dn + b] = src.f[p * sn + a];
    EBB_MOVE(pos, 3)
    EBB_MOVE(vel, 3)
    EBB_MOVE(old_pos, 3)
    EBB_MOVE(old_vel, 3)
    EBB_MOVE(goto_pt, 3)
    EBB_MOVE(last_g, 3)
    EBB_MOVE(mass, 1)
    EBB_MOVE(time_factor, 1)
    EBB_MOVE(last_collision, 1)
    EBB_MOVE(radius, 1)
    EBB_MOVE(max_vel, 1)
    EBB_MOVE(agility, 1)
    EBB_MOVE(speed_fraction, 1)
    EBB_MOVE(follow_range, 1)
    EBB_MOVE(max_ang_vel, 1)
    EBB_MOVE(rot_agility, 1)
    EBB_MOVE(rot_roll, 1)
    EBB_MOVE(rot, 4)
    EBB_MOVE(old_rot, 4)
    EBB_MOVE(ang_vel, 3)
    EBB_MOVE(old_ang_vel, 3)
    EBB_MOVE(torque, 3)
    EBB_MOVE(ids, 1)
    EBB_MOVE(effect_stamp, 1)
    EBB_MOVE(follow_id, 1)
    EBB_MOVE(owner_id, 1)
    EBB_MOVE(clock, 1)
    EBB_MOVE(mode, 1)
    EBB_MOVE(free_, 1)
    EBB_MOVE(moribund, 1)
    EBB_MOVE(massive, 1)
    EBB_MOVE(interactive, 1)
    EBB_MOVE(sensor, 1)
#undef EBB_MOVE
    const int32_t fp = src.follow_ptr[a];
    int64_t q = fp;
    if (fp >= 0) {
        q = (int64_t)fp + (b - a);
        if (q < 0 || q >= dn || q > INT32_MAX) {
            atomicOr(status, 4);
            q = -1;
        }
    }
    dst.follow_ptr[b] = (int32_t)q;
}

// ================================================================================================ set-up kernels

__global__ void snap_kernel(EbbFlightState s, const uint8_t* __restrict__ mask, int fresh) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.n || !mask[i]) return;
    const int64_t n = s.n;
    if (fresh) {                                                      // a new ball: mOldRot = rot x RotationQ(w, -dt|w|)
        const F4 rot = q_identity();
        const F3 w = ldf3(s.ang_vel, i, n);
        const F4 back = q_axis_angle(w, tof(dmul(dneg((double)s.fdt), tod(f3_len(w)))));
        stf4(s.rot, i, n, rot);
        stf4(s.old_rot, i, n, q_mul(rot, back));
    }
    const D3 v = ld3(s.vel, i, n);
    if (!(d3_lensq(v) > 1e-12)) return;
    const F4 r = snap_rotation(v);
    stf4(s.rot, i, n, r);
    stf4(s.old_rot, i, n, r);
    stf3(s.ang_vel, i, n, F3{0.0f, 0.0f, 0.0f});
    stf3(s.old_ang_vel, i, n, F3{0.0f, 0.0f, 0.0f});
}

__global__ void decay_kernel(EbbFlightState s, const uint8_t* __restrict__ mask, double neg_kdt) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.n || !mask[i]) return;
    const double m = dmul(s.mass[i], tod(s.agility[i]));
    s.time_factor[i] = (m <= 0.0) ? 0.0 : lm::exp(ddiv(neg_kdt, m));
}

__global__ void libm_kernel(int func, int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                            double* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double a = x[i];
    double sn, cs;
    switch (func) {
        case 0: out[i] = lm::sin(a); break;
        case 1: out[i] = lm::cos(a); break;
        case 2: out[i] = lm::log(a); break;
        case 3: out[i] = lm::exp(a); break;
        case 4: lm::sincos(a, &sn, &cs); out[i] = sn; break;
        case 5: lm::sincos(a, &sn, &cs); out[i] = cs; break;
        case 6: out[i] = lm::pow(a, y[i]); break;
        case 10: out[i] = tod(lm::expf(tof(a))); break;
        case 11: out[i] = tod(lm::logf(tof(a))); break;
        case 12: out[i] = tod(lm::sinf(tof(a))); break;
        case 13: out[i] = tod(lm::cosf(tof(a))); break;
        case 14: out[i] = tod(lm::acosf(tof(a))); break;
        case 15: out[i] = tod(lm::atanf(tof(a))); break;
        case 16: out[i] = tod(lm::atan2f(tof(y[i]), tof(a))); break;
        case 17: out[i] = tod(lm::powf(tof(a), tof(y[i]))); break;
        default: out[i] = dnan(); break;
    }
}

}  // namespace flight
}  // namespace ebb

// ==================================================================================================== the C ABI

namespace ebb {
namespace combat {
cudaError_t kernel_attributes(cudaFuncAttributes* fa);   // ebb_combat.cu
cudaError_t composed_attributes(cudaFuncAttributes* fa);
}
}  // namespace ebb

namespace {
int launched() {
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}
bool block_ok(int block, int max_block) { return block > 0 && block <= max_block && block % 32 == 0; }
unsigned grid_of(int64_t n, int block) { return (unsigned)((n + block - 1) / block); }
}  // namespace

extern "C" {

int ebb_abi(void) { return EBB_ABI_VERSION; }

const char* ebb_error_string(int code) {
    if (code == EBB_EINVAL) return "refused: invalid arguments (block size, scratch, tiles)";
    if (code == EBB_ETOOBIG) return "refused: more rows than the allocation-free tick holds (EBB_NOALLOC_MAX_ROWS)";
    return cudaGetErrorString((cudaError_t)code);
}

int64_t ebb_flight_scratch_bytes(int64_t n) { return n <= 0 ? 0 : ebb::flight::records_bytes(n); }

int ebb_flight_tick(const EbbFlightState* s, void* scratch, int64_t scratch_bytes, void* stream, int block) {
    if (s == nullptr) return EBB_EINVAL;
    if (s->n <= 0) return 0;
    if (!block_ok(block, 256) || scratch == nullptr || ((uintptr_t)scratch & 255) != 0 ||
        scratch_bytes < ebb_flight_scratch_bytes(s->n))
        return EBB_EINVAL;
    const ebb::flight::Records r = ebb::flight::records_in(scratch, s->n);
    const cudaStream_t st = (cudaStream_t)stream;
    ebb::flight::records_kernel<<<grid_of(s->n, block), block, 0, st>>>(*s, r);
    int rc = launched();
    if (rc) return rc;
    ebb::flight::tick_kernel<<<grid_of(s->n, block), block, 0, st>>>(*s, r);
    return launched();
}

// ebb_flight_tick_noalloc's set-up: the device address of noalloc_records, one a device. In host code the array's
// name stands for a host-side shadow, not device memory, so the kernels get the address cudaGetSymbolAddress gives
// with the device current; it is looked up on the first call on each device and kept.
static std::atomic<uintptr_t> noalloc_address[EBB_NOALLOC_MAX_DEVICES];

int ebb_flight_tick_noalloc(const EbbFlightState* s, void* stream, int block) {
    if (s == nullptr) return EBB_EINVAL;
    if (s->n <= 0) return 0;
    if (s->n > EBB_NOALLOC_MAX_ROWS) return EBB_ETOOBIG;
    if (!block_ok(block, 256)) return EBB_EINVAL;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return (int)e;
    if (dev < 0 || dev >= EBB_NOALLOC_MAX_DEVICES) return EBB_EINVAL;
    uintptr_t addr = noalloc_address[dev].load(std::memory_order_acquire);
    if (addr == 0) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, ebb::flight::noalloc_records);
        if (e != cudaSuccess) return (int)e;
        addr = (uintptr_t)p;
        noalloc_address[dev].store(addr, std::memory_order_release);
    }
    // Every record a tick reads (rows below n) is written by the records pass first: nothing needs clearing.
    const ebb::flight::Records r = ebb::flight::records_in((void*)addr, s->n);
    const cudaStream_t st = (cudaStream_t)stream;
    ebb::flight::records_kernel<<<grid_of(s->n, block), block, 0, st>>>(*s, r);
    int rc = launched();
    if (rc) return rc;
    ebb::flight::tick_kernel<<<grid_of(s->n, block), block, 0, st>>>(*s, r);
    return launched();
}

int ebb_flight_tick_tiled(const EbbFlightState* s, const int64_t* tile_rows, int64_t tiles, int tile_cap,
                          int32_t* status, void* stream, int block, int grid) {
    if (s == nullptr) return EBB_EINVAL;
    if (s->n <= 0 || tiles <= 0) return 0;
    if (!block_ok(block, 256) || tile_cap <= 0 || tile_cap > 4096 || tile_rows == nullptr || status == nullptr ||
        grid <= 0)
        return EBB_EINVAL;
    const size_t smem = ebb::flight::tiled_smem_bytes(tile_cap, block);
    auto kernel = (tile_cap <= block && grid >= tiles) ? ebb::flight::tiled_kernel<true>
                                                         : ebb::flight::tiled_kernel<false>;
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
    }
    kernel<<<(unsigned)grid, block, smem, (cudaStream_t)stream>>>(*s, tile_rows, tiles, tile_cap, status);
    return launched();
}

int ebb_flight_tick_worlds(const EbbFlightState* s, const int64_t* worlds, const int64_t* tile_worlds, int64_t tiles,
                           int tile_cap, const uint8_t* active, int32_t* status, void* stream, int block, int grid) {
    if (s == nullptr) return EBB_EINVAL;
    if (s->n <= 0 || tiles <= 0) return 0;
    if (!block_ok(block, 256) || tile_cap <= 0 || tile_cap > EBB_WORLDS_MAX_TILE || worlds == nullptr ||
        tile_worlds == nullptr || status == nullptr || grid <= 0)
        return EBB_EINVAL;
    const size_t smem = ebb::flight::listed_smem_bytes(tile_cap, block);
    auto kernel = (tile_cap <= block && grid >= tiles) ? ebb::flight::worlds_kernel<true>
                                                         : ebb::flight::worlds_kernel<false>;
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
    }
    kernel<<<(unsigned)grid, block, smem, (cudaStream_t)stream>>>(*s, worlds, tile_worlds, tiles, tile_cap, active,
                                                                  status);
    return launched();
}

int ebb_flight_move(const EbbFlightState* dst, const EbbFlightState* src, const int64_t* src_rows,
                    const int64_t* dst_rows, int64_t m, int32_t* status, void* stream, int block) {
    if (dst == nullptr || src == nullptr) return EBB_EINVAL;
    if (m <= 0) return 0;
    if (!block_ok(block, 1024) || src_rows == nullptr || dst_rows == nullptr || status == nullptr) return EBB_EINVAL;
    ebb::flight::move_kernel<<<grid_of(m, block), block, 0, (cudaStream_t)stream>>>(*dst, *src, src_rows, dst_rows, m,
                                                                                    status);
    return launched();
}

int ebb_flight_snap(const EbbFlightState* s, const uint8_t* mask, int fresh, void* stream, int block) {
    if (s == nullptr || mask == nullptr) return EBB_EINVAL;
    if (s->n <= 0) return 0;
    if (!block_ok(block, 1024)) return EBB_EINVAL;
    ebb::flight::snap_kernel<<<grid_of(s->n, block), block, 0, (cudaStream_t)stream>>>(*s, mask, fresh);
    return launched();
}

int ebb_flight_decay(const EbbFlightState* s, const uint8_t* mask, double neg_kdt, void* stream, int block) {
    if (s == nullptr || mask == nullptr) return EBB_EINVAL;
    if (s->n <= 0) return 0;
    if (!block_ok(block, 1024)) return EBB_EINVAL;
    ebb::flight::decay_kernel<<<grid_of(s->n, block), block, 0, (cudaStream_t)stream>>>(*s, mask, neg_kdt);
    return launched();
}

int ebb_libm(int func, int64_t n, const double* x, const double* y, double* out, void* stream, int block) {
    if (n <= 0) return 0;
    if (!block_ok(block, 1024) || x == nullptr || out == nullptr) return EBB_EINVAL;
    if (!((func >= 0 && func <= 6) || (func >= 10 && func <= 17))) return EBB_EINVAL;
    if ((func == 6 || func == 16 || func == 17) && y == nullptr) return EBB_EINVAL;
    ebb::flight::libm_kernel<<<grid_of(n, block), block, 0, (cudaStream_t)stream>>>(func, n, x, y, out);
    return launched();
}

int ebb_kernel_info(int which, int* regs, int* local_bytes, int* binary_version, int* ptx_version, int* max_threads) {
    cudaFuncAttributes fa;
    cudaError_t e;
    switch (which) {
        case 0: e = cudaFuncGetAttributes(&fa, ebb::flight::tick_kernel); break;
        case 1: e = cudaFuncGetAttributes(&fa, ebb::flight::records_kernel); break;
        case 2: e = cudaFuncGetAttributes(&fa, ebb::flight::tiled_kernel<true>); break;
        case 3: e = cudaFuncGetAttributes(&fa, ebb::flight::worlds_kernel<true>); break;
        case 5: e = cudaFuncGetAttributes(&fa, ebb::flight::tiled_kernel<false>); break;
        case 6: e = cudaFuncGetAttributes(&fa, ebb::flight::worlds_kernel<false>); break;
        case 4: e = cudaFuncGetAttributes(&fa, ebb::flight::move_kernel); break;
        case 7: e = ebb::combat::kernel_attributes(&fa); break;
        case 8: e = ebb::combat::composed_attributes(&fa); break;
        default: return EBB_EINVAL;
    }
    if (e != cudaSuccess) return (int)e;
    *regs = fa.numRegs;
    *local_bytes = (int)fa.localSizeBytes;
    *binary_version = fa.binaryVersion;
    *ptx_version = fa.ptxVersion;
    *max_threads = fa.maxThreadsPerBlock;
    return 0;
}

}  // extern "C"

EBB_OP_COUNTER(ebb_count_ops_flight)
