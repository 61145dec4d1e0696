// TEST INFRASTRUCTURE, NOT THE PRODUCT. The CPU oracle's flight park as its C entry points take it (oracle/flight.cpp;
// oracle/park.py's _State): field for field the reference park's tensors, vectors as [n][3] and rotations as [n][4]
// doubles, row-major. Shared by oracle/space.cpp, whose worlds tick their balls through oracle_flight_tick_hooked.
#pragma once

#include <cstdint>

extern "C" {

struct OracleFlight {
    int64_t n;
    double friction, dt;
    float ffriction, fdt;
    int32_t new_orbit, dynamical;
    double *pos, *vel, *old_pos, *old_vel, *goto_, *last_g;
    double *mass, *time_factor, *last_collision;
    double *radius, *max_vel, *agility, *speed_fraction, *follow_range, *max_ang_vel, *rot_agility, *rot_roll;
    double *rot, *old_rot, *ang_vel, *old_ang_vel, *torque;
    int64_t *ids, *world, *mode, *effect_stamp, *follow_id, *owner_id, *follow_ptr, *clock;
    uint8_t *free_, *moribund, *massive, *interactive, *sensor;
};

int oracle_flight_tick_mt(const OracleFlight* s, int threads);

// A caller's collisions and partition inside the flight tick: at a massive ball's turn in phase 3 (its mLastCollision
// reset to -1) `gradient` is called with its row and leaves the ball's collision acceleration in last_c [n][3] (zeroed
// by the caller before the tick) and its time in last_collision; at a warp's drop-out nearly at rest (the drop-out
// point already the row's position) `drop_out` is called to re-file the row there.
struct OracleTickHooks {
    double* last_c;
    void* world;
    void (*gradient)(void* world, int64_t row);
    void (*drop_out)(void* world, int64_t row);
};

// One tick of every world on the calling thread, with the hooks above. Returns 0.
int oracle_flight_tick_hooked(const OracleFlight* s, const OracleTickHooks* h);

}  // extern "C"
