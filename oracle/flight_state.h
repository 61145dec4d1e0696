// TEST INFRASTRUCTURE, NOT THE PRODUCT. The CPU oracle's flight park as its C entry points take it (oracle/flight.cpp;
// oracle/park.py's _State): field for field the reference park's tensors, vectors as [n][3] and rotations as [n][4]
// doubles, row-major. Shared by oracle/space.cpp, whose worlds tick their balls through oracle_flight_tick_mt.
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

}  // extern "C"
