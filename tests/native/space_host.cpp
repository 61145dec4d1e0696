// SPDX-License-Identifier: MIT
// TEST INFRASTRUCTURE, NOT THE PRODUCT. The space layer's per-world program (exact_ballpark_b200/csrc/ebb_space.cuh,
// which the device kernel runs, one thread a world) compiled for the host with g++, so that the CPU tests hold the
// same source to the oracle (oracle/space.cpp) without a GPU; the product has no host path.
#include "../../exact_ballpark_b200/csrc/ebb_space.cuh"

extern "C" int space_tape_host(const EbbFlightState* p, const EbbSpaceState* s, const EbbSpaceTape* t) {
    for (int64_t w = 0; w < s->worlds; ++w) {
        if (s->pitch > 0)
            ebb::space::run_tape<true>(p, s, t, w);
        else
            ebb::space::run_tape<false>(p, s, t, w);
    }
    return 0;
}

extern "C" int space_query_host(const EbbFlightState* p, const EbbSpaceState* s, const EbbSpaceQuery* q) {
    for (int64_t w = 0; w < s->worlds; ++w) {
        if (s->pitch > 0)
            ebb::space::run_query<true>(p, s, q, w);
        else
            ebb::space::run_query<false>(p, s, q, w);
    }
    return 0;
}
