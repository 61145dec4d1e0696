// SPDX-License-Identifier: LGPL-2.1-or-later
// glibc 2.34's random_r draw (TYPE_3: a table of 31 words, separation 3) as host-and-device code, for the kernels
// that draw a world's rand() (ebb_rand.cu, the space layer's shuffled sensors). glibc's published algorithm
// (stdlib/random_r.c): the sum of the front and rear table words, wrapping at 2^32, stored at the front, returned
// shifted right by one; the indices advance and wrap.
#pragma once

#include <cstdint>

#include "ebb_arith.cuh"

namespace ebb {
namespace grand {

constexpr int DEG = 31, SEP = 3;

EBB_HD int32_t draw(int32_t* t, int32_t& f, int32_t& r) {
    const uint32_t val = (uint32_t)t[f] + (uint32_t)t[r];
    t[f] = (int32_t)val;
    if (++f >= DEG) {
        f = 0;
        ++r;
    } else if (++r >= DEG) {
        r = 0;
    }
    return (int32_t)(val >> 1);
}

}  // namespace grand
}  // namespace ebb
