// SPDX-License-Identifier: LGPL-2.1-or-later
// glibc 2.34's rand() after srand(seed) (random_r / srandom_r, TYPE_3: a table of 31 words, separation 3), one
// generator a world, on the device: destiny's floatrand (Ball.cpp:19) draws it for a shuffled proximity sensor's first
// period (the reference's exact_ballpark/glibc_rand.py:14-45 and vec_space.py:148; glibc's stdlib/random_r.c). The
// steps are glibc's published algorithm: the table seeded by the minimal-standard generator (16807, Schrage's
// decomposition by 127773 and 2836), 310 draws discarded, then each draw the sum of two table words (wrapping at 2^32),
// stored back, returned shifted right by one.
#include <cuda_runtime.h>

#include "../../include/ebb.h"
#include "ebb_rand.cuh"

namespace ebb {
namespace grand {

// srand(seed) for each world: the table, then the front and rear indices (EBB_RAND_WORDS int32 a world)
__global__ void srand_kernel(const int64_t* __restrict__ seeds, int64_t worlds, int32_t* __restrict__ state) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= worlds) return;
    uint32_t seed = (uint32_t)seeds[w];
    if (seed == 0) seed = 1;
    int32_t t[DEG];
    int32_t word = (int32_t)seed;
    t[0] = word;
    for (int i = 1; i < DEG; ++i) {
        const int32_t hi = word / 127773, lo = word % 127773;     // C's division toward zero, as glibc's
        word = 16807 * lo - 2836 * hi;
        if (word < 0) word += 2147483647;
        t[i] = word;
    }
    int32_t f = SEP, r = 0;
    for (int i = 0; i < 10 * DEG; ++i) draw(t, f, r);
    int32_t* out = state + w * EBB_RAND_WORDS;
    for (int i = 0; i < DEG; ++i) out[i] = t[i];
    out[DEG] = f;
    out[DEG + 1] = r;
}

// `draws` values of rand() for each world, its state advanced
__global__ void rand_kernel(int32_t* __restrict__ state, int64_t worlds, int64_t draws, int32_t* __restrict__ out) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= worlds) return;
    int32_t* st = state + w * EBB_RAND_WORDS;
    int32_t t[DEG];
    for (int i = 0; i < DEG; ++i) t[i] = st[i];
    int32_t f = st[DEG], r = st[DEG + 1];
    if (f < 0 || f >= DEG || r < 0 || r >= DEG) return;
    for (int64_t k = 0; k < draws; ++k) out[w * draws + k] = draw(t, f, r);
    for (int i = 0; i < DEG; ++i) st[i] = t[i];
    st[DEG] = f;
    st[DEG + 1] = r;
}

}  // namespace grand
}  // namespace ebb

extern "C" {

int ebb_glibc_srand(const int64_t* seeds, int64_t worlds, int32_t* state, void* stream) {
    if (worlds < 0 || (worlds > 0 && (seeds == nullptr || state == nullptr))) return EBB_EINVAL;
    if (worlds == 0) return 0;
    ebb::grand::srand_kernel<<<(unsigned)((worlds + 127) / 128), 128, 0, (cudaStream_t)stream>>>(seeds, worlds, state);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}

int ebb_glibc_rand(int32_t* state, int64_t worlds, int64_t draws, int32_t* out, void* stream) {
    if (worlds < 0 || draws < 0 || (worlds > 0 && draws > 0 && (state == nullptr || out == nullptr))) return EBB_EINVAL;
    if (worlds == 0 || draws == 0) return 0;
    ebb::grand::rand_kernel<<<(unsigned)((worlds + 127) / 128), 128, 0, (cudaStream_t)stream>>>(state, worlds, draws,
                                                                                               out);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}

}  // extern "C"
