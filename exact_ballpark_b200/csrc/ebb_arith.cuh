// SPDX-License-Identifier: MIT
// Rounding-pinned IEEE arithmetic shared by the device kernels and their host builds.
//
// Every double operation is a single correctly rounded IEEE operation (__dadd_rn ... __dsqrt_rn on the device; plain
// operators on the host, built with -ffp-contract=off so that g++ fuses nothing); every float operation likewise in
// binary32 (__fadd_rn ... on the device; float operators on x86-64 SSE, which round each to binary32). A fused
// multiply-add appears only where a caller writes dfma/ffma: __fma_rn/__fmaf_rn on the device, fma/fmaf on the host,
// both the IEEE fused operation. nvcc builds with -fmad=false -prec-div=true -prec-sqrt=true -ftz=false and no fast
// math, so even plain operators would not be contracted; the explicit intrinsics make the rounding visible in source.
#pragma once

#include <cstdint>
#include <cstring>
#ifndef __CUDACC__
#include <cmath>
#endif

#ifdef __CUDACC__
#define EBB_HD __host__ __device__ __forceinline__
#define EBB_HDNI inline __host__ __device__ __noinline__
#else
#define EBB_HD inline
#define EBB_HDNI inline
#endif

namespace ebb {

// ---- bit casts ----
EBB_HD uint64_t dbits(double x) {
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t u;
    std::memcpy(&u, &x, 8);
    return u;
#endif
}
EBB_HD double dfrom(uint64_t u) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)u);
#else
    double x;
    std::memcpy(&x, &u, 8);
    return x;
#endif
}
EBB_HD uint32_t fbits(float x) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(x);
#else
    uint32_t u;
    std::memcpy(&u, &x, 4);
    return u;
#endif
}
EBB_HD float ffrom(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float x;
    std::memcpy(&x, &u, 4);
    return x;
#endif
}

// ---- the counting build ----
// Built with EBB_COUNT_OPS (a measurement build, never the timed library), every IEEE operation a kernel executes is
// counted by kind into the translation unit's own device array op_count (one atomic add an operation), which the
// unit's ebb_count_ops_* entry point reads and clears: the FLOPs per ship-tick of the algorithm as it runs.
enum OpKind { OP_DADD, OP_DSUB, OP_DMUL, OP_DDIV, OP_DSQRT, OP_DFMA, OP_FADD, OP_FSUB, OP_FMUL, OP_FDIV, OP_FSQRT,
              OP_FFMA, OP_KINDS };
#if defined(EBB_COUNT_OPS) && defined(__CUDACC__)
static __device__ unsigned long long op_count[OP_KINDS];
#endif
#if defined(EBB_COUNT_OPS) && defined(__CUDA_ARCH__)
#define EBB_OP(k) atomicAdd(&op_count[k], 1ull)
#else
#define EBB_OP(k) ((void)0)
#endif
// the unit's reader (the counting build only): its counts into out[OP_KINDS], cleared after when `reset`
#if defined(EBB_COUNT_OPS) && defined(__CUDACC__)
#define EBB_OP_COUNTER(name)                                                                                    \
    extern "C" int name(unsigned long long* out, int reset) {                                                   \
        cudaError_t e = cudaMemcpyFromSymbol(out, ebb::op_count, sizeof(unsigned long long) * ebb::OP_KINDS);   \
        if (e == cudaSuccess && reset) {                                                                        \
            const unsigned long long zero[ebb::OP_KINDS] = {};                                                  \
            e = cudaMemcpyToSymbol(ebb::op_count, zero, sizeof(zero));                                          \
        }                                                                                                       \
        return e == cudaSuccess ? 0 : (int)e;                                                                   \
    }
#else
#define EBB_OP_COUNTER(name)
#endif

// ---- double ----
EBB_HD double dadd(double a, double b) {
#ifdef __CUDA_ARCH__
    EBB_OP(OP_DADD);
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
EBB_HD double dsub(double a, double b) {
#ifdef __CUDA_ARCH__
    EBB_OP(OP_DSUB);
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
EBB_HD double dmul(double a, double b) {
#ifdef __CUDA_ARCH__
    EBB_OP(OP_DMUL);
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
EBB_HD double ddiv(double a, double b) {
#ifdef __CUDA_ARCH__
    EBB_OP(OP_DDIV);
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}
EBB_HD double dsqrt(double a) {
#ifdef __CUDA_ARCH__
    EBB_OP(OP_DSQRT);
    return __dsqrt_rn(a);
#else
    return std::sqrt(a);
#endif
}
EBB_HD double dfma(double a, double b, double c) {   // a b + c, rounded once
#ifdef __CUDA_ARCH__
    EBB_OP(OP_DFMA);
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
EBB_HD double dneg(double a) { return dfrom(dbits(a) ^ 0x8000000000000000ULL); }
EBB_HD double dabs(double a) { return dfrom(dbits(a) & 0x7fffffffffffffffULL); }
EBB_HD double dcopysign(double a, double s) {
    return dfrom((dbits(a) & 0x7fffffffffffffffULL) | (dbits(s) & 0x8000000000000000ULL));
}
EBB_HD bool dfinite(double x) { return (dbits(x) & 0x7ff0000000000000ULL) != 0x7ff0000000000000ULL; }
EBB_HD double dinf() { return dfrom(0x7ff0000000000000ULL); }
EBB_HD double dnan() { return dfrom(0x7ff8000000000000ULL); }
EBB_HD double dtrunc(double x) {                     // toward zero, exact
#ifdef __CUDA_ARCH__
    return trunc(x);
#else
    return std::trunc(x);
#endif
}
// aarch64 frinta: to the nearest integer, ties away from zero (z - trunc(z) is exact)
EBB_HD double frinta(double z) {
    const double t = dtrunc(z);
    const double d = dsub(z, t);
    return d >= 0.5 ? dadd(t, 1.0) : (d <= -0.5 ? dsub(t, 1.0) : t);
}
// (int64_t)x of a double on aarch64 (fcvtzs): toward zero, saturating, NaN to 0
EBB_HD int64_t to_i64(double x) {
    if (x != x) return 0;
    if (x >= 9223372036854775808.0) return INT64_MAX;
    if (x < -9223372036854775808.0) return INT64_MIN;
#ifdef __CUDA_ARCH__
    return (int64_t)__double2ll_rz(x);
#else
    return (int64_t)x;
#endif
}
// (int)x of a float value on aarch64 (fcvtzs): toward zero, saturating, NaN to 0
EBB_HD int32_t to_i32(double x) {
    if (x != x) return 0;
    if (x < -2147483648.0) return INT32_MIN;
    if (x > 2147483647.0) return INT32_MAX;
#ifdef __CUDA_ARCH__
    return __double2int_rz(x);
#else
    return (int32_t)x;
#endif
}
// an int64 as a double, rounded to nearest (exact below 2^53)
EBB_HD double i2d(int64_t v) {
#ifdef __CUDA_ARCH__
    return __ll2double_rn((long long)v);
#else
    return (double)v;
#endif
}

// ---- float ----
EBB_HD float fadd(float a, float b) {
#ifdef __CUDA_ARCH__
    EBB_OP(OP_FADD);
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
EBB_HD float fsub(float a, float b) {
#ifdef __CUDA_ARCH__
    EBB_OP(OP_FSUB);
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}
EBB_HD float fmul(float a, float b) {
#ifdef __CUDA_ARCH__
    EBB_OP(OP_FMUL);
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
EBB_HD float fdiv(float a, float b) {
#ifdef __CUDA_ARCH__
    EBB_OP(OP_FDIV);
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}
EBB_HD float fsqrt(float a) {
#ifdef __CUDA_ARCH__
    EBB_OP(OP_FSQRT);
    return __fsqrt_rn(a);
#else
    return std::sqrt(a);
#endif
}
EBB_HD float ffma(float a, float b, float c) {       // a b + c, rounded once to binary32
#ifdef __CUDA_ARCH__
    EBB_OP(OP_FFMA);
    return __fmaf_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
EBB_HD float fneg(float a) { return ffrom(fbits(a) ^ 0x80000000u); }
EBB_HD float fabs_(float a) { return ffrom(fbits(a) & 0x7fffffffu); }
EBB_HD bool ffinite(float x) { return (fbits(x) & 0x7f800000u) != 0x7f800000u; }
EBB_HD float fnan() { return ffrom(0x7fc00000u); }
EBB_HD float finf() { return ffrom(0x7f800000u); }
EBB_HD float fmax_(float a, float b) { return (a < b) ? b : a; }   // std::max
EBB_HD float fmin_(float a, float b) { return (b < a) ? b : a; }   // std::min
EBB_HD float fceil(float x) {                        // toward +inf, exact
#ifdef __CUDA_ARCH__
    return ceilf(x);
#else
    return std::ceil(x);
#endif
}
// a double rounded to the nearest float (a C++ float parameter or result); beyond the range an infinity
EBB_HD float tof(double x) {
#ifdef __CUDA_ARCH__
    return __double2float_rn(x);
#else
    return (float)x;
#endif
}
EBB_HD double tod(float x) { return (double)x; }     // exact

}  // namespace ebb
