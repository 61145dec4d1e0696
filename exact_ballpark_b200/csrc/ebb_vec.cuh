// SPDX-License-Identifier: MIT
// Vectors of the flight tick with every rounding pinned: Destiny's Vector3d (double) arithmetic and carbonengine's
// float Vector3 / Quaternion / Matrix (the 3x3 part of the 4x4; the rest is 0 0 0 1), each component expression in
// the reference's operation order (exact_ballpark/modes.py:81-91, full.py:140-300).
#pragma once

#include "ebb_arith.cuh"

namespace ebb {

// ---------------------------------------------------------------------------------------------------- double
struct D3 {
    double x, y, z;
};

__device__ __forceinline__ D3 d3(double x, double y, double z) { return D3{x, y, z}; }
__device__ __forceinline__ D3 d3_add(D3 a, D3 b) { return D3{dadd(a.x, b.x), dadd(a.y, b.y), dadd(a.z, b.z)}; }
__device__ __forceinline__ D3 d3_sub(D3 a, D3 b) { return D3{dsub(a.x, b.x), dsub(a.y, b.y), dsub(a.z, b.z)}; }
__device__ __forceinline__ D3 d3_mul(D3 a, double c) { return D3{dmul(a.x, c), dmul(a.y, c), dmul(a.z, c)}; }
// x x + y y + z z, left to right
__device__ __forceinline__ double d3_lensq(D3 v) { return dadd(dadd(dmul(v.x, v.x), dmul(v.y, v.y)), dmul(v.z, v.z)); }
__device__ __forceinline__ double d3_len(D3 v) { return dsqrt(d3_lensq(v)); }
__device__ __forceinline__ double d3_dot(D3 a, D3 b) { return dadd(dadd(dmul(a.x, b.x), dmul(a.y, b.y)), dmul(a.z, b.z)); }
// Vector3d::Normalize: times the reciprocal of the length; a zero vector as it is
__device__ __forceinline__ D3 d3_unit(D3 v) {
    const double n = d3_len(v);
    return n == 0.0 ? v : d3_mul(v, ddiv(1.0, n));
}
__device__ __forceinline__ D3 d3_cross(D3 u, D3 v) {
    return D3{dsub(dmul(u.y, v.z), dmul(u.z, v.y)), dsub(dmul(u.z, v.x), dmul(u.x, v.z)),
              dsub(dmul(u.x, v.y), dmul(u.y, v.x))};
}
__device__ __forceinline__ bool d3_finite(D3 v) { return dfinite(v.x) && dfinite(v.y) && dfinite(v.z); }

// ---------------------------------------------------------------------------------------------------- float
struct F3 {
    float x, y, z;
};
struct F4 {
    float x, y, z, w;
};
struct M3 {                                 // rows r0, r1, r2 of the rotation matrix
    F3 r0, r1, r2;
};

__device__ __forceinline__ F3 f3_mul(F3 a, float f) { return F3{fmul(a.x, f), fmul(a.y, f), fmul(a.z, f)}; }
__device__ __forceinline__ F3 f3_add(F3 a, F3 b) { return F3{fadd(a.x, b.x), fadd(a.y, b.y), fadd(a.z, b.z)}; }
__device__ __forceinline__ F3 f3_sub(F3 a, F3 b) { return F3{fsub(a.x, b.x), fsub(a.y, b.y), fsub(a.z, b.z)}; }
__device__ __forceinline__ F3 f3_div(F3 a, float f) { return f3_mul(a, fdiv(1.0f, f)); }   // times 1.0f / f
__device__ __forceinline__ float f3_dot(F3 a, F3 b) { return fadd(fadd(fmul(a.x, b.x), fmul(a.y, b.y)), fmul(a.z, b.z)); }
__device__ __forceinline__ float f3_len(F3 a) { return fsqrt(f3_dot(a, a)); }
__device__ __forceinline__ F3 f3_cross(F3 a, F3 b) {
    return F3{fsub(fmul(a.y, b.z), fmul(a.z, b.y)), fsub(fmul(a.z, b.x), fmul(a.x, b.z)),
              fsub(fmul(a.x, b.y), fmul(a.y, b.x))};
}
// Vector3::Normalize: scaled by the largest magnitude first, then by the length (a zero length left as it is)
__device__ __forceinline__ F3 f3_unit(F3 v) {
    const float mx = fmax_(fmax_(fabs_(v.x), fabs_(v.y)), fabs_(v.z));
    const F3 m = f3_div(v, mx != 0.0f ? mx : 1.0f);
    const float l = f3_len(m);
    return f3_mul(m, l != 0.0f ? fdiv(1.0f, l) : l);
}
__device__ __forceinline__ F3 f3_of(D3 v) { return F3{tof(v.x), tof(v.y), tof(v.z)}; }
__device__ __forceinline__ D3 d3_of(F3 v) { return D3{tod(v.x), tod(v.y), tod(v.z)}; }

// Quaternion product q o (Quaternion_inline.h)
__device__ __forceinline__ F4 q_mul(F4 q, F4 o) {
    return F4{fsub(fadd(fadd(fmul(o.w, q.x), fmul(o.x, q.w)), fmul(o.y, q.z)), fmul(o.z, q.y)),
              fadd(fadd(fsub(fmul(o.w, q.y), fmul(o.x, q.z)), fmul(o.y, q.w)), fmul(o.z, q.x)),
              fadd(fsub(fadd(fmul(o.w, q.z), fmul(o.x, q.y)), fmul(o.y, q.x)), fmul(o.z, q.w)),
              fsub(fsub(fsub(fmul(o.w, q.w), fmul(o.x, q.x)), fmul(o.y, q.y)), fmul(o.z, q.z))};
}
__device__ __forceinline__ float q_lensq(F4 q) {
    return fadd(fadd(fadd(fmul(q.x, q.x), fmul(q.y, q.y)), fmul(q.z, q.z)), fmul(q.w, q.w));
}
__device__ __forceinline__ F4 q_scale_inv(F4 q, float f) {
    const float d = fdiv(1.0f, f);
    return F4{fmul(q.x, d), fmul(q.y, d), fmul(q.z, d), fmul(q.w, d)};
}
__device__ __forceinline__ F4 q_conj(F4 q) { return F4{fneg(q.x), fneg(q.y), fneg(q.z), q.w}; }
__device__ __forceinline__ F4 q_identity() { return F4{0.0f, 0.0f, 0.0f, 1.0f}; }

// RotationMatrix(Quaternion) (Matrix_inline.h:365)
__device__ __forceinline__ M3 m_of_q(F4 q) {
    const float x = q.x, y = q.y, z = q.z, w = q.w;
    M3 m;
    m.r0 = F3{fsub(1.0f, fmul(2.0f, fadd(fmul(y, y), fmul(z, z)))), fmul(2.0f, fadd(fmul(x, y), fmul(z, w))),
              fmul(2.0f, fsub(fmul(x, z), fmul(y, w)))};
    m.r1 = F3{fmul(2.0f, fsub(fmul(x, y), fmul(z, w))), fsub(1.0f, fmul(2.0f, fadd(fmul(x, x), fmul(z, z)))),
              fmul(2.0f, fadd(fmul(y, z), fmul(x, w)))};
    m.r2 = F3{fmul(2.0f, fadd(fmul(x, z), fmul(y, w))), fmul(2.0f, fsub(fmul(y, z), fmul(x, w))),
              fsub(1.0f, fmul(2.0f, fadd(fmul(x, x), fmul(y, y))))};
    return m;
}
// TransformCoord: the row vector (v, 1) times the matrix, divided by its w (the 0 0 0 1 column keeps every zero's
// sign through the sums)
__device__ __forceinline__ F3 m_apply(F3 v, const M3& m) {
    const float norm = fadd(fadd(fadd(fmul(0.0f, v.x), fmul(0.0f, v.y)), fmul(0.0f, v.z)), 1.0f);
    if (!(norm != 0.0f)) return F3{0.0f, 0.0f, 0.0f};
    return F3{fdiv(fadd(fadd(fadd(fmul(v.x, m.r0.x), fmul(v.y, m.r1.x)), fmul(v.z, m.r2.x)), 0.0f), norm),
              fdiv(fadd(fadd(fadd(fmul(v.x, m.r0.y), fmul(v.y, m.r1.y)), fmul(v.z, m.r2.y)), 0.0f), norm),
              fdiv(fadd(fadd(fadd(fmul(v.x, m.r0.z), fmul(v.y, m.r1.z)), fmul(v.z, m.r2.z)), 0.0f), norm)};
}

}  // namespace ebb
