// SPDX-License-Identifier: LGPL-2.1-or-later
// Derived from the GNU C Library 2.34 (sysdeps/ieee754/dbl-64 and flt-32, including ARM's optimized-routines code
// that glibc carries), as compiled for aarch64 by GCC: the reference transcribed each function operation for
// operation into Python (exact_ballpark/dlibm.py, vec_exp.py, vec_libm.py), and this file restates those
// transcriptions for the device and the host. Copyright notices: glibc's, ARM's (MIT upstream) and Sun's fdlibm.
//
// What Destiny's compiled code calls, bit for bit:
//   double: exp (e_exp.c), log (e_log.c), sin, cos, sincos (s_sin.c with __branred), pow (e_pow.c);
//   float:  expf, logf (e_expf.c, e_logf.c), sinf, cosf (s_sinf.c, s_cosf.c), acosf, atanf, atan2f (fdlibm).
// A fused multiply-add (dfma/ffma) appears exactly where GCC fused one in the aarch64 build, as the transcriptions
// record; every other operation is a single rounded IEEE operation (ebb_arith.cuh). The constants and tables come
// from ebb_libm_tables.h, which gen_libm_tables.py prints from the transcriptions' own values.
//
// Every function is __host__ __device__: the kernels call the device build; the host build serves the C oracle and
// the CPU tests that pin this file to the reference's golden vectors.
#pragma once

#include "ebb_arith.cuh"
#include "ebb_libm_tables.h"

#ifndef EBB_INF
#define EBB_INF (__builtin_inf())
#endif

namespace ebb {
namespace lm {

// ---- the tables, once for the device and once for the host ----
#ifdef __CUDACC__
__device__ const double d_sincostab[] = DL_SINCOSTAB_INIT;
__device__ const double d_br_toverp[] = DL_BR_TOVERP_INIT;
__device__ const double d_log_tab[] = DL_LOG_TAB_INIT;
__device__ const uint64_t d_exp_tab[] = DX_TAB_INIT;
__device__ const uint64_t d_exp2f_tab[] = FL_EXP2F_TAB_INIT;
__device__ const double d_logf_tab[] = FL_LOGF_TAB_INIT;
__device__ const uint32_t d_inv_pio4[] = FL_INV_PIO4_INIT;
__device__ const double d_pow_tab[] = FL_POW_TAB_INIT;
__device__ const double d_powf_invc[] = FL_POWF_INVC_INIT;
__device__ const double d_powf_logc[] = FL_POWF_LOGC_INIT;
#endif
static const double h_sincostab[] = DL_SINCOSTAB_INIT;
static const double h_br_toverp[] = DL_BR_TOVERP_INIT;
static const double h_log_tab[] = DL_LOG_TAB_INIT;
static const uint64_t h_exp_tab[] = DX_TAB_INIT;
static const uint64_t h_exp2f_tab[] = FL_EXP2F_TAB_INIT;
static const double h_logf_tab[] = FL_LOGF_TAB_INIT;
static const uint32_t h_inv_pio4[] = FL_INV_PIO4_INIT;
static const double h_pow_tab[] = FL_POW_TAB_INIT;
static const double h_powf_invc[] = FL_POWF_INVC_INIT;
static const double h_powf_logc[] = FL_POWF_LOGC_INIT;

#ifdef __CUDA_ARCH__
#define EBB_TAB(name, i) (__ldg(&d_##name[(i)]))
#else
#define EBB_TAB(name, i) (h_##name[(i)])
#endif

// ======================================================================================== exp (e_exp.c)

// The special case of exp's main path for 512 <= |x| < 1024 (specialcase in e_exp.c): the scale rebiased so the
// result neither overflows nor underflows early; the subnormal side rounded once through a two-sum with 1.
EBB_HDNI double exp_special(double tmp, uint64_t sbits, uint64_t ki) {
    if ((ki & 0x80000000ULL) == 0) {
        const double scale = dfrom(sbits - (1009ULL << 52));
        return dmul(dfma(tmp, scale, scale), DX_TWO_1009);
    }
    const double scale = dfrom(sbits + (1022ULL << 52));
    const double st = dmul(tmp, scale);                              // not fused in the compiled code
    double y = dadd(scale, st);
    if (y < 1.0) {
        double lo = dadd(dsub(scale, y), st);
        const double hi = dadd(y, 1.0);
        lo = dadd(dadd(dsub(1.0, hi), y), lo);
        y = dsub(dadd(lo, hi), 1.0);
        if (y == 0.0) y = 0.0;
    }
    return dmul(y, DX_TWO_M1022);
}

// glibc's exp (vec_exp.exp): k = round(x 128/ln2), r = x - k ln2/128 in two fused steps, a degree-5 polynomial
// around the table's 2^(k/128)
EBB_HD double exp(double x) {
    const uint64_t bits = dbits(x);
    const uint32_t abstop = (uint32_t)(bits >> 52) & 0x7ff;
    if (abstop < 0x3c9) return dadd(x, 1.0);                         // |x| < 2^-54 (zeros, subnormals)
    if (abstop > 0x408) {                                            // |x| >= 1024, infinities, NaN
        if (bits == 0xfff0000000000000ULL) return 0.0;
        if (abstop == 0x7ff) return dadd(x, 1.0);
        return (bits >> 63) ? 0.0 : dinf();                          // __math_uflow(0), __math_oflow(0)
    }
    const double z = dmul(x, DX_INVLN2N);
    const double kd = frinta(z);
    const uint64_t ki = (uint64_t)(int64_t)kd;
    double r = dfma(kd, DX_NEGLN2HIN, x);
    r = dfma(kd, DX_NEGLN2LON, r);
    const uint32_t idx = 2u * (uint32_t)(ki & 0x7f);
    const double tail = dfrom(EBB_TAB(exp_tab, idx));
    const uint64_t sbits = EBB_TAB(exp_tab, idx + 1) + (ki << 45);
    const double p23 = dfma(r, DX_C3, DX_C2);
    const double p45 = dfma(r, DX_C5, DX_C4);
    const double r2 = dmul(r, r);
    double tmp = dadd(r, tail);
    const double r4 = dmul(r2, r2);
    tmp = dfma(p23, r2, tmp);
    tmp = dfma(r4, p45, tmp);
    if (abstop == 0x408) return exp_special(tmp, sbits, ki);
    const double scale = dfrom(sbits);
    return dfma(tmp, scale, scale);
}

// ======================================================================================== log (e_log.c)

// glibc's log (dlibm.log): near 1 a degree-11 polynomial with r split at 2^27; otherwise x = 2^k z, r = z/c - 1
// against the 128-cell table, log c + k ln2 in two parts
EBB_HD double log(double x) {
    uint64_t ix = dbits(x);
    if (ix + DL_LOG_NEG_LO <= DL_LOG_RANGE) {                        // 1 - 2^-4 <= x < 1 + 0x1.09p-4
        if (ix == 0x3ff0000000000000ULL) return 0.0;
        const double bb[11] = DL_LOG_B_INIT;
        const double r = dsub(x, 1.0);
        double rhi = dfma(r, DL_LOG_TWO27, r);
        const double r2 = dmul(r, r);
        const double p78 = dfma(bb[8], r, bb[7]);
        rhi = dfma(dneg(r), DL_LOG_TWO27, rhi);                      // fmsub: (r + w) - w, w = r 2^27
        const double r3 = dmul(r, r2);
        const double p789 = dfma(bb[9], r2, p78);
        const double p45 = dfma(bb[5], r, bb[4]);
        const double p710 = dfma(bb[10], r3, p789);
        const double rhi2 = dmul(rhi, rhi);
        const double p456 = dfma(bb[6], r2, p45);
        const double hi = dfma(rhi2, bb[0], r);
        const double p12 = dfma(bb[2], r, bb[1]);
        const double p410 = dfma(p710, r3, p456);
        const double rlo = dsub(r, rhi);
        const double rr = dadd(r, rhi);
        const double p123 = dfma(bb[3], r2, p12);
        const double b0rlo = dmul(bb[0], rlo);
        double lo = dsub(r, hi);
        lo = dfma(rhi2, bb[0], lo);
        const double p = dfma(p410, r3, p123);
        lo = dfma(b0rlo, rr, lo);
        const double y = dfma(p, r3, lo);
        return dadd(hi, y);
    }
    const uint64_t top = ix >> 48;
    if (((top - 0x0010) & 0xffffffffULL) >= 0x7fe0) {                // below 2^-1022, negative, infinite or NaN
        if ((ix << 1) == 0) return dneg(dinf());
        if (ix == 0x7ff0000000000000ULL) return x;
        if ((top & 0x8000) || (top & 0x7ff0) == 0x7ff0) return dnan();
        ix = dbits(dmul(x, DL_LOG_TWO52)) + DL_LOG_NEG_52;           // a subnormal normalised by 2^52
    }
    const uint64_t tmp = ix + DL_LOG_NEG_OFF;
    const uint32_t i = (uint32_t)(tmp >> 45) & 127;
    const int64_t k = ((int64_t)tmp) >> 52;
    const uint64_t iz = ix - (tmp & 0xfff0000000000000ULL);
    const double kd = i2d(k);
    const double invc = EBB_TAB(log_tab, 2 * i), logc = EBB_TAB(log_tab, 2 * i + 1);
    const double a[5] = DL_LOG_A_INIT;
    const double w = dfma(DL_LOG_LN2HI, kd, logc);
    const double r = dfma(dfrom(iz), invc, -1.0);
    const double hi = dadd(r, w);
    const double p34 = dfma(a[4], r, a[3]);
    const double p12 = dfma(a[2], r, a[1]);
    const double r2 = dmul(r, r);
    double lo = dsub(w, hi);
    const double r3 = dmul(r, r2);
    lo = dadd(lo, r);
    const double p = dfma(p34, r2, p12);
    lo = dfma(DL_LOG_LN2LO, kd, lo);
    lo = dfma(a[0], r2, lo);
    lo = dfma(r3, p, lo);
    return dadd(lo, hi);
}

// ================================================================================ sin, cos, sincos (s_sin.c)

// TAYLOR_SIN: a + ((POLY(a a) a - da / 2) a a + da)
EBB_HD double taylor_sin(double a, double da) {
    const double xx = dmul(a, a);
    const double poly = dfma(xx, dfma(xx, dfma(xx, dfma(xx, DL_S5, DL_S4), DL_S3), DL_S2), DL_S1);
    const double t = dfma(poly, a, dneg(dmul(da, 0.5)));             // fnmsub: poly a - da/2
    return dadd(dfma(xx, t, da), a);
}

struct SinCell {
    double r, sn, ssn, cs, ccs;
};
// u = big + |x|: the table cell of the nearest 1/128 and the remainder
EBB_HD SinCell sin_cell(double x) {
    const double ax = dabs(x);
    const double u = dadd(DL_BIG, ax);
    const uint32_t k = ((uint32_t)(dbits(u) & 0xffffffffULL)) << 2;
    SinCell c;
    c.r = dsub(ax, dsub(u, DL_BIG));
    c.sn = EBB_TAB(sincostab, k);
    c.ssn = EBB_TAB(sincostab, k + 1);
    c.cs = EBB_TAB(sincostab, k + 2);
    c.ccs = EBB_TAB(sincostab, k + 3);
    return c;
}

// do_sin (s_sin.c): the Taylor polynomial below 0.126, else the table's sin and cos of the nearest cell
EBB_HD double do_sin(double x, double dx) {
    if (dabs(x) < DL_TAYLOR_LIMIT) return taylor_sin(x, dx);
    if (x <= 0.0) dx = dneg(dx);
    const SinCell c = sin_cell(x);
    const double xx = dmul(c.r, c.r);
    const double pc = dfma(xx, DL_CS6, DL_CS4);
    const double ps = dfma(xx, DL_SN5, DL_SN3);
    const double r3 = dmul(c.r, xx);
    const double c1 = dfma(xx, pc, DL_CS2);
    const double s = dadd(c.r, dfma(r3, ps, dx));
    const double cc = dfma(c.r, dx, dmul(xx, c1));
    const double cor = dfma(s, c.cs, dfma(dneg(cc), c.sn, dfma(s, c.ccs, c.ssn)));
    return dcopysign(dadd(c.sn, cor), x);
}

// do_cos (s_sin.c)
EBB_HD double do_cos(double x, double dx) {
    if (x < 0.0) dx = dneg(dx);
    const SinCell c = sin_cell(x);
    const double r = dadd(c.r, dx);
    const double xx = dmul(r, r);
    const double pc = dfma(xx, DL_CS6, DL_CS4);
    const double ps = dfma(xx, DL_SN5, DL_SN3);
    const double r3 = dmul(r, xx);
    const double c1 = dfma(xx, pc, DL_CS2);
    const double s = dfma(r3, ps, r);
    const double cc = dmul(xx, c1);
    const double cor = dfma(dneg(s), c.sn, dfma(dneg(cc), c.cs, dfma(dneg(s), c.ssn, c.ccs)));
    return dadd(c.cs, cor);
}

// x = n pi/2 + a + da
struct Reduced {
    int n;
    double a, da;
};

// reduce_sincos: x = n pi/2 + a + da in four fused steps, n the low bits of round(x 2/pi)
EBB_HD Reduced reduce_sincos(double x) {
    const double t = dfma(x, DL_HPINV, DL_TOINT);
    const double xn = dsub(t, DL_TOINT);
    const double y = dfma(dneg(xn), DL_MP2, dfma(dneg(xn), DL_MP1, x));
    const double t2 = dfma(dneg(xn), DL_PP3, y);
    const double b = dfma(dneg(xn), DL_PP4, t2);
    double db = dfma(dneg(xn), DL_PP3, dsub(y, t2));
    db = dadd(db, dfma(dneg(xn), DL_PP4, dsub(t2, b)));
    return Reduced{(int)(dbits(t) & 3), b, db};
}

// one half of __branred: xh 2/pi from six 24-bit pieces of 2/pi, the integer part split off
struct BranredHalf {
    double sum, b, bb;
};
EBB_HD BranredHalf branred_half(double xh) {
    const uint32_t e = (uint32_t)(dbits(xh) >> 52) & 0x7ff;
    int k = 0;
    if (e > (uint32_t)DL_BR_EXP_LIMIT && e >= (uint32_t)DL_BR_EXP_BIAS) k = (int)((e - (uint32_t)DL_BR_EXP_BIAS) / 24);
    double gor = dfrom(((uint64_t)(((uint32_t)DL_BR_T576_HI - ((uint32_t)(3 * k) << 23)) & 0xffffffffu)) << 32);
    double r[6];
    for (int i = 0; i < 6; ++i) {
        const double piece = (i == 0 && e <= (uint32_t)DL_BR_EXP_LIMIT) ? DL_BR_TOVERP0 : EBB_TAB(br_toverp, k + i);
        r[i] = dmul(dmul(xh, piece), gor);
        gor = dmul(gor, DL_BR_TM24);
    }
    double total = 0.0;
    for (int i = 0; i < 3; ++i) {
        const double s = dsub(dadd(r[i], DL_BR_BIG), DL_BR_BIG);
        total = dadd(total, s);
        r[i] = dsub(r[i], s);
    }
    double t = 0.0;
    for (int i = 0; i < 6; ++i) t = dadd(t, r[5 - i]);
    double bb = dadd(dadd(dadd(dadd(dadd(dsub(r[0], t), r[1]), r[2]), r[3]), r[4]), r[5]);
    double s = dsub(dadd(t, DL_BR_BIG), DL_BR_BIG);
    total = dadd(s, total);
    t = dsub(t, s);
    s = dsub(dadd(total, DL_BR_BIG1), DL_BR_BIG1);
    total = dsub(total, s);
    const double b = dadd(bb, t);
    bb = dadd(dsub(t, b), bb);
    return BranredHalf{total, b, bb};
}

// __branred: x = n pi/2 + a + da for huge x (scaled by 2^-600 and split in two)
EBB_HDNI Reduced branred(double x) {
    x = dmul(x, DL_BR_TM600);
    const double t0 = dmul(x, DL_BR_SPLIT);
    const double x1 = dsub(t0, dsub(t0, x));
    const double x2 = dsub(x, x1);
    const BranredHalf h1 = branred_half(x1), h2 = branred_half(x2);
    const double sum1 = h1.sum, b1 = h1.b, bb1 = h1.bb, sum2 = h2.sum, b2 = h2.b, bb2 = h2.bb;
    double total = dadd(sum1, sum2);
    double b = dadd(b1, b2);
    double bb = (dabs(b1) > dabs(b2)) ? dadd(dsub(b1, b), b2) : dadd(dsub(b2, b), b1);
    if (b > 0.5) {
        b = dsub(b, 1.0);
        total = dadd(total, 1.0);
    } else if (b < -0.5) {
        b = dadd(b, 1.0);
        total = dsub(total, 1.0);
    }
    const double s = dadd(dadd(dadd(bb, bb1), bb2), b);
    const double t = dadd(dadd(dsub(b, s), bb), dadd(bb1, bb2));
    const double sp = dmul(s, DL_BR_SPLIT);
    const double t1 = dsub(sp, dsub(sp, s));
    const double t2 = dsub(s, t1);
    const double bh = dmul(s, DL_BR_HP0);
    const double bl = dadd(dadd(dadd(dsub(dmul(t1, DL_BR_MP1), bh), dmul(t1, DL_BR_MP2)), dmul(t2, DL_BR_MP1)),
                           dadd(dadd(dmul(t2, DL_BR_MP2), dmul(s, DL_BR_HP1)), dmul(t, DL_BR_HP0)));
    const double ss = dadd(bh, bl);
    return Reduced{(int)(to_i64(total) & 3), ss, dadd(dsub(bh, ss), bl)};
}

// do_sincos: do_cos for odd n, else do_sin; negated when n & 2
EBB_HD double sincos_n(double a, double da, int n) {
    const double v = (n & 1) ? do_cos(a, da) : do_sin(a, da);
    return (n & 2) ? dneg(v) : v;
}

EBB_HDNI double sin(double x) {
    const uint32_t k = (uint32_t)(dbits(x) >> 32) & 0x7fffffffu;
    if (k < (uint32_t)DL_K_TINY_SIN) return x;
    if (k < (uint32_t)DL_K_DO_SIN) return do_sin(x, 0.0);
    if (k < (uint32_t)DL_K_MID) return dcopysign(do_cos(dsub(DL_HP0, dabs(x)), DL_HP1), x);
    Reduced r;
    if (k < (uint32_t)DL_K_REDUCE) r = reduce_sincos(x);
    else if (k < (uint32_t)DL_K_HUGE) r = branred(x);
    else return dnan();
    return sincos_n(r.a, r.da, r.n);
}

EBB_HDNI double cos(double x) {
    const uint32_t k = (uint32_t)(dbits(x) >> 32) & 0x7fffffffu;
    if (k < (uint32_t)DL_K_TINY_COS) return 1.0;
    if (k < (uint32_t)DL_K_DO_SIN) return do_cos(x, 0.0);
    if (k < (uint32_t)DL_K_MID) {
        const double y = dsub(DL_HP0, dabs(x));
        const double a = dadd(y, DL_HP1);
        return do_sin(a, dadd(dsub(y, a), DL_HP1));
    }
    Reduced r;
    if (k < (uint32_t)DL_K_REDUCE) r = reduce_sincos(x);
    else if (k < (uint32_t)DL_K_HUGE) r = branred(x);
    else return dnan();
    return sincos_n(r.a, r.da, r.n + 1);
}

struct SinCos {
    double s, c;
};

// sincos as Destiny's compiled code takes a sine and a cosine of one argument: __sin's and __cos's branches, except
// that between 0.855469 and 2.426265 the sine is do_cos after the two-sum of hp0 - |x| and hp1
EBB_HDNI SinCos sincos_v(double x) {
    const uint32_t k = (uint32_t)(dbits(x) >> 32) & 0x7fffffffu;
    if (k < (uint32_t)DL_K_TINY_COS) return SinCos{x, 1.0};
    if (k < (uint32_t)DL_K_DO_SIN) return SinCos{do_sin(x, 0.0), do_cos(x, 0.0)};
    if (k < (uint32_t)DL_K_MID) {
        const double y = dsub(DL_HP0, dabs(x));
        const double a = dadd(y, DL_HP1);
        const double da = dadd(dsub(y, a), DL_HP1);
        return SinCos{dcopysign(do_cos(a, da), x), do_sin(a, da)};
    }
    Reduced r;
    if (k < (uint32_t)DL_K_REDUCE) r = reduce_sincos(x);
    else if (k < (uint32_t)DL_K_HUGE) r = branred(x);
    else return SinCos{dnan(), dnan()};
    return SinCos{sincos_n(r.a, r.da, r.n), sincos_n(r.a, r.da, r.n + 1)};
}
EBB_HD void sincos(double x, double* s_out, double* c_out) {
    const SinCos v = sincos_v(x);
    *s_out = v.s;
    *c_out = v.c;
}

// ======================================================================================== expf, logf

// glibc's expf (e_expf.c): k = round(x 32/ln2), a cubic in the rest around 2^(k/32), rounded to float
EBB_HD float expf(float xf) {
    const uint32_t ix = fbits(xf);
    const uint32_t abstop = (ix >> 20) & 0x7ff;
    const double x = tod(xf);
    if (abstop > 0x42a) {                                            // |x| >= 88 or NaN
        const float oflow = ffrom(FL_EXPF_OFLOW_BITS);
        const float may = ffrom(FL_EXPF_MAY_UFLOW_BITS);
        if (!(xf <= oflow && xf >= may)) {
            if (ix == 0xff800000u) return 0.0f;
            if (abstop >= 0x7f8) return fadd(xf, xf);
            if (xf > oflow) return finf();                           // __math_oflowf
            if (xf < ffrom(FL_EXPF_UFLOW_BITS)) return 0.0f;         // __math_uflowf
            return ffrom(FL_MAY_UFLOWF_BITS);                        // __math_may_uflowf
        }
    }
    const double cc[3] = FL_EXPF_C_INIT;
    const double z = dmul(x, FL_EXPF_INVLN2);
    const double kd = frinta(z);
    const uint64_t ki = (uint64_t)(int64_t)kd;
    const double r = dsub(z, kd);
    const double s = dfrom(EBB_TAB(exp2f_tab, ki & 31) + (ki << 47));
    const double zc = dfma(r, cc[0], cc[1]);
    double y = dfma(r, cc[2], 1.0);
    const double r2 = dmul(r, r);
    y = dfma(zc, r2, y);
    return tof(dmul(y, s));
}

// glibc's logf (e_logf.c): x = 2^k z, r = z/c - 1 fused, a cubic in r, log c + k ln2 fused
EBB_HD float logf(float xf) {
    uint32_t ix = fbits(xf);
    if (ix == 0x3f800000u) return 0.0f;
    if (ix - 0x00800000u >= 0x7f000000u) {                           // below 2^-126, negative, infinite or NaN
        if ((ix & 0x7fffffffu) == 0) return fneg(finf());
        if (ix == 0x7f800000u) return finf();
        if ((ix & 0x80000000u) || (ix & 0x7f800000u) == 0x7f800000u) return fnan();
        ix = fbits(fmul(xf, 8388608.0f)) - (23u << 23);              // a subnormal normalised by 2^23
    }
    const uint32_t tmp = ix - 0x3f330000u;
    const uint32_t i = (tmp >> 19) & 15;
    const int32_t k = ((int32_t)tmp) >> 23;
    const float zf = ffrom(ix - (tmp & 0xff800000u));
    const double z = tod(zf);
    const double invc = EBB_TAB(logf_tab, 2 * i), logc = EBB_TAB(logf_tab, 2 * i + 1);
    const double A[3] = FL_LOGF_A_INIT;
    const double r = dfma(z, invc, -1.0);
    const double y0 = dfma(i2d(k), FL_LOGF_LN2, logc);
    double y = dfma(r, A[1], A[2]);
    const double r2 = dmul(r, r);
    const double ry0 = dadd(r, y0);
    y = dfma(r2, A[0], y);
    return tof(dfma(y, r2, ry0));
}

// ======================================================================================== sinf, cosf

// sinf_poly's sine branch: x3 = x x2, s1 = s2 + x2 s3, x7 = x2 x3, (x + x3 s1) + s1 x7
EBB_HD double sinf_sin_poly(double x, double x2) {
    const double S[3] = FL_SINF_S_INIT;
    const double x3 = dmul(x, x2);
    const double s1 = dfma(x2, S[2], S[1]);
    const double x7 = dmul(x2, x3);
    const double s = dfma(x3, S[0], x);
    return dfma(s1, x7, s);
}
// sinf_poly's cosine branch: c1 = c0 + x2 c1, c2 = c3 + x2 c4, x4 = x2 x2, x6 = x2 x4, (c1 + x4 c2) + c2 x6
EBB_HD double sinf_cos_poly(double x2) {
    const double C[5] = FL_COSF_C_INIT;
    const double c1 = dfma(x2, C[1], C[0]);
    const double c2 = dfma(x2, C[4], C[3]);
    const double x4 = dmul(x2, x2);
    const double x6 = dmul(x2, x4);
    const double c = dfma(x4, C[2], c1);
    return dfma(c2, x6, c);
}

// reduce_large (sincosf.h): x 4/pi in 62-bit fixed point from __inv_pio4
struct ReducedF {
    int n;
    double x;
};
EBB_HD ReducedF sinf_reduce_large(uint32_t xi) {
    const uint32_t idx = (xi >> 26) & 15;
    const int shift = (xi >> 23) & 7;
    const uint32_t m = ((xi & 0x7fffffu) | 0x800000u) << shift;
    uint64_t res0 = (uint64_t)(uint32_t)(m * EBB_TAB(inv_pio4, idx));
    const uint64_t res1 = (uint64_t)m * EBB_TAB(inv_pio4, idx + 4);
    const uint64_t res2 = (uint64_t)m * EBB_TAB(inv_pio4, idx + 8);
    res0 = (res2 >> 32) | (res0 << 32);
    res0 += res1;
    const uint64_t n = (res0 + (1ULL << 61)) >> 62;
    res0 -= n << 62;
    return ReducedF{(int)n, dmul(i2d((int64_t)res0), FL_PI63)};
}

// glibc's sinf (cosine = false) and cosf (cosine = true): the polynomial at x below pi/4 (x or 1 below 2^-12);
// reduce_fast below 120, reduce_large above; the quadrant's sign, the polynomial by n's parity, the second table's
// negated cosine applied as the result's sign (exact)
EBB_HD float sincosf_one(float y, bool cosine) {
    const uint32_t ix = fbits(y);
    const uint32_t abstop = (ix >> 20) & 0x7ff;
    const double x = tod(y);
    if (abstop < 0x3f4) {
        if (abstop < 0x398) return cosine ? 1.0f : y;
        const double xx = dmul(x, x);
        return tof(cosine ? sinf_cos_poly(xx) : sinf_sin_poly(x, xx));
    }
    if (abstop >= 0x7f8) return fnan();
    const double SIGN[4] = FL_SINCOSF_SIGN_INIT;
    int n, q;
    double xr;
    if (abstop < 0x42f) {
        const double kd = frinta(dmul(x, FL_HPI_INV));
        xr = dfma(kd, dneg(FL_HPI), x);
        n = (int)(int64_t)kd;
        q = n;
    } else {
        const ReducedF rl = sinf_reduce_large(ix);
        xr = rl.x;
        n = rl.n;
        q = n + (int)(ix >> 31);
    }
    const double s = SIGN[q & 3];
    const double x2 = dmul(xr, xr);
    const bool use_cos = cosine ? ((n & 1) == 0) : ((n & 1) == 1);
    double v;
    if (use_cos) {
        v = sinf_cos_poly(x2);
        if (q & 2) v = dneg(v);
    } else {
        v = sinf_sin_poly(dmul(xr, s), x2);
    }
    return tof(v);
}
EBB_HD float sinf(float x) { return sincosf_one(x, false); }
EBB_HD float cosf(float x) { return sincosf_one(x, true); }

// ======================================================================================== acosf, atanf, atan2f

// e_acosf.c's r = p/q, every step fused as compiled
EBB_HD float acosf_r(float z) {
    const float p4 = ffma(z, ffrom(FL_ACOSF_PS5_BITS), ffrom(FL_ACOSF_PS4_BITS));
    const float q3 = ffma(z, ffrom(FL_ACOSF_QS4_BITS), ffrom(FL_ACOSF_QS3_BITS));
    const float p3 = ffma(p4, z, ffrom(FL_ACOSF_PS3_BITS));
    const float q2 = ffma(q3, z, ffrom(FL_ACOSF_QS2_BITS));
    const float p2 = ffma(p3, z, ffrom(FL_ACOSF_PS2_BITS));
    const float q1 = ffma(q2, z, ffrom(FL_ACOSF_QS1_BITS));
    const float p1 = ffma(p2, z, ffrom(FL_ACOSF_PS1_BITS));
    const float q = ffma(q1, z, 1.0f);
    const float p0 = ffma(p1, z, ffrom(FL_ACOSF_PS0_BITS));
    const float p = fmul(p0, z);
    return fdiv(p, q);
}

// fdlibm's acosf (e_acosf.c) as glibc 2.34 aarch64 compiled it
EBB_HDNI float acosf(float x) {
    const uint32_t hx = fbits(x);
    const uint32_t ix = hx & 0x7fffffffu;
    const float pi = ffrom(FL_ACOSF_PI_BITS), pio2_hi = ffrom(FL_ACOSF_PIO2_HI_BITS);
    const float pio2_lo = ffrom(FL_ACOSF_PIO2_LO_BITS);
    if (ix == 0x3f800000u) return (hx >> 31) ? fadd(pi, ffrom(FL_ACOSF_TWO_PIO2_LO_BITS)) : 0.0f;
    if (ix > 0x3f800000u) return fnan();
    if (ix < 0x3f000000u) {                                          // |x| < 0.5
        if (ix <= 0x32800000u) return fadd(pio2_hi, pio2_lo);
        const float z = fmul(x, x);
        const float t = ffma(fneg(x), acosf_r(z), pio2_lo);
        return fsub(pio2_hi, fsub(x, t));
    }
    if (hx >> 31) {                                                  // x < -0.5
        const float z = fmul(fadd(x, 1.0f), 0.5f);
        const float r = acosf_r(z);
        const float s = fsqrt(z);
        const float w = ffma(s, r, ffrom(FL_ACOSF_NEG_PIO2_LO_BITS));
        return ffma(fneg(fadd(s, w)), 2.0f, pi);
    }
    const float z = fmul(fsub(1.0f, x), 0.5f);                       // x > 0.5
    const float s = fsqrt(z);
    const float df = ffrom(fbits(s) & 0xfffff000u);
    const float c = fdiv(ffma(fneg(df), df, z), fadd(s, df));
    const float w = ffma(s, acosf_r(z), c);
    return fadd(fadd(df, w), fadd(df, w));
}

// fdlibm's atanf (s_atanf.c) as glibc 2.34 aarch64 compiled it
EBB_HDNI float atanf(float x) {
    const uint32_t hx = fbits(x);
    const uint32_t ix = hx & 0x7fffffffu;
    if (ix > 0x4bffffffu) {                                          // |x| >= 2^25
        if (ix > 0x7f800000u) return fadd(x, x);
        const float hi3 = ffrom(FL_ATANF_HI3_BITS), lo3 = ffrom(FL_ATANF_LO3_BITS);
        return (hx >> 31) ? fsub(fneg(hi3), lo3) : fadd(hi3, lo3);
    }
    int id = -1;
    float xr = x;
    if (ix <= 0x3edfffffu) {                                         // |x| < 7/16
        if (ix <= 0x30ffffffu) return x;                             // |x| < 2^-29
    } else {
        const float ax = fabs_(x);
        if (ix <= 0x3f97ffffu) {
            if (ix <= 0x3f2fffffu) {
                id = 0;
                xr = fdiv(ffma(ax, 2.0f, -1.0f), fadd(ax, 2.0f));
            } else {
                id = 1;
                xr = fdiv(fsub(ax, 1.0f), fadd(ax, 1.0f));
            }
        } else if (ix <= 0x401bffffu) {
            id = 2;
            xr = fdiv(fsub(ax, 1.5f), ffma(ax, 1.5f, 1.0f));
        } else {
            id = 3;
            xr = fdiv(-1.0f, ax);
        }
    }
    const float z = fmul(xr, xr);
    const float w = fmul(z, z);
    const float t8 = ffma(w, ffrom(FL_ATANF_T10_BITS), ffrom(FL_ATANF_T8_BITS));
    const float t7 = ffma(w, ffrom(FL_ATANF_T9_BITS), ffrom(FL_ATANF_T7_BITS));
    const float t6 = ffma(t8, w, ffrom(FL_ATANF_T6_BITS));
    const float t5 = ffma(t7, w, ffrom(FL_ATANF_T5_BITS));
    const float t4 = ffma(t6, w, ffrom(FL_ATANF_T4_BITS));
    const float t3 = ffma(t5, w, ffrom(FL_ATANF_T3_BITS));
    const float t2 = ffma(t4, w, ffrom(FL_ATANF_T2_BITS));
    const float t1 = ffma(t3, w, ffrom(FL_ATANF_T1_BITS));
    const float t0 = ffma(t2, w, ffrom(FL_ATANF_T0_BITS));
    const float s12 = ffma(t0, z, fmul(t1, w));
    const float xs12 = fmul(xr, s12);
    if (id < 0) return fsub(xr, xs12);
    const double HI[4] = FL_ATANF_HI_INIT;
    const double LO[4] = FL_ATANF_LO_INIT;
    const float zz = fsub(tof(HI[id]), fsub(fsub(xs12, tof(LO[id])), xr));
    return (hx >> 31) ? fneg(zz) : zz;
}

// fdlibm's atan2f (e_atan2f.c) as glibc 2.34 aarch64 compiled it
EBB_HDNI float atan2f(float y, float x) {
    const uint32_t hx = fbits(x), hy = fbits(y);
    const uint32_t ix = hx & 0x7fffffffu, iy = hy & 0x7fffffffu;
    if (ix > 0x7f800000u || iy > 0x7f800000u) return fadd(x, y);
    if (hx == 0x3f800000u) return atanf(y);
    const uint32_t m = ((hx >> 30) & 2u) | (hy >> 31);
    const float pi = ffrom(FL_ATAN2F_PI_BITS), tiny = ffrom(FL_ATAN2F_TINY_BITS);
    const float pi_t = fadd(pi, tiny), mpi_t = fsub(ffrom(FL_ATAN2F_NEG_PI_BITS), tiny);
    const float pio2_t = (hy >> 31) ? fsub(ffrom(FL_ATAN2F_NEG_PIO2_BITS), tiny) : fadd(ffrom(FL_ATAN2F_PIO2_BITS), tiny);
    if (iy == 0) return m <= 1 ? y : (m == 2 ? pi_t : mpi_t);
    if (ix == 0) return pio2_t;
    if (ix == 0x7f800000u) {
        if (iy == 0x7f800000u) {
            const float pio4 = ffrom(FL_ATAN2F_PIO4_BITS);
            if (m == 0) return fadd(pio4, tiny);
            if (m == 1) return fsub(ffrom(FL_ATAN2F_NEG_PIO4_BITS), tiny);
            if (m == 2) return ffma(3.0f, pio4, tiny);
            return ffma(-3.0f, pio4, ffrom(FL_ATAN2F_NEG_TINY_BITS));
        }
        if (m == 0) return 0.0f;
        if (m == 1) return -0.0f;
        return m == 2 ? pi_t : mpi_t;
    }
    if (iy == 0x7f800000u) return pio2_t;
    const int32_t k = ((int32_t)iy - (int32_t)ix) >> 23;
    float z;
    if (k > 60) z = fsub(ffrom(FL_ATAN2F_PIO2_BITS), ffrom(FL_ATAN2F_NEG_HALF_PI_LO_BITS));
    else if ((hx >> 31) && k < -60) z = 0.0f;
    else z = atanf(fabs_(fdiv(y, x)));
    if (m == 0) return z;
    if (m == 1) return fneg(z);
    const float zl = fadd(z, ffrom(FL_ATAN2F_NEG_PI_LO_BITS));       // z - pi_lo
    return m == 2 ? fsub(pi, zl) : fsub(zl, pi);
}

// ======================================================================================== pow (e_pow.c)

// checkint: 0 if y is not an integer, 1 if odd, 2 if even
EBB_HD int pow_checkint(uint64_t iy) {
    const int e = (int)(iy >> 52) & 0x7ff;
    if (e < 0x3ff) return 0;
    if (e > 0x3ff + 52) return 2;
    if (iy & ((1ULL << (0x3ff + 52 - e)) - 1)) return 0;
    if (iy & (1ULL << (0x3ff + 52 - e))) return 1;
    return 2;
}

struct HiLo {
    double hi, lo;
};
// log_inline: log x as hi + lo, every step as compiled
EBB_HD HiLo pow_log_inline(uint64_t ix) {
    const uint64_t tmp = ix - FL_POW_OFF;
    const uint32_t i = (uint32_t)(tmp >> 45) & 127;
    const double kd = i2d(((int64_t)tmp) >> 52);
    const double z = dfrom(ix - (tmp & 0xfff0000000000000ULL));
    const double invc = EBB_TAB(pow_tab, 3 * i), logc = EBB_TAB(pow_tab, 3 * i + 1);
    const double logctail = EBB_TAB(pow_tab, 3 * i + 2);
    const double A[7] = FL_POW_A_INIT;
    const double t1 = dfma(kd, FL_POW_LN2HI, logc);
    const double r = dfma(z, invc, -1.0);
    const double lo1 = dfma(kd, FL_POW_LN2LO, logctail);
    const double ar = dmul(r, A[0]);
    const double a56 = dfma(r, A[6], A[5]);
    const double t2 = dadd(r, t1);
    const double a34 = dfma(r, A[4], A[3]);
    const double a12 = dfma(r, A[2], A[1]);
    const double ar2 = dmul(r, ar);
    const double d = dsub(t1, t2);
    const double lo3 = dfma(ar, r, dneg(ar2));
    const double a3456 = dfma(ar2, a56, a34);
    const double hi = dadd(t2, ar2);
    const double lo2 = dadd(d, r);
    const double ar3 = dmul(r, ar2);
    const double e = dsub(t2, hi);
    double s = dadd(lo1, lo2);
    const double poly = dfma(ar2, a3456, a12);
    const double lo4 = dadd(e, ar2);
    s = dadd(s, lo3);
    s = dadd(s, lo4);
    const double lo = dfma(ar3, poly, s);
    const double y = dadd(hi, lo);
    return HiLo{y, dadd(dsub(hi, y), lo)};
}

// exp_inline: sign x exp(ehi + elo), the sign through the scale's sign bit
EBB_HD double pow_exp_inline(double ehi, double elo, bool negative) {
    const uint32_t abstop = (uint32_t)(dbits(ehi) >> 52) & 0x7ff;
    if (abstop < 0x3c9) {
        const double one = dadd(ehi, 1.0);
        return negative ? dneg(one) : one;
    }
    if (abstop > 0x408) {
        const double f = ehi < 0.0 ? 0.0 : dinf();
        return negative ? dneg(f) : f;
    }
    const double kd = frinta(dmul(ehi, DX_INVLN2N));
    const uint64_t ki = (uint64_t)(int64_t)kd;
    double r = dfma(kd, DX_NEGLN2HIN, ehi);
    r = dfma(kd, DX_NEGLN2LON, r);
    const uint32_t idx = 2u * (uint32_t)(ki & 0x7f);
    const double tail = dfrom(EBB_TAB(exp_tab, idx));
    const uint64_t base = EBB_TAB(exp_tab, idx + 1) + (ki << 45);
    const uint64_t sgn = negative ? 0x8000000000000000ULL : 0;
    r = dadd(elo, r);
    const double p23 = dfma(r, DX_C3, DX_C2);
    const double p45 = dfma(r, DX_C5, DX_C4);
    const double r2 = dmul(r, r);
    const double t = dadd(r, tail);
    const double r4 = dmul(r2, r2);
    double tmp = dfma(r2, p23, t);
    tmp = dfma(r4, p45, tmp);
    if (abstop != 0x408) {
        const double scale = dfrom(base ^ sgn);
        return dfma(tmp, scale, scale);
    }
    if ((ki & 0x80000000ULL) == 0) {
        const double sc = dfrom((base - (1009ULL << 52)) ^ sgn);
        return dmul(dfma(tmp, sc, sc), DX_TWO_1009);
    }
    const uint64_t sb = (base + (1022ULL << 52)) ^ sgn;
    const double sc = dfrom(sb);
    const double st = dmul(tmp, sc);                                 // not fused in the compiled code
    double y = dadd(sc, st);
    if (dabs(y) < 1.0) {
        const double one = y < 0.0 ? -1.0 : 1.0;
        double lo = dadd(dsub(sc, y), st);
        const double hi = dadd(y, one);
        lo = dadd(dadd(dsub(one, hi), y), lo);
        y = dsub(dadd(lo, hi), one);
        if (y == 0.0) y = dfrom(sb & 0x8000000000000000ULL);
    }
    return dmul(y, DX_TWO_M1022);
}

// glibc's pow: log_inline, y log x in two parts (fused), exp_inline; the special cases in glibc's order
EBB_HDNI double pow(double x, double y) {
    uint64_t ix = dbits(x);
    const uint64_t iy = dbits(y);
    uint32_t topx = (uint32_t)(ix >> 52);
    const uint32_t topy = (uint32_t)(iy >> 52);
    bool negative = false;
    const uint64_t one_bits = 0x3ff0000000000000ULL, inf_bits = 0x7ff0000000000000ULL;
    if (topx - 0x001 >= 0x7ff - 0x001 || (topy & 0x7ff) - 0x3be >= 0x43e - 0x3be) {
        if (2 * iy - 1 >= 2 * inf_bits - 1) {                        // y zero, infinite or NaN
            if (2 * iy == 0) return 1.0;
            if (ix == one_bits) return 1.0;
            if (2 * ix > 2 * inf_bits || 2 * iy > 2 * inf_bits) return dadd(x, y);
            if (2 * ix == 2 * one_bits) return 1.0;
            if ((2 * ix < 2 * one_bits) == !(iy >> 63)) return 0.0;
            return dmul(y, y);
        }
        if (2 * ix - 1 >= 2 * inf_bits - 1) {                        // x zero, infinite or NaN
            double x2 = dmul(x, x);
            if ((ix >> 63) && pow_checkint(iy) == 1) x2 = dneg(x2);
            return (iy >> 63) ? ddiv(1.0, x2) : x2;
        }
        if (ix >> 63) {                                              // finite x < 0
            const int yint = pow_checkint(iy);
            if (yint == 0) return dnan();
            if (yint == 1) negative = true;
            ix &= 0x7fffffffffffffffULL;
            topx &= 0x7ff;
        }
        if ((topy & 0x7ff) - 0x3be >= 0x43e - 0x3be) {               // |y| below 2^-65 or at 2^63 and beyond
            if (ix == one_bits) return 1.0;
            if ((topy & 0x7ff) < 0x3be) return ix > one_bits ? dadd(1.0, y) : dsub(1.0, y);
            return (ix > one_bits) == (topy < 0x800) ? dinf() : 0.0;
        }
        if (topx == 0) {                                             // a subnormal x normalised
            ix = dbits(dmul(x, 4503599627370496.0)) & 0x7fffffffffffffffULL;
            ix -= 52ULL << 52;
        }
    }
    const HiLo hl = pow_log_inline(ix);
    const double hi = hl.hi, lo = hl.lo;
    const double ehi = dmul(y, hi);
    const double elo = dfma(y, lo, dfma(y, hi, dneg(ehi)));
    return pow_exp_inline(ehi, elo, negative);
}

// ---- powf: glibc 2.34's e_powf.c (ARM's optimized-routines), as the aarch64 build computes it ----
// x = 2^k z with z within a 16th of an octave of a table point c: log2 x (times 32) is k + log2 c plus a quintic in
// r = z/c - 1, all in double; y log2 x then goes through exp2's 32-entry table and a cubic, rounded to float once.
// Six multiply-adds are fused in the logarithm and three in the exponential, the ones the aarch64 build fuses.

// log2(x) x 32 for the bits ix of a positive normal (or normalised) x
EBB_HD double powf_log2(uint32_t ix) {
    const uint32_t tmp = ix - 0x3f330000u;                           // ix - OFF: z in [OFF, 2 OFF)
    const int i = (int)((tmp >> 19) & 15u);
    const uint32_t top = tmp & 0xff800000u;
    const uint32_t iz = ix - top;
    const int32_t k = (int32_t)top >> 18;                             // the exponent, times 32
    const double a[5] = FL_POWF_A_INIT;
    const double invc = EBB_TAB(powf_invc, i), logc = EBB_TAB(powf_logc, i);
    const double z = tod(ffrom(iz));
    const double r = dfma(invc, z, -1.0);
    const double y0 = dadd((double)k, logc);
    const double p = dfma(r, a[2], a[3]);
    double q = dfma(r, a[4], y0);
    const double r2 = dmul(r, r);
    const double yy = dfma(r, a[0], a[1]);
    const double r4 = dmul(r2, r2);
    q = dfma(r2, p, q);
    return dfma(yy, r4, q);
}
// 2^(xd / 32) rounded to float, negative when sign_bias says so (expf's table and cubic)
EBB_HD float powf_exp2(double xd, uint64_t sign_bias) {
    const double cc[3] = FL_EXPF_C_INIT;
    const double kd = frinta(xd);
    const uint64_t ki = (uint64_t)(int64_t)kd;
    const double r = dsub(xd, kd);
    double y = dfma(r, cc[2], 1.0);
    const double zc = dfma(r, cc[0], cc[1]);
    const double r2 = dmul(r, r);
    const uint64_t t = EBB_TAB(exp2f_tab, ki & 31) + ((ki + sign_bias) << 47);
    y = dfma(zc, r2, y);
    return tof(dmul(y, dfrom(t)));
}
// 1 for an odd integer y, 2 for an even one, 0 for none (its bits iy)
EBB_HD int powf_checkint(uint32_t iy) {
    const int e = (int)((iy >> 23) & 0xff);
    if (e < 0x7f) return 0;
    if (e > 0x7f + 23) return 2;
    const uint32_t bit = 1u << (0x7f + 23 - e);
    if (iy & (bit - 1)) return 0;
    return (iy & bit) ? 1 : 2;
}
EBB_HD bool powf_signaling(uint32_t u) { return ((u ^ 0x00400000u) & 0x7fffffffu) > 0x7fc00000u; }
// __math_oflowf, __math_uflowf, __math_may_uflowf: (sign ? -t : t) t in float
EBB_HD float powf_xflow(uint64_t sign_bias, uint32_t tbits) {
    const float t = ffrom(tbits);
    return fmul(sign_bias ? fneg(t) : t, t);
}
EBB_HD float powf(float x, float y) {
    uint32_t ix = fbits(x);
    const uint32_t iy = fbits(y);
    const bool zinf_y = 2u * iy - 1u >= 2u * 0x7f800000u - 1u;       // y zero, infinite or NaN
    uint64_t sign_bias = 0;
    if (ix - 0x00800000u >= 0x7f800000u - 0x00800000u || zinf_y) {
        if (zinf_y) {
            if (2u * iy == 0) return powf_signaling(ix) ? fadd(x, y) : 1.0f;
            if (ix == 0x3f800000u) return powf_signaling(iy) ? fadd(x, y) : 1.0f;
            if (2u * ix > 2u * 0x7f800000u || 2u * iy > 2u * 0x7f800000u) return fadd(x, y);
            if (2u * ix == 2u * 0x3f800000u) return 1.0f;
            if ((2u * ix < 2u * 0x3f800000u) == !(iy & 0x80000000u)) return 0.0f;   // |x|<1 to +inf, |x|>1 to -inf
            return fmul(y, y);
        }
        if (2u * ix - 1u >= 2u * 0x7f800000u - 1u) {                 // x zero, infinite or NaN
            float x2 = fmul(x, x);
            if ((ix & 0x80000000u) && powf_checkint(iy) == 1) x2 = fneg(x2);
            return (iy & 0x80000000u) ? fdiv(1.0f, x2) : x2;
        }
        if (ix & 0x80000000u) {                                      // a finite x < 0
            const int yint = powf_checkint(iy);
            if (yint == 0) return fnan();                            // __math_invalidf
            if (yint == 1) sign_bias = 0x10000u;
            ix &= 0x7fffffffu;
        }
        if (ix < 0x00800000u) {                                      // a subnormal x normalised by 2^23
            ix = fbits(fmul(x, 8388608.0f)) & 0x7fffffffu;
            ix -= 23u << 23;
        }
    }
    const double ylogx = dmul(tod(y), powf_log2(ix));
    if (((dbits(ylogx) >> 47) & 0xffff) >= (dbits(126.0 * 32.0) >> 47)) {   // |y log2 x| >= 126: over or under
        if (ylogx > FL_POWF_OFLOW) return powf_xflow(sign_bias, FL_POWF_OFLOWF_X);
        if (ylogx <= dfrom(FL_POWF_UFLOW_BITS)) return powf_xflow(sign_bias, FL_POWF_UFLOWF_X);
        if (ylogx < dfrom(FL_POWF_MAY_UFLOW_BITS)) return powf_xflow(sign_bias, FL_POWF_MAY_UFLOWF_X);
    }
    return powf_exp2(ylogx, sign_bias);
}


}  // namespace lm
}  // namespace ebb
