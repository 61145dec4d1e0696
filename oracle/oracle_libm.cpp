// The oracle's libm entry: glibc 2.34 aarch64's functions (exact_ballpark_b200/csrc/ebb_libm.cuh, host build),
// elementwise over arrays, for the CPU tests that pin them to the reference's golden vectors and for the flight
// oracle. Test infrastructure only.
#include <cstdint>

#include "../exact_ballpark_b200/csrc/ebb_libm.cuh"

extern "C" {

// func: 0 sin, 1 cos, 2 log, 3 exp, 4 sincos's sine, 5 sincos's cosine, 6 pow(x, y); 10 expf, 11 logf, 12 sinf,
// 13 cosf, 14 acosf, 15 atanf, 16 atan2f(y, x), 17 powf(x, y) (floats held in doubles). Returns -1 for an unknown
// func.
int oracle_libm(int func, int64_t n, const double* x, const double* y, double* out) {
    using namespace ebb;
    for (int64_t i = 0; i < n; ++i) {
        const double a = x[i];
        double s, c;
        switch (func) {
            case 0: out[i] = lm::sin(a); break;
            case 1: out[i] = lm::cos(a); break;
            case 2: out[i] = lm::log(a); break;
            case 3: out[i] = lm::exp(a); break;
            case 4: lm::sincos(a, &s, &c); out[i] = s; break;
            case 5: lm::sincos(a, &s, &c); out[i] = c; break;
            case 6: out[i] = lm::pow(a, y[i]); break;
            case 10: out[i] = tod(lm::expf(tof(a))); break;
            case 11: out[i] = tod(lm::logf(tof(a))); break;
            case 12: out[i] = tod(lm::sinf(tof(a))); break;
            case 13: out[i] = tod(lm::cosf(tof(a))); break;
            case 14: out[i] = tod(lm::acosf(tof(a))); break;
            case 15: out[i] = tod(lm::atanf(tof(a))); break;
            case 16: out[i] = tod(lm::atan2f(tof(y[i]), tof(a))); break;
            case 17: out[i] = tod(lm::powf(tof(a), tof(y[i]))); break;
            default: return -1;
        }
    }
    return 0;
}

}  // extern "C"
