// zj_math.h -- FP64 reciprocal and square root on the FMA pipe.
//
// An FP64 division or square root is a long dependent instruction sequence
// with a special-case path; the residual kernels take several per state.
// These two functions use Newton-Raphson iterations from integer-arithmetic
// seeds, so they are short branch-free chains of FP64 FMAs and integer ops:
//   reciprocal: seed = bits(0x7FDE623822FC16E6 - bits(x)) (relative error
//     below 1/8 for normal x), then e = 1 - x*y, y += y*e five times
//     (error squares each step: 2^-3 -> below 2^-60);
//   inverse square root: Lomont's seed bits(0x5FE6EB50C7B537A9 - bits(a)/2)
//     (relative error below 4%), then y += y/2 * (1 - a*y*y) four times;
//   square root: s = a*y and one Newton correction s += (a - s*s) * y/2.
// Results are within 2 ulp of the correctly rounded value on the domains
// below (tests/test_zj_math.py checks the bound over 2^20 samples).
// zj_rcp: 2^-1020 < x < 2^1020 (the residual passes floored densities).
// zj_sqrt: any a >= 0; sqrt(0) = 0, NaN and +inf propagate, a < 0 gives NaN.
#pragma once

#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define ZJ_MATH_HD __host__ __device__ __forceinline__
#else
#define ZJ_MATH_HD inline
#endif

namespace zj {

ZJ_MATH_HD int64_t zj_bits(double x) {
#ifdef __CUDA_ARCH__
    return __double_as_longlong(x);
#else
    int64_t i;
    std::memcpy(&i, &x, sizeof(i));
    return i;
#endif
}

ZJ_MATH_HD double zj_from_bits(int64_t i) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double(i);
#else
    double x;
    std::memcpy(&x, &i, sizeof(x));
    return x;
#endif
}

ZJ_MATH_HD double zj_fma(double a, double b, double c) {
#ifdef __CUDA_ARCH__
    return __fma_rn(a, b, c);
#else
    return __builtin_fma(a, b, c);
#endif
}

// 1/x for positive normal x (the floored densities of the residual).
ZJ_MATH_HD double zj_rcp(double x) {
    double y = zj_from_bits(0x7FDE623822FC16E6LL - zj_bits(x));
#pragma unroll
    for (int it = 0; it < 5; ++it) {
        const double e = zj_fma(-x, y, 1.0);
        y = zj_fma(y, e, y);
    }
    return y;
}

// sqrt(a) for a >= 0.
ZJ_MATH_HD double zj_sqrt(double a) {
    if (!(a > 0.0) || !(a < 1.7976931348623157e308)) {
        if (a == 0.0) return 0.0;
        return (a < 0.0) ? zj_from_bits(0x7FF8000000000000LL) : a + a;
    }
    double y = zj_from_bits(0x5FE6EB50C7B537A9LL - (zj_bits(a) >> 1));
#pragma unroll
    for (int it = 0; it < 4; ++it) {
        const double e = zj_fma(-a, y * y, 1.0);
        y = zj_fma(0.5 * y, e, y);
    }
    double s = a * y;
    const double r = zj_fma(-s, s, a);
    return zj_fma(r, 0.5 * y, s);
}

}  // namespace zj
