// zj_math.h -- FP64 reciprocal, square root and x^0.7 on the FMA pipe.
//
// An FP64 division or square root is a long dependent instruction sequence
// with a special-case path; the residual kernels take several per state.
// These two functions use Newton-Raphson iterations, so they are short
// branch-free chains of FP64 FMAs:
//   reciprocal: e = 1 - x*y, y += y*e (the error squares each step) from the
//     hardware's approximate FP64 reciprocal (rcp.approx.ftz.f64) on the
//     device, two steps; on the host from the integer seed
//     bits(0x7FDE623822FC16E6 - bits(x)) (relative error below 1/8), five
//     steps (2^-3 -> below 2^-60);
//   inverse square root: y += y/2 * (1 - a*y*y) from rsqrt.approx.ftz.f64 on
//     the device, two steps; on the host from Lomont's seed
//     bits(0x5FE6EB50C7B537A9 - bits(a)/2) (relative error below 4%), four;
//   square root: s = a*y and one Newton correction s += (a - s*s) * y/2.
// Results are within 2 ulp of the correctly rounded value on the domains
// below (tests/test_zj_math.py checks the host side, tests/test_zj_math_gpu.py
// the device side, over 2^20 samples each).
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
#ifdef __CUDA_ARCH__
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
#pragma unroll
    for (int it = 0; it < 2; ++it) {
        const double e = zj_fma(-x, y, 1.0);
        y = zj_fma(y, e, y);
    }
    return y;
#else
    double y = zj_from_bits(0x7FDE623822FC16E6LL - zj_bits(x));
#pragma unroll
    for (int it = 0; it < 5; ++it) {
        const double e = zj_fma(-x, y, 1.0);
        y = zj_fma(y, e, y);
    }
    return y;
#endif
}

// sqrt(a) for a >= 0.
ZJ_MATH_HD double zj_sqrt(double a) {
    if (!(a > 0.0) || !(a < 1.7976931348623157e308)) {
        if (a == 0.0) return 0.0;
        return (a < 0.0) ? zj_from_bits(0x7FF8000000000000LL) : a + a;
    }
#ifdef __CUDA_ARCH__
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
    constexpr int kIt = 2;
#else
    double y = zj_from_bits(0x5FE6EB50C7B537A9LL - (zj_bits(a) >> 1));
    constexpr int kIt = 4;
#endif
#pragma unroll
    for (int it = 0; it < kIt; ++it) {
        const double e = zj_fma(-a, y * y, 1.0);
        y = zj_fma(0.5 * y, e, y);
    }
    double s = a * y;
    const double r = zj_fma(-s, s, a);
    return zj_fma(r, 0.5 * y, s);
}

// x^a for positive normal x with a = 0.7 as a double (0.7 - d, d = 4.44e-17:
// the exponent pow(T, 0.7) sees in the viscosity law mu = T^0.7 / Re), from
// two textbook series instead of a general pow:
//   x = 2^k m, m in [sqrt(1/2), sqrt(2));
//   ln m = 2 atanh(s) = 2 (s + s^3/3 + ... + s^21/21), s = (m-1)/(m+1),
//     |s| <= 0.172, so the truncation is below 1e-17 relative;
//   a k = n + r/10 - d k with n = floor(7k/10), r = 7k - 10n in integers, so
//     the large part of the exponent carries no rounding;
//   g = r/10 - d k + (a/ln 2) ln m in [-0.35, 1.25]; j = 1 if g >= 1/2 else 0;
//   2^(g-j) = exp((g-j) ln 2) by its Taylor series to degree 13 (argument
//     below 0.35 in magnitude: truncation below 1e-17 relative);
//   x^0.7 = 2^(g-j) 2^(n+j), the scaling applied to the exponent bits.
// Within 2 ulp of pow(x, 0.7) on [1e-300, 1e300] (tests/test_zj_math.py);
// zero, subnormal, negative and non-finite inputs take the library pow.
ZJ_MATH_HD double zj_pow07(double x) {
    const int64_t b = zj_bits(x);
    const int64_t be = (b >> 52) & 0x7FF;
    if (b <= 0 || be == 0 || be == 0x7FF) {
#ifdef __CUDA_ARCH__
        return pow(x, 0.7);
#else
        return __builtin_pow(x, 0.7);
#endif
    }
    int64_t k = be - 1023;
    double m = zj_from_bits((b & 0x000FFFFFFFFFFFFFLL) | 0x3FF0000000000000LL);
    if (m > 1.4142135623730951) {
        m *= 0.5;
        k += 1;
    }
    const double s = (m - 1.0) * zj_rcp(m + 1.0);
    const double z = s * s;
    double p = 1.0 / 21.0;
    p = zj_fma(p, z, 1.0 / 19.0);
    p = zj_fma(p, z, 1.0 / 17.0);
    p = zj_fma(p, z, 1.0 / 15.0);
    p = zj_fma(p, z, 1.0 / 13.0);
    p = zj_fma(p, z, 1.0 / 11.0);
    p = zj_fma(p, z, 1.0 / 9.0);
    p = zj_fma(p, z, 1.0 / 7.0);
    p = zj_fma(p, z, 1.0 / 5.0);
    p = zj_fma(p, z, 1.0 / 3.0);
    p = zj_fma(p, z, 1.0);
    const double lnm = 2.0 * s * p;
    const int64_t q = 7 * k;
    const int64_t n = (q >= 0) ? q / 10 : -((-q + 9) / 10);
    const int64_t r = q - 10 * n;                           // 0..9
    const double g = zj_fma(lnm, 1.0098865286222742, zj_fma(-4.4408920985006264e-17, (double)k, (double)r * 0.1));
    const int64_t j = (g >= 0.5) ? 1 : 0;
    const double t = (g - (double)j) * 0.6931471805599453;
    double e = 1.0 / 6227020800.0;                          // 1/13!
    e = zj_fma(e, t, 1.0 / 479001600.0);
    e = zj_fma(e, t, 1.0 / 39916800.0);
    e = zj_fma(e, t, 1.0 / 3628800.0);
    e = zj_fma(e, t, 1.0 / 362880.0);
    e = zj_fma(e, t, 1.0 / 40320.0);
    e = zj_fma(e, t, 1.0 / 5040.0);
    e = zj_fma(e, t, 1.0 / 720.0);
    e = zj_fma(e, t, 1.0 / 120.0);
    e = zj_fma(e, t, 1.0 / 24.0);
    e = zj_fma(e, t, 1.0 / 6.0);
    e = zj_fma(e, t, 0.5);
    e = zj_fma(e, t, 1.0);
    e = zj_fma(e, t, 1.0);
    return zj_from_bits(zj_bits(e) + (n + j) * (int64_t(1) << 52));
}

}  // namespace zj
