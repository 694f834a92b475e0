// zj_dual.cuh -- forward-mode dual numbers (value + one tangent) for the
// Jacobian-vector product of the residual and for the local Jacobian
// columns the adjoint kernels need.  Every helper the physics templates use
// (rcp_any, sqrt_any, pow_any, div_any, fma_any, max_any, abs_any) has a dual
// overload here, so the residual kernels, the Riemann solvers, the ghost
// states and the viscous flux instantiate with T = Dual unchanged: the value
// part repeats the FP64 arithmetic, the tangent part carries d/d(eps) of every
// intermediate along the input tangent.
#pragma once

#include <cuda_runtime.h>

#include "zj_device.cuh"

namespace zj {

struct Dual {
    double v, d;
    __host__ __device__ constexpr Dual() : v(0.0), d(0.0) {}
    __host__ __device__ constexpr Dual(double x) : v(x), d(0.0) {}
    __host__ __device__ constexpr Dual(double x, double t) : v(x), d(t) {}
    __host__ __device__ explicit operator double() const { return v; }
    __device__ Dual& operator+=(const Dual& b) { v += b.v; d += b.d; return *this; }
    __device__ Dual& operator-=(const Dual& b) { v -= b.v; d -= b.d; return *this; }
    __device__ Dual& operator*=(const Dual& b) { d = fma(d, b.v, v * b.d); v *= b.v; return *this; }
};

__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, fma(a.d, b.v, a.v * b.d)); }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
struct Dual4 { Dual x, y, z, w; };

template <typename T> struct IsDual { static constexpr bool value = false; };
template <> struct IsDual<Dual> { static constexpr bool value = true; };

__device__ __forceinline__ bool operator<(Dual a, Dual b) { return a.v < b.v; }
__device__ __forceinline__ bool operator>(Dual a, Dual b) { return a.v > b.v; }
__device__ __forceinline__ bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
__device__ __forceinline__ bool operator>=(Dual a, Dual b) { return a.v >= b.v; }

// The helpers live in namespace zj, Dual's own namespace, so the physics
// templates find them by argument-dependent lookup at instantiation.
__device__ __forceinline__ Dual rcp_any(Dual x) {
    const double r = dev::rcp_any(x.v);
    return Dual(r, -x.d * r * r);
}
__device__ __forceinline__ Dual sqrt_any(Dual a) {
    const double s = dev::sqrt_any(a.v);
    return Dual(s, (s > 0.0) ? 0.5 * a.d / s : 0.0);
}
__device__ __forceinline__ Dual sqrt_ieee(Dual a) {
    const double s = sqrt(a.v);
    return Dual(s, (s > 0.0) ? 0.5 * a.d / s : 0.0);
}
__device__ __forceinline__ Dual pow_any(Dual a, Dual b) {
    const double p = pow(a.v, b.v);
    double t = (a.d != 0.0) ? b.v * pow(a.v, b.v - 1.0) * a.d : 0.0;
    if (b.d != 0.0) t += p * log(a.v) * b.d;
    return Dual(p, t);
}
__device__ __forceinline__ Dual visc_pow(Dual a) {
    const double p = zj_pow07(a.v);
    return Dual(p, (a.d != 0.0) ? 0.7 * p / a.v * a.d : 0.0);
}
__device__ __forceinline__ Dual div_any(Dual a, Dual b) { return a / b; }
__device__ __forceinline__ Dual fma_any(Dual a, Dual b, Dual c) {
    return Dual(__fma_rn(a.v, b.v, c.v), fma(a.d, b.v, fma(a.v, b.d, c.d)));
}
// max/abs: the derivative of the selected branch (the reference's floors are
// max() selections).
__device__ __forceinline__ Dual max_any(Dual a, Dual b) { return (a.v >= b.v) ? a : b; }
__device__ __forceinline__ Dual abs_any(Dual a) { return (a.v < 0.0) ? -a : a; }

__device__ __forceinline__ void load4(const Dual* p, Dual* v) {
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const double2 t = q[i];
        v[i] = Dual(t.x, t.y);
    }
}
__device__ __forceinline__ void load4_nc(const Dual* p, Dual* v) { load4(p, v); }
__device__ __forceinline__ void store4(Dual* p, const Dual* v) {
    double2* q = reinterpret_cast<double2*>(p);
#pragma unroll
    for (int i = 0; i < 4; ++i) q[i] = make_double2(v[i].v, v[i].d);
}
// The global-row helpers of the FP64 and FP32 kernels, on dual numbers.
__device__ __forceinline__ void gload4(const Dual* p, Dual* v) { load4(p, v); }
__device__ __forceinline__ void gstore4(Dual* p, const Dual* v) { store4(p, v); }
__device__ __forceinline__ void gload8_nc(const Dual* p, Dual* v) {
    load4(p, v);
    load4(p + 4, v + 4);
}
__device__ __forceinline__ void gstore8(Dual* p, const Dual* v) {
    store4(p, v);
    store4(p + 4, v + 4);
}
__device__ __forceinline__ Dual ldg_any(const Dual* p) { return *p; }
__device__ __forceinline__ void load_normal(const Dual4* p, Dual* n) {
    n[0] = p->x; n[1] = p->y; n[2] = p->z;
}
template <int N>
__device__ __forceinline__ void load_row(const Dual* row, Dual* out) {
#pragma unroll
    for (int m = 0; m < N; ++m) out[m] = row[m];
}

}  // namespace zj
