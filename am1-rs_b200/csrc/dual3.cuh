// Forward-mode dual number with three derivative components: a value and its gradient with
// respect to the pair displacement (delta_x, delta_y, delta_z).  The integral and overlap
// templates of integrals_t.cuh instantiated with D3 give the exact derivatives of the quantities
// the SCF evaluates (the reference's Dual, src/dual.rs, carries the same three components for
// the same purpose).  Only the operations the integral code uses are defined.
#pragma once

#include <cuda_runtime.h>

namespace am1 {

struct D3 {
    double v;
    double d[3];
};

__device__ __forceinline__ D3 d3c(double v) { return D3{v, {0.0, 0.0, 0.0}}; }
__device__ __forceinline__ double val(double x) { return x; }
__device__ __forceinline__ double val(const D3& x) { return x.v; }

__device__ __forceinline__ D3 operator+(const D3& a, const D3& b) { return D3{a.v + b.v, {a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2]}}; }
__device__ __forceinline__ D3 operator-(const D3& a, const D3& b) { return D3{a.v - b.v, {a.d[0] - b.d[0], a.d[1] - b.d[1], a.d[2] - b.d[2]}}; }
__device__ __forceinline__ D3 operator-(const D3& a) { return D3{-a.v, {-a.d[0], -a.d[1], -a.d[2]}}; }
__device__ __forceinline__ D3 operator*(const D3& a, const D3& b) {
    return D3{a.v * b.v, {a.d[0] * b.v + a.v * b.d[0], a.d[1] * b.v + a.v * b.d[1], a.d[2] * b.v + a.v * b.d[2]}};
}
__device__ __forceinline__ D3 operator/(const D3& a, const D3& b) {
    const double q = a.v / b.v, ib = 1.0 / b.v;
    return D3{q, {(a.d[0] - q * b.d[0]) * ib, (a.d[1] - q * b.d[1]) * ib, (a.d[2] - q * b.d[2]) * ib}};
}
__device__ __forceinline__ D3 operator+(const D3& a, double b) { return D3{a.v + b, {a.d[0], a.d[1], a.d[2]}}; }
__device__ __forceinline__ D3 operator+(double a, const D3& b) { return b + a; }
__device__ __forceinline__ D3 operator-(const D3& a, double b) { return D3{a.v - b, {a.d[0], a.d[1], a.d[2]}}; }
__device__ __forceinline__ D3 operator-(double a, const D3& b) { return D3{a - b.v, {-b.d[0], -b.d[1], -b.d[2]}}; }
__device__ __forceinline__ D3 operator*(const D3& a, double b) { return D3{a.v * b, {a.d[0] * b, a.d[1] * b, a.d[2] * b}}; }
__device__ __forceinline__ D3 operator*(double a, const D3& b) { return b * a; }
__device__ __forceinline__ D3 operator/(const D3& a, double b) { return D3{a.v / b, {a.d[0] / b, a.d[1] / b, a.d[2] / b}}; }
__device__ __forceinline__ D3 operator/(double a, const D3& b) {
    const double q = a / b.v, s = -q / b.v;
    return D3{q, {s * b.d[0], s * b.d[1], s * b.d[2]}};
}
__device__ __forceinline__ D3& operator+=(D3& a, const D3& b) { return a = a + b; }
__device__ __forceinline__ D3& operator-=(D3& a, const D3& b) { return a = a - b; }
__device__ __forceinline__ D3& operator*=(D3& a, const D3& b) { return a = a * b; }
__device__ __forceinline__ D3& operator*=(D3& a, double b) { return a = a * b; }

// The double overloads forward to the CUDA math functions: inside this namespace the D3 overloads
// below would otherwise hide them.
__device__ __forceinline__ double exp(double x) { return ::exp(x); }
__device__ __forceinline__ double sqrt(double x) { return ::sqrt(x); }
__device__ __forceinline__ double pow(double x, double p) { return ::pow(x, p); }

// f(x) with f' = df at x: the chain rule on the three components
__device__ __forceinline__ D3 d3_chain(const D3& x, double f, double df) { return D3{f, {df * x.d[0], df * x.d[1], df * x.d[2]}}; }

__device__ __forceinline__ D3 exp(const D3& x) {
    const double e = ::exp(x.v);
    return d3_chain(x, e, e);
}
__device__ __forceinline__ D3 sqrt(const D3& x) {
    const double s = ::sqrt(x.v);
    return d3_chain(x, s, 0.5 / s);
}
// x^p for a constant p (x > 0)
__device__ __forceinline__ D3 pow(const D3& x, double p) {
    const double f = ::pow(x.v, p);
    return d3_chain(x, f, p * f / x.v);
}

}  // namespace am1
