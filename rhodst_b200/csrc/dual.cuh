// dual.cuh -- forward-mode dual numbers for the discrete adjoint.
//
// Dual<K> carries a value and K directional derivatives.  The per-face
// arithmetic of the residual (flux schemes, reconstruction, boundary
// conditions) is templated on its scalar type; evaluated on Dual<K> inputs
// seeded with unit directions it returns the exact local Jacobian columns,
// from which the adjoint kernels form the transposed products.  Branches
// and switches (pos/neg masks, min/max, the limiter guards) take the branch
// of the value, so the result is the derivative of the branch the primal
// evaluation takes.
#pragma once

#include <math.h>

namespace rdst {

// the double overloads stay visible next to the Dual ones declared here
using ::fabs;
using ::fmax;
using ::fmin;
using ::pow;
using ::sqrt;

template <int K>
struct Dual {
    double v;
    double d[K];
    __device__ __forceinline__ Dual() {}
    __device__ __forceinline__ Dual(double x) : v(x) {
#pragma unroll
        for (int k = 0; k < K; ++k) d[k] = 0.0;
    }
    // x with unit derivative in direction k (no derivative when k is out of range)
    __device__ __forceinline__ static Dual seed(double x, int k) {
        Dual r(x);
#pragma unroll
        for (int j = 0; j < K; ++j) r.d[j] = (j == k) ? 1.0 : 0.0;
        return r;
    }
};

__device__ __forceinline__ double val(double x) { return x; }
template <int K> __device__ __forceinline__ double val(const Dual<K>& x) { return x.v; }

// value with derivative dfdx * x'
template <int K>
__device__ __forceinline__ Dual<K> chain(double value, const Dual<K>& x, double dfdx) {
    Dual<K> r;
    r.v = value;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = dfdx * x.d[k];
    return r;
}

template <int K> __device__ __forceinline__ Dual<K> operator-(const Dual<K>& a) {
    Dual<K> r; r.v = -a.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = -a.d[k];
    return r;
}
template <int K> __device__ __forceinline__ Dual<K> operator+(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r; r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int K> __device__ __forceinline__ Dual<K> operator-(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r; r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int K> __device__ __forceinline__ Dual<K> operator*(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r; r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int K> __device__ __forceinline__ Dual<K> operator/(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r; r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
}
template <int K> __device__ __forceinline__ Dual<K> operator+(const Dual<K>& a, double b) { Dual<K> r = a; r.v += b; return r; }
template <int K> __device__ __forceinline__ Dual<K> operator+(double a, const Dual<K>& b) { return b + a; }
template <int K> __device__ __forceinline__ Dual<K> operator-(const Dual<K>& a, double b) { Dual<K> r = a; r.v -= b; return r; }
template <int K> __device__ __forceinline__ Dual<K> operator-(double a, const Dual<K>& b) { Dual<K> r = -b; r.v += a; return r; }
template <int K> __device__ __forceinline__ Dual<K> operator*(const Dual<K>& a, double b) {
    Dual<K> r; r.v = a.v * b;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b;
    return r;
}
template <int K> __device__ __forceinline__ Dual<K> operator*(double a, const Dual<K>& b) { return b * a; }
template <int K> __device__ __forceinline__ Dual<K> operator/(const Dual<K>& a, double b) {
    Dual<K> r; r.v = a.v / b;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] / b;
    return r;
}
template <int K> __device__ __forceinline__ Dual<K> operator/(double a, const Dual<K>& b) {
    Dual<K> r; r.v = a / b.v;
    const double s = -r.v / b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = s * b.d[k];
    return r;
}
template <int K> __device__ __forceinline__ Dual<K>& operator+=(Dual<K>& a, const Dual<K>& b) { a = a + b; return a; }
template <int K> __device__ __forceinline__ Dual<K>& operator-=(Dual<K>& a, const Dual<K>& b) { a = a - b; return a; }
template <int K> __device__ __forceinline__ Dual<K>& operator*=(Dual<K>& a, const Dual<K>& b) { a = a * b; return a; }
template <int K> __device__ __forceinline__ Dual<K>& operator*=(Dual<K>& a, double b) { a = a * b; return a; }
template <int K> __device__ __forceinline__ Dual<K>& operator+=(Dual<K>& a, double b) { a.v += b; return a; }

template <int K> __device__ __forceinline__ Dual<K> sqrt(const Dual<K>& a) {
    const double s = ::sqrt(a.v);
    return chain(s, a, s > 0 ? 0.5 / s : 0.0);
}
template <int K> __device__ __forceinline__ Dual<K> fabs(const Dual<K>& a) { return a.v >= 0 ? a : -a; }
template <int K> __device__ __forceinline__ Dual<K> fmax(const Dual<K>& a, const Dual<K>& b) { return a.v >= b.v ? a : b; }
template <int K> __device__ __forceinline__ Dual<K> fmin(const Dual<K>& a, const Dual<K>& b) { return a.v <= b.v ? a : b; }
template <int K> __device__ __forceinline__ Dual<K> fmax(const Dual<K>& a, double b) { return a.v >= b ? a : Dual<K>(b); }
template <int K> __device__ __forceinline__ Dual<K> fmax(double a, const Dual<K>& b) { return a >= b.v ? Dual<K>(a) : b; }
template <int K> __device__ __forceinline__ Dual<K> fmin(const Dual<K>& a, double b) { return a.v <= b ? a : Dual<K>(b); }
template <int K> __device__ __forceinline__ Dual<K> fmin(double a, const Dual<K>& b) { return a <= b.v ? Dual<K>(a) : b; }
// x^c for a constant exponent
template <int K> __device__ __forceinline__ Dual<K> pow(const Dual<K>& a, double c) {
    const double p = ::pow(a.v, c);
    return chain(p, a, c * ::pow(a.v, c - 1.0));
}

}  // namespace rdst
