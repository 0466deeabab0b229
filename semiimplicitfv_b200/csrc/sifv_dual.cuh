// sifv_dual.cuh -- forward-mode dual numbers for the local Jacobians of the
// discrete adjoint and the tangent of the explicit step.
//
// Dual<N> carries a value and N partial derivatives.  Instantiating the
// reconstruction and Riemann templates of sifv_device.cuh with T = Dual<N>
// differentiates exactly the arithmetic the forward step executes: every
// comparison (wave-speed estimates, HLLC branch selection, smax/smin
// clamps) acts on the value, so the derivative is the one of the branch the
// forward pass took.  sqrt and fabs at 0 use the zero subgradient.
#pragma once

#include <cuda_runtime.h>

namespace sifv {

template <int N>
struct Dual {
    double v;
    double d[N];
    __device__ __forceinline__ Dual() {}
    __device__ __forceinline__ Dual(double x) : v(x) {
#pragma unroll
        for (int q = 0; q < N; ++q) d[q] = 0.0;
    }
    __device__ __forceinline__ static Dual seed(double x, int q) {
        Dual r(x);
        r.d[q] = 1.0;
        return r;
    }
    __device__ __forceinline__ Dual& operator+=(const Dual& b) {
        v += b.v;
#pragma unroll
        for (int q = 0; q < N; ++q) d[q] += b.d[q];
        return *this;
    }
    __device__ __forceinline__ Dual& operator-=(const Dual& b) {
        v -= b.v;
#pragma unroll
        for (int q = 0; q < N; ++q) d[q] -= b.d[q];
        return *this;
    }
    __device__ __forceinline__ Dual& operator*=(const Dual& b) {
#pragma unroll
        for (int q = 0; q < N; ++q) d[q] = d[q] * b.v + v * b.d[q];
        v *= b.v;
        return *this;
    }
    __device__ __forceinline__ Dual& operator/=(const Dual& b) {
        const double inv = 1.0 / b.v;
        const double r = v * inv;
#pragma unroll
        for (int q = 0; q < N; ++q) d[q] = (d[q] - r * b.d[q]) * inv;
        v = r;
        return *this;
    }
};

template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int q = 0; q < N; ++q) r.d[q] = -a.d[q];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(Dual<N> a, const Dual<N>& b) { return a += b; }
template <int N>
__device__ __forceinline__ Dual<N> operator-(Dual<N> a, const Dual<N>& b) { return a -= b; }
template <int N>
__device__ __forceinline__ Dual<N> operator*(Dual<N> a, const Dual<N>& b) { return a *= b; }
template <int N>
__device__ __forceinline__ Dual<N> operator/(Dual<N> a, const Dual<N>& b) { return a /= b; }

// mixed with plain doubles
template <int N>
__device__ __forceinline__ Dual<N> operator+(Dual<N> a, double b) { a.v += b; return a; }
template <int N>
__device__ __forceinline__ Dual<N> operator+(double b, Dual<N> a) { a.v += b; return a; }
template <int N>
__device__ __forceinline__ Dual<N> operator-(Dual<N> a, double b) { a.v -= b; return a; }
template <int N>
__device__ __forceinline__ Dual<N> operator-(double b, const Dual<N>& a) { Dual<N> r = -a; r.v += b; return r; }
template <int N>
__device__ __forceinline__ Dual<N> operator*(Dual<N> a, double b) {
    a.v *= b;
#pragma unroll
    for (int q = 0; q < N; ++q) a.d[q] *= b;
    return a;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(double b, Dual<N> a) { return a * b; }
template <int N>
__device__ __forceinline__ Dual<N> operator/(Dual<N> a, double b) {
    const double inv = 1.0 / b;
    a.v /= b;
#pragma unroll
    for (int q = 0; q < N; ++q) a.d[q] *= inv;
    return a;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(double b, const Dual<N>& a) { return Dual<N>(b) / a; }

// comparisons act on values
template <int N> __device__ __forceinline__ bool operator<(const Dual<N>& a, const Dual<N>& b) { return a.v < b.v; }
template <int N> __device__ __forceinline__ bool operator>(const Dual<N>& a, const Dual<N>& b) { return a.v > b.v; }
template <int N> __device__ __forceinline__ bool operator<=(const Dual<N>& a, const Dual<N>& b) { return a.v <= b.v; }
template <int N> __device__ __forceinline__ bool operator>=(const Dual<N>& a, const Dual<N>& b) { return a.v >= b.v; }
template <int N> __device__ __forceinline__ bool operator<(const Dual<N>& a, double b) { return a.v < b; }
template <int N> __device__ __forceinline__ bool operator>(const Dual<N>& a, double b) { return a.v > b; }
template <int N> __device__ __forceinline__ bool operator<=(const Dual<N>& a, double b) { return a.v <= b; }
template <int N> __device__ __forceinline__ bool operator>=(const Dual<N>& a, double b) { return a.v >= b; }
template <int N> __device__ __forceinline__ bool operator<(double a, const Dual<N>& b) { return a < b.v; }
template <int N> __device__ __forceinline__ bool operator>(double a, const Dual<N>& b) { return a > b.v; }

template <int N>
__device__ __forceinline__ Dual<N> sqrt(const Dual<N>& a) {
    Dual<N> r;
    r.v = ::sqrt(a.v);
    const double h = (r.v > 0.0) ? 0.5 / r.v : 0.0;
#pragma unroll
    for (int q = 0; q < N; ++q) r.d[q] = h * a.d[q];
    return r;
}

template <int N>
__device__ __forceinline__ Dual<N> fabs(const Dual<N>& a) {
    if (a.v > 0.0) return a;
    if (a.v < 0.0) return -a;
    return Dual<N>(0.0);
}

}  // namespace sifv
