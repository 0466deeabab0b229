// sifv_dual.cuh -- forward-mode dual numbers for the local Jacobians of the
// discrete adjoint and the tangent of the explicit step.
//
// Dual<N, S> carries a value and N partial derivatives in scalar type S
// (double, or float for the FP32 reverse sweep).  Instantiating the
// reconstruction and Riemann templates of sifv_device.cuh with T = Dual<N>
// differentiates exactly the arithmetic the forward step executes: every
// comparison (wave-speed estimates, HLLC branch selection, smax/smin
// clamps) acts on the value, so the derivative is the one of the branch the
// forward pass took.  sqrt and fabs at 0 use the zero subgradient.
#pragma once

#include <cuda_runtime.h>

namespace sifv {

template <int N, typename S = double>
struct Dual {
    S v;
    S d[N];
    __device__ __forceinline__ Dual() {}
    __device__ __forceinline__ Dual(double x) : v((S)x) {
#pragma unroll
        for (int q = 0; q < N; ++q) d[q] = S(0);
    }
    __device__ __forceinline__ static Dual seed(double x, int q) {
        Dual r(x);
        r.d[q] = S(1);
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
        const S inv = S(1) / b.v;
        const S r = v * inv;
#pragma unroll
        for (int q = 0; q < N; ++q) d[q] = (d[q] - r * b.d[q]) * inv;
        v = r;
        return *this;
    }
};

template <int N, typename S>
__device__ __forceinline__ Dual<N, S> operator-(const Dual<N, S>& a) {
    Dual<N, S> r;
    r.v = -a.v;
#pragma unroll
    for (int q = 0; q < N; ++q) r.d[q] = -a.d[q];
    return r;
}
template <int N, typename S>
__device__ __forceinline__ Dual<N, S> operator+(Dual<N, S> a, const Dual<N, S>& b) { return a += b; }
template <int N, typename S>
__device__ __forceinline__ Dual<N, S> operator-(Dual<N, S> a, const Dual<N, S>& b) { return a -= b; }
template <int N, typename S>
__device__ __forceinline__ Dual<N, S> operator*(Dual<N, S> a, const Dual<N, S>& b) { return a *= b; }
template <int N, typename S>
__device__ __forceinline__ Dual<N, S> operator/(Dual<N, S> a, const Dual<N, S>& b) { return a /= b; }

// mixed with plain doubles
template <int N, typename S>
__device__ __forceinline__ Dual<N, S> operator+(Dual<N, S> a, double b) { a.v += b; return a; }
template <int N, typename S>
__device__ __forceinline__ Dual<N, S> operator+(double b, Dual<N, S> a) { a.v += b; return a; }
template <int N, typename S>
__device__ __forceinline__ Dual<N, S> operator-(Dual<N, S> a, double b) { a.v -= b; return a; }
template <int N, typename S>
__device__ __forceinline__ Dual<N, S> operator-(double b, const Dual<N, S>& a) { Dual<N, S> r = -a; r.v += b; return r; }
template <int N, typename S>
__device__ __forceinline__ Dual<N, S> operator*(Dual<N, S> a, double b) {
    const S sb = (S)b;
    a.v *= sb;
#pragma unroll
    for (int q = 0; q < N; ++q) a.d[q] *= sb;
    return a;
}
template <int N, typename S>
__device__ __forceinline__ Dual<N, S> operator*(double b, Dual<N, S> a) { return a * b; }
template <int N, typename S>
__device__ __forceinline__ Dual<N, S> operator/(Dual<N, S> a, double b) {
    const S sb = (S)b;
    const S inv = S(1) / sb;
    a.v /= sb;
#pragma unroll
    for (int q = 0; q < N; ++q) a.d[q] *= inv;
    return a;
}
template <int N, typename S>
__device__ __forceinline__ Dual<N, S> operator/(double b, const Dual<N, S>& a) { return Dual<N, S>(b) / a; }

// comparisons act on values
template <int N, typename S> __device__ __forceinline__ bool operator<(const Dual<N, S>& a, const Dual<N, S>& b) { return a.v < b.v; }
template <int N, typename S> __device__ __forceinline__ bool operator>(const Dual<N, S>& a, const Dual<N, S>& b) { return a.v > b.v; }
template <int N, typename S> __device__ __forceinline__ bool operator<=(const Dual<N, S>& a, const Dual<N, S>& b) { return a.v <= b.v; }
template <int N, typename S> __device__ __forceinline__ bool operator>=(const Dual<N, S>& a, const Dual<N, S>& b) { return a.v >= b.v; }
template <int N, typename S> __device__ __forceinline__ bool operator<(const Dual<N, S>& a, double b) { return a.v < b; }
template <int N, typename S> __device__ __forceinline__ bool operator>(const Dual<N, S>& a, double b) { return a.v > b; }
template <int N, typename S> __device__ __forceinline__ bool operator<=(const Dual<N, S>& a, double b) { return a.v <= b; }
template <int N, typename S> __device__ __forceinline__ bool operator>=(const Dual<N, S>& a, double b) { return a.v >= b; }
template <int N, typename S> __device__ __forceinline__ bool operator<(double a, const Dual<N, S>& b) { return a < b.v; }
template <int N, typename S> __device__ __forceinline__ bool operator>(double a, const Dual<N, S>& b) { return a > b.v; }

template <int N, typename S>
__device__ __forceinline__ Dual<N, S> sqrt(const Dual<N, S>& a) {
    Dual<N, S> r;
    r.v = ::sqrt(a.v);
    const S h = (r.v > S(0)) ? S(0.5) / r.v : S(0);
#pragma unroll
    for (int q = 0; q < N; ++q) r.d[q] = h * a.d[q];
    return r;
}

template <int N, typename S>
__device__ __forceinline__ Dual<N, S> fabs(const Dual<N, S>& a) {
    if (a.v > S(0)) return a;
    if (a.v < S(0)) return -a;
    return Dual<N, S>(0.0);
}

}  // namespace sifv
