// sifv_fastmath.cuh -- arithmetic building blocks of the fast-FP64 and
// mixed-precision paths (never used by the reference-ordered path): fast
// reciprocal / square root, and both WENO5 face values of a cell from one
// set of smoothness indicators.
#pragma once

#include <cuda_runtime.h>

namespace sifv {

// Fast reciprocal and square root of the fast / mixed paths.  FP64: the
// hardware approximation (rcp.approx.ftz.f64 / rsqrt.approx.ftz.f64, about
// 2^-20 relative error, measured) refined by one third-order step: with
// e = 1 - x y, 1/x = y / (1 - e) = y (1 + e + e^2) + O(e^3); with
// e = 1 - x y^2, 1/sqrt(x) = y (1 - e)^(-1/2) = y (1 + e/2 + 3 e^2 / 8) + O(e^3),
// O(e^3) ~ 2^-60, below half an ulp (one step where two Newton-Raphson steps
// y <- y + y e took four fused operations); sqrt(x) = x * (1 / sqrt(x))
// with one correction s <- s + (x - s^2) y / 2.  Within 1 ulp of the IEEE
// results (checked against them by sifv_fastmath_selftest).  FP32: the
// single-instruction approximations (about 1 ulp).  The reference-ordered
// path never uses these.
__device__ __forceinline__ double frcp(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x, y, 1.0);
    return fma(y, fma(e, e, e), y);
}
__device__ __forceinline__ float frcp(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// sqrt of a positive normal argument
__device__ __forceinline__ double fsqrt_pos(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x * y, y, 1.0);
    y = fma(y, e * fma(e, 0.375, 0.5), y);
    double sq = x * y;
    double r = fma(-sq, sq, x);
    return fma(r, 0.5 * y, sq);
}
__device__ __forceinline__ float fsqrt_pos(float x) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// 1 / sqrt(x) of a positive normal argument: the hardware approximation
// refined by the third-order step above (FP64; within 1 ulp of IEEE
// 1 / sqrt(x), checked by sifv_fastmath_selftest), the single-instruction
// approximation in FP32.
__device__ __forceinline__ double frsqrt_pos(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x * y, y, 1.0);
    return fma(y, e * fma(e, 0.375, 0.5), y);
}
__device__ __forceinline__ float frsqrt_pos(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Both WENO5 face values of the cell whose 5-cell stencil is v0..v4
// (v2 = the cell): L = value at its right face from the left,
// R = value at its left face from the right.
__device__ __forceinline__ void weno5_pair(double v0, double v1, double v2, double v3, double v4, double eps,
                                           double& L, double& R) {
    double t0 = v0 - 2.0 * v1 + v2, s0 = v0 - 4.0 * v1 + 3.0 * v2;
    double t1 = v1 - 2.0 * v2 + v3, s1 = v1 - v3;
    double t2 = v2 - 2.0 * v3 + v4, s2 = 3.0 * v2 - 4.0 * v3 + v4;
    double q0 = eps + ((13.0 / 12.0) * t0 * t0 + 0.25 * s0 * s0);
    double q1 = eps + ((13.0 / 12.0) * t1 * t1 + 0.25 * s1 * s1);
    double q2 = eps + ((13.0 / 12.0) * t2 * t2 + 0.25 * s2 * s2);
    q0 *= q0; q1 *= q1; q2 *= q2;
    // a_k = d_k / q_k; multiplying through by q0 q1 q2 leaves one division per side
    double m01 = q0 * q1, m02 = q0 * q2, m12 = q1 * q2;
    // candidate polynomials times 6; the 1/6 goes into the normalisation
    double pL0 = 2.0 * v0 - 7.0 * v1 + 11.0 * v2;
    double pL1 = -v1 + 5.0 * v2 + 2.0 * v3;
    double pL2 = 2.0 * v2 + 5.0 * v3 - v4;
    double pR0 = 2.0 * v4 - 7.0 * v3 + 11.0 * v2;
    double pR1 = -v3 + 5.0 * v2 + 2.0 * v1;
    double pR2 = 2.0 * v2 + 5.0 * v1 - v0;
    double wL0 = 0.1 * m12, wL1 = 0.6 * m02, wL2 = 0.3 * m01;   // L: d = (.1,.6,.3) on (b0,b1,b2)
    double wR0 = 0.1 * m01, wR1 = 0.6 * m02, wR2 = 0.3 * m12;   // R: d = (.1,.6,.3) on (b2,b1,b0)
    L = (wL0 * pL0 + wL1 * pL1 + wL2 * pL2) * frcp(6.0 * (wL0 + wL1 + wL2));
    R = (wR0 * pR0 + wR1 * pR1 + wR2 * pR2) * frcp(6.0 * (wR0 + wR1 + wR2));
}

// FP32 version: the product form would overflow single precision for
// large-valued fields (q ~ (dp^2)^2), so the weights use reciprocals.
__device__ __forceinline__ void weno5_pair(float v0, float v1, float v2, float v3, float v4, float eps, float& L,
                                           float& R) {
    float t0 = v0 - 2.0f * v1 + v2, s0 = v0 - 4.0f * v1 + 3.0f * v2;
    float t1 = v1 - 2.0f * v2 + v3, s1 = v1 - v3;
    float t2 = v2 - 2.0f * v3 + v4, s2 = 3.0f * v2 - 4.0f * v3 + v4;
    float q0 = eps + ((13.0f / 12.0f) * t0 * t0 + 0.25f * s0 * s0);
    float q1 = eps + ((13.0f / 12.0f) * t1 * t1 + 0.25f * s1 * s1);
    float q2 = eps + ((13.0f / 12.0f) * t2 * t2 + 0.25f * s2 * s2);
    float r0 = frcp(q0 * q0), r1 = frcp(q1 * q1), r2 = frcp(q2 * q2);
    float pL0 = (2.0f * v0 - 7.0f * v1 + 11.0f * v2) * (1.0f / 6.0f);
    float pL1 = (-v1 + 5.0f * v2 + 2.0f * v3) * (1.0f / 6.0f);
    float pL2 = (2.0f * v2 + 5.0f * v3 - v4) * (1.0f / 6.0f);
    float pR0 = (2.0f * v4 - 7.0f * v3 + 11.0f * v2) * (1.0f / 6.0f);
    float pR1 = (-v3 + 5.0f * v2 + 2.0f * v1) * (1.0f / 6.0f);
    float pR2 = (2.0f * v2 + 5.0f * v1 - v0) * (1.0f / 6.0f);
    float aL0 = 0.1f * r0, aL1 = 0.6f * r1, aL2 = 0.3f * r2;
    float aR0 = 0.1f * r2, aR1 = 0.6f * r1, aR2 = 0.3f * r0;
    L = (aL0 * pL0 + aL1 * pL1 + aL2 * pL2) * frcp(aL0 + aL1 + aL2);
    R = (aR0 * pR0 + aR1 * pR1 + aR2 * pR2) * frcp(aR0 + aR1 + aR2);
}

template <typename T>
__device__ __forceinline__ T trsqrt(T x) { return frsqrt_pos(x); }

template <typename T>
__device__ __forceinline__ T trcp(T x);
template <>
__device__ __forceinline__ double trcp<double>(double x) { return frcp(x); }
template <>
__device__ __forceinline__ float trcp<float>(float x) { return frcp(x); }


}  // namespace sifv
