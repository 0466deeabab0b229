// sifv_ensemble.cuh -- batched ensembles of independent 1D problems of
// different sizes, advanced to a common end time in ONE kernel launch.
//
// One CTA owns one instance and runs that instance's whole time loop
// (the explicit step of ExplicitSolver::step, src/ExplicitSolver.cpp:68-203,
// with the targetDt = tEnd - t cap of the reference's time loop,
// src/RKTimeStepping.cpp:258-266): its own acoustic dt (block-wide minimum),
// then per SSP-RK stage three phases separated by __syncthreads:
//   1. conservative -> primitive of the interior and the ghost fill,
//   2. face reconstruction + Riemann flux (+ upwinded partial-density flux),
//   3. flux divergence, sources and the stage update.
// Blocks never wait on each other, so instances of any size (and step
// count) retire independently; the host orders instances by cost (N^2) so
// the longest start first.  State arrays are packed per instance with
// ghosts, x fastest (offsets in EnsArgs).
//
// T is the arithmetic of the reconstruction / Riemann bulk (double: the
// reference's operation order, bit-identical to the single-instance path;
// float: mixed precision).  Primitive recovery (including the mixture
// pressure from total energy), dt, the divergence and the update are FP64.
#pragma once

#include "sifv_common.cuh"

namespace sifv {

struct EnsArgs {
    Params P;                 // per-instance values nx / nxT are set per block
    int nInst;
    const int* order;         // block -> instance (cost-sorted)
    const int* n;             // interior cells per instance
    const long long* off;     // packed cell offset per instance (ghosts included)
    const long long* foff;    // packed face offset per instance (n + 1 faces)
    // packed fields (ghosts included)
    double *rho, *rhoU, *rhoE, *velU, *pres;
    double* alphaRho[MAXPH];
    double* alpha[MAXPH];
    double *rho0, *rhoU0, *rhoE0, *pres0;
    double* alphaRho0[MAXPH];
    double* alpha0[MAXPH];
    const double* dx;         // packed cell widths (ghosts included)
    // packed face scratch
    double *fMass, *fMom, *fEnergy, *fVel;
    double* fAlpha[MAXPH];
    double* fAR[MAXPH];
    // per instance
    double* time;
    int* steps;
    double* lastDt;
    int* status;              // 0 ok, 1 the time step was not positive (state blew up)
    double cfl, maxDt, constDt, tEnd;
    int maxSteps;
};

// std::min(dt, x) over a block, NaN ignored; result broadcast to all threads.
__device__ __forceinline__ double block_min_bcast(double v, double* sm) {
    if (!(v == v)) v = __longlong_as_double(0x7ff0000000000000LL);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = smin(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) sm[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (lane < nw) ? sm[lane] : __longlong_as_double(0x7ff0000000000000LL);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = smin(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) sm[32] = v;
    }
    __syncthreads();
    return sm[32];
}

template <typename T, int NPH>
__global__ void __launch_bounds__(512) k_ensemble(EnsArgs A) {
    __shared__ double red[33];
    const int inst = A.order[blockIdx.x];
    const int n = A.n[inst];
    const long long base = A.off[inst];
    const long long fb = A.foff[inst];
    Params P = A.P;
    const int ng = P.ngx;
    P.nx = n;
    P.nxT = n + 2 * ng;
    const int RK = P.RKOrder;
    const double eps = P.wenoEps;
    const bool weno = (P.reconOrder == SIFV_WENO5);
    double t = A.time[inst];
    int steps = A.steps[inst];
    double dtLast = 0.0;
    // cell q (may be a ghost) -> packed index
    auto at = [&](int q) -> long long { return base + ng + q; };

    while (t < A.tEnd && steps < A.maxSteps) {
        // ---- dt: computeAcousticTimeStep (src/RKTimeStepping.cpp:43-123) ----
        double dt;
        if (A.constDt > 0) {
            dt = A.constDt;
        } else {
            double v = __longlong_as_double(0x7ff0000000000000LL);
            for (int q = threadIdx.x; q < n; q += blockDim.x) {
                long long c = at(q);
                double cs;
                if (NPH > 0) {
                    double a[NPH > 0 ? NPH : 1], ar[NPH > 0 ? NPH : 1];
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph) {
                        a[ph] = (ph < P.nPh) ? A.alpha[ph][c] : 0.0;
                        ar[ph] = (ph < P.nPh) ? A.alphaRho[ph][c] : 0.0;
                    }
                    cs = mixture_sound_speed<NPH>(P, A.rho[c], A.pres[c], a, ar);
                } else {
                    cs = single_sound_speed(P, A.rho[c], A.pres[c]);
                }
                v = smin(v, A.cfl * (A.dx[c] / (fabs(A.velU[c]) + cs)));
            }
            double m = block_min_bcast(v, red);
            dt = smin(A.maxDt, m);
        }
        const double target = A.tEnd - t;
        if (target > 0) dt = smin(dt, target);
        if (!(dt > 0.0)) {   // a non-finite wave speed: stop instead of stepping in place
            if (threadIdx.x == 0) A.status[inst] = 1;
            break;
        }

        for (int s = 0; s < RK; ++s) {
            // SSP-RK coefficients, src/ExplicitSolver.cpp:92-103
            double c1, c2, c3, c4;
            if (RK == 1) { c1 = 1.0; c2 = 0.0; c3 = 1.0; c4 = 1.0; }
            else if (RK == 2) {
                if (s == 0) { c1 = 1.0; c2 = 0.0; c3 = 1.0; c4 = 1.0; } else { c1 = 1.0; c2 = 1.0; c3 = 1.0; c4 = 2.0; }
            } else {
                if (s == 0) { c1 = 1.0; c2 = 0.0; c3 = 1.0; c4 = 1.0; }
                else if (s == 1) { c1 = 1.0; c2 = 3.0; c3 = 1.0; c4 = 4.0; }
                else { c1 = 2.0; c2 = 1.0; c3 = 2.0; c4 = 3.0; }
            }
            // ---- phase 1: cons -> prim (interior), then PRIM ghost fill ----
            for (int q = threadIdx.x; q < n; q += blockDim.x) {
                long long c = at(q);
                if (NPH > 0) {
                    double rho = 0.0;
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph)
                        if (ph < P.nPh) rho += A.alphaRho[ph][c];
                    double rs = smax(rho, 1e-14);
                    A.rho[c] = rs;
                    double u = A.rhoU[c] / rs;
                    A.velU[c] = u;
                    double ke = 0.5 * rs * u * u;
                    double a[NPH > 0 ? NPH : 1];
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph) a[ph] = (ph < P.nPh) ? A.alpha[ph][c] : 0.0;
                    A.pres[c] = mixture_pressure<NPH>(P, A.rhoE[c] - ke, a);
                } else {
                    double rho = smax(A.rho[c], 1e-14);
                    double u = A.rhoU[c] / rho;
                    double ke = 0.0 + u * u;
                    ke *= 0.5 * rho;
                    double e = A.rhoE[c] - ke;
                    A.velU[c] = u;
                    A.pres[c] = P.eosStiffened ? (P.gamma - 1.0) * e - P.gamma * P.pInf
                                               : smax((P.gamma - 1.0) * e, 1e-14);
                }
            }
            __syncthreads();
            for (int g = threadIdx.x; g < 2 * ng; g += blockDim.x) {
                int q = (g < ng) ? -1 - g : n + (g - ng);
                double sn, sa;
                int sq = prim_src(q, n, P.bc[0], P.bc[1], sn, sa);
                long long d = at(q), sc = at(sq);
                A.rho[d] = A.rho[sc];
                A.velU[d] = (sn * sa) * A.velU[sc];
                A.pres[d] = A.pres[sc];
#pragma unroll
                for (int ph = 0; ph < NPH; ++ph)
                    if (ph < P.nPh) { A.alphaRho[ph][d] = A.alphaRho[ph][sc]; A.alpha[ph][d] = A.alpha[ph][sc]; }
            }
            __syncthreads();
            // ---- phase 2: faces f in [0, n]: left cell f-1, right cell f ----
            for (int f = threadIdx.x; f <= n; f += blockDim.x) {
                FaceState<NPH, T> L, R;
                L.u[1] = L.u[2] = R.u[1] = R.u[2] = T(0.0);
                L.sigma = R.sigma = T(0.0);
                long long c = at(f);
                auto rec = [&](const double* fld, T& l, T& r) {
                    T v0 = T(fld[c - 3]), v1 = T(fld[c - 2]), v2 = T(fld[c - 1]), v3 = T(fld[c]),
                      v4 = T(fld[c + 1]), v5 = T(fld[c + 2]);
                    if (weno) { l = weno5L<T>(v0, v1, v2, v3, v4, T(eps)); r = weno5R<T>(v1, v2, v3, v4, v5, T(eps)); }
                    else { l = upwind5L<T>(v0, v1, v2, v3, v4); r = upwind5R<T>(v1, v2, v3, v4, v5); }
                };
                rec(A.rho, L.rho, R.rho);
                rec(A.velU, L.u[0], R.u[0]);
                rec(A.pres, L.p, R.p);
#pragma unroll
                for (int ph = 0; ph < NPH; ++ph) {
                    L.alpha[ph] = R.alpha[ph] = T(0.0);
                    if (ph < P.nPh) rec(A.alpha[ph], L.alpha[ph], R.alpha[ph]);
                }
                if (NPH > 0) {
                    eff_gamma_piinf<NPH, T>(P, L.alpha, L.gEff, L.piEff);
                    eff_gamma_piinf<NPH, T>(P, R.alpha, R.gEff, R.piEff);
                } else {
                    L.gEff = R.gEff = T(P.gamma);
                    L.piEff = R.piEff = T(P.pInf);
                }
                FaceFlux<NPH, T> Fx;
                switch (P.riemann) {
                    case SIFV_HLLC: hllc_flux<0, NPH, T>(P, L, R, Fx); break;
                    case SIFV_RUSANOV: rusanov_flux<0, NPH, T>(P, L, R, Fx); break;
                    default: lf_flux<0, NPH, T>(P, L, R, Fx); break;
                }
                const long long fi = fb + f;
                A.fMass[fi] = (double)Fx.mass;
                A.fMom[fi] = (double)Fx.mom[0];
                A.fEnergy[fi] = (double)Fx.energy;
                if (NPH > 0) {
                    A.fVel[fi] = (double)Fx.fvel;
                    long long upw = ((double)Fx.mass >= 0) ? c - 1 : c;
                    double rhoUpw = smax(A.rho[upw], 1e-14);
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph) {
                        if (ph < P.nPh) {
                            A.fAlpha[ph][fi] = (double)Fx.alpha[ph];
                            A.fAR[ph][fi] = (A.alphaRho[ph][upw] / rhoUpw) * (double)Fx.mass;
                        }
                    }
                }
            }
            __syncthreads();
            // ---- phase 3: divergence (src/ExplicitSolver.cpp:294-496) + update (127-188) ----
            for (int q = threadIdx.x; q < n; q += blockDim.x) {
                long long c = at(q);
                const long long fl = fb + q, fh = fb + q + 1;
                double coeff = (1.0 * 1.0) / ((A.dx[c] * 1.0) * 1.0);
                double rR = 0.0, rU = 0.0, rE = 0.0;
                rR += coeff * A.fMass[fl]; rR -= coeff * A.fMass[fh];
                rU += coeff * A.fMom[fl]; rU -= coeff * A.fMom[fh];
                rE += coeff * A.fEnergy[fl]; rE -= coeff * A.fEnergy[fh];
                double rAR[NPH > 0 ? NPH : 1], rA[NPH > 0 ? NPH : 1];
                if (NPH > 0) {
                    double divU = 0.0;
                    divU -= coeff * A.fVel[fl];
                    divU += coeff * A.fVel[fh];
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph) {
                        if (ph < P.nPh) {
                            double r1 = 0.0, r2 = 0.0;
                            r1 += coeff * A.fAR[ph][fl]; r1 -= coeff * A.fAR[ph][fh];
                            r2 += coeff * A.fAlpha[ph][fl]; r2 -= coeff * A.fAlpha[ph][fh];
                            r2 += A.alpha[ph][c] * divU;
                            rAR[ph] = r1;
                            rA[ph] = r2;
                        }
                    }
                }
                if (s == 0 && RK > 1) {
                    A.rho0[c] = A.rho[c]; A.rhoU0[c] = A.rhoU[c]; A.rhoE0[c] = A.rhoE[c]; A.pres0[c] = A.pres[c];
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph)
                        if (ph < P.nPh) { A.alphaRho0[ph][c] = A.alphaRho[ph][c]; A.alpha0[ph][c] = A.alpha[ph][c]; }
                }
                if (RK == 1) {
                    A.rho[c] += dt * rR;
                    A.rhoU[c] += dt * rU;
                    A.rhoE[c] += dt * rE;
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph)
                        if (ph < P.nPh) A.alphaRho[ph][c] += dt * rAR[ph];
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph)
                        if (ph < P.nPh) A.alpha[ph][c] += dt * rA[ph];
                } else {
                    A.rho[c] = (c1 * A.rho[c] + c2 * A.rho0[c] + c3 * dt * rR) / c4;
                    A.rhoU[c] = (c1 * A.rhoU[c] + c2 * A.rhoU0[c] + c3 * dt * rU) / c4;
                    A.rhoE[c] = (c1 * A.rhoE[c] + c2 * A.rhoE0[c] + c3 * dt * rE) / c4;
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph)
                        if (ph < P.nPh)
                            A.alphaRho[ph][c] = (c1 * A.alphaRho[ph][c] + c2 * A.alphaRho0[ph][c] + c3 * dt * rAR[ph]) / c4;
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph)
                        if (ph < P.nPh) A.alpha[ph][c] = (c1 * A.alpha[ph][c] + c2 * A.alpha0[ph][c] + c3 * dt * rA[ph]) / c4;
                }
                if (NPH > 0) {   // src/ExplicitSolver.cpp:169-185
                    double rhoSum = 0.0;
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph) {
                        if (ph < P.nPh) {
                            double v = smax(A.alphaRho[ph][c], 1e-14);
                            A.alphaRho[ph][c] = v;
                            rhoSum += v;
                        }
                    }
                    A.rho[c] = rhoSum;
                    double a[NPH > 0 ? NPH : 1];
                    double aSum = 0.0;
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph)
                        if (ph < P.nPh) a[ph] = smax(A.alpha[ph][c], P.alphaMin);
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph)
                        if (ph < P.nPh) aSum += a[ph];
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph)
                        if (ph < P.nPh) A.alpha[ph][c] = a[ph] / aSum;
                }
            }
            __syncthreads();
        }
        // ---- final cons -> prim + ghosts (src/ExplicitSolver.cpp:192-200) ----
        for (int q = threadIdx.x; q < n; q += blockDim.x) {
            long long c = at(q);
            if (NPH > 0) {
                double rho = 0.0;
#pragma unroll
                for (int ph = 0; ph < NPH; ++ph)
                    if (ph < P.nPh) rho += A.alphaRho[ph][c];
                double rs = smax(rho, 1e-14);
                A.rho[c] = rs;
                double u = A.rhoU[c] / rs;
                A.velU[c] = u;
                double ke = 0.5 * rs * u * u;
                double a[NPH > 0 ? NPH : 1];
#pragma unroll
                for (int ph = 0; ph < NPH; ++ph) a[ph] = (ph < P.nPh) ? A.alpha[ph][c] : 0.0;
                A.pres[c] = mixture_pressure<NPH>(P, A.rhoE[c] - ke, a);
            } else {
                double rho = smax(A.rho[c], 1e-14);
                double u = A.rhoU[c] / rho;
                double ke = 0.0 + u * u;
                ke *= 0.5 * rho;
                double e = A.rhoE[c] - ke;
                A.velU[c] = u;
                A.pres[c] = P.eosStiffened ? (P.gamma - 1.0) * e - P.gamma * P.pInf : smax((P.gamma - 1.0) * e, 1e-14);
            }
        }
        __syncthreads();
        for (int g = threadIdx.x; g < 2 * ng; g += blockDim.x) {
            int q = (g < ng) ? -1 - g : n + (g - ng);
            double sn, sa;
            int sq = prim_src(q, n, P.bc[0], P.bc[1], sn, sa);
            long long d = at(q), sc = at(sq);
            A.rho[d] = A.rho[sc];
            A.velU[d] = (sn * sa) * A.velU[sc];
            A.pres[d] = A.pres[sc];
#pragma unroll
            for (int ph = 0; ph < NPH; ++ph)
                if (ph < P.nPh) { A.alphaRho[ph][d] = A.alphaRho[ph][sc]; A.alpha[ph][d] = A.alpha[ph][sc]; }
        }
        __syncthreads();
        t += dt;
        ++steps;
        dtLast = dt;
    }
    if (threadIdx.x == 0) {
        A.time[inst] = t;
        A.steps[inst] = steps;
        A.lastDt[inst] = dtLast;
    }
}

}  // namespace sifv
