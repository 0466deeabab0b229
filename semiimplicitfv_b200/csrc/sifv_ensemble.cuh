// sifv_ensemble.cuh -- batched ensembles of independent 1D problems of
// different sizes, advanced to a common end time in ONE kernel launch.
//
// One CTA owns one instance and runs that instance's whole time loop
// (the explicit step of ExplicitSolver::step, src/ExplicitSolver.cpp:68-203,
// with the targetDt = tEnd - t cap of the reference's time loop,
// src/RKTimeStepping.cpp:258-266): its own acoustic dt (block-wide minimum
// over the stored primitives), then per SSP-RK stage the instance is walked
// in chunks of blockDim cells; per chunk, separated by __syncthreads:
//   1. the primitives of the chunk and its 3-cell halo (ghosts through the
//      PRIM ghost map, src/RectilinearMesh.cpp:498-524) are computed from the
//      stage input into shared memory (FP64 conversion, T copies for the
//      reconstruction),
//   2. every face of the chunk: reconstruction + Riemann flux (+ upwinded
//      partial-density flux), into shared memory,
//   3. every cell: flux divergence, sources, the stage update and the
//      multiphase clamps, written to the stage output; the last stage also
//      writes the primitives of the new state.
// The stage input and output are different packed states (S[0] the state,
// S[1], S[2] scratch; the last stage writes S[0], which only the cell itself
// reads there as U0), so chunks never see each other's updates.  Blocks never
// wait on each other, so instances of any size (and step count) retire
// independently; the host orders instances by cost (N^2) so the longest
// start first.  State arrays are packed per instance with ghosts, x fastest.
//
// T is the arithmetic of the reconstruction / Riemann bulk (double: the
// reference's operation order, bit-identical to the single-instance path;
// float: mixed precision).  Primitive recovery (including the mixture
// pressure from total energy), dt, the divergence and the update are FP64.
#pragma once

#include "sifv_common.cuh"
#include "sifv_fastmath.cuh"

namespace sifv {

struct EnsState {             // one packed conservative state
    double *rho, *rhoU, *rhoE;
    double* alphaRho[MAXPH];
    double* alpha[MAXPH];
};

struct EnsArgs {
    Params P;                 // per-instance values nx / nxT are set per block
    int nInst;
    const int* order;         // block -> instance (cost-sorted)
    const int* n;             // interior cells per instance
    const long long* off;     // packed cell offset per instance (ghosts included)
    EnsState S[3];            // S[0]: the state; S[1], S[2]: stage outputs
    double *velU, *pres;      // primitives of the state (rho: S[0].rho)
    const double* dx;         // packed cell widths (ghosts included)
    // per instance
    double* time;
    int* steps;
    double* lastDt;
    int* status;              // 0 ok, 1 the time step was not positive (state blew up)
    double cfl, maxDt, constDt, tEnd;
    int maxSteps;
    const int* stepLimit;     // per-instance step limit (autotuner probes), may be null
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

// Dynamic shared memory of one block of `threads` threads (chunks of
// threads - 6 cells): staged primitives (T), FP64 density / partial
// densities (multiphase), the face values (FP64) and, with FP32 bulk
// arithmetic, both face values of every staged cell (T).
template <typename T, int NPH>
__host__ __device__ constexpr size_t ens_smem_bytes(int threads) {
    return ((size_t)(3 + NPH) * threads * sizeof(T) + 7) / 8 * 8 +
           (NPH > 0 ? (size_t)(1 + NPH) * threads * sizeof(double) : 0) +
           (size_t)(4 + 2 * NPH) * (threads - 5) * sizeof(double) +
           (sizeof(T) == 4 ? ((size_t)2 * (3 + NPH) * threads * sizeof(T) + 7) / 8 * 8 : 0);
}

// Largest block: 1024 threads with FP32 bulk arithmetic (fits the register
// file at <= 64 registers per thread), 512 with FP64.
template <typename T>
struct EnsMaxThreads {
    static constexpr int value = (sizeof(T) == 4) ? 1024 : 512;
};

template <typename T, int NPH>
__global__ void __launch_bounds__(EnsMaxThreads<T>::value) k_ensemble(EnsArgs A) {
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double red[33];
    constexpr int NVR = 3 + NPH;       // reconstructed: rho, u, p, alpha[NPH]
    const int CH = blockDim.x - 6;     // cells per chunk: the chunk and its 3-cell halo fill the block
    const int W = CH + 6;              // staged positions
    T* sW = reinterpret_cast<T*>(smraw);
    double* sD = reinterpret_cast<double*>(smraw + ((size_t)NVR * W * sizeof(T) + 7) / 8 * 8);
    double* sF = sD + (NPH > 0 ? (1 + NPH) * W : 0);   // face values (4 + 2 NPH rows of CH + 1):
                                                         // mass, mom, energy, fvel, alpha[NPH], AR[NPH]
    // FP32 bulk: per staged cell its high-face (sHi) and low-face (sLo) values
    // from one set of WENO5 smoothness indicators (mixed precision only)
    T* sHi = reinterpret_cast<T*>(sF + (4 + 2 * NPH) * (CH + 1));
    T* sLo = sHi + NVR * W;
    constexpr bool kPair = sizeof(T) == 4;

    const int inst = A.order[blockIdx.x];
    const int n = A.n[inst];
    const long long base = A.off[inst];
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
    auto at = [&](int q) -> long long { return base + ng + q; };
    const EnsState& S0 = A.S[0];

    const int limit = A.stepLimit ? min(A.maxSteps, A.stepLimit[inst]) : A.maxSteps;
    while (t < A.tEnd && steps < limit) {
        // ---- dt: computeAcousticTimeStep (src/RKTimeStepping.cpp:43-123) on the stored primitives ----
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
                        a[ph] = (ph < P.nPh) ? S0.alpha[ph][c] : 0.0;
                        ar[ph] = (ph < P.nPh) ? S0.alphaRho[ph][c] : 0.0;
                    }
                    cs = mixture_sound_speed<NPH>(P, S0.rho[c], A.pres[c], a, ar);
                } else {
                    cs = single_sound_speed(P, S0.rho[c], A.pres[c]);
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
            // stage input / output: S0 -> S1 (-> S2) -> S0; RK1 writes S1 and copies it back
            const EnsState& In = A.S[s];
            const bool lastStage = (s == RK - 1);
            const EnsState& Out = (lastStage && RK > 1) ? A.S[0] : A.S[s + 1];
            const bool writePrim = lastStage && RK > 1;

            for (int c0 = 0; c0 < n; c0 += CH) {
                // ---- 1. primitives of positions c0-3 .. c0+CH+2 ----
                for (int k = threadIdx.x; k < W; k += blockDim.x) {
                    const int q = c0 - 3 + k;
                    if (q >= n + 3) {
#pragma unroll
                        for (int v = 0; v < NVR; ++v) sW[v * W + k] = T(0.0);
                        continue;
                    }
                    double sn, sa;
                    const int sq = prim_src(q, n, P.bc[0], P.bc[1], sn, sa);
                    const long long c = at(sq);
                    double rhoP, u, p;
                    double a[NPH > 0 ? NPH : 1];
                    if (NPH > 0) {
                        double rho = 0.0;
#pragma unroll
                        for (int ph = 0; ph < NPH; ++ph)
                            if (ph < P.nPh) rho += In.alphaRho[ph][c];
                        const double rs = smax(rho, 1e-14);
                        rhoP = rs;
                        u = In.rhoU[c] / rs;
                        const double ke = 0.5 * rs * u * u;
#pragma unroll
                        for (int ph = 0; ph < NPH; ++ph) a[ph] = (ph < P.nPh) ? In.alpha[ph][c] : 0.0;
                        p = mixture_pressure<NPH>(P, In.rhoE[c] - ke, a);
                        sD[k] = rs;
#pragma unroll
                        for (int ph = 0; ph < NPH; ++ph) sD[(1 + ph) * W + k] = (ph < P.nPh) ? In.alphaRho[ph][c] : 0.0;
                    } else {
                        const double rc = In.rho[c];
                        const double rho = smax(rc, 1e-14);
                        u = In.rhoU[c] / rho;
                        double ke = 0.0 + u * u;
                        ke *= 0.5 * rho;
                        const double e = In.rhoE[c] - ke;
                        p = P.eosStiffened ? (P.gamma - 1.0) * e - P.gamma * P.pInf : smax((P.gamma - 1.0) * e, 1e-14);
                        rhoP = rc;
                    }
                    sW[k] = T(rhoP);
                    sW[W + k] = T((sn * sa) * u);
                    sW[2 * W + k] = T(p);
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph) sW[(3 + ph) * W + k] = T(a[ph]);
                }
                __syncthreads();
                if (kPair && weno) {   // staged cells 2 .. CH+3 (left cells and right cells of the faces)
                    for (int k = threadIdx.x + 2; k <= CH + 3; k += blockDim.x) {
#pragma unroll
                        for (int v = 0; v < NVR; ++v) {
                            if (v >= 3 && v - 3 >= P.nPh) continue;
                            const T* w = sW + v * W + k - 2;
                            weno5_pair(w[0], w[1], w[2], w[3], w[4], T(eps), sHi[v * W + k], sLo[v * W + k]);
                        }
                    }
                    __syncthreads();
                }
                // ---- 2. faces f = c0 .. c0+CH (left cell f-1, right cell f) ----
                for (int k = threadIdx.x; k <= CH; k += blockDim.x) {
                    const int f = c0 + k;
                    if (f > n) continue;
                    FaceState<NPH, T> L, R;
                    L.u[1] = L.u[2] = R.u[1] = R.u[2] = T(0.0);
                    L.sigma = R.sigma = T(0.0);
                    auto rec = [&](int v, T& l, T& r) {
                        const T* w = sW + v * W + k;   // cells f-3 .. f+2
                        if (kPair && weno) { l = sHi[v * W + k + 2]; r = sLo[v * W + k + 3]; }
                        else if (weno) { l = weno5L<T>(w[0], w[1], w[2], w[3], w[4], T(eps)); r = weno5R<T>(w[1], w[2], w[3], w[4], w[5], T(eps)); }
                        else { l = upwind5L<T>(w[0], w[1], w[2], w[3], w[4]); r = upwind5R<T>(w[1], w[2], w[3], w[4], w[5]); }
                    };
                    rec(0, L.rho, R.rho);
                    rec(1, L.u[0], R.u[0]);
                    rec(2, L.p, R.p);
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph) {
                        L.alpha[ph] = R.alpha[ph] = T(0.0);
                        if (ph < P.nPh) rec(3 + ph, L.alpha[ph], R.alpha[ph]);
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
                    const int ldF = CH + 1;
                    sF[k] = (double)Fx.mass;
                    sF[ldF + k] = (double)Fx.mom[0];
                    sF[2 * ldF + k] = (double)Fx.energy;
                    if (NPH > 0) {
                        sF[3 * ldF + k] = (double)Fx.fvel;
                        const int upw = ((double)Fx.mass >= 0) ? k + 2 : k + 3;   // staged index of cell f-1 or f
                        const double rhoUpw = smax(sD[upw], 1e-14);
#pragma unroll
                        for (int ph = 0; ph < NPH; ++ph) {
                            if (ph < P.nPh) {
                                sF[(4 + ph) * ldF + k] = (double)Fx.alpha[ph];
                                sF[(4 + NPH + ph) * ldF + k] = (sD[(1 + ph) * W + upw] / rhoUpw) * (double)Fx.mass;
                            }
                        }
                    }
                }
                __syncthreads();
                // ---- 3. cells: divergence (src/ExplicitSolver.cpp:294-496) + update (127-188) ----
                for (int k = threadIdx.x; k < CH; k += blockDim.x) {
                    const int q = c0 + k;
                    if (q >= n) continue;
                    const long long c = at(q);
                    const int ldF = CH + 1;
                    const int fl = k, fh = k + 1;
                    double coeff = (1.0 * 1.0) / ((A.dx[c] * 1.0) * 1.0);
                    double rR = 0.0, rU = 0.0, rE = 0.0;
                    rR += coeff * sF[fl]; rR -= coeff * sF[fh];
                    rU += coeff * sF[ldF + fl]; rU -= coeff * sF[ldF + fh];
                    rE += coeff * sF[2 * ldF + fl]; rE -= coeff * sF[2 * ldF + fh];
                    double rAR[NPH > 0 ? NPH : 1], rA[NPH > 0 ? NPH : 1];
                    if (NPH > 0) {
                        double divU = 0.0;
                        divU -= coeff * sF[3 * ldF + fl];
                        divU += coeff * sF[3 * ldF + fh];
#pragma unroll
                        for (int ph = 0; ph < NPH; ++ph) {
                            if (ph < P.nPh) {
                                double r1 = 0.0, r2 = 0.0;
                                r1 += coeff * sF[(4 + NPH + ph) * ldF + fl]; r1 -= coeff * sF[(4 + NPH + ph) * ldF + fh];
                                r2 += coeff * sF[(4 + ph) * ldF + fl]; r2 -= coeff * sF[(4 + ph) * ldF + fh];
                                r2 += In.alpha[ph][c] * divU;
                                rAR[ph] = r1;
                                rA[ph] = r2;
                            }
                        }
                    }
                    // the stage input's density: the primitive (mixture: max(sum alphaRho, 1e-14))
                    const double rhoIn = (NPH > 0) ? sD[k + 3] : In.rho[c];
                    double nRho, nU, nE, nAR[NPH > 0 ? NPH : 1], nA[NPH > 0 ? NPH : 1];
                    if (RK == 1) {
                        nRho = rhoIn + dt * rR;
                        nU = In.rhoU[c] + dt * rU;
                        nE = In.rhoE[c] + dt * rE;
#pragma unroll
                        for (int ph = 0; ph < NPH; ++ph)
                            if (ph < P.nPh) nAR[ph] = In.alphaRho[ph][c] + dt * rAR[ph];
#pragma unroll
                        for (int ph = 0; ph < NPH; ++ph)
                            if (ph < P.nPh) nA[ph] = In.alpha[ph][c] + dt * rA[ph];
                    } else {
                        // U0 = the step-start state S0 (its density the step-start primitive)
                        const double rho0 = (s == 0) ? rhoIn : S0.rho[c];
                        nRho = (c1 * rhoIn + c2 * rho0 + c3 * dt * rR) / c4;
                        nU = (c1 * In.rhoU[c] + c2 * S0.rhoU[c] + c3 * dt * rU) / c4;
                        nE = (c1 * In.rhoE[c] + c2 * S0.rhoE[c] + c3 * dt * rE) / c4;
#pragma unroll
                        for (int ph = 0; ph < NPH; ++ph)
                            if (ph < P.nPh)
                                nAR[ph] = (c1 * In.alphaRho[ph][c] + c2 * S0.alphaRho[ph][c] + c3 * dt * rAR[ph]) / c4;
#pragma unroll
                        for (int ph = 0; ph < NPH; ++ph)
                            if (ph < P.nPh) nA[ph] = (c1 * In.alpha[ph][c] + c2 * S0.alpha[ph][c] + c3 * dt * rA[ph]) / c4;
                    }
                    if (NPH > 0) {   // src/ExplicitSolver.cpp:169-185
                        double rhoSum = 0.0;
#pragma unroll
                        for (int ph = 0; ph < NPH; ++ph) {
                            if (ph < P.nPh) {
                                double v = smax(nAR[ph], 1e-14);
                                nAR[ph] = v;
                                rhoSum += v;
                            }
                        }
                        nRho = rhoSum;
                        double a[NPH > 0 ? NPH : 1];
                        double aSum = 0.0;
#pragma unroll
                        for (int ph = 0; ph < NPH; ++ph)
                            if (ph < P.nPh) a[ph] = smax(nA[ph], P.alphaMin);
#pragma unroll
                        for (int ph = 0; ph < NPH; ++ph)
                            if (ph < P.nPh) aSum += a[ph];
#pragma unroll
                        for (int ph = 0; ph < NPH; ++ph)
                            if (ph < P.nPh) nA[ph] = a[ph] / aSum;
                    }
                    Out.rho[c] = nRho;
                    Out.rhoU[c] = nU;
                    Out.rhoE[c] = nE;
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph)
                        if (ph < P.nPh) { Out.alphaRho[ph][c] = nAR[ph]; Out.alpha[ph][c] = nA[ph]; }
                    if (writePrim) {   // final cons -> prim (src/ExplicitSolver.cpp:192-200)
                        if (NPH > 0) {
                            double rho = 0.0;
#pragma unroll
                            for (int ph = 0; ph < NPH; ++ph)
                                if (ph < P.nPh) rho += nAR[ph];
                            const double rs = smax(rho, 1e-14);
                            Out.rho[c] = rs;
                            const double u = nU / rs;
                            A.velU[c] = u;
                            const double ke = 0.5 * rs * u * u;
                            double a[NPH > 0 ? NPH : 1];
#pragma unroll
                            for (int ph = 0; ph < NPH; ++ph) a[ph] = (ph < P.nPh) ? nA[ph] : 0.0;
                            A.pres[c] = mixture_pressure<NPH>(P, nE - ke, a);
                        } else {
                            const double rho = smax(nRho, 1e-14);
                            const double u = nU / rho;
                            double ke = 0.0 + u * u;
                            ke *= 0.5 * rho;
                            const double e = nE - ke;
                            A.velU[c] = u;
                            A.pres[c] = P.eosStiffened ? (P.gamma - 1.0) * e - P.gamma * P.pInf
                                                       : smax((P.gamma - 1.0) * e, 1e-14);
                        }
                    }
                }
                __syncthreads();
            }
            if (lastStage && RK == 1) {   // S1 -> S0 and the primitives of the new state
                const EnsState& S1 = A.S[1];
                for (int q = threadIdx.x; q < n; q += blockDim.x) {
                    const long long c = at(q);
                    double nAR[NPH > 0 ? NPH : 1], nA[NPH > 0 ? NPH : 1];
                    const double nU = S1.rhoU[c], nE = S1.rhoE[c];
                    S0.rhoU[c] = nU;
                    S0.rhoE[c] = nE;
#pragma unroll
                    for (int ph = 0; ph < NPH; ++ph)
                        if (ph < P.nPh) {
                            nAR[ph] = S1.alphaRho[ph][c];
                            nA[ph] = S1.alpha[ph][c];
                            S0.alphaRho[ph][c] = nAR[ph];
                            S0.alpha[ph][c] = nA[ph];
                        }
                    if (NPH > 0) {
                        double rho = 0.0;
#pragma unroll
                        for (int ph = 0; ph < NPH; ++ph)
                            if (ph < P.nPh) rho += nAR[ph];
                        const double rs = smax(rho, 1e-14);
                        S0.rho[c] = rs;
                        const double u = nU / rs;
                        A.velU[c] = u;
                        const double ke = 0.5 * rs * u * u;
                        double a[NPH > 0 ? NPH : 1];
#pragma unroll
                        for (int ph = 0; ph < NPH; ++ph) a[ph] = (ph < P.nPh) ? nA[ph] : 0.0;
                        A.pres[c] = mixture_pressure<NPH>(P, nE - ke, a);
                    } else {
                        const double nRho = S1.rho[c];
                        S0.rho[c] = nRho;
                        const double rho = smax(nRho, 1e-14);
                        const double u = nU / rho;
                        double ke = 0.0 + u * u;
                        ke *= 0.5 * rho;
                        const double e = nE - ke;
                        A.velU[c] = u;
                        A.pres[c] = P.eosStiffened ? (P.gamma - 1.0) * e - P.gamma * P.pInf
                                                   : smax((P.gamma - 1.0) * e, 1e-14);
                    }
                }
                __syncthreads();
            }
        }
        t += dt;
        ++steps;
        dtLast = dt;
    }
    // PRIM ghost fill of the state (src/RectilinearMesh.cpp:498-524), for the caller
    for (int g = threadIdx.x; g < 2 * ng; g += blockDim.x) {
        int q = (g < ng) ? -1 - g : n + (g - ng);
        double sn, sa;
        int sq = prim_src(q, n, P.bc[0], P.bc[1], sn, sa);
        long long d = at(q), sc = at(sq);
        S0.rho[d] = S0.rho[sc];
        A.velU[d] = (sn * sa) * A.velU[sc];
        A.pres[d] = A.pres[sc];
#pragma unroll
        for (int ph = 0; ph < NPH; ++ph)
            if (ph < P.nPh) { S0.alphaRho[ph][d] = S0.alphaRho[ph][sc]; S0.alpha[ph][d] = S0.alpha[ph][sc]; }
    }
    if (threadIdx.x == 0) {
        A.time[inst] = t;
        A.steps[inst] = steps;
        A.lastDt[inst] = dtLast;
    }
}

}  // namespace sifv
