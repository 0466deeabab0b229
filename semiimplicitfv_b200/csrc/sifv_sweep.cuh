// sifv_sweep.cuh -- fused dimension-sweep kernels of the explicit step for
// the fast-FP64 and mixed-precision paths (T = double or float for the
// reconstruction / Riemann bulk; state, primitive recovery, flux
// divergence and the RK update stay FP64).
//
// Per RK stage, one kernel per direction:
//   x sweep  (k_sweep_x): conservative -> primitive (FP64, written back as
//            the stage's primitive state), WENO5 + Riemann flux along x,
//            x flux divergence; a warp marches along one row, 32 cells per
//            step, neighbours exchanged by warp shuffles.
//   y / z    (k_sweep_line): primitive stencil from the x sweep's output,
//            flux divergence along y or z; each thread marches along one
//            line segment keeping a 5-cell register window, lanes are
//            consecutive x so every load is coalesced.
// The last direction adds the divergence of the earlier ones and applies
// the SSP-RK stage update in place (ExplicitSolver::step,
// src/ExplicitSolver.cpp:127-188); earlier directions write / accumulate
// the FP64 rhs buffer.
//
// Each cell's reconstruction yields both its right-face value (from the
// left, weno5Left) and its left-face value (from the right, weno5Right)
// from one set of smoothness indicators: the indicators of the two
// reconstructions of a 5-cell stencil are the same three numbers in mirror
// order (src/Reconstruction.cpp:119-168).
#pragma once

#include "sifv_common.cuh"
#include "sifv_fastmath.cuh"
#include "sifv_sweep_api.h"

namespace sifv {

template <typename T>
struct Prim5 {
    T rho, u, v, w, p;
};

template <typename T>
__device__ __forceinline__ T tmax(T a, T b) { return (a < b) ? b : a; }
template <typename T>
__device__ __forceinline__ T tmin(T a, T b) { return (b < a) ? b : a; }

template <typename T>
struct Flux4 {
    T mass, m0, m1, m2, energy;
};

// Single-phase face flux on the normal axis D: HLLC (src/HLLCSolver.cpp:7-161),
// Rusanov (src/RusanovSolver.cpp:7-83) or LF (src/LFSolver.cpp:8-75), with
// pressure (explicit step).  The HLLC arithmetic is rearranged to need two
// reciprocals per face: the sound speed sqrt(g p' / rho) is evaluated as
// g p' / sqrt(g p' rho) (one reciprocal square root, no 1 / rho), and in the
// star state rho* e = (s - u) rhoE / (s - s*) and rho* p / a = p / (s - s*)
// (a = rho (s - u)), so neither 1 / rho nor 1 / a is formed.
template <int D, int DIM, typename T>
__device__ __forceinline__ void face_flux(int riemann, const FluxConsts& C, const Prim5<T>& L, const Prim5<T>& R,
                                          Flux4<T>& F) {
    const T g = (T)C.gamma, pinf = (T)C.pInf, invGm1 = (T)C.invGm1, gPinf = (T)C.gPinf;
    const T tiny = (T)1e-14;
    T uL[3] = {L.u, L.v, L.w}, uR[3] = {R.u, R.v, R.w};
    T unL = uL[D], unR = uR[D];
    T q2L = L.u * L.u, q2R = R.u * R.u;
    if (DIM >= 2) { q2L += L.v * L.v; q2R += R.v * R.v; }
    if (DIM >= 3) { q2L += L.w * L.w; q2R += R.w * R.w; }
    T rhoEL = (L.p + gPinf) * invGm1 + (T)0.5 * L.rho * q2L;
    T rhoER = (R.p + gPinf) * invGm1 + (T)0.5 * R.rho * q2R;
    const T gpL = g * tmax(L.p + pinf, tiny), gpR = g * tmax(R.p + pinf, tiny);
    T cL = gpL * trsqrt(gpL * tmax(L.rho, tiny)), cR = gpR * trsqrt(gpR * tmax(R.rho, tiny));
    if (riemann == SIFV_HLLC) {
        T sL = tmin(unL - cL, unR - cR);
        T sR = tmax(unL + cL, unR + cR);
        T aL = L.rho * (sL - unL), aR = R.rho * (sR - unR);
        T sStar = (R.p - L.p + aL * unL - aR * unR) * trcp(aL - aR);
        if (sL >= (T)0) {
            F.mass = L.rho * unL;
            F.m0 = F.mass * L.u; F.m1 = F.mass * L.v; F.m2 = F.mass * L.w;
            F.energy = (rhoEL + L.p) * unL;
            if (D == 0) F.m0 += L.p; else if (D == 1) F.m1 += L.p; else F.m2 += L.p;
        } else if (sR <= (T)0) {
            F.mass = R.rho * unR;
            F.m0 = F.mass * R.u; F.m1 = F.mass * R.v; F.m2 = F.mass * R.w;
            F.energy = (rhoER + R.p) * unR;
            if (D == 0) F.m0 += R.p; else if (D == 1) F.m1 += R.p; else F.m2 += R.p;
        } else {
            const bool left = sStar >= (T)0;
            const Prim5<T>& W = left ? L : R;
            T s = left ? sL : sR, un = left ? unL : unR, rhoE = left ? rhoEL : rhoER, a = left ? aL : aR;
            T inv = trcp(s - sStar);
            T rhoStar = a * inv;                    // rho (s - u) / (s - s*)
            T fm = W.rho * un;
            F.mass = fm + s * (rhoStar - W.rho);
            T du = sStar - un;
            T w0 = W.u, w1 = W.v, w2 = W.w;
            T ws[3] = {w0, w1, w2};
            ws[D] += du;
            F.m0 = fm * w0 + s * (rhoStar * ws[0] - W.rho * w0);
            F.m1 = fm * w1 + s * (rhoStar * ws[1] - W.rho * w1);
            F.m2 = fm * w2 + s * (rhoStar * ws[2] - W.rho * w2);
            if (D == 0) F.m0 += W.p; else if (D == 1) F.m1 += W.p; else F.m2 += W.p;
            // rho* (e + du (s* + p / a)) with e = rhoE / rho
            T EStar = (s - un) * inv * rhoE + du * (rhoStar * sStar + W.p * inv);
            F.energy = (rhoE + W.p) * un + s * (EStar - rhoE);
        }
    } else {
        T sMax;
        if (riemann == SIFV_RUSANOV) {
            sMax = tmax(fabs(unL) + cL, fabs(unR) + cR);
        } else {
            T sL2 = sqrt(q2L), sR2 = sqrt(q2R);
            sMax = tmax(sL2, sR2) + tmax(cL, cR);
        }
        T fmL = L.rho * unL, fmR = R.rho * unR;
        T h = (T)0.5, hs = (T)0.5 * sMax;
        F.mass = h * (fmL + fmR) - hs * (R.rho - L.rho);
        F.m0 = h * (fmL * L.u + fmR * R.u) - hs * (R.rho * R.u - L.rho * L.u);
        F.m1 = h * (fmL * L.v + fmR * R.v) - hs * (R.rho * R.v - L.rho * L.v);
        F.m2 = h * (fmL * L.w + fmR * R.w) - hs * (R.rho * R.w - L.rho * L.w);
        T pm = h * (L.p + R.p);
        if (D == 0) F.m0 += pm; else if (D == 1) F.m1 += pm; else F.m2 += pm;
        F.energy = h * ((rhoEL + L.p) * unL + (rhoER + R.p) * unR) - hs * (rhoER - rhoEL);
    }
}

// Conservative -> primitive of one cell in FP64 with velocity signs of its
// ghost mapping (1 for interior cells).
__device__ __forceinline__ Prim5<double> load_cons_prim(const Params& P, const Fields& F, size_t src,
                                                        const double sg[3]) {
    double rho, u[3], p;
    cons_to_prim_cell<0>(P, F, src, rho, u, p);
    Prim5<double> r;
    r.rho = rho;
    r.u = sg[0] * u[0];
    r.v = sg[1] * u[1];
    r.w = sg[2] * u[2];
    r.p = p;
    return r;
}

template <int DIM>
__device__ __forceinline__ Prim5<double> load_prim(const Fields& F, const double* rhoP, size_t src,
                                                   const double sg[3]) {
    Prim5<double> r;
    r.rho = rhoP[src];
    r.u = sg[0] * F.velU[src];
    r.v = (DIM >= 2) ? sg[1] * F.velV[src] : 0.0;
    r.w = (DIM >= 3) ? sg[2] * F.velW[src] : 0.0;
    r.p = F.pres[src];
    return r;
}

template <typename T>
__device__ __forceinline__ Prim5<T> to_t(const Prim5<double>& a) {
    return Prim5<T>{(T)a.rho, (T)a.u, (T)a.v, (T)a.w, (T)a.p};
}

template <int DIM, typename T>
__device__ __forceinline__ void recon_cell(const Prim5<T>& a, const Prim5<T>& b, const Prim5<T>& c,
                                           const Prim5<T>& d, const Prim5<T>& e, T eps, Prim5<T>& L, Prim5<T>& R) {
    weno5_pair(a.rho, b.rho, c.rho, d.rho, e.rho, eps, L.rho, R.rho);
    weno5_pair(a.u, b.u, c.u, d.u, e.u, eps, L.u, R.u);
    if (DIM >= 2) weno5_pair(a.v, b.v, c.v, d.v, e.v, eps, L.v, R.v);
    else { L.v = R.v = (T)0; }
    if (DIM >= 3) weno5_pair(a.w, b.w, c.w, d.w, e.w, eps, L.w, R.w);
    else { L.w = R.w = (T)0; }
    weno5_pair(a.p, b.p, c.p, d.p, e.p, eps, L.p, R.p);
}

template <int DIM>
__device__ __forceinline__ void rk_apply(const Fields& F, size_t c, const RKUpdate& K, double dt, double rR,
                                         double rU, double rV, double rW, double rE) {
    const double a3 = K.a3 * dt;
    double r = F.rho[c], ru = F.rhoU[c], re = F.rhoE[c];
    double rv = (DIM >= 2) ? F.rhoV[c] : 0.0, rw = (DIM >= 3) ? F.rhoW[c] : 0.0;
    if (K.save) {
        F.rho0[c] = r; F.rhoU0[c] = ru; F.rhoE0[c] = re;
        if (DIM >= 2) F.rhoV0[c] = rv;
        if (DIM >= 3) F.rhoW0[c] = rw;
        F.pres0[c] = F.pres[c];
    }
    double nr = K.a1 * r + a3 * rR, nu = K.a1 * ru + a3 * rU, ne = K.a1 * re + a3 * rE;
    double nv = K.a1 * rv + a3 * rV, nw = K.a1 * rw + a3 * rW;
    if (K.useU0) {
        nr += K.a2 * F.rho0[c]; nu += K.a2 * F.rhoU0[c]; ne += K.a2 * F.rhoE0[c];
        if (DIM >= 2) nv += K.a2 * F.rhoV0[c];
        if (DIM >= 3) nw += K.a2 * F.rhoW0[c];
    }
    F.rho[c] = nr; F.rhoU[c] = nu; F.rhoE[c] = ne;
    if (DIM >= 2) F.rhoV[c] = nv;
    if (DIM >= 3) F.rhoW[c] = nw;
}

// x sweep: each warp takes one segment [x0, x0 + seg) of one row (seg = 32 m
// - 2, so the seg + 2 positions whose face values are needed, x0-1 .. x0+seg,
// fill m steps of 32 lanes exactly); lane l handles position
// q = x0 - 1 + 32 t + l at step t.  The conservative values of step t+2 are
// loaded during step t and converted to primitives at its end, so their
// memory latency is hidden behind a step of arithmetic.  Writes the
// stage's primitive state (the density into the stage copy) and the x flux
// divergence (rhs buffer); it never updates the conservative state, so
// periodic ghosts read at the end of a row still see the stage-start values.
struct RawCons {
    double rho, ru, rv, rw, re;
    double sg0, sg1, sg2;
    int valid;
};

template <int DIM, typename T>
__global__ void __launch_bounds__(128) k_sweep_x(SweepArgs A) {
    const Params& P = A.P;
    const Fields& F = A.F;
    if (A.ctl->skip) return;
    const int lane = threadIdx.x & 31;
    const int nx = P.nx;
    const int segs = (nx + A.segx - 1) / A.segx;
    const long long wid = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (wid >= (long long)P.ny * P.nz * segs) return;
    const int sIdx = (int)(wid % segs);
    const long long row = wid / segs;
    const int j = (int)(row % P.ny), k = (int)(row / P.ny);
    const int x0 = sIdx * A.segx;
    const int xe = min(x0 + A.segx, nx);          // cells [x0, xe)
    const size_t rowBase = cidx(P, 0, j, k);
    const T eps = (T)A.eps;

    // raw conservative values of position q (ghosts through the x ghost map)
    auto fetch = [&](int q) -> RawCons {
        RawCons r;
        r.valid = (q >= -P.ngx && q < nx + P.ngx);
        r.sg0 = r.sg1 = r.sg2 = 1.0;
        if (!r.valid) { r.rho = r.ru = r.rv = r.rw = r.re = 0.0; return r; }
        double sn, sa;
        int s = prim_src(q, nx, P.bc[0], P.bc[1], sn, sa);
        if (s != q) { r.sg0 = sn * sa; r.sg1 = sa; r.sg2 = sa; }
        size_t c = rowBase + (size_t)s;
        r.rho = F.rho[c];
        r.ru = F.rhoU[c];
        r.rv = (DIM >= 2) ? F.rhoV[c] : 0.0;
        r.rw = (DIM >= 3) ? F.rhoW[c] : 0.0;
        r.re = F.rhoE[c];
        return r;
    };
    // conservative -> primitive in FP64 (SolutionState::convertConservativeToPrimitiveVariables,
    // src/SolutionState.cpp:187-205 with src/IdealGasEOS.cpp:46-64 / src/StiffenedGasEOS.cpp:47-64)
    auto convert = [&](const RawCons& r) -> Prim5<double> {
        if (!r.valid) return Prim5<double>{0.0, 0.0, 0.0, 0.0, 0.0};
        const int dim = DIM;
        double rho = (r.rho < 1e-14) ? 1e-14 : r.rho;
        double ir = frcp(rho);
        double u = r.ru * ir, v = r.rv * ir, w = r.rw * ir;
        double ke = u * u;
        if (dim >= 2) ke += v * v;
        if (dim >= 3) ke += w * w;
        ke *= 0.5 * rho;
        double e = r.re - ke;
        double p = P.eosStiffened ? (P.gamma - 1.0) * e - P.gamma * P.pInf : (P.gamma - 1.0) * e;
        if (!P.eosStiffened && p < 1e-14) p = 1e-14;
        return Prim5<double>{r.rho, r.sg0 * u, r.sg1 * v, r.sg2 * w, p};
    };

    const int nsteps = (xe - x0 + 2 + 31) / 32;
    Prim5<double> curD = convert(fetch(x0 - 1 + lane));
    Prim5<T> prev = to_t<T>(convert(fetch(x0 - 33 + lane)));
    Prim5<T> cur = to_t<T>(curD);
    Prim5<double> nextD = convert(fetch(x0 + 31 + lane));
    Prim5<T> next = to_t<T>(nextD);
    RawCons raw = fetch(x0 + 63 + lane);
    Prim5<T> Lprev31 = Prim5<T>{(T)0, (T)0, (T)0, (T)0, (T)0};
    Flux4<T> Fprev31 = Flux4<T>{(T)0, (T)0, (T)0, (T)0, (T)0};
    for (int t = 0; t < nsteps; ++t) {
        const int q = x0 - 1 + 32 * t + lane;
        if (q >= x0 && q < xe) {
            size_t c = rowBase + q;
            A.rhoP[c] = curD.rho;
            F.velU[c] = curD.u;
            if (DIM >= 2) F.velV[c] = curD.v;
            if (DIM >= 3) F.velW[c] = curD.w;
            F.pres[c] = curD.p;
        }
        // stencil q-2 .. q+2
        Prim5<T> sm2, sm1, sp1, sp2;
#define SHUF_FIELD(fld)                                                                      \
        {                                                                                    \
            T a2 = __shfl_sync(0xffffffffu, cur.fld, (lane + 30) & 31);                       \
            T b2 = __shfl_sync(0xffffffffu, prev.fld, (lane + 30) & 31);                      \
            sm2.fld = (lane >= 2) ? a2 : b2;                                                 \
            T a1 = __shfl_sync(0xffffffffu, cur.fld, (lane + 31) & 31);                       \
            T b1 = __shfl_sync(0xffffffffu, prev.fld, (lane + 31) & 31);                      \
            sm1.fld = (lane >= 1) ? a1 : b1;                                                 \
            T c1 = __shfl_sync(0xffffffffu, cur.fld, (lane + 1) & 31);                        \
            T d1 = __shfl_sync(0xffffffffu, next.fld, (lane + 1) & 31);                       \
            sp1.fld = (lane <= 30) ? c1 : d1;                                                \
            T c2 = __shfl_sync(0xffffffffu, cur.fld, (lane + 2) & 31);                        \
            T d2 = __shfl_sync(0xffffffffu, next.fld, (lane + 2) & 31);                       \
            sp2.fld = (lane <= 29) ? c2 : d2;                                                \
        }
        SHUF_FIELD(rho)
        SHUF_FIELD(u)
        if (DIM >= 2) SHUF_FIELD(v)
        if (DIM >= 3) SHUF_FIELD(w)
        SHUF_FIELD(p)
#undef SHUF_FIELD
        if (DIM < 2) { sm2.v = sm1.v = sp1.v = sp2.v = (T)0; }
        if (DIM < 3) { sm2.w = sm1.w = sp1.w = sp2.w = (T)0; }
        Prim5<T> L, R;
        recon_cell<DIM, T>(sm2, sm1, cur, sp1, sp2, eps, L, R);
        // face q: left state L(q-1), right state R(q)
        Prim5<T> Lm;
        Lm.rho = __shfl_sync(0xffffffffu, L.rho, (lane + 31) & 31);
        Lm.u = __shfl_sync(0xffffffffu, L.u, (lane + 31) & 31);
        Lm.v = __shfl_sync(0xffffffffu, L.v, (lane + 31) & 31);
        Lm.w = __shfl_sync(0xffffffffu, L.w, (lane + 31) & 31);
        Lm.p = __shfl_sync(0xffffffffu, L.p, (lane + 31) & 31);
        if (lane == 0) Lm = Lprev31;
        Flux4<T> Fq;
        face_flux<0, DIM, T>(P.riemann, A.C, Lm, R, Fq);
        // divergence of cell q-1: faces q-1 and q
        Flux4<T> Fm;
        Fm.mass = __shfl_sync(0xffffffffu, Fq.mass, (lane + 31) & 31);
        Fm.m0 = __shfl_sync(0xffffffffu, Fq.m0, (lane + 31) & 31);
        Fm.m1 = __shfl_sync(0xffffffffu, Fq.m1, (lane + 31) & 31);
        Fm.m2 = __shfl_sync(0xffffffffu, Fq.m2, (lane + 31) & 31);
        Fm.energy = __shfl_sync(0xffffffffu, Fq.energy, (lane + 31) & 31);
        if (lane == 0) Fm = Fprev31;
        const int cq = q - 1;
        if (cq >= x0 && cq < xe) {
            size_t c = rowBase + cq;
            double ci = A.inv[0][cq + P.ngx];
            A.rhs[0][c] = ci * ((double)Fm.mass - (double)Fq.mass);
            A.rhs[1][c] = ci * ((double)Fm.m0 - (double)Fq.m0);
            if (DIM >= 2) A.rhs[2][c] = ci * ((double)Fm.m1 - (double)Fq.m1);
            if (DIM >= 3) A.rhs[3][c] = ci * ((double)Fm.m2 - (double)Fq.m2);
            A.rhs[4][c] = ci * ((double)Fm.energy - (double)Fq.energy);
        }
        // carry lane 31's L and flux to the next step's lane 0
        Lprev31.rho = __shfl_sync(0xffffffffu, L.rho, 31);
        Lprev31.u = __shfl_sync(0xffffffffu, L.u, 31);
        Lprev31.v = __shfl_sync(0xffffffffu, L.v, 31);
        Lprev31.w = __shfl_sync(0xffffffffu, L.w, 31);
        Lprev31.p = __shfl_sync(0xffffffffu, L.p, 31);
        Fprev31.mass = __shfl_sync(0xffffffffu, Fq.mass, 31);
        Fprev31.m0 = __shfl_sync(0xffffffffu, Fq.m0, 31);
        Fprev31.m1 = __shfl_sync(0xffffffffu, Fq.m1, 31);
        Fprev31.m2 = __shfl_sync(0xffffffffu, Fq.m2, 31);
        Fprev31.energy = __shfl_sync(0xffffffffu, Fq.energy, 31);
        // advance the window by 32 positions; convert the prefetched step,
        // then start loading the one after it
        prev = cur;
        cur = next;
        curD = nextD;
        nextD = convert(raw);
        next = to_t<T>(nextD);
        if (t + 3 < nsteps + 1) raw = fetch(x0 + 32 * (t + 3) - 1 + lane);
    }
}

// y or z sweep: each thread marches along one line segment [s0, s0 + seg)
// of axis DIR at fixed x = i (consecutive lanes, coalesced) keeping the
// 5-cell window of positions q-2 .. q+2 in registers.  The primitive values
// of position q+3 and the update inputs of cell q-1 are loaded before the
// arithmetic of step q so their latency overlaps it.
template <int DIR, int DIM, typename T, bool LAST>
__global__ void __launch_bounds__(128) k_sweep_line(SweepArgs A) {
    const Params& P = A.P;
    const Fields& F = A.F;
    if (A.ctl->skip) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.nx) return;
    const int nLine = (DIR == 1) ? P.ny : P.nz;
    const int other = blockIdx.z;   // k for DIR == 1, j for DIR == 2
    const int s0 = blockIdx.y * A.seg;
    if (s0 >= nLine) return;
    const int s1 = min(s0 + A.seg, nLine);
    const long st = (DIR == 1) ? (long)P.nxT : (long)P.nxT * P.nyT;
    const size_t lineBase = (DIR == 1) ? cidx(P, i, 0, other) : cidx(P, i, other, 0);
    const int ng = (DIR == 1) ? P.ngy : P.ngz;
    const int bcLo = P.bc[2 * DIR], bcHi = P.bc[2 * DIR + 1];
    const T eps = (T)A.eps;
    const double dt = A.ctl->dt;

    auto loadq = [&](int q) -> Prim5<double> {
        if (q < -ng || q >= nLine + ng) return Prim5<double>{0.0, 0.0, 0.0, 0.0, 0.0};
        double sn, sa;
        int s = prim_src(q, nLine, bcLo, bcHi, sn, sa);
        double sg[3] = {1.0, 1.0, 1.0};
        if (s != q) { sg[0] = sa; sg[1] = sa; sg[2] = sa; sg[DIR] = sn * sa; }
        return load_prim<DIM>(F, A.rhoP, lineBase + (long)s * st, sg);
    };

    Prim5<T> w0 = to_t<T>(loadq(s0 - 3)), w1 = to_t<T>(loadq(s0 - 2)), w2 = to_t<T>(loadq(s0 - 1));
    Prim5<T> w3 = to_t<T>(loadq(s0)), w4 = to_t<T>(loadq(s0 + 1));
    Prim5<double> ahead = loadq(s0 + 2);
    Prim5<T> Lm;
    Flux4<T> Fm;
    // position s0 - 1: only its right-face value is needed
    {
        Prim5<T> R;
        recon_cell<DIM, T>(w0, w1, w2, w3, w4, eps, Lm, R);
    }
    for (int q = s0; q <= s1; ++q) {
        w0 = w1; w1 = w2; w2 = w3; w3 = w4;
        w4 = to_t<T>(ahead);
        ahead = loadq(q + 3);
        // update inputs of cell q-1
        const bool emit = q > s0;
        const int cq = q - 1;
        const size_t c = lineBase + (long)cq * st;
        double pr[5] = {0, 0, 0, 0, 0}, U[5] = {0, 0, 0, 0, 0}, U0[5] = {0, 0, 0, 0, 0}, pres = 0.0;
        if (emit) {
            pr[0] = A.rhs[0][c]; pr[1] = A.rhs[1][c]; pr[4] = A.rhs[4][c];
            if (DIM >= 2) pr[2] = A.rhs[2][c];
            if (DIM >= 3) pr[3] = A.rhs[3][c];
            if (LAST) {
                U[0] = F.rho[c]; U[1] = F.rhoU[c]; U[4] = F.rhoE[c];
                if (DIM >= 2) U[2] = F.rhoV[c];
                if (DIM >= 3) U[3] = F.rhoW[c];
                if (A.K.useU0) {
                    U0[0] = F.rho0[c]; U0[1] = F.rhoU0[c]; U0[4] = F.rhoE0[c];
                    if (DIM >= 2) U0[2] = F.rhoV0[c];
                    if (DIM >= 3) U0[3] = F.rhoW0[c];
                }
                if (A.K.save) pres = F.pres[c];
            }
        }
        Prim5<T> L, R;
        recon_cell<DIM, T>(w0, w1, w2, w3, w4, eps, L, R);
        Flux4<T> Fq;
        face_flux<DIR, DIM, T>(P.riemann, A.C, Lm, R, Fq);
        if (emit) {
            double ci = A.inv[DIR][cq + ng];
            double rR = ci * ((double)Fm.mass - (double)Fq.mass) + pr[0];
            double rU = ci * ((double)Fm.m0 - (double)Fq.m0) + pr[1];
            double rV = ci * ((double)Fm.m1 - (double)Fq.m1) + pr[2];
            double rW = ci * ((double)Fm.m2 - (double)Fq.m2) + pr[3];
            double rE = ci * ((double)Fm.energy - (double)Fq.energy) + pr[4];
            if (LAST) {
                const RKUpdate& K = A.K;
                if (K.save) {
                    F.rho0[c] = U[0]; F.rhoU0[c] = U[1]; F.rhoE0[c] = U[4];
                    if (DIM >= 2) F.rhoV0[c] = U[2];
                    if (DIM >= 3) F.rhoW0[c] = U[3];
                    F.pres0[c] = pres;
                }
                const double a3 = K.a3 * dt;
                double nr = K.a1 * U[0] + a3 * rR, nu = K.a1 * U[1] + a3 * rU, ne = K.a1 * U[4] + a3 * rE;
                double nv = K.a1 * U[2] + a3 * rV, nw = K.a1 * U[3] + a3 * rW;
                if (K.useU0) {
                    nr += K.a2 * U0[0]; nu += K.a2 * U0[1]; ne += K.a2 * U0[4];
                    nv += K.a2 * U0[2]; nw += K.a2 * U0[3];
                }
                F.rho[c] = nr; F.rhoU[c] = nu; F.rhoE[c] = ne;
                if (DIM >= 2) F.rhoV[c] = nv;
                if (DIM >= 3) F.rhoW[c] = nw;
            } else {
                A.rhs[0][c] = rR;
                A.rhs[1][c] = rU;
                if (DIM >= 2) A.rhs[2][c] = rV;
                if (DIM >= 3) A.rhs[3][c] = rW;
                A.rhs[4][c] = rE;
            }
        }
        Lm = L;
        Fm = Fq;
    }
}

// Stage update from the complete rhs buffer (1D, where the x sweep is the
// only direction).
template <int DIM>
__global__ void __launch_bounds__(256) k_rk_update(SweepArgs A) {
    if (A.ctl->skip) return;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!int_coords(A.P, t, i, j, k)) return;
    size_t c = cidx(A.P, i, j, k);
    rk_apply<DIM>(A.F, c, A.K, A.ctl->dt, A.rhs[0][c], A.rhs[1][c], (DIM >= 2) ? A.rhs[2][c] : 0.0,
                  (DIM >= 3) ? A.rhs[3][c] : 0.0, A.rhs[4][c]);
}

// End of step: primitive state of the updated cells (interior), as the
// reference's final convertConservativeToPrimitiveVariables.
__global__ void __launch_bounds__(256) k_cons_to_prim_interior(Params P, Fields F, const Ctl* ctl) {
    if (ctl->skip) return;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!int_coords(P, t, i, j, k)) return;
    size_t c = cidx(P, i, j, k);
    double rho, u[3], p;
    cons_to_prim_cell<0>(P, F, c, rho, u, p);
    F.velU[c] = u[0];
    if (P.dim >= 2) F.velV[c] = u[1];
    if (P.dim >= 3) F.velW[c] = u[2];
    F.pres[c] = p;
}

}  // namespace sifv
