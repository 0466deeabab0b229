// sifv_adjoint.cuh -- discrete adjoint (reverse) and tangent (forward) of
// the explicit single-phase step: cons -> prim, PRIM ghost fill, WENO5 /
// UPWIND5 reconstruction, Riemann flux, flux divergence and the SSP-RK stage
// update of ExplicitSolver::step (src/ExplicitSolver.cpp:68-203,
// src/Reconstruction.cpp:119-200, src/HLLCSolver.cpp:7-161,
// src/RusanovSolver.cpp:7-83, src/LFSolver.cpp:8-75), linearised about the
// forward trajectory with the time-step sequence held fixed.
//
// Reverse of one stage U' = (c1 U + c2 U0 + c3 dt R(U)) / c4, given
// lam = dJ/dU':
//   k_adj_face  per face: mu = coeff_R lam_R - coeff_L lam_L (dJ/dF), the
//               flux Jacobian w.r.t. both reconstructed states (Dual<2 nv>
//               through the Riemann template), the reconstruction gradient
//               w.r.t. the stencil (Dual<5> through the WENO5 template), and
//               the product: per stencil cell and primitive variable, its
//               share of dJ/dW, written per face (no atomics);
//   k_adj_cell  per interior cell: gathers the shares of every face whose
//               stencil holds the cell or one of its ghost images (ghost
//               velocity signs applied), multiplies by the cons -> prim
//               Jacobian, and updates lam <- (c1/c4) lam + (c3 dt/c4) g,
//               acc0 += (c2/c4) lam_in (dJ/dU0 through the RK combination).
// The tangent runs the same linearisation forwards: k_tan_prim (dW from dU
// incl. ghosts), k_tan_face (dF with Dual<1>), k_tan_update.
#pragma once

#include "sifv_adjoint_api.h"
#include "sifv_common.cuh"
#include "sifv_dual.cuh"

namespace sifv {

// number of primitive (rho, u.., p) and conservative variables
template <int DIM>
struct NV {
    static constexpr int n = DIM + 2;
};

// cons slot of each primitive-velocity / flux component: 0 rho, 1..DIM mom, DIM+1 energy
__device__ __forceinline__ double* cons_ptr(const Fields& F, int q, int dim) {
    if (q == 0) return F.rho;
    if (q == dim + 1) return F.rhoE;
    return (q == 1) ? F.rhoU : (q == 2) ? F.rhoV : F.rhoW;
}
__device__ __forceinline__ const double* prim_ptr(const Fields& F, int q, int dim) {
    if (q == 0) return F.rho;
    if (q == dim + 1) return F.pres;
    return (q == 1) ? F.velU : (q == 2) ? F.velV : F.velW;
}

template <int DIR>
__device__ __forceinline__ double face_coeff(const Params& P, const Fields& F, int i, int j, int k) {
    double dxi = F.dx[i + P.ngx], dyj = F.dy[j + P.ngy], dzk = F.dz[k + P.ngz];
    double vol = dxi * dyj * dzk;
    return (DIR == 0) ? (dyj * dzk) / vol : (DIR == 1) ? (dxi * dzk) / vol : (dxi * dyj) / vol;
}

template <int DIR>
__device__ __forceinline__ long long face_index(const Params& P, int i, int j, int k) {
    const long long fnx = P.nx + (DIR == 0), fny = P.ny + (DIR == 1);
    return (long long)i + fnx * ((long long)j + fny * (long long)k);
}

// Face states + Riemann flux in arithmetic T (double or Dual<N>).
template <int DIR, typename T>
__device__ __forceinline__ void riemann_T(const Params& P, const FaceState<0, T>& L, const FaceState<0, T>& R,
                                          FaceFlux<0, T>& Fx) {
    switch (P.riemann) {
        case SIFV_HLLC: hllc_flux<DIR, 0, T>(P, L, R, Fx); break;
        case SIFV_RUSANOV: rusanov_flux<DIR, 0, T>(P, L, R, Fx); break;
        default: lf_flux<DIR, 0, T>(P, L, R, Fx); break;
    }
}

template <typename T>
__device__ __forceinline__ void recon5(bool weno, double eps, const T* v, T& l, T& r) {
    if (weno) {
        l = weno5L<T>(v[0], v[1], v[2], v[3], v[4], T(eps));
        r = weno5R<T>(v[1], v[2], v[3], v[4], v[5], T(eps));
    } else {
        l = upwind5L<T>(v[0], v[1], v[2], v[3], v[4]);
        r = upwind5R<T>(v[1], v[2], v[3], v[4], v[5]);
    }
}

// flux component q (cons order) of a FaceFlux
template <typename T>
__device__ __forceinline__ const T& flux_comp(const FaceFlux<0, T>& Fx, int q, int dim) {
    if (q == 0) return Fx.mass;
    if (q == dim + 1) return Fx.energy;
    return Fx.mom[q - 1];
}

// ---------------------------------------------------------------------------
// Reverse: per-face shares of dJ/dW.
// share layout (direction DIR): slot (side * 5 + k) * NVN + v, face-major SoA
//   side 0: left state, stencil cells f-3..f+1 (k = 0..4)
//   side 1: right state, stencil cells f-2..f+2
// ---------------------------------------------------------------------------
// S: the arithmetic of the local Jacobians (double; float for the FP32
// reverse sweep, whose shares are still stored and gathered in FP64).
template <int DIR, int DIM, typename S>
__global__ void __launch_bounds__(128) k_adj_face(AdjArgs A) {
    constexpr int NVN = NV<DIM>::n;
    constexpr int ND = 2 * NVN;
    const Params& P = A.P;
    const Fields& F = A.F;
    const int fnx = P.nx + (DIR == 0), fny = P.ny + (DIR == 1), fnz = P.nz + (DIR == 2);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long tot = (long long)fnx * fny * fnz;
    if (t >= tot) return;
    int i, j, k;
    split3(t, fnx, fny, i, j, k);
    const size_t base = cidx(P, i, j, k);   // right cell of the face
    const long st = (DIR == 0) ? 1L : (DIR == 1) ? (long)P.nxT : (long)P.nxT * P.nyT;
    const int pos = (DIR == 0) ? i : (DIR == 1) ? j : k;
    const int nd = (DIR == 0) ? P.nx : (DIR == 1) ? P.ny : P.nz;
    const int dim = DIM;

    // mu = dJ/dF (cons order)
    S mu[NVN];
    {
        const bool rIn = pos < nd, lIn = pos >= 1;
        const int li = (DIR == 0) ? i - 1 : i, lj = (DIR == 1) ? j - 1 : j, lk = (DIR == 2) ? k - 1 : k;
        const double cR = rIn ? face_coeff<DIR>(P, F, i, j, k) : 0.0;
        const double cL = lIn ? face_coeff<DIR>(P, F, li, lj, lk) : 0.0;
#pragma unroll
        for (int q = 0; q < NVN; ++q) {
            double lr = rIn ? A.lam[q][base] : 0.0;
            double ll = lIn ? A.lam[q][base - st] : 0.0;
            mu[q] = (S)(cR * lr - cL * ll);
        }
    }
    const bool weno = (P.reconOrder == SIFV_WENO5);
    // reconstruction values and stencil gradients
    S WL[NVN], WR[NVN], dL[NVN][5], dR[NVN][5];
#pragma unroll
    for (int v = 0; v < NVN; ++v) {
        const double* f = prim_ptr(F, v, dim);
        S s[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) s[q] = (S)f[base + (q - 3) * st];
        // left state: stencil cells 0..4, right state: cells 1..5 (each seeded 0..4)
        using D5 = Dual<5, S>;
        D5 x[5], l, rr;
        const D5 e5(P.wenoEps);
#pragma unroll
        for (int q = 0; q < 5; ++q) x[q] = D5::seed(s[q], q);
        l = weno ? weno5L<D5>(x[0], x[1], x[2], x[3], x[4], e5) : upwind5L<D5>(x[0], x[1], x[2], x[3], x[4]);
#pragma unroll
        for (int q = 0; q < 5; ++q) x[q] = D5::seed(s[q + 1], q);
        rr = weno ? weno5R<D5>(x[0], x[1], x[2], x[3], x[4], e5) : upwind5R<D5>(x[0], x[1], x[2], x[3], x[4]);
        WL[v] = l.v;
        WR[v] = rr.v;
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            dL[v][q] = l.d[q];
            dR[v][q] = rr.d[q];
        }
    }
    // flux Jacobian w.r.t. (WL, WR)
    FaceState<0, Dual<ND, S>> L, R;
    L.rho = Dual<ND, S>::seed(WL[0], 0);
    R.rho = Dual<ND, S>::seed(WR[0], NVN);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        L.u[d] = (d < DIM) ? Dual<ND, S>::seed(WL[1 + d], 1 + d) : Dual<ND, S>(0.0);
        R.u[d] = (d < DIM) ? Dual<ND, S>::seed(WR[1 + d], NVN + 1 + d) : Dual<ND, S>(0.0);
    }
    L.p = Dual<ND, S>::seed(WL[DIM + 1], DIM + 1);
    R.p = Dual<ND, S>::seed(WR[DIM + 1], NVN + DIM + 1);
    L.sigma = R.sigma = Dual<ND, S>(0.0);
    L.gEff = R.gEff = Dual<ND, S>(P.gamma);
    L.piEff = R.piEff = Dual<ND, S>(P.pInf);
    FaceFlux<0, Dual<ND, S>> Fx;
    riemann_T<DIR, Dual<ND, S>>(P, L, R, Fx);
    S gW[ND];
#pragma unroll
    for (int a = 0; a < ND; ++a) gW[a] = S(0);
#pragma unroll
    for (int q = 0; q < NVN; ++q) {
        const Dual<ND, S>& fq = flux_comp(Fx, q, dim);
#pragma unroll
        for (int a = 0; a < ND; ++a) gW[a] += mu[q] * fq.d[a];
    }
    double* const sh = A.share[DIR];
#pragma unroll
    for (int v = 0; v < NVN; ++v) {
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            sh[(size_t)((0 * 5 + q) * NVN + v) * tot + t] = (double)(gW[v] * dL[v][q]);
            sh[(size_t)((1 * 5 + q) * NVN + v) * tot + t] = (double)(gW[NVN + v] * dR[v][q]);
        }
    }
}

// ghost images of interior index c along one axis: positions g in the
// ghost ranges whose PRIM source is c (with the axis's sn, sa)
__device__ __forceinline__ int axis_images(int c, int n, int ng, int bcLo, int bcHi, int* pos, double* sn,
                                           double* sa) {
    int m = 0;
    pos[m] = c; sn[m] = 1.0; sa[m] = 1.0; ++m;
    for (int g = -ng; g < 0; ++g) {
        double a, b;
        if (prim_src(g, n, bcLo, bcHi, a, b) == c) { pos[m] = g; sn[m] = a; sa[m] = b; ++m; }
    }
    for (int g = n; g < n + ng; ++g) {
        double a, b;
        if (prim_src(g, n, bcLo, bcHi, a, b) == c) { pos[m] = g; sn[m] = a; sa[m] = b; ++m; }
    }
    return m;
}

// sum of the direction-DIR shares at stencil position p (image cell (pi, pj, pk))
template <int DIR, int DIM>
__device__ __forceinline__ void gather_dir(const AdjArgs& A, int pi, int pj, int pk, double* acc) {
    constexpr int NVN = NV<DIM>::n;
    const Params& P = A.P;
    // faces exist only at interior transverse positions
    if (DIR != 0 && (pi < 0 || pi >= P.nx)) return;
    if (DIR != 1 && DIM >= 2 && (pj < 0 || pj >= P.ny)) return;
    if (DIR != 2 && DIM >= 3 && (pk < 0 || pk >= P.nz)) return;
    const int p = (DIR == 0) ? pi : (DIR == 1) ? pj : pk;
    const int nd = (DIR == 0) ? P.nx : (DIR == 1) ? P.ny : P.nz;
    const int fnx = P.nx + (DIR == 0), fny = P.ny + (DIR == 1), fnz = P.nz + (DIR == 2);
    const long long tot = (long long)fnx * fny * fnz;
    const double* sh = A.share[DIR];
    for (int f = p - 2; f <= p + 3; ++f) {
        if (f < 0 || f > nd) continue;
        const long long t = (DIR == 0) ? face_index<0>(P, f, pj, pk)
                            : (DIR == 1) ? face_index<1>(P, pi, f, pk) : face_index<2>(P, pi, pj, f);
        const int kl = p - f + 3;   // left stencil position (cells f-3..f+1)
        const int kr = p - f + 2;   // right stencil position (cells f-2..f+2)
#pragma unroll
        for (int v = 0; v < NVN; ++v) {
            if (kl >= 0 && kl <= 4) acc[v] += sh[(size_t)((0 * 5 + kl) * NVN + v) * tot + t];
            if (kr >= 0 && kr <= 4) acc[v] += sh[(size_t)((1 * 5 + kr) * NVN + v) * tot + t];
        }
    }
}

template <int DIM>
__global__ void __launch_bounds__(128) k_adj_cell(AdjArgs A) {
    constexpr int NVN = NV<DIM>::n;
    const Params& P = A.P;
    const Fields& F = A.F;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!int_coords(P, t, i, j, k)) return;
    const size_t c = cidx(P, i, j, k);
    // images along each axis
    // at most 1 + 2 nGhost images per axis (nGhost <= 7 is checked by the host)
    int px[16], py[16], pz[16];
    double snx[16], sax[16], sny[16], say[16], snz[16], saz[16];
    const int mx = axis_images(i, P.nx, P.ngx, P.bc[0], P.bc[1], px, snx, sax);
    const int my = (DIM >= 2) ? axis_images(j, P.ny, P.ngy, P.bc[2], P.bc[3], py, sny, say) : 1;
    const int mz = (DIM >= 3) ? axis_images(k, P.nz, P.ngz, P.bc[4], P.bc[5], pz, snz, saz) : 1;
    if (DIM < 2) { py[0] = j; sny[0] = say[0] = 1.0; }
    if (DIM < 3) { pz[0] = k; snz[0] = saz[0] = 1.0; }
    double gW[NVN];
#pragma unroll
    for (int v = 0; v < NVN; ++v) gW[v] = 0.0;
    for (int a = 0; a < mx; ++a)
        for (int b = 0; b < my; ++b)
            for (int e = 0; e < mz; ++e) {
                double acc[NVN];
#pragma unroll
                for (int v = 0; v < NVN; ++v) acc[v] = 0.0;
                gather_dir<0, DIM>(A, px[a], py[b], pz[e], acc);
                if (DIM >= 2) gather_dir<1, DIM>(A, px[a], py[b], pz[e], acc);
                if (DIM >= 3) gather_dir<2, DIM>(A, px[a], py[b], pz[e], acc);
                // ghost velocity signs (composition of prim_source)
                double sg[3] = {1.0, 1.0, 1.0};
                if (a > 0) { sg[0] *= snx[a] * sax[a]; sg[1] *= sax[a]; sg[2] *= sax[a]; }
                if (b > 0) { sg[0] *= say[b]; sg[1] *= sny[b] * say[b]; sg[2] *= say[b]; }
                if (e > 0) { sg[0] *= saz[e]; sg[1] *= saz[e]; sg[2] *= snz[e] * saz[e]; }
                gW[0] += acc[0];
#pragma unroll
                for (int d = 0; d < DIM; ++d) gW[1 + d] += sg[d] * acc[1 + d];
                gW[DIM + 1] += acc[DIM + 1];
            }
    // cons -> prim Jacobian (IdealGasEOS / StiffenedGasEOS::toPrimitive):
    // rho_W = rho; u = m / max(rho, 1e-14); ke = 0.5 r sum u^2;
    // p = (g - 1)(E - ke) [- g pInf]  (ideal: max(., 1e-14))
    const double rho = F.rho[c];
    const bool rAct = rho > 1e-14;
    const double r = rAct ? rho : 1e-14;
    double u[3] = {0.0, 0.0, 0.0}, u2 = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        u[d] = cons_ptr(F, 1 + d, DIM)[c] / r;
        u2 += u[d] * u[d];
    }
    const double gm1 = P.gamma - 1.0;
    bool pAct = true;
    if (!P.eosStiffened) {
        double e = F.rhoE[c] - 0.5 * r * u2;
        pAct = gm1 * e > 1e-14;
    }
    const double gp = pAct ? gW[DIM + 1] : 0.0;
    double g[NVN];
    g[0] = gW[0] + (rAct ? gp * gm1 * 0.5 * u2 : 0.0);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        if (rAct) g[0] -= gW[1 + d] * u[d] / r;
        g[1 + d] = gW[1 + d] / r - gp * gm1 * u[d];
    }
    g[DIM + 1] = gp * gm1;
    // RK combination
#pragma unroll
    for (int q = 0; q < NVN; ++q) {
        const double lin = A.lam[q][c];
        double ln = A.a1 * lin + A.a3 * A.dt * g[q];
        double a0 = A.acc0[q][c] + A.a2 * lin;
        if (A.stage0) {
            ln += a0;
            a0 = 0.0;
        }
        A.lam[q][c] = ln;
        A.acc0[q][c] = a0;
    }
}

// ---------------------------------------------------------------------------
// Tangent (forward mode).
// ---------------------------------------------------------------------------
// dW of every cell (ghosts: the source cell's dW with the velocity signs)
template <int DIM>
__global__ void __launch_bounds__(256) k_tan_prim(AdjArgs A) {
    const Params& P = A.P;
    const Fields& F = A.F;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!ext_coords(P, t, i, j, k)) return;
    const size_t d = cidx(P, i, j, k);
    double sg[3] = {1.0, 1.0, 1.0};
    const size_t s = is_interior(P, i, j, k) ? d : prim_source(P, i, j, k, sg);
    const double rho = F.rho[s];
    const bool rAct = rho > 1e-14;
    const double r = rAct ? rho : 1e-14;
    double u[3] = {0.0, 0.0, 0.0}, u2 = 0.0;
#pragma unroll
    for (int q = 0; q < DIM; ++q) {
        u[q] = cons_ptr(F, 1 + q, DIM)[s] / r;
        u2 += u[q] * u[q];
    }
    const double gm1 = P.gamma - 1.0;
    bool pAct = true;
    if (!P.eosStiffened) pAct = gm1 * (F.rhoE[s] - 0.5 * r * u2) > 1e-14;
    const double dr = A.tan[0][s];
    double dp = A.tan[DIM + 1][s] + (rAct ? 0.5 * u2 * dr : 0.0);
    A.tanW[0][d] = dr;
#pragma unroll
    for (int q = 0; q < DIM; ++q) {
        const double dm = A.tan[1 + q][s];
        double du = dm / r - (rAct ? u[q] * dr / r : 0.0);
        dp -= u[q] * dm;
        A.tanW[1 + q][d] = sg[q] * du;
    }
    A.tanW[DIM + 1][d] = pAct ? gm1 * dp : 0.0;
}

template <int DIR, int DIM>
__global__ void __launch_bounds__(128) k_tan_face(AdjArgs A) {
    constexpr int NVN = NV<DIM>::n;
    const Params& P = A.P;
    const Fields& F = A.F;
    const int fnx = P.nx + (DIR == 0), fny = P.ny + (DIR == 1), fnz = P.nz + (DIR == 2);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long tot = (long long)fnx * fny * fnz;
    if (t >= tot) return;
    int i, j, k;
    split3(t, fnx, fny, i, j, k);
    const size_t base = cidx(P, i, j, k);
    const long st = (DIR == 0) ? 1L : (DIR == 1) ? (long)P.nxT : (long)P.nxT * P.nyT;
    const bool weno = (P.reconOrder == SIFV_WENO5);
    const int dim = DIM;
    Dual<1> WL[NVN], WR[NVN];
#pragma unroll
    for (int v = 0; v < NVN; ++v) {
        const double* f = prim_ptr(F, v, dim);
        const double* df = A.tanW[v];
        Dual<1> s[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            s[q].v = f[base + (q - 3) * st];
            s[q].d[0] = df[base + (q - 3) * st];
        }
        recon5<Dual<1>>(weno, P.wenoEps, s, WL[v], WR[v]);
    }
    FaceState<0, Dual<1>> L, R;
    L.rho = WL[0];
    R.rho = WR[0];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        L.u[d] = (d < DIM) ? WL[1 + d] : Dual<1>(0.0);
        R.u[d] = (d < DIM) ? WR[1 + d] : Dual<1>(0.0);
    }
    L.p = WL[DIM + 1];
    R.p = WR[DIM + 1];
    L.sigma = R.sigma = Dual<1>(0.0);
    L.gEff = R.gEff = Dual<1>(P.gamma);
    L.piEff = R.piEff = Dual<1>(P.pInf);
    FaceFlux<0, Dual<1>> Fx;
    riemann_T<DIR, Dual<1>>(P, L, R, Fx);
#pragma unroll
    for (int q = 0; q < NVN; ++q) A.tanF[DIR][q][t] = flux_comp(Fx, q, dim).d[0];
}

template <int DIM>
__global__ void __launch_bounds__(256) k_tan_update(AdjArgs A, int save) {
    constexpr int NVN = NV<DIM>::n;
    const Params& P = A.P;
    const Fields& F = A.F;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!int_coords(P, t, i, j, k)) return;
    const size_t c = cidx(P, i, j, k);
    const double dt = A.dtDev ? *A.dtDev : A.dt;
    double dR[NVN];
#pragma unroll
    for (int q = 0; q < NVN; ++q) dR[q] = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        const double co = (d == 0) ? face_coeff<0>(P, F, i, j, k)
                          : (d == 1) ? face_coeff<1>(P, F, i, j, k) : face_coeff<2>(P, F, i, j, k);
        const long long lo = (d == 0) ? face_index<0>(P, i, j, k)
                             : (d == 1) ? face_index<1>(P, i, j, k) : face_index<2>(P, i, j, k);
        const long long hi = (d == 0) ? face_index<0>(P, i + 1, j, k)
                             : (d == 1) ? face_index<1>(P, i, j + 1, k) : face_index<2>(P, i, j, k + 1);
#pragma unroll
        for (int q = 0; q < NVN; ++q) dR[q] += co * A.tanF[d][q][lo] - co * A.tanF[d][q][hi];
    }
#pragma unroll
    for (int q = 0; q < NVN; ++q) {
        const double du = A.tan[q][c];
        if (save) A.tan0[q][c] = du;
        const double du0 = (A.a2 != 0.0) ? A.tan0[q][c] : 0.0;
        A.tan[q][c] = A.a1 * du + A.a2 * du0 + A.a3 * dt * dR[q];
    }
}

}  // namespace sifv
