// sifv_tile2d.cuh -- one fused kernel per SSP-RK stage for the 2D explicit
// step of the fast-FP64 and mixed-precision paths.
//
// A block owns a TX x TY tile of cells.  It stages the conservative state of
// the tile and its 3-cell halo (ghosts through the PRIM ghost map with the
// velocity signs, src/RectilinearMesh.cpp:127-131) as primitives in shared
// memory (FP64 conversion, src/SolutionState.cpp:187-205), reconstructs both
// face values of every cell along x (one set of WENO5 smoothness indicators
// per cell, src/Reconstruction.cpp:119-168), solves the x-face Riemann
// problems, does the same along y, and applies the flux divergence and the
// stage update U' = a1 U + a2 U0 + a3 dt R (src/ExplicitSolver.cpp:127-188)
// to its own cells.  Per stage the state is read once (plus the halo, from
// L2) and written once: no face arrays, no rhs or primitive round trips.
// The stage input and output are different arrays (neighbouring tiles read
// the input's halo while the output is written); the last stage writes the
// step's state over the step-start state, which only the cell itself reads
// there (U0), and writes the primitives of the updated cells.
#pragma once

#include "sifv_sweep.cuh"

namespace sifv {

template <int TX, int TY, typename T>
struct TileSmem {
    static constexpr int HX = TX + 6, HY = TY + 6;              // primitives incl. halo
    static constexpr int RX = (TX + 2) * TY, RY = TX * (TY + 2);  // reconstruction positions
    static constexpr int RN = (RX > RY) ? RX : RY;
    T w[4][HY][HX];       // rho, u, v, p
    T rl[4][RN];          // value at the cell's high face (from below)
    T rr[4][RN];          // value at the cell's low face (from above)
    T fx[4][TY][TX + 1];  // x-face fluxes: mass, mom x, mom y, energy
    T fy[4][TY + 1][TX];
};

// Threads per block: FP64 512 (2 blocks of 96 KB per SM: 32 warps), FP32
// 256 (4 blocks of 48 KB per SM).
template <typename T>
struct TileThreads {
    static constexpr int value = (sizeof(T) == 8) ? 512 : 256;
    static constexpr int blocks = (sizeof(T) == 8) ? 2 : 4;
};

template <int TX, int TY, typename T>
__global__ void __launch_bounds__(TileThreads<T>::value, TileThreads<T>::blocks) k_tile2d(TileArgs A) {
    using S = TileSmem<TX, TY, T>;
    extern __shared__ __align__(16) unsigned char smemRaw[];
    S& sm = *reinterpret_cast<S*>(smemRaw);
    if (A.ctl->skip) return;
    const Params& P = A.P;
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
    const int nx = P.nx, ny = P.ny;
    const T eps = (T)A.eps;

    // ---- stage the primitives of the tile and its halo (corners unused) ----
    for (int it = threadIdx.x; it < S::HX * S::HY; it += blockDim.x) {
        const int xl = it % S::HX - 3, yl = it / S::HX - 3;
        int gi = i0 + xl, gj = j0 + yl;
        const bool xin = xl >= 0 && xl < TX, yin = yl >= 0 && yl < TY;
        T* w0 = &sm.w[0][yl + 3][xl + 3];
        if ((!xin && !yin) || gi >= nx + 3 || gj >= ny + 3) {   // corner / past a ragged edge: unused
            w0[0] = w0[S::HX * S::HY] = w0[2 * S::HX * S::HY] = w0[3 * S::HX * S::HY] = (T)0;
            continue;
        }
        double sgu = 1.0, sgv = 1.0, sn, sa;
        const int si = prim_src(gi, nx, P.bc[0], P.bc[1], sn, sa);
        if (si != gi) { sgu *= sn * sa; sgv *= sa; }
        const int sj = prim_src(gj, ny, P.bc[2], P.bc[3], sn, sa);
        if (sj != gj) { sgu *= sa; sgv *= sn * sa; }
        const size_t c = cidx(P, si, sj, 0);
        const double r = A.in[0][c], ru = A.in[1][c], rv = A.in[2][c], re = A.in[3][c];
        const double rho = (r < 1e-14) ? 1e-14 : r;
        const double ir = frcp(rho);
        const double u = ru * ir, v = rv * ir;
        double ke = u * u;
        ke += v * v;
        ke *= 0.5 * rho;
        const double e = re - ke;
        double p = P.eosStiffened ? (P.gamma - 1.0) * e - P.gamma * P.pInf : (P.gamma - 1.0) * e;
        if (!P.eosStiffened && p < 1e-14) p = 1e-14;
        sm.w[0][yl + 3][xl + 3] = (T)r;
        sm.w[1][yl + 3][xl + 3] = (T)(sgu * u);
        sm.w[2][yl + 3][xl + 3] = (T)(sgv * v);
        sm.w[3][yl + 3][xl + 3] = (T)p;
    }
    __syncthreads();

    // ---- x: both face values of positions -1 .. TX of each row ----
    for (int it = threadIdx.x; it < S::RX; it += blockDim.x) {
        const int xl = it % (TX + 2) - 1, yl = it / (TX + 2);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const T* s = &sm.w[v][yl + 3][xl + 1];
            weno5_pair(s[0], s[1], s[2], s[3], s[4], eps, sm.rl[v][it], sm.rr[v][it]);
        }
    }
    __syncthreads();
    for (int it = threadIdx.x; it < (TX + 1) * TY; it += blockDim.x) {
        const int f = it % (TX + 1), yl = it / (TX + 1);   // face between cells f-1 and f
        const int lo = yl * (TX + 2) + f, hi = lo + 1;     // positions f-1 and f
        Prim5<T> L{sm.rl[0][lo], sm.rl[1][lo], sm.rl[2][lo], (T)0, sm.rl[3][lo]};
        Prim5<T> R{sm.rr[0][hi], sm.rr[1][hi], sm.rr[2][hi], (T)0, sm.rr[3][hi]};
        Flux4<T> Fq;
        face_flux<0, 2, T>(P.riemann, A.C, L, R, Fq);
        sm.fx[0][yl][f] = Fq.mass;
        sm.fx[1][yl][f] = Fq.m0;
        sm.fx[2][yl][f] = Fq.m1;
        sm.fx[3][yl][f] = Fq.energy;
    }
    __syncthreads();

    // ---- y: both face values of positions -1 .. TY of each column ----
    for (int it = threadIdx.x; it < S::RY; it += blockDim.x) {
        const int xl = it % TX, yl = it / TX - 1;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const T a = sm.w[v][yl + 1][xl + 3], b = sm.w[v][yl + 2][xl + 3], c = sm.w[v][yl + 3][xl + 3];
            const T d = sm.w[v][yl + 4][xl + 3], e = sm.w[v][yl + 5][xl + 3];
            weno5_pair(a, b, c, d, e, eps, sm.rl[v][it], sm.rr[v][it]);
        }
    }
    __syncthreads();
    for (int it = threadIdx.x; it < TX * (TY + 1); it += blockDim.x) {
        const int xl = it % TX, g = it / TX;        // face between cells g-1 and g of column xl
        const int lo = g * TX + xl, hi = lo + TX;   // positions g-1 and g
        Prim5<T> L{sm.rl[0][lo], sm.rl[1][lo], sm.rl[2][lo], (T)0, sm.rl[3][lo]};
        Prim5<T> R{sm.rr[0][hi], sm.rr[1][hi], sm.rr[2][hi], (T)0, sm.rr[3][hi]};
        Flux4<T> Fq;
        face_flux<1, 2, T>(P.riemann, A.C, L, R, Fq);
        sm.fy[0][g][xl] = Fq.mass;
        sm.fy[1][g][xl] = Fq.m0;
        sm.fy[2][g][xl] = Fq.m1;
        sm.fy[3][g][xl] = Fq.energy;
    }
    __syncthreads();

    // ---- divergence + stage update of the tile's cells ----
    const double a3 = A.a3 * A.ctl->dt;
    for (int it = threadIdx.x; it < TX * TY; it += blockDim.x) {
        const int xl = it % TX, yl = it / TX;
        const int gi = i0 + xl, gj = j0 + yl;
        if (gi >= nx || gj >= ny) continue;
        const size_t c = cidx(P, gi, gj, 0);
        const double cx = A.inv[0][gi + P.ngx], cy = A.inv[1][gj + P.ngy];
        double nw[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double rx = cx * ((double)sm.fx[q][yl][xl] - (double)sm.fx[q][yl][xl + 1]);
            const double r = cy * ((double)sm.fy[q][yl][xl] - (double)sm.fy[q][yl + 1][xl]) + rx;
            double n = A.a1 * A.in[q][c] + a3 * r;
            if (A.u0[0]) n += A.a2 * A.u0[q][c];
            nw[q] = n;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) A.out[q][c] = nw[q];
        if (A.last) {   // primitives of the new state (cons_to_prim_cell, single phase)
            const double rho = (nw[0] < 1e-14) ? 1e-14 : nw[0];
            const double u = nw[1] / rho, v = nw[2] / rho;
            double ke = 0.0;
            ke += u * u;
            ke += v * v;
            ke *= 0.5 * rho;
            const double e = nw[3] - ke;
            A.velU[c] = u;
            A.velV[c] = v;
            A.pres[c] = P.eosStiffened ? (P.gamma - 1.0) * e - P.gamma * P.pInf
                                       : ((P.gamma - 1.0) * e < 1e-14 ? 1e-14 : (P.gamma - 1.0) * e);
        }
    }
}

// Stage output copied over the state (RK1, whose only stage cannot update
// in place).
struct Copy4 {
    const double* src[4];
    double* dst[4];
};
__global__ void k_copy4(const Ctl* ctl, Copy4 A, size_t n) {
    if (ctl->skip) return;
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
#pragma unroll
    for (int q = 0; q < 4; ++q) A.dst[q][t] = A.src[q][t];
}

}  // namespace sifv
