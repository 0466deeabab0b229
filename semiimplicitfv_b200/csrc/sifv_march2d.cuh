// sifv_march2d.cuh -- one fused kernel per SSP-RK stage for the 2D explicit
// step of the fast-FP64 and mixed-precision paths: every warp marches up a
// strip of 30 columns, one cell row per step.
//
// A warp owns a strip [x0, x0 + 30) x [y0, y1) of cells.  Its 32 lanes
// hold the x positions x0 - 1 .. x0 + 30 (the strip and one position on
// each side).  It keeps a warp-private ring of six rows of primitives in
// shared memory (each row: the strip with its 3-cell halo on both sides,
// 36 positions), and per row step j:
//   1. converts row j + 3 (conservative -> primitive in FP64, ghosts through
//      the PRIM ghost map with the velocity signs, src/RectilinearMesh.cpp:
//      127-131, src/SolutionState.cpp:187-205) from a cp.async staging
//      buffer into the ring, and starts the copy of row j + 4;
//   2. reconstructs both WENO5 face values of its column at row j + 1 (one
//      set of smoothness indicators, src/Reconstruction.cpp:119-168) and
//      solves the y-face Riemann problem between rows j and j + 1 (the
//      row-j value from below was reconstructed one step earlier);
//   3. reconstructs row j along x at its position, solves the x-face
//      Riemann problem with its neighbour lane's value (warp shuffle);
//   4. updates cell (column, j) from the two x fluxes (shuffle) and the two
//      y fluxes (registers): U' = a1 U + a2 U0 + a3 dt R
//      (src/ExplicitSolver.cpp:127-188).
// Every primitive is converted once per strip (plus the 6-position halo),
// every cell is reconstructed once per direction (plus the two halo
// positions of a strip), and no step waits on another warp: warps share
// nothing, so there is no block-wide barrier.
//
// The stage input and output are different arrays (neighbouring strips
// read the input's halo while the output is written); the last stage writes
// the step's state over the step-start state, which only the cell itself
// reads there (U0), and writes the primitives of the updated cells.
//
// T = double: fast FP64.  T = float: mixed precision -- the primitives are
// recovered in FP64 and rounded to FP32 for the reconstruction, the Riemann
// fluxes and the flux divergence (FP32 accumulation); the FP32 divergence
// is added to the FP64 state in FP64, which keeps the low-order bits that
// an FP32 state would lose (the role compensated summation plays for an
// FP32 accumulator).
#pragma once

#include "sifv_sweep.cuh"

namespace sifv {

// Resident blocks per SM of the FP64 kernel (launch bounds): 5 blocks of 4
// warps leave 96 registers per thread.
#ifndef SIFV_MARCH_FP64_BLOCKS
#define SIFV_MARCH_FP64_BLOCKS 5
#endif

template <typename T>
struct MarchShape {
    static constexpr int warps = 4;      // warps per block
    static constexpr int cols = 30;      // cells per strip row
    static constexpr int pos = 36;       // ring positions per row: strip + 3-cell halo each side
    static constexpr int rows = 5;       // ring rows: j-2 .. j+2 before step j (row j+3 replaces row j-2)
    static constexpr int blocks = (sizeof(T) == 8) ? SIFV_MARCH_FP64_BLOCKS : 8;   // resident blocks per SM
};

// One warp's shared memory: the primitive ring (rho, u, v, p) and the
// two-row staging buffer of raw conservative values (cp.async).
template <typename T>
struct MarchWarpSmem {
    T ring[MarchShape<T>::rows][4][MarchShape<T>::pos];
    double stage[2][4][MarchShape<T>::pos];
};

__device__ __forceinline__ void march_cp8(double* smemDst, const double* gmemSrc) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smemDst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gmemSrc) : "memory");
}
__device__ __forceinline__ void march_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void march_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Per lane and strip: the x part of the ghost map of the (up to two) ring
// positions the lane loads and converts -- source column, velocity signs,
// and whether an interior row / a ghost row needs the position.
struct MarchCol {
    int q;         // ring position (-1: none)
    int src;       // source column (interior index, or the column itself on an exchange face)
    int flags;     // bit 0: needed on interior rows, 1: needed on ghost rows, 2: negate u, 3: negate v
};

__device__ __forceinline__ MarchCol march_col(const Params& P, int x0, int lane, int round) {
    MarchCol m;
    m.q = (round == 0) ? lane + 2 : (lane < 2 ? lane : (lane < 4 ? lane + 32 : -1));
    m.src = 0;
    m.flags = 0;
    if (m.q < 0) return m;
    const int x = x0 - 3 + m.q;
    if (x < P.nx + 3) m.flags |= 1;                        // interior rows: up to the third ghost column
    if (m.q >= 3 && m.q < 33 && x < P.nx) m.flags |= 2;    // ghost rows: the strip's own columns
    double sn, sa;
    m.src = prim_src(x, P.nx, P.bc[0], P.bc[1], sn, sa);
    if (m.src != x) {
        if (sn * sa < 0.0) m.flags |= 4;
        if (sa < 0.0) m.flags |= 8;
    }
    return m;
}

template <typename T, int RS>
__global__ void __launch_bounds__(128, MarchShape<T>::blocks) k_march2d(TileArgs A) {
    using S = MarchShape<T>;
    extern __shared__ __align__(16) unsigned char smemRaw[];
    if (A.ctl->skip) return;
    const int lane = threadIdx.x & 31;
    MarchWarpSmem<T>& W = reinterpret_cast<MarchWarpSmem<T>*>(smemRaw)[threadIdx.x >> 5];
    const Params& P = A.P;
    const int nx = P.nx, ny = P.ny;
    const T eps = (T)A.eps;
    const double a3dt = A.a3 * A.ctl->dt;
    const bool useU0 = A.u0[0] != nullptr;
    const long long units = (long long)A.strips * A.segs;
    const long long nWarps = (long long)gridDim.x * S::warps;
    const long long rowStride = P.nxT;

    for (long long unit = (long long)blockIdx.x * S::warps + (threadIdx.x >> 5); unit < units; unit += nWarps) {
        const int x0 = (int)(unit % A.strips) * S::cols;
        const int y0 = (int)(unit / A.strips) * A.segRows;
        const int y1 = min(y0 + A.segRows, ny);
        const MarchCol c0 = march_col(P, x0, lane, 0), c1 = march_col(P, x0, lane, 1);

        // start of row r's cells in the arrays (ghost rows through the y map), and its velocity signs
        auto row_map = [&](int r, long long& off, int& negFlags, bool& ghost) {
            double sn, sa;
            const int sy = prim_src(r, ny, P.bc[2], P.bc[3], sn, sa);
            off = (long long)P.ngx + rowStride * ((long long)sy + P.ngy);
            negFlags = 0;
            if (sy != r) {
                if (sa < 0.0) negFlags |= 4;          // u: tangential
                if (sn * sa < 0.0) negFlags |= 8;     // v: normal
            }
            ghost = r < 0 || r >= ny;
        };
        // cp.async of the raw conservative values of row r into staging slot b
        auto issue_row = [&](int r, int b) {
            long long off;
            int nf;
            bool ghost;
            row_map(r, off, nf, ghost);
            const int need = ghost ? 2 : 1;
            if (c0.flags & need) {
#pragma unroll
                for (int v = 0; v < 4; ++v) march_cp8(&W.stage[b][v][c0.q], A.in[v] + off + c0.src);
            }
            if (c1.q >= 0 && (c1.flags & need)) {
#pragma unroll
                for (int v = 0; v < 4; ++v) march_cp8(&W.stage[b][v][c1.q], A.in[v] + off + c1.src);
            }
            march_commit();
        };
        // conservative -> primitive of staging slot b (row r) into ring row `dst`
        auto convert_pos = [&](const MarchCol& m, int b, int need, int negRow, T* dst) {
            T w0 = (T)0, w1 = (T)0, w2 = (T)0, w3 = (T)0;
            if (m.flags & need) {
                const int neg = (m.flags ^ negRow);
                const double rr = W.stage[b][0][m.q], ru = W.stage[b][1][m.q];
                const double rv = W.stage[b][2][m.q], re = W.stage[b][3][m.q];
                const double rho = (rr < 1e-14) ? 1e-14 : rr;
                const double ir = frcp(rho);
                const double u = ru * ir, v = rv * ir;
                double ke = u * u;
                ke += v * v;
                ke *= 0.5 * rho;
                const double e = re - ke;
                double p = P.eosStiffened ? (P.gamma - 1.0) * e - P.gamma * P.pInf : (P.gamma - 1.0) * e;
                if (!P.eosStiffened && p < 1e-14) p = 1e-14;
                w0 = (T)rr;
                w1 = (T)((neg & 4) ? -u : u);
                w2 = (T)((neg & 8) ? -v : v);
                w3 = (T)p;
            }
            dst[m.q] = w0;
            dst[S::pos + m.q] = w1;
            dst[2 * S::pos + m.q] = w2;
            dst[3 * S::pos + m.q] = w3;
        };
        auto convert_row = [&](int r, int b, T* dst) {
            long long off;
            int nf;
            bool ghost;
            row_map(r, off, nf, ghost);
            const int need = ghost ? 2 : 1;
            convert_pos(c0, b, need, nf, dst);
            if (c1.q >= 0) convert_pos(c1, b, need, nf, dst);
        };

        // ring rows j-2 .. j+2 before step j: R0 .. R4 (rotated every step)
        T* R0 = &W.ring[0][0][0];
        T* R1 = &W.ring[1][0][0];
        T* R2 = &W.ring[2][0][0];
        T* R3 = &W.ring[3][0][0];
        T* R4 = &W.ring[4][0][0];

        // the lane's cell column and its x metric (constant along the strip)
        const int cx = x0 + lane - 1;
        const bool colActive = lane >= 1 && lane <= S::cols && cx < nx;
        const T invx = colActive ? (T)A.inv[0][cx + P.ngx] : (T)0;

        double dtMin = __longlong_as_double(0x7ff0000000000000LL);   // next step's dt over the lane's cells
        Prim5<T> Lc;    // value at the high face of the current row, from below
        Flux4<T> Fc;    // y flux at the low face of the current row
        Lc = Prim5<T>{(T)0, (T)0, (T)0, (T)0, (T)0};
        Fc = Flux4<T>{(T)0, (T)0, (T)0, (T)0, (T)0};

        // Steps y0-5 .. y0-3 only convert rows y0-2 .. y0 (rows y0-3 .. y0-1
        // are converted by the first steps' ... ) -- see the phase tests below.
        issue_row(y0 - 3, (y0 - 3) & 1);
        for (int j = y0 - 6; j < y1; ++j) {
            // 1. row j+3 into the ring (its copy was started a step ago); start row j+4
            if (j + 4 < y1 + 3) issue_row(j + 4, (j + 4) & 1);
            else march_commit();                          // keep one group per step
            march_wait<1>();
            __syncwarp();                                  // ring row j-2 is no longer read
            convert_row(j + 3, (j + 3) & 1, R0);
            {   // rotate: rows j-1 .. j+3
                T* t = R0;
                R0 = R1; R1 = R2; R2 = R3; R3 = R4; R4 = t;
            }
            __syncwarp();
            if (j < y0 - 2) continue;                      // the ring is filling

            // 2. y: face values of row j+1 (rows j-1 .. j+3), flux at the face between rows j and j+1
            const int q = lane + 2;
            Prim5<T> Ln, Rn;
            {
                T l[4], rr[4];
#pragma unroll
                for (int v = 0; v < 4; ++v)
                    weno5_pair(R0[v * S::pos + q], R1[v * S::pos + q], R2[v * S::pos + q], R3[v * S::pos + q],
                               R4[v * S::pos + q], eps, l[v], rr[v]);
                Ln = Prim5<T>{l[0], l[1], l[2], (T)0, l[3]};
                Rn = Prim5<T>{rr[0], rr[1], rr[2], (T)0, rr[3]};
            }
            Flux4<T> Fy;
            face_flux<1, 2, T>(RS, A.C, Lc, Rn, Fy);
            Lc = Ln;
            if (j < y0) {                                  // rows y0-2, y0-1: only the carried y state
                Fc = Fy;
                continue;
            }

            // 3. x: both face values at the lane's position of row j (ring row R1), flux at its right face
            Prim5<T> Lx, Rx;
            {
                T l[4], rr[4];
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const T* row = R1 + v * S::pos + q - 2;
                    weno5_pair(row[0], row[1], row[2], row[3], row[4], eps, l[v], rr[v]);
                }
                Lx = Prim5<T>{l[0], l[1], l[2], (T)0, l[3]};
                Rx = Prim5<T>{rr[0], rr[1], rr[2], (T)0, rr[3]};
            }
            // face between positions lane-1 and lane: L from this lane, R from the next
            Prim5<T> Rr;
            Rr.rho = __shfl_down_sync(0xffffffffu, Rx.rho, 1);
            Rr.u = __shfl_down_sync(0xffffffffu, Rx.u, 1);
            Rr.v = __shfl_down_sync(0xffffffffu, Rx.v, 1);
            Rr.w = (T)0;
            Rr.p = __shfl_down_sync(0xffffffffu, Rx.p, 1);
            Flux4<T> Fx;   // x flux at the right face of the lane's position
            face_flux<0, 2, T>(RS, A.C, Lx, Rr, Fx);
            Flux4<T> Fxl;  // ... and at its left face (previous lane's right face)
            Fxl.mass = __shfl_up_sync(0xffffffffu, Fx.mass, 1);
            Fxl.m0 = __shfl_up_sync(0xffffffffu, Fx.m0, 1);
            Fxl.m1 = __shfl_up_sync(0xffffffffu, Fx.m1, 1);
            Fxl.energy = __shfl_up_sync(0xffffffffu, Fx.energy, 1);

            // 4. divergence (FP32 accumulation in the mixed form) + stage update in FP64
            if (colActive) {
                const size_t c = (size_t)((long long)P.ngx + cx + rowStride * ((long long)j + P.ngy));
                const T invy = (T)A.inv[1][j + P.ngy];
                const T fl[4] = {Fxl.mass, Fxl.m0, Fxl.m1, Fxl.energy};
                const T fr[4] = {Fx.mass, Fx.m0, Fx.m1, Fx.energy};
                const T gl[4] = {Fc.mass, Fc.m0, Fc.m1, Fc.energy};
                const T gr[4] = {Fy.mass, Fy.m0, Fy.m1, Fy.energy};
                double nw[4];
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const T rx = invx * (fl[v] - fr[v]);
                    const T r = invy * (gl[v] - gr[v]) + rx;
                    double n = A.a1 * A.in[v][c] + a3dt * (double)r;
                    if (useU0) n += A.a2 * A.u0[v][c];
                    nw[v] = n;
                }
#pragma unroll
                for (int v = 0; v < 4; ++v) A.out[v][c] = nw[v];
                if (A.last) {   // primitives of the new state (cons_to_prim_cell, single phase)
                    const double rho = (nw[0] < 1e-14) ? 1e-14 : nw[0];
                    const double ir = frcp(rho);
                    const double u = nw[1] * ir, v = nw[2] * ir;
                    double ke = u * u;
                    ke += v * v;
                    ke *= 0.5 * rho;
                    const double e = nw[3] - ke;
                    const double p = P.eosStiffened ? (P.gamma - 1.0) * e - P.gamma * P.pInf
                                                    : ((P.gamma - 1.0) * e < 1e-14 ? 1e-14 : (P.gamma - 1.0) * e);
                    A.velU[c] = u;
                    A.velV[c] = v;
                    A.pres[c] = p;
                    if (A.dtNext) {   // computeAcousticTimeStep's cell term, as k_dt_acoustic evaluates it
                        const double cs = single_sound_speed(P, nw[0], p);
                        double dtCell = A.dx[cx + P.ngx] / (fabs(u) + cs);
                        dtCell = smin(dtCell, A.dy[j + P.ngy] / (fabs(v) + cs));
                        dtMin = smin(dtMin, A.cfl * dtCell);   // a NaN candidate leaves dtMin
                    }
                }
            }
            Fc = Fy;
        }
        march_wait<0>();
        __syncwarp();
        if (A.dtNext) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) dtMin = smin(dtMin, __shfl_xor_sync(0xffffffffu, dtMin, o));
            if (lane == 0) atomicMin(&A.ctl->dtBits, d2bits(dtMin));
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
