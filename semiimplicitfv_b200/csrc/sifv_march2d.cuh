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
// ... and of the packed-FP32 mixed kernel (7: 72 registers per thread).
#ifndef SIFV_MARCH_MIXED_BLOCKS
#define SIFV_MARCH_MIXED_BLOCKS 7
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

// ---------------------------------------------------------------------------
// Mixed precision on packed FP32: the same march with the FP32 bulk in
// two-wide vector arithmetic (Blackwell's FFMA2 / FADD2 / FMUL2: two FP32
// operations per instruction).  The ring holds (rho, u) and (v, p) pairs, so
// each WENO5 call reconstructs two variables at once; the Riemann solver
// pairs the left and right states; the flux divergence runs on (mass, x
// momentum) and (y momentum, energy) pairs.  Reciprocals and reciprocal
// square roots stay per component (the FP32 special-function unit).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 rcp2(float2 a) { return make_float2(frcp(a.x), frcp(a.y)); }
__device__ __forceinline__ float2 max2(float2 a, float2 b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }

// weno5_pair (FP32 reciprocal-weight form) on two variables at once.
__device__ __forceinline__ void weno5_pair2(float2 v0, float2 v1, float2 v2, float2 v3, float2 v4, float2 eps,
                                            float2& L, float2& R) {
    const float2 t0 = fma2(f2(-2.f), v1, add2(v0, v2)), s0 = fma2(f2(3.f), v2, fma2(f2(-4.f), v1, v0));
    const float2 t1 = fma2(f2(-2.f), v2, add2(v1, v3)), s1 = sub2(v1, v3);
    const float2 t2 = fma2(f2(-2.f), v3, add2(v2, v4)), s2 = fma2(f2(3.f), v2, fma2(f2(-4.f), v3, v4));
    const float2 q0 = fma2(mul2(f2(13.f / 12.f), t0), t0, fma2(mul2(f2(0.25f), s0), s0, eps));
    const float2 q1 = fma2(mul2(f2(13.f / 12.f), t1), t1, fma2(mul2(f2(0.25f), s1), s1, eps));
    const float2 q2 = fma2(mul2(f2(13.f / 12.f), t2), t2, fma2(mul2(f2(0.25f), s2), s2, eps));
    const float2 r0 = rcp2(mul2(q0, q0)), r1 = rcp2(mul2(q1, q1)), r2 = rcp2(mul2(q2, q2));
    // candidate polynomials times 6; the 1/6 goes into the normalisation
    const float2 pL0 = fma2(f2(11.f), v2, fma2(f2(-7.f), v1, mul2(f2(2.f), v0)));
    const float2 pL1 = fma2(f2(2.f), v3, fma2(f2(5.f), v2, mul2(f2(-1.f), v1)));
    const float2 pL2 = fma2(f2(-1.f), v4, fma2(f2(5.f), v3, mul2(f2(2.f), v2)));
    const float2 pR0 = fma2(f2(11.f), v2, fma2(f2(-7.f), v3, mul2(f2(2.f), v4)));
    const float2 pR1 = fma2(f2(2.f), v1, fma2(f2(5.f), v2, mul2(f2(-1.f), v3)));
    const float2 pR2 = fma2(f2(-1.f), v0, fma2(f2(5.f), v1, mul2(f2(2.f), v2)));
    const float2 aL0 = mul2(f2(0.1f), r0), aM = mul2(f2(0.6f), r1), aL2 = mul2(f2(0.3f), r2);
    const float2 aR0 = mul2(f2(0.1f), r2), aR2 = mul2(f2(0.3f), r0);
    const float2 nL = fma2(aL2, pL2, fma2(aM, pL1, mul2(aL0, pL0)));
    const float2 nR = fma2(aR2, pR2, fma2(aM, pR1, mul2(aR0, pR0)));
    const float2 dL = mul2(f2(6.f), add2(add2(aL0, aM), aL2));
    const float2 dR = mul2(f2(6.f), add2(add2(aR0, aM), aR2));
    L = mul2(nL, rcp2(dL));
    R = mul2(nR, rcp2(dR));
}

// Single-phase face flux on the normal axis D (HLLC, Rusanov or LF with
// pressure) of face_flux, on FP32 pairs.  In: left / right states as
// (rho, u), (v, p) pairs.  Out: (mass, x momentum), (y momentum, energy).
// The transverse momentum flux is written as u_t * mass (the same value as
// fm u_t + s (rho* u_t - rho u_t)).
template <int D, int RS>
__device__ __forceinline__ void face_flux2(const FluxConsts& C, float2 lru, float2 lvp, float2 rru, float2 rvp,
                                           float2& fA, float2& fB) {
    const float g = (float)C.gamma, pinf = (float)C.pInf, invGm1 = (float)C.invGm1, gPinf = (float)C.gPinf;
    const float tiny = 1e-14f;
    const float2 RHO = make_float2(lru.x, rru.x), U = make_float2(lru.y, rru.y);
    const float2 V = make_float2(lvp.x, rvp.x), Pp = make_float2(lvp.y, rvp.y);
    const float2 UN = (D == 0) ? U : V, UT = (D == 0) ? V : U;
    const float2 q2 = fma2(V, V, mul2(U, U));
    const float2 rhoE = fma2(mul2(f2(0.5f), RHO), q2, mul2(add2(Pp, f2(gPinf)), f2(invGm1)));
    const float2 gp = mul2(f2(g), max2(add2(Pp, f2(pinf)), f2(tiny)));
    const float2 rg = mul2(gp, max2(RHO, f2(tiny)));
    const float2 c = mul2(gp, make_float2(frsqrt_pos(rg.x), frsqrt_pos(rg.y)));
    float mass, mn, energy;
    if (RS == SIFV_HLLC) {
        const float2 lo = sub2(UN, c), hi = add2(UN, c);
        const float sL = fminf(lo.x, lo.y), sR = fmaxf(hi.x, hi.y);
        const float2 A2 = mul2(RHO, sub2(make_float2(sL, sR), UN));
        const float sStar = (Pp.y - Pp.x + A2.x * UN.x - A2.y * UN.y) * frcp(A2.x - A2.y);
        if (sL >= 0.f || sR <= 0.f) {
            const bool l = sL >= 0.f;
            const float rho = l ? RHO.x : RHO.y, un = l ? UN.x : UN.y, p = l ? Pp.x : Pp.y;
            const float e = l ? rhoE.x : rhoE.y;
            mass = rho * un;
            mn = mass * un + p;
            energy = (e + p) * un;
        } else {
            const bool l = sStar >= 0.f;
            const float s = l ? sL : sR, un = l ? UN.x : UN.y, e = l ? rhoE.x : rhoE.y, a = l ? A2.x : A2.y;
            const float rho = l ? RHO.x : RHO.y, p = l ? Pp.x : Pp.y;
            const float inv = frcp(s - sStar);
            const float rhoStar = a * inv;
            const float fm = rho * un;
            mass = fm + s * (rhoStar - rho);
            const float rs = rhoStar * sStar;
            mn = fm * un + s * (rs - rho * un) + p;
            const float EStar = (s - un) * inv * e + (sStar - un) * (rs + p * inv);
            energy = (e + p) * un + s * (EStar - e);
        }
        const float ut = (sL >= 0.f) ? UT.x : (sR <= 0.f) ? UT.y : (sStar >= 0.f ? UT.x : UT.y);
        const float mt = ut * mass;
        fA = make_float2(mass, D == 0 ? mn : mt);
        fB = make_float2(D == 0 ? mt : mn, energy);
    } else {
        float sMax;
        if (RS == SIFV_RUSANOV) {
            sMax = fmaxf(fabsf(UN.x) + c.x, fabsf(UN.y) + c.y);
        } else {
            sMax = fmaxf(sqrtf(q2.x), sqrtf(q2.y)) + fmaxf(c.x, c.y);
        }
        const float2 FM = mul2(RHO, UN);                 // (fmL, fmR)
        const float2 FN = fma2(FM, UN, Pp);              // normal momentum flux
        const float2 FT = mul2(FM, UT);                  // transverse momentum flux
        const float2 FE = mul2(add2(rhoE, Pp), UN);      // energy flux
        const float2 MN = mul2(RHO, UN), MT = mul2(RHO, UT);
        const float hs = 0.5f * sMax;
        mass = 0.5f * (FM.x + FM.y) - hs * (RHO.y - RHO.x);
        mn = 0.5f * (FN.x + FN.y) - hs * (MN.y - MN.x);
        const float mt = 0.5f * (FT.x + FT.y) - hs * (MT.y - MT.x);
        energy = 0.5f * (FE.x + FE.y) - hs * (rhoE.y - rhoE.x);
        fA = make_float2(mass, D == 0 ? mn : mt);
        fB = make_float2(D == 0 ? mt : mn, energy);
    }
}

template <int RS>
__global__ void __launch_bounds__(128, SIFV_MARCH_MIXED_BLOCKS) k_march2d_mixed(TileArgs A) {
    constexpr int NW = 4, COLS = 30, POS = 36, ROWS = 5;
    struct WarpSmem {
        float2 ring[ROWS][2][POS];     // (rho, u), (v, p)
        double stage[2][4][POS];
    };
    extern __shared__ __align__(16) unsigned char smemRaw[];
    if (A.ctl->skip) return;
    const int lane = threadIdx.x & 31;
    WarpSmem& W = reinterpret_cast<WarpSmem*>(smemRaw)[threadIdx.x >> 5];
    const Params& P = A.P;
    const int nx = P.nx, ny = P.ny;
    const float2 eps = f2((float)A.eps);
    const double a3dt = A.a3 * A.ctl->dt;
    const bool useU0 = A.u0[0] != nullptr;
    const long long units = (long long)A.strips * A.segs;
    const long long nWarps = (long long)gridDim.x * NW;
    const long long rowStride = P.nxT;

    for (long long unit = (long long)blockIdx.x * NW + (threadIdx.x >> 5); unit < units; unit += nWarps) {
        const int x0 = (int)(unit % A.strips) * COLS;
        const int y0 = (int)(unit / A.strips) * A.segRows;
        const int y1 = min(y0 + A.segRows, ny);
        const MarchCol c0 = march_col(P, x0, lane, 0), c1 = march_col(P, x0, lane, 1);
        auto row_map = [&](int r, long long& off, int& negFlags, bool& ghost) {
            double sn, sa;
            const int sy = prim_src(r, ny, P.bc[2], P.bc[3], sn, sa);
            off = (long long)P.ngx + rowStride * ((long long)sy + P.ngy);
            negFlags = 0;
            if (sy != r) {
                if (sa < 0.0) negFlags |= 4;
                if (sn * sa < 0.0) negFlags |= 8;
            }
            ghost = r < 0 || r >= ny;
        };
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
        // FP64 primitive recovery, rounded to FP32 pairs
        auto convert_pos = [&](const MarchCol& m, int b, int need, int negRow, float2 (*dst)[POS]) {
            float2 ru = make_float2(0.f, 0.f), vp = make_float2(0.f, 0.f);
            if (m.flags & need) {
                const int neg = (m.flags ^ negRow);
                const double rr = W.stage[b][0][m.q], rmu = W.stage[b][1][m.q];
                const double rmv = W.stage[b][2][m.q], re = W.stage[b][3][m.q];
                const double rho = (rr < 1e-14) ? 1e-14 : rr;
                const double ir = frcp(rho);
                const double u = rmu * ir, v = rmv * ir;
                double ke = u * u;
                ke += v * v;
                ke *= 0.5 * rho;
                const double e = re - ke;
                double p = P.eosStiffened ? (P.gamma - 1.0) * e - P.gamma * P.pInf : (P.gamma - 1.0) * e;
                if (!P.eosStiffened && p < 1e-14) p = 1e-14;
                ru = make_float2((float)rr, (float)((neg & 4) ? -u : u));
                vp = make_float2((float)((neg & 8) ? -v : v), (float)p);
            }
            dst[0][m.q] = ru;
            dst[1][m.q] = vp;
        };
        auto convert_row = [&](int r, int b, float2 (*dst)[POS]) {
            long long off;
            int nf;
            bool ghost;
            row_map(r, off, nf, ghost);
            const int need = ghost ? 2 : 1;
            convert_pos(c0, b, need, nf, dst);
            if (c1.q >= 0) convert_pos(c1, b, need, nf, dst);
        };
        float2 (*R0)[POS] = W.ring[0];
        float2 (*R1)[POS] = W.ring[1];
        float2 (*R2)[POS] = W.ring[2];
        float2 (*R3)[POS] = W.ring[3];
        float2 (*R4)[POS] = W.ring[4];
        const int cx = x0 + lane - 1;
        const bool colActive = lane >= 1 && lane <= COLS && cx < nx;
        const float invx = colActive ? (float)A.inv[0][cx + P.ngx] : 0.f;
        double dtMin = __longlong_as_double(0x7ff0000000000000LL);
        float2 Lru = make_float2(0.f, 0.f), Lvp = make_float2(0.f, 0.f);   // row value at its high face, from below
        float2 FcA = make_float2(0.f, 0.f), FcB = make_float2(0.f, 0.f);   // y flux at the row's low face
        issue_row(y0 - 3, (y0 - 3) & 1);
        for (int j = y0 - 6; j < y1; ++j) {
            if (j + 4 < y1 + 3) issue_row(j + 4, (j + 4) & 1);
            else march_commit();
            march_wait<1>();
            __syncwarp();
            convert_row(j + 3, (j + 3) & 1, R0);
            {
                float2 (*t)[POS] = R0;
                R0 = R1; R1 = R2; R2 = R3; R3 = R4; R4 = t;
            }
            __syncwarp();
            if (j < y0 - 2) continue;
            const int q = lane + 2;
            // y: both face values of row j+1 (rows j-1 .. j+3 = R0 .. R4)
            float2 nLru, nRru, nLvp, nRvp;
            weno5_pair2(R0[0][q], R1[0][q], R2[0][q], R3[0][q], R4[0][q], eps, nLru, nRru);
            weno5_pair2(R0[1][q], R1[1][q], R2[1][q], R3[1][q], R4[1][q], eps, nLvp, nRvp);
            float2 FyA, FyB;
            face_flux2<1, RS>(A.C, Lru, Lvp, nRru, nRvp, FyA, FyB);
            Lru = nLru;
            Lvp = nLvp;
            if (j < y0) {
                FcA = FyA;
                FcB = FyB;
                continue;
            }
            // x: both face values at the lane's position of row j (R1)
            float2 xLru, xRru, xLvp, xRvp;
            {
                const float2* a = &R1[0][q - 2];
                const float2* b = &R1[1][q - 2];
                weno5_pair2(a[0], a[1], a[2], a[3], a[4], eps, xLru, xRru);
                weno5_pair2(b[0], b[1], b[2], b[3], b[4], eps, xLvp, xRvp);
            }
            float2 rru, rvp;   // the right state of the lane's right face: the next lane's low-face value
            rru.x = __shfl_down_sync(0xffffffffu, xRru.x, 1);
            rru.y = __shfl_down_sync(0xffffffffu, xRru.y, 1);
            rvp.x = __shfl_down_sync(0xffffffffu, xRvp.x, 1);
            rvp.y = __shfl_down_sync(0xffffffffu, xRvp.y, 1);
            float2 FxA, FxB;
            face_flux2<0, RS>(A.C, xLru, xLvp, rru, rvp, FxA, FxB);
            float2 FlA, FlB;   // the lane's left face: the previous lane's right face
            FlA.x = __shfl_up_sync(0xffffffffu, FxA.x, 1);
            FlA.y = __shfl_up_sync(0xffffffffu, FxA.y, 1);
            FlB.x = __shfl_up_sync(0xffffffffu, FxB.x, 1);
            FlB.y = __shfl_up_sync(0xffffffffu, FxB.y, 1);
            if (colActive) {
                const size_t c = (size_t)((long long)P.ngx + cx + rowStride * ((long long)j + P.ngy));
                const float invy = (float)A.inv[1][j + P.ngy];
                // FP32 divergence of the (mass, x momentum) and (y momentum, energy) pairs
                const float2 rA = fma2(f2(invy), sub2(FcA, FyA), mul2(f2(invx), sub2(FlA, FxA)));
                const float2 rB = fma2(f2(invy), sub2(FcB, FyB), mul2(f2(invx), sub2(FlB, FxB)));
                const double r[4] = {(double)rA.x, (double)rA.y, (double)rB.x, (double)rB.y};
                double nw[4];
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    double n = A.a1 * A.in[v][c] + a3dt * r[v];
                    if (useU0) n += A.a2 * A.u0[v][c];
                    nw[v] = n;
                }
#pragma unroll
                for (int v = 0; v < 4; ++v) A.out[v][c] = nw[v];
                if (A.last) {
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
                    if (A.dtNext) {
                        const double cs = single_sound_speed(P, nw[0], p);
                        double dtCell = A.dx[cx + P.ngx] / (fabs(u) + cs);
                        dtCell = smin(dtCell, A.dy[j + P.ngy] / (fabs(v) + cs));
                        dtMin = smin(dtMin, A.cfl * dtCell);
                    }
                }
            }
            FcA = FyA;
            FcB = FyB;
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

inline size_t march_mixed_smem() { return 4 * (5 * 2 * 36 * sizeof(float2) + 2 * 4 * 36 * sizeof(double)); }

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
