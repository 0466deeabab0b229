// sifv_gs_march.cuh -- 2D Gauss-Seidel iterations as one persistent
// wavefront (GaussSeidelPressureSolver::solve, src/GaussSeidelPressureSolver.cpp:60-100,
// on a 2D mesh without halo exchange).  Included by sifv_capi.cu after
// sifv_kernels.cuh (gs_cell's arithmetic, div_markstein, igr_fast_*).
//
// The lexicographic sweep (x fastest) computes cell (x, j) from the new
// values at (x-1, j), (x, j-1) and the old ones at (x+1, j), (x, j+1), so
// the pair of cells (2h, 2h+1) of row j may run at wavefront time h + j.
// One warp owns 32 consecutive rows (a group); lane b takes row 32 g + b - 1
// and at step t updates the pair h = t - b, cell 2h then cell 2h+1, so the
// warp walks the wavefront along x: the new pair of the row below arrives by
// a shuffle from lane b - 1 (computed at step t - 1), the old pair of the row
// above is lane b + 1's next prefetched pair.  Lane 0 reads the row below
// from the group below (shared memory within a CTA, global memory across
// CTAs) and lane 31 the old row above from the group above; a group trails
// the one below by a little over 32 steps.  Sweep k + 1 of a group follows
// its sweep k, so all groups run consecutive sweeps in a pipeline and every
// iterate stays in its own buffer (nb buffers in rotation): the arithmetic
// of each cell, its operands and their order are those of the in-place
// sweep, bit for bit.
//
// Layout ("skewed"): row r = j + 1 (r = 0 and r = ny + 1 are the ghost
// rows), group g = r / 32, lane b = r % 32, pair h = x / 2 in slot s = h + b;
// the pair at double2 index ((g SW + s) 32 + b), SW = ceil(nx / 2) + 32, so
// the 32 lanes of a step read and write one contiguous 512-byte run.
// Records (per cell 4 x 16 bytes: x-, x+ coefficients; y-, y+; coeff,
// denom; 1 / denom, rhs) at double2 (((g SW + s) 8 + 4 v + ch) 32 + b) for
// cell v of the pair, streamed through a shared-memory ring with cp.async.
// The first ghost layer (periodic wrap or zero-gradient copy,
// fillScalarGhosts, src/RectilinearMesh.cpp:424-492) is never stored: the
// ghost columns come from the source cells read at the start of each sweep,
// and the lanes standing for the ghost rows load their source row's pairs
// (the group's own rows, or row ny - 1 / row 0 across a periodic face).
// Deeper ghost layers of the result are filled at the end.
//
// Orientation: the dependencies are the same along x and y (only the order
// of the two neighbour pairs in a cell's formula is fixed), so the warps may
// equally own 32 columns and walk along y (TR): the "march" axis m and the
// "row" axis n of the description above are then y and x.  A periodic march
// axis costs nothing (each row is walked whole before its next sweep); a
// periodic row axis makes each sweep wait for the far group's previous one.
//
// Segments: without a periodic face the rows may be cut into S segments of
// L pairs along the march axis, a warp per (segment, group).  A segment
// starts sweep k once the segment to its left finished sweep k (its first
// pair reads that segment's new last cell) and the one to its right did the
// first 32 steps of sweep k - 1 (its last pair reads that segment's old
// first cell), so the segments work on consecutive sweeps at once.
//
// Synchronization: each compute warp publishes its progress (steps done,
// counted across sweeps) in shared memory after each batch of D
// steps; warp kMarchWarps of the CTA (the helper) turns those into
// device-wide progress counters after a fence, so no compute warp waits on a
// device-wide fence.  A compute warp reads the counters of groups in other
// CTAs itself, one batch ahead of their use.  A sweep starts once every group finished the sweep
// that last used its output buffer, and no group starts a sweep after one
// that is complete and converged.  All CTAs are co-resident (cooperative
// launch), every wait is bounded (kMarchTimeoutNs) and a wait that gives up
// stops all groups and leaves an error code for the host.
// ---------------------------------------------------------------------------

namespace sifv {

#ifndef SIFV_MARCH_WARPS
#define SIFV_MARCH_WARPS 2
#endif
constexpr int kMarchWarps = SIFV_MARCH_WARPS;  // compute warps per CTA
// Prefetch distance and batch length D (steps): 8 (fewer waits per cell),
// or 4 when the row axis is periodic and the groups' lags add up to more
// than a sweep (each group trails the one below by about 32 + 2 D steps,
// and a periodic row axis makes the sweep period the sum of those lags).
// The record ring holds two batches.
#ifndef SIFV_MARCH_SHORT_D
#define SIFV_MARCH_SHORT_D 4
#endif
constexpr int kMarchShortD = SIFV_MARCH_SHORT_D;
constexpr int kMarchRE = 256;                  // lane-31 pairs kept for the warp above (power of 2)
constexpr int kMarchMaxBufs = 32;
constexpr int kMarchFin = 0x7fffffff;          // progress of a finished group
constexpr unsigned long long kMarchTimeoutNs = 2000000000ull;

struct GsMarch {
    // extents nx (march axis m) and ny (row axis n); x and y when !TR, y and x when TR
    const double2* rec;
    double2* q[kMarchMaxBufs];   // iterate n in q[n % nb]
    int* prog;                   // [S][G] device-wide progress per segment and group
    int* done;                   // [maxIter] groups through sweep k
    int* flags;                  // [0] stop, [1] error code (1: a wait timed out)
    const int* slowRecs;
    int nb, G, GA, SW, NS, NH, maxIter;
    int nx, ny;
    int xsLo, xsHi;              // source cells of the ghosts along the march axis
    int perLoY, perHiY;          // the ghost rows across the row axis wrap around
    double tol;
    const double* ghost0;        // IGR: the stored field, whose ghost cells sweep 0 reads
    const double* wRow;          // IGR: the metric weight along the row axis (ady2, or adx2 when TR), per row
    int wRowOff;                 // its ghost offset
    int S, L;                    // segments along the march axis and their length in pairs (S = 1: whole rows)
    int ctasPerSeg;              // CTAs of one segment (its row groups)
};

__host__ __device__ __forceinline__ size_t march_q(int SW, int g, int s, int b) {
    return ((size_t)g * SW + s) * 32 + b;
}
// record chunks (16 bytes) per cell: Gauss-Seidel 4, IGR 6
__host__ __device__ constexpr int march_chunks(int kind) { return kind ? 6 : 4; }
inline size_t march_smem(int D, int kind) {
    return ((size_t)kMarchWarps * 2 * D * 2 * march_chunks(kind) * 32 + (size_t)kMarchWarps * kMarchRE) *
           sizeof(double2);
}

__device__ __forceinline__ unsigned long long march_now() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Predicated 16-byte global load (L2, no L1 allocation) into dst, left
// unchanged when !pred: no select on the loaded value, so the load stays in
// flight until its value is used (a prefetch several steps ahead).
__device__ __forceinline__ void march_ld(double2& dst, const double2* p, bool pred) {
    asm volatile("{\n .reg .pred q;\n setp.ne.b32 q, %3, 0;\n @q ld.global.cg.v2.f64 {%0, %1}, [%2];\n}\n"
                 : "+d"(dst.x), "+d"(dst.y)
                 : "l"(p), "r"((int)pred));
}
// predicated stores (no branch around them)
__device__ __forceinline__ void march_st(double2* p, double2 v, bool pred) {
    asm volatile("{\n .reg .pred q;\n setp.ne.b32 q, %3, 0;\n @q st.global.v2.f64 [%0], {%1, %2};\n}\n" ::"l"(p),
                 "d"(v.x), "d"(v.y), "r"((int)pred));
}
__device__ __forceinline__ void march_sts(double2* p, double2 v, bool pred) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("{\n .reg .pred q;\n setp.ne.b32 q, %3, 0;\n @q st.shared.v2.f64 [%0], {%1, %2};\n}\n" ::"r"(a),
                 "d"(v.x), "d"(v.y), "r"((int)pred));
}
__device__ __forceinline__ double2 march_shfl_up(double2 v) {
    return make_double2(__shfl_up_sync(0xffffffffu, v.x, 1), __shfl_up_sync(0xffffffffu, v.y, 1));
}
__device__ __forceinline__ double2 march_shfl_down(double2 v) {
    return make_double2(__shfl_down_sync(0xffffffffu, v.x, 1), __shfl_down_sync(0xffffffffu, v.y, 1));
}

// gs_cell's update from record (c0, c1, c2, c3) and the four neighbours
// along the march axis (pL, pR) and the row axis (pD, pU); an inactive cell
// evaluates 1 / 1 (no operand of the slow path).
template <bool TR>
__device__ __forceinline__ double march_cell(bool act, bool fastRecs, double2 c0, double2 c1, double2 c2, double2 c3,
                                             double pL, double pR, double pD, double pU) {
    // gs_cell's order: od = cf0 p(x-) + cf1 p(x+), then the y pair
    const double xm = TR ? pD : pL, xp = TR ? pU : pR, ym = TR ? pL : pD, yp = TR ? pR : pU;
    double od = 0.0;
    od += c0.x * xm + c0.y * xp;
    od += c1.x * ym + c1.y * yp;
    const double num = act ? c3.y + c2.x * od : 1.0;
    const double dv = act ? c2.y : 1.0, rdv = act ? c3.x : 1.0;
    return (fastRecs && igr_fast_operand(num)) ? div_markstein(num, dv, rdv) : div_rn_plain(num, dv);
}

// The IGR update of one cell (igr_cell, src/IGR.cpp:110-156, 2D) from its
// record r (face densities and their reciprocals per face, the metric
// weights, rhs, diagonal and its reciprocal) and the four sigma neighbours:
// div_markstein's correctly rounded quotients when every operand and
// reciprocal is in range, plain divisions otherwise.  Inactive cells take
// the fast path on whatever they hold (their result is discarded).
__device__ __noinline__ double igr_cell_plain2(double sxm, double sxp, double sym, double syp, double rflx, double rfrx,
                                               double rfly, double rfry, double ax, double ay, double rhs,
                                               double diag) {
    double off = 0.0;
    off += ax * (sxm / rflx + sxp / rfrx);
    off += ay * (sym / rfly + syp / rfry);
    return (rhs + off) / diag;
}
// The record holds the march axis' metric weight; the row axis' one (wn) is
// constant along the row.
template <bool TR>
__device__ __forceinline__ double igr_march_cell(bool act, bool fastRecs, const double2* r, double wn, double pL,
                                                 double pR, double pD, double pU) {
    const double sxm = TR ? pD : pL, sxp = TR ? pU : pR, sym = TR ? pL : pD, syp = TR ? pR : pU;
    const double ax = TR ? wn : r[4].x, ay = TR ? r[4].x : wn;
    if (!act || (fastRecs && igr_fast_operand(sxm) && igr_fast_operand(sxp) && igr_fast_operand(sym) &&
                 igr_fast_operand(syp))) {
        double off = 0.0;
        off += ax * (div_markstein(sxm, r[0].x, r[0].y) + div_markstein(sxp, r[1].x, r[1].y));
        off += ay * (div_markstein(sym, r[2].x, r[2].y) + div_markstein(syp, r[3].x, r[3].y));
        const double num = r[4].y + off;
        return (!act || igr_fast_operand(num)) ? div_markstein(num, r[5].x, r[5].y) : div_rn_plain(num, r[5].x);
    }
    return igr_cell_plain2(sxm, sxp, sym, syp, r[0].x, r[1].x, r[2].x, r[3].x, ax, ay, r[4].y, r[5].x);
}

// IGR records and iterate 0 (interior pairs, and the stored first ghost
// layer in the ghost rows' slots, which sweep 0 reads).  Record of a cell:
// (rho_f, 1 / rho_f) of the x-, x+, y-, y+ faces with the sweep's
// expressions 0.5 (rho_i + rho_nb), (the march axis' metric weight, rhs),
// (diag, 1 / diag).
__global__ void k_march_igr_setup(Params P, Fields F, double2* __restrict__ rec, double2* __restrict__ q0, int SW,
                                  long long total, int* __restrict__ slowRecs, int tr) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= total) return;
    const int b = (int)(id & 31);
    const long long gs = id >> 5;
    const int s = (int)(gs % SW), g = (int)(gs / SW);
    const int h = s - b, n = 32 * g + b - 1;
    const int Nm = tr ? P.ny : P.nx, Nn = tr ? P.nx : P.ny;
    double v[2] = {0.0, 0.0};
    if (n >= -1 && n <= Nn && h >= 0 && 2 * h < Nm) {
        const size_t sy = (size_t)P.nxT;
        for (int e = 0; e < 2; ++e) {
            const int m = 2 * h + e;
            if (m >= Nm) break;
            const int i = tr ? n : m, j = tr ? m : n;
            const size_t c = cidx(P, i, j, 0);
            v[e] = F.sigma[c];
            if (n < 0 || n >= Nn) continue;   // a ghost row: its stored value only
            const double rho_i = F.rho[c];
            const double rflx = 0.5 * (rho_i + F.rho[c - 1]), rfrx = 0.5 * (rho_i + F.rho[c + 1]);
            const double rfly = 0.5 * (rho_i + F.rho[c - sy]), rfry = 0.5 * (rho_i + F.rho[c + sy]);
            const double rxl = 1.0 / rflx, rxr = 1.0 / rfrx, ryl = 1.0 / rfly, ryr = 1.0 / rfry;
            const double diag = F.igrDiag[c], rd = 1.0 / diag;
            double2* o = rec + ((size_t)gs * 12 + 6 * e) * 32 + b;
            o[0] = make_double2(rflx, rxl);
            o[32] = make_double2(rfrx, rxr);
            o[64] = make_double2(rfly, ryl);
            o[96] = make_double2(rfry, ryr);
            o[128] = make_double2(tr ? F.ady2[j + P.ngy] : F.adx2[i + P.ngx], F.igrRhs[c]);
            o[160] = make_double2(diag, rd);
            if (!(igr_fast_recip(rxl) && igr_fast_recip(rxr) && igr_fast_recip(ryl) && igr_fast_recip(ryr) &&
                  igr_fast_recip(rd)))
                atomicOr(slowRecs, 1);
        }
    }
    q0[id] = make_double2(v[0], v[1]);
}

// Records and iterate 0 (interior pairs; ghost cells are read from their sources).
__global__ void k_march_gs_setup(Params P, const double* __restrict__ coef, size_t nc, const double* __restrict__ rhs,
                                 const double* __restrict__ p0, double2* __restrict__ rec, double2* __restrict__ q0,
                                 int SW, long long total, int* __restrict__ slowRecs, int tr) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= total) return;
    const int b = (int)(id & 31);
    const long long gs = id >> 5;
    const int s = (int)(gs % SW), g = (int)(gs / SW);
    const int h = s - b, n = 32 * g + b - 1;
    const int Nm = tr ? P.ny : P.nx, Nn = tr ? P.nx : P.ny;
    double v[2] = {0.0, 0.0};
    if (n >= 0 && n < Nn && h >= 0 && 2 * h < Nm) {
        for (int e = 0; e < 2; ++e) {
            const int m = 2 * h + e;
            if (m >= Nm) break;
            const size_t c = tr ? cidx(P, n, m, 0) : cidx(P, m, n, 0);
            v[e] = p0[c];
            const double denom = coef[5 * nc + c];
            const double rd = 1.0 / denom;
            double2* o = rec + ((size_t)gs * 8 + 4 * e) * 32 + b;
            o[0] = make_double2(coef[c], coef[nc + c]);
            o[32] = make_double2(coef[2 * nc + c], coef[3 * nc + c]);
            o[64] = make_double2(coef[4 * nc + c], denom);
            o[96] = make_double2(rd, rhs[c]);
            if (!igr_fast_recip(rd)) atomicOr(slowRecs, 1);
        }
    }
    q0[id] = make_double2(v[0], v[1]);
}

// The result in the mesh layout: interior from iterate `fin`, every ghost
// cell from iterate fin - 1 (the fill before the last sweep).
__global__ void k_march_gs_out(Params P, const double2* __restrict__ qFin, const double2* __restrict__ qPrev,
                               double* __restrict__ out, int SW, int tr) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (long long)P.nxT * P.nyT) return;
    const int i = (int)(id % P.nxT) - P.ngx, j = (int)(id / P.nxT) - P.ngy;
    const bool in = i >= 0 && i < P.nx && j >= 0 && j < P.ny;
    const int xs = in ? i : scalar_src(i, P.nx, P.bc[0], P.bc[1]);
    const int ys = in ? j : scalar_src(j, P.ny, P.bc[2], P.bc[3]);
    const int m = tr ? ys : xs, r = (tr ? xs : ys) + 1;
    const double2 v = (in ? qFin : qPrev)[march_q(SW, r >> 5, (m >> 1) + (r & 31), r & 31)];
    out[cidx(P, i, j, 0)] = (m & 1) ? v.y : v.x;
}

// KIND 0: Gauss-Seidel pressure iterations (residual, convergence);
// KIND 1: IGR sweeps (a fixed count; sweep 0 reads the stored ghost cells).
template <int W, int D, bool TR, int KIND>
__global__ void __launch_bounds__(32 * (W + 1), 1) k_march_gs(Params P, GsMarch M, Ctl* ctl) {
    constexpr int R = 2 * D, RE = kMarchRE;
    constexpr int CH = march_chunks(KIND), PC = 2 * CH;   // record chunks per cell and per pair
    extern __shared__ __align__(16) unsigned char marchSmem[];
    double2* ringAll = reinterpret_cast<double2*>(marchSmem);   // [W][R][PC][32]
    double2* eRing = ringAll + (size_t)W * R * PC * 32;         // [W][RE]
    __shared__ volatile int sp[W];    // compute progress (this CTA)
    __shared__ volatile int pub[W];   // the same, once visible device-wide
    __shared__ volatile int stopS;
    const int warp = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31);
    // CTA -> segment `seg` of the march axis and its row groups g0 .. g0 + W - 1; a warp's progress counter
    // is prog[seg G + g]
    const int seg = (int)blockIdx.x / M.ctasPerSeg, g0 = ((int)blockIdx.x % M.ctasPerSeg) * W;
    const int pbase = seg * M.G;
    const int NH = M.NH;
    const int hs0 = seg * M.L, hs1 = min(NH, hs0 + M.L);   // this segment's pairs
    auto seg_steps = [&](int s) { return min(NH, (s + 1) * M.L) - s * M.L + 31; };
    const int NS = hs1 - hs0 + 31, SW = M.SW;              // steps per sweep of this segment
    const int nWarps = M.G * M.S;                           // warps that count a sweep done
    if (threadIdx.x < W) {
        sp[threadIdx.x] = (g0 + (int)threadIdx.x < M.G) ? 0 : kMarchFin;
        pub[threadIdx.x] = sp[threadIdx.x];
    }
    if (threadIdx.x == 0) stopS = 0;
    __syncthreads();
    const int topR = M.ny;   // r of row ny - 1 (source of the periodic low ghost row)

    if (warp == W) {   // helper
        if (lane != 0) return;
        int last[W];
#pragma unroll
        for (int w = 0; w < W; ++w) last[w] = -1;
        unsigned long long tLast = march_now();
        for (unsigned it = 0;; ++it) {
            int cur[W];
            bool fin = true, changed = false;
#pragma unroll
            for (int w = 0; w < W; ++w) {
                cur[w] = sp[w];
                fin = fin && cur[w] == kMarchFin;
                changed = changed || cur[w] != last[w];
            }
            if (changed) {
                __threadfence();   // the compute warps' stores before their progress, device-wide
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    if (cur[w] != last[w]) {
                        if (g0 + w < M.G) *(volatile int*)&M.prog[pbase + g0 + w] = cur[w];
                        pub[w] = cur[w];
                        last[w] = cur[w];
                    }
                }
                tLast = march_now();
            }
            if ((it & 63) == 0 && *(volatile int*)&M.flags[0]) stopS = 1;
            if (fin) break;
            if (march_now() - tLast > 2 * kMarchTimeoutNs) {   // compute warps stuck past their own limits
                atomicOr(&M.flags[1], 1);
                *(volatile int*)&M.flags[0] = 1;
                stopS = 1;
                break;
            }
        }
        return;
    }

    const int g = g0 + warp;
    if (g >= M.G) return;
    double2* ring = ringAll + (size_t)warp * R * PC * 32 + lane;   // slot q, chunk ch at ring[(PC q + ch) 32]
    double2* eMine = eRing + (size_t)warp * RE;
    const double2* eBelow = eRing + (size_t)(warp > 0 ? warp - 1 : 0) * RE;
    const int r = 32 * g + lane;
    const bool rowIn = r >= 1 && r <= M.ny;
    const double wn = (KIND == 1 && rowIn) ? M.wRow[r - 1 + M.wRowOff] : 0.0;   // IGR: row axis' metric weight
    const int nx = M.nx;
    const bool fastRecs = *M.slowRecs == 0;
    const int gT = (M.ny + 1) >> 5, bT = (M.ny + 1) & 31;   // the high ghost row r = ny + 1
    const bool hasAbove = g + 1 < M.G;                        // group above with interior rows
    const int topG = topR >> 5, topB = topR & 31;
    const bool lowGhostLane = (g == 0 && lane == 0);
    const bool topGhostLane = (g == gT && lane == bT && bT >= 1);
    // per-lane step windows: step t updates pair h = hs0 + t - lane
    const int nP = hs1 - hs0;
    // own pairs are loaded through step NS - 1, or NS before another segment (lane 31's last pair then
    // reads that segment's first pair)
    const int tPEnd = NS + (hs1 < NH ? 1 : 0);
    const int tAct0 = rowIn ? lane : NS, tAct1 = rowIn ? lane + nP : NS;
    const int hLastX = (nx - 1) >> 1;   // the pair holding x = nx - 1, and its step (last segment only)
    const int tLast = (hLastX >= hs0 && hLastX < hs1) ? lane + hLastX - hs0 : -1;
    const bool lastOdd = ((nx - 1) & 1) != 0;   // x = nx - 1 is the second cell of its pair
    // the edge pair of step t at eP[32 t] for t in [eLo, eHi): lane 0 the new pair of the row below
    // (group below in another CTA) or of row ny - 1 (periodic low ghost row), lane 31 the old pair of the
    // row above (or of its own row / row 0 when the row above is the high ghost row)
    int eKind = 0, eLo = 0, eHi = 0;
    if (lane == 0 && warp == 0 && g > 0) { eKind = 1; eHi = nP; }
    else if (lowGhostLane && M.perLoY) { eKind = 2; eHi = nP; }
    else if (lane == 31 && hasAbove) { eKind = 3; eLo = 31; eHi = nP + 31; }
    else if (lane == 31 && g + 1 == gT && bT == 0) { eKind = 4; eLo = 31; eHi = nP + 31; }
    const bool eBelowLane = lane == 0 && warp > 0;
    const bool eWriter = lane == 31 && warp < W - 1 && rowIn;
    // the lane's own pair loads: its row, or the source row of the ghost row it stands for, from step pLo
    int pLo = 0;
    if (topGhostLane) pLo = M.perHiY ? max(0, bT - 1) : 1;
    bool ok = true;
    int chk = 0;

    // device-wide progress of the groups in other CTAs this warp waits on -- the group below (lane 0's
    // edge), the group above (lane 31's edge) and the top row's group (periodic low ghost row) -- as last
    // read (extV) and as read one batch ahead of its use (extN); lane 0 only
    const bool inCta0 = g - 1 >= g0, inCta1 = g + 1 < g0 + W, inCta2 = topG >= g0 && topG < g0 + W;
    const int extG[3] = {(g > 0 && !inCta0) ? g - 1 : -1, (hasAbove && !inCta1) ? g + 1 : -1,
                         (g == 0 && M.perLoY && topG != 0 && !inCta2) ? topG : -1};
    int extV[3] = {0, 0, 0}, extN[3] = {0, 0, 0};
    auto ext_issue = [&]() {
#pragma unroll
        for (int q = 0; q < 3; ++q)
            if (extG[q] >= 0) extN[q] = *(volatile int*)&M.prog[pbase + extG[q]];
    };
    auto progress_of = [&](int hgrp) -> int {
        if (hgrp >= g0 && hgrp < g0 + W) return pub[hgrp - g0];
#pragma unroll
        for (int q = 0; q < 3; ++q)
            if (extG[q] == hgrp) return extV[q];
        return -1;   // not reached: every external group a wait names is in extG (a wait on it would time out)
    };

    for (int k = 0; k < M.maxIter && ok; ++k) {
        const int base = k * NS, prevBase = base - NS;
        // ---- sweep start: buffer reuse, the high ghost row across a periodic face, then stop and
        // convergence of the complete sweeps (sweep k + 1 - nb among them, so a started sweep never
        // writes the buffer of a converged iterate or of its predecessor)
        if (lane == 0) {
            bool go = !stopS && !*(volatile int*)&M.flags[0];
            const int kw = k + 1 - M.nb;
            const unsigned long long tw = march_now();
            while (go) {
                const bool a = kw < 0 || *(volatile int*)&M.done[kw] >= nWarps;
                const bool b = !(M.perHiY && g == M.G - 1 && g != 0) || *(volatile int*)&M.prog[pbase] >= base;
                // the segment to the left through sweep k (this row's first pair reads its new last cell),
                // the one to the right through the first pairs of sweep k - 1 (every lane's first pair is
                // done after 32 steps; this row's last pair reads its old first cell)
                const bool sl = seg == 0 || *(volatile int*)&M.prog[pbase - M.G + g] >= (k + 1) * seg_steps(seg - 1);
                const bool sr = seg == M.S - 1 || k == 0 ||
                                *(volatile int*)&M.prog[pbase + M.G + g] >= (k - 1) * seg_steps(seg + 1) + 32;
                if (a && b && sl && sr) break;
                if (stopS || *(volatile int*)&M.flags[0]) go = false;
                else if (march_now() - tw > kMarchTimeoutNs) {
                    atomicOr(&M.flags[1], 1);
                    *(volatile int*)&M.flags[0] = 1;
                    go = false;
                }
            }
            if (go) __threadfence();
            while (KIND == 0 && go && chk < k) {
                if (*(volatile int*)&M.done[chk] < nWarps) break;
                __threadfence();
                if (bits2d(*(volatile unsigned long long*)&ctl->res[chk]) < M.tol) {
                    *(volatile int*)&M.flags[0] = 1;
                    go = false;
                }
                ++chk;
            }
            if (go && *(volatile int*)&M.flags[0]) go = false;
            ok = go;
        }
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        if (!ok) break;
        const double2* __restrict__ Qk = M.q[k % M.nb];
        double2* __restrict__ Qn = M.q[(k + 1) % M.nb];
        const double2* rowK = Qk + march_q(SW, g, 0, lane);   // slot s at rowK[32 s]
        const double2* rowKs = rowK + 32 * hs0;                // step t's slot at rowKs[32 t]
        double2* outP = Qn + march_q(SW, g, hs0, lane);        // step t's pair at outP[32 t]
        // step t, chunk ch at recP[(PC t + ch) 32]
        const double2* recP = M.rec + march_q(SW, g, hs0, 0) * PC + lane;
        // IGR sweep 0 reads the ghost cells as stored (the ghost rows' own slots, the stored ghost columns);
        // every other sweep reads them from their source cells in iterate k
        const bool stored0 = KIND == 1 && k == 0;
        // own pair of step t at pP[32 t]
        const double2* pP = rowKs;
        int pLoK = pLo;
        if (!stored0) {
            if (lowGhostLane && !M.perLoY) pP = Qk + march_q(SW, 0, hs0 + 1, 1);   // row 0's pair h = hs0 + t
            if (topGhostLane)   // row 0's / row ny - 1's pair h = hs0 + t + 1 - bT
                pP = M.perHiY ? Qk + march_q(SW, 0, hs0 + 1, 1) - 32 * (ptrdiff_t)bT
                              : Qk + march_q(SW, gT, hs0, bT - 1) - 32;
        } else {
            pLoK = 0;
        }
        const double2* eP = (eKind == 1)   ? Qn + march_q(SW, g - 1, hs0 + 31, 31)
                            : (eKind == 2) ? Qk + march_q(SW, topG, hs0 + topB, topB)
                            : (eKind == 3) ? Qk + march_q(SW, g + 1, hs0, 0) - 32 * 31
                            : (eKind == 4) ? (stored0 ? Qk + march_q(SW, g + 1, hs0, 0) - 32 * 31
                                              : M.perHiY ? Qk + march_q(SW, 0, hs0 + 1, 1) - 32 * 31 : rowKs)
                                           : rowKs;
        const bool lowFromEdge = M.perLoY && !stored0;   // the low ghost pair from row ny - 1
        // the ghost columns of this row in iterate k: sources xsLo, xsHi; a segment after the first starts
        // from the new value of the left segment's last cell instead
        double gL, gR;
        if (hs0 > 0) {
            gL = __ldcg(Qn + march_q(SW, g, hs0 - 1 + lane, lane)).y;
            gR = 0.0;   // x = nx - 1 lies in the last segment only
            if (tLast >= 0) {
                const double2 gRp = __ldcg(rowK + 32 * ((M.xsHi >> 1) + lane));
                gR = (M.xsHi & 1) ? gRp.y : gRp.x;
            }
            if (stored0) gR = M.ghost0[TR ? cidx(P, rowIn ? r - 1 : 0, M.nx, 0) : cidx(P, M.nx, rowIn ? r - 1 : 0, 0)];
        } else if (stored0) {
            const int n = r - 1, nn = rowIn ? n : 0, Nm = M.nx;
            gL = M.ghost0[TR ? cidx(P, nn, -1, 0) : cidx(P, -1, nn, 0)];
            gR = M.ghost0[TR ? cidx(P, nn, Nm, 0) : cidx(P, Nm, nn, 0)];
        } else {
            const double2 gLp = __ldcg(rowK + 32 * ((M.xsLo >> 1) + lane));
            const double2 gRp = __ldcg(rowK + 32 * ((M.xsHi >> 1) + lane));
            gL = (M.xsLo & 1) ? gLp.y : gLp.x;
            gR = (M.xsHi & 1) ? gRp.y : gRp.x;
        }
        const int eOff = base & (RE - 1);

        // lane 0 waits before using steps up to tu and prefetching edges up to tp
        auto batch_wait = [&](int tu, int tp) -> bool {
            bool good = true;
            if (lane == 0) {
#pragma unroll
                for (int q = 0; q < 3; ++q) extV[q] = extN[q];   // read one batch ago
                const int n0 = (warp > 0) ? base + min(tu + 32, NS) : -1;
                const int n1 = (warp == 0 && g > 0) ? base + min(tp + 32, NS) : -1;
                const int n2 = (g == 0 && lowFromEdge && topG != 0) ? prevBase + min(tp + topB + 1, NS) : -1;
                const int n3 = (hasAbove && tp - 30 > 0) ? prevBase + min(tp - 30, NS) : -1;
                const int n4 = (warp < W - 1 && hasAbove) ? base + tu - 30 - RE : -1;
                auto met = [&]() {
                    return (n0 < 0 || sp[warp - 1] >= n0) && (n1 < 0 || progress_of(g - 1) >= n1) &&
                           (n2 < 0 || progress_of(topG) >= n2) && (n3 < 0 || progress_of(g + 1) >= n3) &&
                           (n4 < 0 || sp[warp + 1] >= n4);
                };
                if (!met()) {
                    const unsigned long long tw = march_now();
                    for (;;) {
                        ext_issue();
#pragma unroll
                        for (int q = 0; q < 3; ++q) extV[q] = extN[q];
                        if (met()) break;
                        if (stopS) { good = false; break; }
                        if (march_now() - tw > kMarchTimeoutNs) {
                            atomicOr(&M.flags[1], 1);
                            *(volatile int*)&M.flags[0] = 1;
                            stopS = 1;
                            good = false;
                            break;
                        }
                    }
                }
                ext_issue();   // for the next batch
            }
            const bool res = __shfl_sync(0xffffffffu, good ? 1 : 0, 0) != 0;
            asm volatile("" ::: "memory");   // no load of the batch moves above the wait
            return res;
        };
        // the records of the batch of steps t0 .. t0 + D - 1 into ring slots (t0 mod 2 D) .. + D - 1, one group
        auto issue_records = [&](int t0) {
            double2* dst = ring + (size_t)(t0 & (R - 1)) * PC * 32;
            const double2* src = recP + (size_t)t0 * PC * 32;
#pragma unroll
            for (int u = 0; u < D; ++u)
                if (t0 + u < NS) {
#pragma unroll
                    for (int ch = 0; ch < PC; ++ch) cp_async16(dst + (PC * u + ch) * 32, src + (PC * u + ch) * 32);
                }
            cp_async_commit();
        };

        // ---- prime
        if (!batch_wait(-1, D - 1)) { ok = false; break; }
        issue_records(0);
        double2 pr[D], er[D];
#pragma unroll
        for (int u = 0; u < D; ++u) {
            pr[u] = make_double2(0.0, 0.0);
            er[u] = make_double2(0.0, 0.0);
            march_ld(pr[u], pP + 32 * u, u >= pLoK);
            march_ld(er[u], eP + 32 * u, (unsigned)(u - eLo) < (unsigned)(eHi - eLo));
        }
        double2 newPair = make_double2(0.0, 0.0);
        double maxRes = 0.0;
        for (int t0 = 0; t0 < NS; t0 += D) {
            if (!batch_wait(t0 + D - 1, t0 + 2 * D - 1)) { ok = false; break; }
            issue_records(t0 + D);        // the next batch (slots of the batch before this one)
            cp_async_wait_group<1>();     // this batch's records landed
            const double2* rb = ring + (size_t)(t0 & (R - 1)) * PC * 32;
            const double2* pPb = pP + 32 * (size_t)(t0 + D);
            const double2* ePb = eP + 32 * (size_t)(t0 + D);
            double2* outB = outP + 32 * (size_t)t0;
#pragma unroll
            for (int u = 0; u < D; ++u) {
                const int t = t0 + u;
                if (t < NS) {
                    const double2 Pt = pr[u];                 // old pair h (or the ghost row's source pair)
                    const double2 Pn = pr[(u + 1) % D];       // old pair h + 1
                    const double2 eg = er[u];
                    const int tn = t + D;
                    march_ld(pr[u], pPb + 32 * u, tn < tPEnd && tn >= pLoK);
                    march_ld(er[u], ePb + 32 * u, tn < NS && (unsigned)(tn - eLo) < (unsigned)(eHi - eLo));
                    const double2 up = march_shfl_up(newPair);
                    const double2 down = march_shfl_down(Pn);
                    const double2 eb = eBelow[(eOff + t) & (RE - 1)];
                    const double2 pD = (lane == 0) ? (eBelowLane ? eb : eg) : up;
                    const double2 pU = (lane == 31) ? eg : down;
                    double2 ra[CH], rc[CH];   // records of the pair's two cells
#pragma unroll
                    for (int ch = 0; ch < CH; ++ch) {
                        ra[ch] = rb[(PC * u + ch) * 32];
                        rc[ch] = rb[(PC * u + CH + ch) * 32];
                    }
                    const bool act0 = t >= tAct0 && t < tAct1;
                    const bool act1 = act0 && !(t == tLast && !lastOdd);   // the pair's second cell exists
                    // cell 2h: left is the previous pair's second cell (ghost at h = 0), right the pair's second
                    // cell (ghost past the last cell)
                    const double pL0 = (t == lane) ? gL : newPair.y;
                    const double pR0 = (t == tLast && !lastOdd) ? gR : Pt.y;
                    const double pn0 = KIND == 0 ? march_cell<TR>(act0, fastRecs, ra[0], ra[1], ra[2], ra[3], pL0, pR0,
                                                                  pD.x, pU.x)
                                                 : igr_march_cell<TR>(act0, fastRecs, ra, wn, pL0, pR0, pD.x, pU.x);
                    // cell 2h + 1: left is cell 2h's new value, right the next pair's first cell
                    const double pR1 = (t == tLast) ? gR : Pn.x;
                    const double pn1 = KIND == 0 ? march_cell<TR>(act1, fastRecs, rc[0], rc[1], rc[2], rc[3], pn0, pR1,
                                                                  pD.y, pU.y)
                                                 : igr_march_cell<TR>(act1, fastRecs, rc, wn, pn0, pR1, pD.y, pU.y);
                    const double2 pn = make_double2(pn0, pn1);
                    if (KIND == 0) {
                        maxRes = act0 ? smax(maxRes, fabs(pn0 - Pt.x)) : maxRes;
                        maxRes = act1 ? smax(maxRes, fabs(pn1 - Pt.y)) : maxRes;
                    }
                    march_st(outB + 32 * u, pn, act0);
                    march_sts(eMine + ((eOff + t - 31) & (RE - 1)), pn, act0 && eWriter);
                    // the low ghost lane hands lane 1 the ghost pair h = t
                    newPair = act0 ? pn : (lowGhostLane ? (lowFromEdge ? eg : Pt) : newPair);
                }
            }
            asm volatile("" ::: "memory");
            __syncwarp();
            if (lane == 0) {
                __threadfence_block();
                sp[warp] = base + min(t0 + D, NS);
            }
        }
        cp_async_wait_group<0>();
        if (!ok) break;
        // ---- residual of the sweep, then the group counts as through sweep k
        double v = maxRes;
        if (!(v == v)) v = 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = smax(v, __shfl_xor_sync(0xffffffffu, v, o));
        __syncwarp();
        if (lane == 0) {
            if (KIND == 0) atomicMax(&ctl->res[k], d2bits(v));
            __threadfence();
            atomicAdd(&M.done[k], 1);
        }
    }
    cp_async_wait_group<0>();
    __syncwarp();
    if (lane == 0) {
        __threadfence_block();
        sp[warp] = kMarchFin;
    }
}

}  // namespace sifv
