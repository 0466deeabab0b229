// sifv_common.cuh -- device helpers shared by the reference-ordered kernels
// (sifv_kernels.cuh) and the fused sweep kernels (sifv_sweep.cuh): index
// decoding, the ghost-cell source map, conservative -> primitive of one
// cell, per-cell face coefficients and block reductions.
#pragma once

#include "sifv_device.cuh"

namespace sifv {

__device__ __forceinline__ double bits2d(unsigned long long b) { return __longlong_as_double((long long)b); }
__device__ __forceinline__ unsigned long long d2bits(double d) { return (unsigned long long)__double_as_longlong(d); }

// Split a linear id t = a + n0 (b + n1 c) into (a, b, c); 32-bit unsigned
// division when t fits (every grid up to 2^32 cells), 64-bit otherwise.
__device__ __forceinline__ void split3(long long t, int n0, int n1, int& a, int& b, int& c) {
    if (t < 0x100000000LL) {
        const unsigned u = (unsigned)t, m0 = (unsigned)n0, m1 = (unsigned)n1;
        const unsigned r = u / m0;
        a = (int)(u - r * m0);
        const unsigned q = r / m1;
        b = (int)(r - q * m1);
        c = (int)q;
    } else {
        const long long r = t / n0;
        a = (int)(t - r * n0);
        const long long q = r / n1;
        b = (int)(r - q * n1);
        c = (int)q;
    }
}

// Decode a linear id over the extended grid into (i, j, k) with ghosts
// (i in [-ngx, nx+ngx), ...).  Returns false past the end.
__device__ __forceinline__ bool ext_coords(const Params& P, long long t, int& i, int& j, int& k) {
    long long tot = (long long)P.nxT * P.nyT * P.nzT;
    if (t >= tot) return false;
    int ii, jj, kk;
    split3(t, P.nxT, P.nyT, ii, jj, kk);
    i = ii - P.ngx;
    j = jj - P.ngy;
    k = kk - P.ngz;
    return true;
}

// Decode a linear id over the ghost cells only: the two z slabs (full x-y
// planes), then per interior z the two y slabs (full rows), then per
// interior (y, z) the two x slabs.  Returns false past the end.
__host__ __device__ __forceinline__ long long ghost_count(const Params& P) {
    return 2LL * P.ngz * P.nxT * P.nyT + (long long)P.nz * (2LL * P.ngy * P.nxT) +
           (long long)P.nz * P.ny * (2LL * P.ngx);
}
__device__ __forceinline__ bool ghost_coords(const Params& P, long long t, int& i, int& j, int& k) {
    const long long zs = 2LL * P.ngz * P.nxT * P.nyT;
    if (t < zs) {
        const long long plane = (long long)P.nxT * P.nyT;
        const int g = (int)(t / plane);
        const long long r = t - g * plane;
        j = (int)(r / P.nxT) - P.ngy;
        i = (int)(r % P.nxT) - P.ngx;
        k = (g < P.ngz) ? g - P.ngz : P.nz + (g - P.ngz);
        return true;
    }
    t -= zs;
    const long long ys = (long long)P.nz * (2LL * P.ngy * P.nxT);
    if (t < ys) {
        const long long per = 2LL * P.ngy * P.nxT;
        k = (int)(t / per);
        const long long r = t - k * per;
        const int g = (int)(r / P.nxT);
        i = (int)(r % P.nxT) - P.ngx;
        j = (g < P.ngy) ? g - P.ngy : P.ny + (g - P.ngy);
        return true;
    }
    t -= ys;
    const long long per = 2LL * P.ngx;
    if (t >= (long long)P.nz * P.ny * per) return false;
    const long long line = t / per;
    const int g = (int)(t - line * per);
    j = (int)(line % P.ny);
    k = (int)(line / P.ny);
    i = (g < P.ngx) ? g - P.ngx : P.nx + (g - P.ngx);
    return true;
}

__device__ __forceinline__ bool int_coords(const Params& P, long long t, int& i, int& j, int& k) {
    long long tot = (long long)P.nx * P.ny * P.nz;
    if (t >= tot) return false;
    split3(t, P.nx, P.ny, i, j, k);
    return true;
}

// ---------------------------------------------------------------------------
// Conservative -> primitive of one cell.
// SolutionState::convertConservativeToPrimitiveVariables with
// IdealGasEOS / StiffenedGasEOS::toPrimitive (src/SolutionState.cpp:187-205,
// src/IdealGasEOS.cpp:46-64, src/StiffenedGasEOS.cpp:47-64), or
// MixtureEOS::convertConservativeToPrimitive (src/MixtureEOS.cpp:99-143).
// ---------------------------------------------------------------------------
template <int NPH>
__device__ __forceinline__ void cons_to_prim_cell(const Params& P, const Fields& F, size_t s, double& rhoOut,
                                                  double u[3], double& p) {
    const int dim = P.dim;
    if (NPH == 0) {
        double U[3] = {F.rhoU[s], (dim >= 2) ? F.rhoV[s] : 0.0, (dim >= 3) ? F.rhoW[s] : 0.0};
        double rho = smax(F.rho[s], 1e-14);
        u[0] = u[1] = u[2] = 0.0;
        DIMLOOP(d) u[d] = U[d] / rho;
        double ke = 0.0;
        DIMLOOP(d) ke += u[d] * u[d];
        ke *= 0.5 * rho;
        double e = F.rhoE[s] - ke;
        p = P.eosStiffened ? (P.gamma - 1.0) * e - P.gamma * P.pInf : smax((P.gamma - 1.0) * e, 1e-14);
        rhoOut = F.rho[s];
    } else {
        double rho = 0.0;
#pragma unroll
        for (int ph = 0; ph < NPH; ++ph)
            if (ph < P.nPh) rho += F.alphaRho[ph][s];
        double rs = smax(rho, 1e-14);
        u[0] = F.rhoU[s] / rs;
        u[1] = (dim >= 2) ? F.rhoV[s] / rs : 0.0;
        u[2] = (dim >= 3) ? F.rhoW[s] / rs : 0.0;
        double ke = 0.5 * rs * u[0] * u[0];
        if (dim >= 2) ke += 0.5 * rs * u[1] * u[1];
        if (dim >= 3) ke += 0.5 * rs * u[2] * u[2];
        double a[NPH > 0 ? NPH : 1];
#pragma unroll
        for (int ph = 0; ph < NPH; ++ph) a[ph] = (ph < P.nPh) ? F.alpha[ph][s] : 0.0;
        p = mixture_pressure<NPH>(P, F.rhoE[s] - ke, a);
        rhoOut = rs;
    }
}

// Composed ghost source of cell (i,j,k) for the PRIM fill (onion peel
// x -> y -> z, src/RectilinearMesh.cpp:127-131) and the velocity signs.
__device__ __forceinline__ size_t prim_source(const Params& P, int i, int j, int k, double sg[3]) {
    double sn, sa;
    sg[0] = sg[1] = sg[2] = 1.0;
    int si = prim_src(i, P.nx, P.bc[0], P.bc[1], sn, sa);
    if (si != i) { sg[0] *= sn * sa; sg[1] *= sa; sg[2] *= sa; }
    int sj = j, sk = k;
    if (P.dim >= 2) {
        sj = prim_src(j, P.ny, P.bc[2], P.bc[3], sn, sa);
        if (sj != j) { sg[0] *= sa; sg[1] *= sn * sa; sg[2] *= sa; }
    }
    if (P.dim >= 3) {
        sk = prim_src(k, P.nz, P.bc[4], P.bc[5], sn, sa);
        if (sk != k) { sg[0] *= sa; sg[1] *= sa; sg[2] *= sn * sa; }
    }
    return cidx(P, si, sj, sk);
}

__device__ __forceinline__ bool is_interior(const Params& P, int i, int j, int k) {
    return i >= 0 && i < P.nx && j >= 0 && j < P.ny && k >= 0 && k < P.nz;
}

struct StageCoef {
    double c1, c2, c3, c4;
    int s;
    double accel[3];   // body force accelerations (host-evaluated), or 0
    int hasBodyForce;
};

struct CellFaces {
    long long lo[3];
    long long hiOff[3];
    double coeff[3];
};

__device__ __forceinline__ void cell_faces(const Params& P, const Fields& F, int i, int j, int k, CellFaces& cf) {
    double dxi = F.dx[i + P.ngx], dyj = F.dy[j + P.ngy], dzk = F.dz[k + P.ngz];
    double vol = dxi * dyj * dzk;
    cf.coeff[0] = (dyj * dzk) / vol;
    cf.coeff[1] = (dxi * dzk) / vol;
    cf.coeff[2] = (dxi * dyj) / vol;
    cf.lo[0] = (long long)i + (long long)(P.nx + 1) * ((long long)j + (long long)P.ny * k);
    cf.hiOff[0] = 1;
    cf.lo[1] = (long long)i + (long long)P.nx * ((long long)j + (long long)(P.ny + 1) * k);
    cf.hiOff[1] = P.nx;
    cf.lo[2] = (long long)i + (long long)P.nx * ((long long)j + (long long)P.ny * k);
    cf.hiOff[2] = (long long)P.nx * P.ny;
}

// Block-wide minimum of non-negative doubles, NaN ignored (std::min(dt, x)
// keeps dt when x is NaN), folded into *acc with an integer atomicMin on the
// bit pattern (order-preserving for non-negative doubles).
__device__ __forceinline__ void block_min_to(double v, unsigned long long* acc) {
    __shared__ double sm[32];
    // v may be NaN: replace by +inf so it cannot win
    if (!(v == v)) v = __longlong_as_double(0x7ff0000000000000LL);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = smin(v, __shfl_xor_sync(0xffffffffu, v, o));
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sm[w] = v;
    __syncthreads();
    if (w == 0) {
        int nw = (blockDim.x + 31) >> 5;
        v = (lane < nw) ? sm[lane] : __longlong_as_double(0x7ff0000000000000LL);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = smin(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) atomicMin(acc, d2bits(v));
    }
}

// Block-wide maximum of non-negative doubles, NaN ignored (std::max(m, x)
// keeps m when x is NaN), folded into *acc with atomicMax on the bits.
__device__ __forceinline__ void block_max_to(double v, unsigned long long* acc) {
    __shared__ double sm[32];
    if (!(v == v)) v = 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = smax(v, __shfl_xor_sync(0xffffffffu, v, o));
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sm[w] = v;
    __syncthreads();
    if (w == 0) {
        int nw = (blockDim.x + 31) >> 5;
        v = (lane < nw) ? sm[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = smax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) atomicMax(acc, d2bits(v));
    }
}

}  // namespace sifv
