// sifv_mg.cuh -- conjugate gradients preconditioned by one geometric
// multigrid V-cycle for the semi-implicit pressure system, the solver the
// reference offers through Hypre (HyprePressureSolver: PCG with one PFMG
// V-cycle of weighted-Jacobi relaxation as preconditioner, two-norm
// relative-residual stopping, src/HyprePressureSolver.cpp:124-139, 360-381).
//
// System (HyprePressureSolver::assembleSystem, src/HyprePressureSolver.cpp:154-279):
//   (1 + c_i sum_f k_f) p_i - c_i sum_f k_f p_nb(f) = rhs_i,
//   c_i = rhoc2_i dt^2,  k_f = 1 / (max(rho_f, 1e-14) d_f w_i),
// with k_f = 0 on physical (non-periodic) boundary faces.  Row i multiplied
// by m_i = vol_i / c_i gives a symmetric positive definite form
//   (m_i + sum_f T_f) p_i - sum_f T_f p_nb = m_i rhs_i,
//   T_f = A_f / (max(rho_f, 1e-14) d_f)  (one value per face),
// on which CG runs; convergence is tested on the unscaled residual
// (r_i / m_i), as Hypre tests its own system.
//
// Level layout: compact x-fastest arrays without ghosts.  tx[c] is T of the
// low-x face of cell c (the face to c - 1, wrapped on periodic axes, 0 on a
// physical boundary); the high-x face of c is tx of c + 1 (wrapped: for a
// physical boundary that is tx of cell 0, which is 0).  Coarse levels halve
// every axis longer than 1 (ceil), aggregate 2^dim cells, and take the
// Galerkin operator of piecewise-constant transfer: summed masses, summed
// face T across each coarse face.
#pragma once

#include "sifv_common.cuh"

namespace sifv {

struct MgLevel {
    int nx, ny, nz;
    long long n;
    double *m, *tx, *ty, *tz, *diag;
    double *x, *b, *r, *t;
};

__device__ __forceinline__ void mg_split(const MgLevel& L, long long c, int& i, int& j, int& k) {
    i = (int)(c % L.nx);
    long long q = c / L.nx;
    j = (int)(q % L.ny);
    k = (int)(q / L.ny);
}

// Fine level from the context's state: masses, face T, the scaled right-hand
// side b = m rhs, the initial guess x = p (interior).  dt from the control block.
__global__ void __launch_bounds__(256) k_mg_fine(Params P, Fields F, const double* __restrict__ rho,
                                                 const double* __restrict__ rhoc2, const double* __restrict__ rhs,
                                                 const double* __restrict__ p0, const Ctl* __restrict__ ctl, MgLevel L,
                                                 double* __restrict__ wInv) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= L.n) return;
    int i, j, k;
    mg_split(L, t, i, j, k);
    const int dim = P.dim;
    const size_t c = cidx(P, i, j, k);
    const double dt = ctl->dt;
    const double dxi = F.dx[i + P.ngx], dyj = F.dy[j + P.ngy], dzk = F.dz[k + P.ngz];
    const double vol = dxi * dyj * dzk;
    const double coeff = rhoc2[c] * (dt * dt);
    const double m = vol / coeff;
    L.m[t] = m;
    wInv[t] = 1.0 / m;
    L.b[t] = m * rhs[c];
    L.x[t] = p0[c];
    {   // low-x face: between i-1 and i
        const bool phys = (i == 0) && P.bc[0] != SIFV_BC_PERIODIC;
        const double rf = 0.5 * (rho[c] + rho[cidx(P, i - 1, j, k)]);
        const double d = 0.5 * (F.dx[i - 1 + P.ngx] + dxi);
        L.tx[t] = phys ? 0.0 : (dyj * dzk) / (smax(rf, 1e-14) * d);
    }
    if (dim >= 2) {
        const bool phys = (j == 0) && P.bc[2] != SIFV_BC_PERIODIC;
        const double rf = 0.5 * (rho[c] + rho[cidx(P, i, j - 1, k)]);
        const double d = 0.5 * (F.dy[j - 1 + P.ngy] + dyj);
        L.ty[t] = phys ? 0.0 : (dxi * dzk) / (smax(rf, 1e-14) * d);
    }
    if (dim >= 3) {
        const bool phys = (k == 0) && P.bc[4] != SIFV_BC_PERIODIC;
        const double rf = 0.5 * (rho[c] + rho[cidx(P, i, j, k - 1)]);
        const double d = 0.5 * (F.dz[k - 1 + P.ngz] + dzk);
        L.tz[t] = phys ? 0.0 : (dxi * dyj) / (smax(rf, 1e-14) * d);
    }
}

// Galerkin coarsening of piecewise-constant aggregates.
__global__ void __launch_bounds__(256) k_mg_coarsen(MgLevel Fn, MgLevel Cs, int dim) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= Cs.n) return;
    int I, J, K;
    mg_split(Cs, t, I, J, K);
    const int fx = (Fn.nx > 1) ? 2 : 1, fy = (Fn.ny > 1) ? 2 : 1, fz = (Fn.nz > 1) ? 2 : 1;
    double m = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
    for (int c = 0; c < fz; ++c)
        for (int b = 0; b < fy; ++b)
            for (int a = 0; a < fx; ++a) {
                const int i = I * fx + a, j = J * fy + b, k = K * fz + c;
                if (i >= Fn.nx || j >= Fn.ny || k >= Fn.nz) continue;
                const long long f = i + (long long)Fn.nx * (j + (long long)Fn.ny * k);
                m += Fn.m[f];
                if (a == 0) sx += Fn.tx[f];
                if (dim >= 2 && b == 0) sy += Fn.ty[f];
                if (dim >= 3 && c == 0) sz += Fn.tz[f];
            }
    Cs.m[t] = m;
    Cs.tx[t] = sx;
    if (dim >= 2) Cs.ty[t] = sy;
    if (dim >= 3) Cs.tz[t] = sz;
}

struct MgNb {
    long long xm, xp, ym, yp, zm, zp;
    double txl, txh, tyl, tyh, tzl, tzh;
};

__device__ __forceinline__ void mg_nb(const MgLevel& L, int dim, long long c, MgNb& q) {
    int i, j, k;
    mg_split(L, c, i, j, k);
    const long long sy = L.nx, sz = (long long)L.nx * L.ny;
    q.xm = c + ((i == 0) ? (L.nx - 1) : -1);
    q.xp = c + ((i == L.nx - 1) ? -(L.nx - 1) : 1);
    q.txl = L.tx[c];
    q.txh = L.tx[q.xp];
    q.ym = q.yp = q.zm = q.zp = c;
    q.tyl = q.tyh = q.tzl = q.tzh = 0.0;
    if (dim >= 2) {
        q.ym = c + ((j == 0) ? (L.ny - 1) * sy : -sy);
        q.yp = c + ((j == L.ny - 1) ? -(L.ny - 1) * sy : sy);
        q.tyl = L.ty[c];
        q.tyh = L.ty[q.yp];
    }
    if (dim >= 3) {
        q.zm = c + ((k == 0) ? (L.nz - 1) * sz : -sz);
        q.zp = c + ((k == L.nz - 1) ? -(L.nz - 1) * sz : sz);
        q.tzl = L.tz[c];
        q.tzh = L.tz[q.zp];
    }
}

__global__ void __launch_bounds__(256) k_mg_diag(MgLevel L, int dim) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= L.n) return;
    MgNb q;
    mg_nb(L, dim, t, q);
    L.diag[t] = L.m[t] + q.txl + q.txh + q.tyl + q.tyh + q.tzl + q.tzh;
}

__device__ __forceinline__ double mg_apply(const MgLevel& L, int dim, long long c, const double* __restrict__ x) {
    MgNb q;
    mg_nb(L, dim, c, q);
    double off = q.txl * x[q.xm] + q.txh * x[q.xp];
    if (dim >= 2) off += q.tyl * x[q.ym] + q.tyh * x[q.yp];
    if (dim >= 3) off += q.tzl * x[q.zm] + q.tzh * x[q.zp];
    return L.diag[c] * x[c] - off;
}

// Block partial sums for the deterministic two-pass reductions.
__device__ __forceinline__ void block_sum_to(double v, double* out) {
    __shared__ double sm[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sm[w] = v;
    __syncthreads();
    if (w == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        v = (lane < nw) ? sm[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) *out = v;
    }
}

// y = M x; partial[block] = sum p . y  (p may equal x)
__global__ void __launch_bounds__(256) k_mg_matvec_dot(MgLevel L, int dim, const double* __restrict__ x,
                                                       double* __restrict__ y, double* __restrict__ partial) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (t < L.n) {
        const double a = mg_apply(L, dim, t, x);
        y[t] = a;
        v = x[t] * a;
    }
    block_sum_to(v, partial + blockIdx.x);
}

// r = b - M x; partial[block] = sum (r / m)^2 (unscaled residual)
__global__ void __launch_bounds__(256) k_mg_residual0(MgLevel L, int dim, const double* __restrict__ wInv,
                                                      double* __restrict__ r, double* __restrict__ partial) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (t < L.n) {
        const double rr = L.b[t] - mg_apply(L, dim, t, L.x);
        r[t] = rr;
        const double u = rr * wInv[t];
        v = u * u;
    }
    block_sum_to(v, partial + blockIdx.x);
}

// partial[block] = sum (b / m)^2 (the unscaled right-hand side)
__global__ void __launch_bounds__(256) k_mg_bnorm(long long n, const double* __restrict__ b,
                                                  const double* __restrict__ wInv, double* __restrict__ partial) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (t < n) {
        const double u = b[t] * wInv[t];
        v = u * u;
    }
    block_sum_to(v, partial + blockIdx.x);
}

// partial[block] = sum a . b
__global__ void __launch_bounds__(256) k_mg_dot(long long n, const double* __restrict__ a,
                                                const double* __restrict__ b, double* __restrict__ partial) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    block_sum_to(t < n ? a[t] * b[t] : 0.0, partial + blockIdx.x);
}

// out[slot] = sum of partial[0 .. nb) (one block, fixed order)
__global__ void __launch_bounds__(1024) k_mg_sum(const double* __restrict__ partial, int nb, double* __restrict__ out,
                                                 int slot) {
    double v = 0.0;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) v += partial[q];
    __shared__ double tmp[1024];
    tmp[threadIdx.x] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) tmp[threadIdx.x] += tmp[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[slot] = tmp[0];
}

// Scalars of one CG iteration, on the device:
//   s[0] = r.z (current), s[1] = p.q, s[2] = |r/m|^2, s[3] = r.z (new)
// x += alpha p; r -= alpha q; partial = sum (r/m)^2, alpha = s[0] / s[1]
__global__ void __launch_bounds__(256) k_cg_update(long long n, const double* __restrict__ s, double* __restrict__ x,
                                                   double* __restrict__ r, const double* __restrict__ p,
                                                   const double* __restrict__ q, const double* __restrict__ wInv,
                                                   double* __restrict__ partial) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const double alpha = s[0] / s[1];
    double v = 0.0;
    if (t < n) {
        x[t] += alpha * p[t];
        const double rr = r[t] - alpha * q[t];
        r[t] = rr;
        const double u = rr * wInv[t];
        v = u * u;
    }
    block_sum_to(v, partial + blockIdx.x);
}

// p = z + beta p, beta = s[3] / s[0] (then k_cg_shift: s[0] = s[3])
__global__ void __launch_bounds__(256) k_cg_direction(long long n, const double* __restrict__ s,
                                                      const double* __restrict__ z, double* __restrict__ p, int first) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    p[t] = first ? z[t] : z[t] + (s[3] / s[0]) * p[t];
}

__global__ void k_cg_shift(double* s) { s[0] = s[3]; }

// Weighted Jacobi from x = 0: x = omega b / diag.
__global__ void __launch_bounds__(256) k_mg_smooth0(MgLevel L, double omega) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= L.n) return;
    L.x[t] = omega * L.b[t] / L.diag[t];
}

// Weighted Jacobi: out = x + omega (b - M x) / diag.
__global__ void __launch_bounds__(256) k_mg_smooth(MgLevel L, int dim, const double* __restrict__ x,
                                                   double* __restrict__ out, double omega) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= L.n) return;
    out[t] = x[t] + omega * (L.b[t] - mg_apply(L, dim, t, x)) / L.diag[t];
}

// Residual r = b - M x of a level, then summed into the coarse right-hand side.
__global__ void __launch_bounds__(256) k_mg_residual(MgLevel L, int dim) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= L.n) return;
    L.r[t] = L.b[t] - mg_apply(L, dim, t, L.x);
}

__global__ void __launch_bounds__(256) k_mg_restrict(MgLevel Fn, MgLevel Cs) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= Cs.n) return;
    int I, J, K;
    mg_split(Cs, t, I, J, K);
    const int fx = (Fn.nx > 1) ? 2 : 1, fy = (Fn.ny > 1) ? 2 : 1, fz = (Fn.nz > 1) ? 2 : 1;
    double s = 0.0;
    for (int c = 0; c < fz; ++c)
        for (int b = 0; b < fy; ++b)
            for (int a = 0; a < fx; ++a) {
                const int i = I * fx + a, j = J * fy + b, k = K * fz + c;
                if (i < Fn.nx && j < Fn.ny && k < Fn.nz) s += Fn.r[i + (long long)Fn.nx * (j + (long long)Fn.ny * k)];
            }
    Cs.b[t] = s;
}

__global__ void __launch_bounds__(256) k_mg_prolong(MgLevel Fn, MgLevel Cs) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= Fn.n) return;
    int i, j, k;
    mg_split(Fn, t, i, j, k);
    const int fx = (Fn.nx > 1) ? 2 : 1, fy = (Fn.ny > 1) ? 2 : 1, fz = (Fn.nz > 1) ? 2 : 1;
    Fn.x[t] += Cs.x[i / fx + (long long)Cs.nx * (j / fy + (long long)Cs.ny * (k / fz))];
}

// Coarsest level: weighted-Jacobi sweeps in one block (the level is small).
__global__ void __launch_bounds__(1024) k_mg_coarsest(MgLevel L, int dim, double omega, int sweeps) {
    for (long long t = threadIdx.x; t < L.n; t += blockDim.x) L.x[t] = omega * L.b[t] / L.diag[t];
    __syncthreads();
    for (int s = 0; s < sweeps; ++s) {
        for (long long t = threadIdx.x; t < L.n; t += blockDim.x)
            L.t[t] = L.x[t] + omega * (L.b[t] - mg_apply(L, dim, t, L.x)) / L.diag[t];
        __syncthreads();
        for (long long t = threadIdx.x; t < L.n; t += blockDim.x) L.x[t] = L.t[t];
        __syncthreads();
    }
}

// Solution back into the context's pressure array (interior cells only, as
// HyprePressureSolver copies back, src/HyprePressureSolver.cpp:388-396).
__global__ void __launch_bounds__(256) k_mg_scatter(Params P, MgLevel L, double* __restrict__ p) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= L.n) return;
    int i, j, k;
    mg_split(L, t, i, j, k);
    p[cidx(P, i, j, k)] = L.x[t];
}

}  // namespace sifv
