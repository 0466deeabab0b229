// sifv_device.cuh -- device-side data layout and the per-cell / per-face
// physics of the SemiImplicitFV finite-volume step, for sm_100a.
//
// Layout in HBM: structure of arrays, one FP64 array of totalCells per
// field, x fastest, ghosts included (the reference's SolutionState layout,
// include/SolutionState.hpp:73-113, indexed as RectilinearMesh::index,
// include/RectilinearMesh.hpp:70-73).  Face fluxes are SoA per direction
// with the reference's face indexing (src/Reconstruction.cpp:71-81).
//
// Arithmetic: every expression is evaluated in the order the reference
// writes it.  The parity build compiles this header with --fmad=false so a
// kernel's output is bit-identical to the reference compiled without FMA
// contraction.
#pragma once

#include <cstddef>
#include <cstdint>

#include "sifv.h"

// Loop over the active axes 0..dim-1, unrolled to 3 with a uniform guard so
// per-axis arrays stay in registers.
#define DIMLOOP(v) _Pragma("unroll") for (int v = 0; v < 3; ++v) if (v < dim)

namespace sifv {

constexpr int MAXPH = SIFV_MAX_PHASES;

// Flux component slots of one face (per direction).
enum FluxSlot : int {
    FS_MASS = 0,
    FS_MOMX = 1,
    FS_MOMY = 2,
    FS_MOMZ = 3,
    FS_ENERGY = 4,
    FS_PFLUX = 5,   // pressureFlux (semi-implicit)
    FS_FVEL = 6,    // faceVelocity (semi-implicit, multi-phase)
    FS_ALPHA = 7,   // alphaFlux[ph]         7 .. 7+MAXPH-1
    FS_AR = 7 + MAXPH,  // upwinded alphaRho flux[ph]
    FS_VISC = 7 + 2 * MAXPH,   // viscous stress on the face: tau.x, tau.y, tau.z, work (4 slots)
    FS_CAP = 11 + 2 * MAXPH,   // capillary stress on the face, same layout (4 slots)
    FS_COUNT = 15 + 2 * MAXPH
};

struct Params {
    int dim;
    int nx, ny, nz;          // physical cells
    int ngx, ngy, ngz;       // ghosts per axis (0 on inactive axes)
    int nxT, nyT, nzT;       // extents incl. ghosts
    int bc[6];
    int nPh;
    int reconOrder;          // SIFV_WENO* / SIFV_UPWIND*
    int riemann;             // SIFV_LF / SIFV_RUSANOV / SIFV_HLLC
    int includePressure;     // !semiImplicit
    int useIGR;
    int reconSigma;          // sigma affects the flux (LF with IGR)
    int eosStiffened;
    int RKOrder;
    double wenoEps;
    double gamma, pInf;
    double phaseGamma[MAXPH], phasePInf[MAXPH];
    double alphaMin;
    int visc;                // viscous stress on (SimulationConfig::hasViscosity)
    int perPhaseMu;          // per-phase viscosities (else the scalar mu)
    double mu;
    double phaseMu[MAXPH];
    int cap;                 // capillary stress on (SimulationConfig::hasSurfaceTension)
    double stSigma, stEps;
};

struct Fields {
    double *rho, *rhoU, *rhoV, *rhoW, *rhoE;
    double *velU, *velV, *velW, *pres, *sigma;
    double* alphaRho[MAXPH];
    double* alpha[MAXPH];
    double *rho0, *rhoU0, *rhoV0, *rhoW0, *rhoE0, *pres0;
    double* alphaRho0[MAXPH];
    double* alpha0[MAXPH];
    double *rhoUStar, *rhoVStar, *rhoWStar, *rhoEstar, *pAdvected, *rhoc2;
    double* flux[3][FS_COUNT];   // per direction, per slot (nullptr when unused)
    double *pA, *pB, *pRhs, *divUstar;
    double *igrRhs, *igrDiag;
    const double *dx, *dy, *dz;     // per cell incl. ghosts (dx(i) at [i + ngx])
    const double *adx2, *ady2, *adz2;  // alpha / (d*d) per cell (IGR)
    const unsigned char* solid;        // immersed-boundary CellType per cell (nonzero: solid), or nullptr
};

// Immersed-boundary ghost cells on the device (GhostCellInfo,
// include/ImmersedBoundary.hpp:96-103), entry q: cell[q], wall[q] (0
// no-slip, 1 slip), normal[3q..3q+2], n[q] stencil cells interp[8q..],
// weights w[8q..].  sequential: some stencil reads another ghost cell, so
// the entries run one after another in list order.
struct IbDev {
    int count, sequential;
    const long long* cell;
    const int* wall;
    const double* normal;
    const int* n;
    const long long* interp;
    const double* w;
};

// Step control block in device memory.
struct Ctl {
    unsigned long long dtBits;   // reduction accumulator (non-negative doubles order as integers)
    double dt;                   // dt of the current step
    double time;                 // physical time (device-resident loops)
    double tEnd;
    int skip;                    // nonzero: remaining work of this step is a no-op
    int jacobiDone;              // iterations taken when converged, else 0
    int stepsTaken;
    int errFlag;
    // device-resident time loop (runTimeLoop): next output time, interval,
    // and the flag set by the step that reaches an output
    double nextOutput;
    double outInterval;
    int outputDue;
    int pad0;
    unsigned long long nanCode;  // NaN scan: min over (interior cell * 8 + field order)
    unsigned long long res[1];   // per-iteration max residual bits (sized at allocation)
};

// std::max / std::min semantics (the first argument unless the comparison
// says otherwise; NaN handling follows from that).
template <typename T>
__device__ __forceinline__ T smax(T a, T b) { return (a < b) ? b : a; }
template <typename T>
__device__ __forceinline__ T smin(T a, T b) { return (b < a) ? b : a; }

__device__ __forceinline__ size_t cidx(const Params& P, int i, int j, int k) {
    return (size_t)(i + P.ngx) + (size_t)P.nxT * ((size_t)(j + P.ngy) + (size_t)P.nyT * (size_t)(k + P.ngz));
}

// Ghost source along one axis for the PRIM fill (the BoundaryCondition
// switch of fillGhostX/Y/Z, src/RectilinearMesh.cpp:147-166, 188-207).
// Returns the interior index (the ghost index itself on an exchange face,
// whose ghost layers hold the neighbouring rank's cells); sn multiplies the
// normal velocity, sa all velocity components.  Requires n >= nGhost.
__device__ __forceinline__ int prim_src(int i, int n, int bcLo, int bcHi, double& sn, double& sa) {
    sn = 1.0;
    sa = 1.0;
    if (i < 0) {
        int g = -i;
        switch (bcLo) {
            case SIFV_BC_EXCHANGE: return i;   // the neighbour's cells, held in the ghost layers
            case SIFV_BC_SYMMETRY: return g - 1;
            case SIFV_BC_PERIODIC: return n - g;
            case SIFV_BC_SLIPWALL: sn = -1.0; return g - 1;
            case SIFV_BC_NOSLIPWALL: sa = -1.0; return g - 1;
            default: return 0;
        }
    }
    if (i >= n) {
        int g = i - n + 1;
        switch (bcHi) {
            case SIFV_BC_EXCHANGE: return i;
            case SIFV_BC_SYMMETRY: return n - g;
            case SIFV_BC_PERIODIC: return g - 1;
            case SIFV_BC_SLIPWALL: sn = -1.0; return n - g;
            case SIFV_BC_NOSLIPWALL: sa = -1.0; return n - g;
            default: return n - 1;
        }
    }
    return i;
}

// Ghost source along one axis for the scalar fill
// (RectilinearMesh::fillScalarGhosts, src/RectilinearMesh.cpp:424-492):
// periodic wrap, otherwise zero gradient.
__device__ __forceinline__ int scalar_src(int i, int n, int bcLo, int bcHi) {
    if (i < 0) return (bcLo == SIFV_BC_PERIODIC) ? n + i : (bcLo == SIFV_BC_EXCHANGE) ? i : 0;
    if (i >= n) return (bcHi == SIFV_BC_PERIODIC) ? i - n : (bcHi == SIFV_BC_EXCHANGE) ? i : n - 1;
    return i;
}

__device__ __forceinline__ size_t scalar_idx(const Params& P, int i, int j, int k) {
    return cidx(P, scalar_src(i, P.nx, P.bc[0], P.bc[1]), (P.dim >= 2) ? scalar_src(j, P.ny, P.bc[2], P.bc[3]) : j,
                (P.dim >= 3) ? scalar_src(k, P.nz, P.bc[4], P.bc[5]) : k);
}

// ---------------------------------------------------------------------------
// EOS
// ---------------------------------------------------------------------------

// MixtureEOS::effectiveGammaAndPiInf, src/MixtureEOS.cpp:18-31
template <int NPH, typename T = double>
__device__ __forceinline__ void eff_gamma_piinf(const Params& P, const T* a, T& gEff, T& piEff) {
    T sumInvGm1 = T(0.0), sumPi = T(0.0);
#pragma unroll
    for (int ph = 0; ph < NPH; ++ph) {
        if (ph < P.nPh) {
            T gk = T(P.phaseGamma[ph]);
            T gm1 = gk - T(1.0);
            sumInvGm1 += a[ph] / gm1;
            sumPi += a[ph] * gk * T(P.phasePInf[ph]) / gm1;
        }
    }
    gEff = T(1.0) + T(1.0) / sumInvGm1;
    piEff = (gEff - T(1.0)) / gEff * sumPi;
}

// MixtureEOS::mixtureSoundSpeed (Wood), src/MixtureEOS.cpp:48-63
template <int NPH>
__device__ __forceinline__ double mixture_sound_speed(const Params& P, double rho, double p, const double* a,
                                                      const double* ar) {
    double sumInv = 0.0;
#pragma unroll
    for (int ph = 0; ph < NPH; ++ph) {
        if (ph < P.nPh) {
            double rho_k = smax(ar[ph], 1e-14) / smax(a[ph], 1e-14);
            double ck2 = P.phaseGamma[ph] * (p + P.phasePInf[ph]) / rho_k;
            sumInv += a[ph] / (rho_k * smax(ck2, 1e-14));
        }
    }
    double c2 = 1.0 / (rho * smax(sumInv, 1e-30));
    return sqrt(smax(c2, 0.0));
}

// MixtureEOS::mixturePressure, src/MixtureEOS.cpp:35-46
template <int NPH>
__device__ __forceinline__ double mixture_pressure(const Params& P, double rhoEint, const double* a) {
    double sumInvGm1 = 0.0, sumPi = 0.0;
#pragma unroll
    for (int ph = 0; ph < NPH; ++ph) {
        if (ph < P.nPh) {
            double gm1 = P.phaseGamma[ph] - 1.0;
            sumInvGm1 += a[ph] / gm1;
            sumPi += a[ph] * P.phaseGamma[ph] * P.phasePInf[ph] / gm1;
        }
    }
    return (rhoEint - sumPi) / sumInvGm1;
}

// MixtureEOS::mixtureTotalEnergy, src/MixtureEOS.cpp:65-76
template <int NPH>
__device__ __forceinline__ double mixture_total_energy(const Params& P, double p, const double* a, double ke) {
    double r = ke;
#pragma unroll
    for (int ph = 0; ph < NPH; ++ph) {
        if (ph < P.nPh) {
            double gm1 = P.phaseGamma[ph] - 1.0;
            r += a[ph] * (p + P.phaseGamma[ph] * P.phasePInf[ph]) / gm1;
        }
    }
    return r;
}

// Single-phase sound speed used by computeAcousticTimeStep
// (src/RKTimeStepping.cpp:61-62) and solvePressure (src/SemiImplicitSolver.cpp:553-554).
__device__ __forceinline__ double single_sound_speed(const Params& P, double rho, double p) {
    return sqrt(P.gamma * smax(p + P.pInf, 1e-14) / smax(rho, 1e-14));
}

// ---------------------------------------------------------------------------
// Reconstruction kernels, src/Reconstruction.cpp:83-200
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T weno5L(T v0, T v1, T v2, T v3, T v4, T eps) {
    T p0 = (T(1.0) / T(3.0)) * v0 - (T(7.0) / T(6.0)) * v1 + (T(11.0) / T(6.0)) * v2;
    T p1 = -(T(1.0) / T(6.0)) * v1 + (T(5.0) / T(6.0)) * v2 + (T(1.0) / T(3.0)) * v3;
    T p2 = (T(1.0) / T(3.0)) * v2 + (T(5.0) / T(6.0)) * v3 - (T(1.0) / T(6.0)) * v4;
    T t0 = v0 - T(2.0) * v1 + v2, s0 = v0 - T(4.0) * v1 + T(3.0) * v2;
    T t1 = v1 - T(2.0) * v2 + v3, s1 = v1 - v3;
    T t2 = v2 - T(2.0) * v3 + v4, s2 = T(3.0) * v2 - T(4.0) * v3 + v4;
    T b0 = (T(13.0) / T(12.0)) * t0 * t0 + (T(1.0) / T(4.0)) * s0 * s0;
    T b1 = (T(13.0) / T(12.0)) * t1 * t1 + (T(1.0) / T(4.0)) * s1 * s1;
    T b2 = (T(13.0) / T(12.0)) * t2 * t2 + (T(1.0) / T(4.0)) * s2 * s2;
    T e0 = eps + b0, e1 = eps + b1, e2 = eps + b2;
    T a0 = (T(1.0) / T(10.0)) / (e0 * e0);
    T a1 = (T(6.0) / T(10.0)) / (e1 * e1);
    T a2 = (T(3.0) / T(10.0)) / (e2 * e2);
    T aSum = a0 + a1 + a2;
    return (a0 * p0 + a1 * p1 + a2 * p2) / aSum;
}

template <typename T>
__device__ __forceinline__ T weno5R(T v0, T v1, T v2, T v3, T v4, T eps) {
    T p0 = (T(1.0) / T(3.0)) * v4 - (T(7.0) / T(6.0)) * v3 + (T(11.0) / T(6.0)) * v2;
    T p1 = -(T(1.0) / T(6.0)) * v3 + (T(5.0) / T(6.0)) * v2 + (T(1.0) / T(3.0)) * v1;
    T p2 = (T(1.0) / T(3.0)) * v2 + (T(5.0) / T(6.0)) * v1 - (T(1.0) / T(6.0)) * v0;
    T t0 = v4 - T(2.0) * v3 + v2, s0 = v4 - T(4.0) * v3 + T(3.0) * v2;
    T t1 = v3 - T(2.0) * v2 + v1, s1 = v3 - v1;
    T t2 = v2 - T(2.0) * v1 + v0, s2 = T(3.0) * v2 - T(4.0) * v1 + v0;
    T b0 = (T(13.0) / T(12.0)) * t0 * t0 + (T(1.0) / T(4.0)) * s0 * s0;
    T b1 = (T(13.0) / T(12.0)) * t1 * t1 + (T(1.0) / T(4.0)) * s1 * s1;
    T b2 = (T(13.0) / T(12.0)) * t2 * t2 + (T(1.0) / T(4.0)) * s2 * s2;
    T e0 = eps + b0, e1 = eps + b1, e2 = eps + b2;
    T a0 = (T(1.0) / T(10.0)) / (e0 * e0);
    T a1 = (T(6.0) / T(10.0)) / (e1 * e1);
    T a2 = (T(3.0) / T(10.0)) / (e2 * e2);
    T aSum = a0 + a1 + a2;
    return (a0 * p0 + a1 * p1 + a2 * p2) / aSum;
}

template <typename T>
__device__ __forceinline__ T upwind5L(T v0, T v1, T v2, T v3, T v4) {
    T p0 = (T(1.0) / T(3.0)) * v0 - (T(7.0) / T(6.0)) * v1 + (T(11.0) / T(6.0)) * v2;
    T p1 = -(T(1.0) / T(6.0)) * v1 + (T(5.0) / T(6.0)) * v2 + (T(1.0) / T(3.0)) * v3;
    T p2 = (T(1.0) / T(3.0)) * v2 + (T(5.0) / T(6.0)) * v3 - (T(1.0) / T(6.0)) * v4;
    return (T(1.0) / T(10.0)) * p0 + (T(6.0) / T(10.0)) * p1 + (T(3.0) / T(10.0)) * p2;
}

template <typename T>
__device__ __forceinline__ T upwind5R(T v0, T v1, T v2, T v3, T v4) {
    T p0 = (T(1.0) / T(3.0)) * v4 - (T(7.0) / T(6.0)) * v3 + (T(11.0) / T(6.0)) * v2;
    T p1 = -(T(1.0) / T(6.0)) * v3 + (T(5.0) / T(6.0)) * v2 + (T(1.0) / T(3.0)) * v1;
    T p2 = (T(1.0) / T(3.0)) * v2 + (T(5.0) / T(6.0)) * v1 - (T(1.0) / T(6.0)) * v0;
    return (T(1.0) / T(10.0)) * p0 + (T(6.0) / T(10.0)) * p1 + (T(3.0) / T(10.0)) * p2;
}

template <typename T>
__device__ __forceinline__ T weno3L(T v0, T v1, T v2, T eps) {
    T p0 = -T(0.5) * v0 + T(1.5) * v1;
    T p1 = T(0.5) * v1 + T(0.5) * v2;
    T b0 = (v1 - v0) * (v1 - v0);
    T b1 = (v2 - v1) * (v2 - v1);
    T e0 = eps + b0, e1 = eps + b1;
    T a0 = (T(1.0) / T(3.0)) / (e0 * e0);
    T a1 = (T(2.0) / T(3.0)) / (e1 * e1);
    T aSum = a0 + a1;
    return (a0 * p0 + a1 * p1) / aSum;
}

template <typename T>
__device__ __forceinline__ T weno3R(T v0, T v1, T v2, T eps) {
    T p0 = T(0.5) * v0 + T(0.5) * v1;
    T p1 = T(1.5) * v1 - T(0.5) * v2;
    T b0 = (v1 - v0) * (v1 - v0);
    T b1 = (v2 - v1) * (v2 - v1);
    T e0 = eps + b0, e1 = eps + b1;
    T a0 = (T(2.0) / T(3.0)) / (e0 * e0);
    T a1 = (T(1.0) / T(3.0)) / (e1 * e1);
    T aSum = a0 + a1;
    return (a0 * p0 + a1 * p1) / aSum;
}

template <typename T>
__device__ __forceinline__ T upwind3L(T v0, T v1, T v2) {
    T p0 = -T(0.5) * v0 + T(1.5) * v1;
    T p1 = T(0.5) * v1 + T(0.5) * v2;
    return (T(1.0) / T(3.0)) * p0 + (T(2.0) / T(3.0)) * p1;
}

template <typename T>
__device__ __forceinline__ T upwind3R(T v0, T v1, T v2) {
    T p0 = T(0.5) * v0 + T(0.5) * v1;
    T p1 = T(1.5) * v1 - T(0.5) * v2;
    return (T(2.0) / T(3.0)) * p0 + (T(1.0) / T(3.0)) * p1;
}

// Left and right face values of one field at the face whose right cell is
// `base`, cells strided by `st` along the sweep direction
// (reconstructScalar, src/Reconstruction.cpp:11-28: the left state uses
// cells -3..+1, the right state -2..+2 for WENO5).
template <int W, typename T>
__device__ __forceinline__ void recon_pair(const T* __restrict__ f, size_t base, long st, bool weno, T eps,
                                           T& L, T& R) {
    if (W == 1) {
        L = f[base - st];
        R = f[base];
    } else if (W == 3) {
        T v0 = f[base - 2 * st], v1 = f[base - st], v2 = f[base], v3 = f[base + st];
        if (weno) {
            L = weno3L(v0, v1, v2, eps);
            R = weno3R(v1, v2, v3, eps);
        } else {
            L = upwind3L(v0, v1, v2);
            R = upwind3R(v1, v2, v3);
        }
    } else {
        T v0 = f[base - 3 * st], v1 = f[base - 2 * st], v2 = f[base - st], v3 = f[base], v4 = f[base + st],
               v5 = f[base + 2 * st];
        if (weno) {
            L = weno5L(v0, v1, v2, v3, v4, eps);
            R = weno5R(v1, v2, v3, v4, v5, eps);
        } else {
            L = upwind5L(v0, v1, v2, v3, v4);
            R = upwind5R(v1, v2, v3, v4, v5);
        }
    }
}

// ---------------------------------------------------------------------------
// Riemann solvers
// ---------------------------------------------------------------------------
template <int NPH, typename T = double>
struct FaceState {
    T rho, u[3], p, sigma, gEff, piEff;
    T alpha[NPH > 0 ? NPH : 1];
};

template <int NPH, typename T = double>
struct FaceFlux {
    T mass, mom[3], energy, pflux, fvel;
    T alpha[NPH > 0 ? NPH : 1];
};

// soundSpeedDirect / rhoEFromState, include/RiemannSolver.hpp:70-78
template <int NPH, typename T>
__device__ __forceinline__ T sound_speed_direct(const FaceState<NPH, T>& W) {
    return sqrt(W.gEff * smax(W.p + W.piEff, T(1e-14)) / smax(W.rho, T(1e-14)));
}
template <int NPH, typename T>
__device__ __forceinline__ T rhoE_from_state(const FaceState<NPH, T>& W) {
    T ke = T(0.5) * W.rho * (W.u[0] * W.u[0] + W.u[1] * W.u[1] + W.u[2] * W.u[2]);
    return (W.p + W.gEff * W.piEff) / (W.gEff - T(1.0)) + ke;
}

// normalVelocity (include/RiemannSolver.hpp:59-64) for the unit normal of
// axis D: 0 + u_D*1 + sum of u_d*0 over the other active axes.
template <int D, int NPH, typename T>
__device__ __forceinline__ T normal_velocity(const FaceState<NPH, T>& W, int dim) {
    T vn = T(0.0);
    DIMLOOP(d) vn += W.u[d] * ((d == D) ? T(1.0) : T(0.0));
    return vn;
}

// computeHLLCFlux, src/HLLCSolver.cpp:7-161
template <int D, int NPH, typename T>
__device__ __forceinline__ void hllc_flux(const Params& P, const FaceState<NPH, T>& L, const FaceState<NPH, T>& R,
                                          FaceFlux<NPH, T>& F) {
    const int dim = P.dim;
    const bool incP = P.includePressure;
    const T n[3] = {D == 0 ? T(1.0) : T(0.0), D == 1 ? T(1.0) : T(0.0), D == 2 ? T(1.0) : T(0.0)};
    F.mass = T(0.0); F.mom[0] = F.mom[1] = F.mom[2] = T(0.0); F.energy = T(0.0); F.pflux = T(0.0); F.fvel = T(0.0);
    T uL = normal_velocity<D>(L, dim), uR = normal_velocity<D>(R, dim);
    T rhoEL = rhoE_from_state(L), rhoER = rhoE_from_state(R);
    T sL, sR, sStar;
    if (incP) {
        T cL = sound_speed_direct(L), cR = sound_speed_direct(R);
        sL = smin(uL - cL, uR - cR);
        sR = smax(uL + cL, uR + cR);
        sStar = (R.p - L.p + L.rho * uL * (sL - uL) - R.rho * uR * (sR - uR)) /
                (L.rho * (sL - uL) - R.rho * (sR - uR));
    } else {
        sL = smin(uL, uR);
        sR = smax(uL, uR);
        sStar = T(0.5) * (uL + uR);
    }
    if (sL >= 0) {
        F.mass = L.rho * uL;
        DIMLOOP(i) F.mom[i] = L.rho * L.u[i] * uL;
        F.energy = rhoEL * uL;
        if (incP) {
            DIMLOOP(i) F.mom[i] += L.p * n[i];
            F.energy += L.p * uL;
        }
    } else if (sR <= 0) {
        F.mass = R.rho * uR;
        DIMLOOP(i) F.mom[i] = R.rho * R.u[i] * uR;
        F.energy = rhoER * uR;
        if (incP) {
            DIMLOOP(i) F.mom[i] += R.p * n[i];
            F.energy += R.p * uR;
        }
    } else if (sStar >= 0) {
        T rhoStarL = L.rho * (sL - uL) / (sL - sStar);
        F.mass = L.rho * uL + sL * (rhoStarL - L.rho);
        if (incP) {
            DIMLOOP(i) {
                T rhoUStarL = rhoStarL * (L.u[i] + (sStar - uL) * n[i]);
                F.mom[i] = L.rho * L.u[i] * uL + L.p * n[i] + sL * (rhoUStarL - L.rho * L.u[i]);
            }
            T eL = rhoEL / L.rho;
            T EStarL = rhoStarL * (eL + (sStar - uL) * (sStar + L.p / (L.rho * (sL - uL))));
            F.energy = (rhoEL + L.p) * uL + sL * (EStarL - rhoEL);
        } else {
            DIMLOOP(i) {
                T rhoUStarL = rhoStarL * (L.u[i] + (sStar - uL) * n[i]);
                F.mom[i] = L.rho * L.u[i] * uL + sL * (rhoUStarL - L.rho * L.u[i]);
            }
            T eL = rhoEL / L.rho;
            T EStarL = rhoStarL * (eL + (sStar - uL) * sStar);
            F.energy = rhoEL * uL + sL * (EStarL - rhoEL);
        }
    } else {
        T rhoStarR = R.rho * (sR - uR) / (sR - sStar);
        F.mass = R.rho * uR + sR * (rhoStarR - R.rho);
        if (incP) {
            DIMLOOP(i) {
                T rhoUStarR = rhoStarR * (R.u[i] + (sStar - uR) * n[i]);
                F.mom[i] = R.rho * R.u[i] * uR + R.p * n[i] + sR * (rhoUStarR - R.rho * R.u[i]);
            }
            T eR = rhoER / R.rho;
            T EStarR = rhoStarR * (eR + (sStar - uR) * (sStar + R.p / (R.rho * (sR - uR))));
            F.energy = (rhoER + R.p) * uR + sR * (EStarR - rhoER);
        } else {
            DIMLOOP(i) {
                T rhoUStarR = rhoStarR * (R.u[i] + (sStar - uR) * n[i]);
                F.mom[i] = R.rho * R.u[i] * uR + sR * (rhoUStarR - R.rho * R.u[i]);
            }
            T eR = rhoER / R.rho;
            T EStarR = rhoStarR * (eR + (sStar - uR) * sStar);
            F.energy = rhoER * uR + sR * (EStarR - rhoER);
        }
    }
    if (sL >= 0) {
        F.fvel = uL;
        F.pflux = L.p * uL;
#pragma unroll
        for (int ph = 0; ph < NPH; ++ph) F.alpha[ph] = L.alpha[ph] * uL;
    } else if (sR <= 0) {
        F.fvel = uR;
        F.pflux = R.p * uR;
#pragma unroll
        for (int ph = 0; ph < NPH; ++ph) F.alpha[ph] = R.alpha[ph] * uR;
    } else {
        F.fvel = sStar;
        if (sStar >= 0) {
            F.pflux = L.p * sStar;
#pragma unroll
            for (int ph = 0; ph < NPH; ++ph) F.alpha[ph] = L.alpha[ph] * sStar;
        } else {
            F.pflux = R.p * sStar;
#pragma unroll
            for (int ph = 0; ph < NPH; ++ph) F.alpha[ph] = R.alpha[ph] * sStar;
        }
    }
}

// computeRusanovFlux, src/RusanovSolver.cpp:7-83
template <int D, int NPH, typename T>
__device__ __forceinline__ void rusanov_flux(const Params& P, const FaceState<NPH, T>& L, const FaceState<NPH, T>& R,
                                             FaceFlux<NPH, T>& F) {
    const int dim = P.dim;
    const bool incP = P.includePressure;
    const T n[3] = {D == 0 ? T(1.0) : T(0.0), D == 1 ? T(1.0) : T(0.0), D == 2 ? T(1.0) : T(0.0)};
    F.mom[0] = F.mom[1] = F.mom[2] = T(0.0);
    T uL = normal_velocity<D>(L, dim), uR = normal_velocity<D>(R, dim);
    T absUL = fabs(uL), absUR = fabs(uR);
    T sMax;
    if (incP) {
        T cL = sound_speed_direct(L), cR = sound_speed_direct(R);
        sMax = smax(absUL + cL, absUR + cR);
    } else {
        sMax = smax(absUL, absUR);
    }
    T rhoEL = rhoE_from_state(L), rhoER = rhoE_from_state(R);
    T mL = L.rho * uL, mR = R.rho * uR;
    T momL[3] = {T(0.0), T(0.0), T(0.0)}, momR[3] = {T(0.0), T(0.0), T(0.0)};
    DIMLOOP(i) {
        momL[i] = L.rho * L.u[i] * uL;
        momR[i] = R.rho * R.u[i] * uR;
    }
    T eL = rhoEL * uL, eR = rhoER * uR;
    if (incP) {
        DIMLOOP(i) {
            momL[i] += L.p * n[i];
            momR[i] += R.p * n[i];
        }
        eL += L.p * uL;
        eR += R.p * uR;
    }
    F.mass = T(0.5) * (mL + mR) - T(0.5) * sMax * (R.rho - L.rho);
    DIMLOOP(i)
        F.mom[i] = T(0.5) * (momL[i] + momR[i]) - T(0.5) * sMax * (R.rho * R.u[i] - L.rho * L.u[i]);
    F.energy = T(0.5) * (eL + eR) - T(0.5) * sMax * (rhoER - rhoEL);
    F.fvel = T(0.5) * (uL + uR);
    F.pflux = T(0.5) * (L.p * uL + R.p * uR) - T(0.5) * sMax * (R.p - L.p);
#pragma unroll
    for (int ph = 0; ph < NPH; ++ph)
        F.alpha[ph] = T(0.5) * (L.alpha[ph] * uL + R.alpha[ph] * uR) - T(0.5) * sMax * (R.alpha[ph] - L.alpha[ph]);
}

// computeLFFlux, src/LFSolver.cpp:8-75
template <int D, int NPH, typename T>
__device__ __forceinline__ void lf_flux(const Params& P, const FaceState<NPH, T>& L, const FaceState<NPH, T>& R,
                                        FaceFlux<NPH, T>& F) {
    const int dim = P.dim;
    const bool incP = P.includePressure;
    const T n[3] = {D == 0 ? T(1.0) : T(0.0), D == 1 ? T(1.0) : T(0.0), D == 2 ? T(1.0) : T(0.0)};
    F.mom[0] = F.mom[1] = F.mom[2] = T(0.0);
    T uL = normal_velocity<D>(L, dim), uR = normal_velocity<D>(R, dim);
    T uLS = T(0.0), uRS = T(0.0);
    DIMLOOP(i) {
        uLS += L.u[i] * L.u[i];
        uRS += R.u[i] * R.u[i];
    }
    uLS = sqrt(uLS);
    uRS = sqrt(uRS);
    T C;
    if (incP) {
        T cL = sound_speed_direct(L), cR = sound_speed_direct(R);
        C = smax(uLS, uRS) + smax(cL, cR);
    } else {
        C = smax(uLS, uRS);
    }
    F.mass = T(0.5) * (L.rho * uL + R.rho * uR) - T(0.5) * C * (R.rho - L.rho);
    DIMLOOP(i)
        F.mom[i] = T(0.5) * (L.rho * L.u[i] * uL + R.rho * R.u[i] * uR) - T(0.5) * C * (R.rho * R.u[i] - L.rho * L.u[i]);
    T rhoEL = rhoE_from_state(L), rhoER = rhoE_from_state(R);
    F.energy = T(0.5) * (rhoEL * uL + rhoER * uR) - T(0.5) * C * (rhoER - rhoEL);
    if (incP) {
        DIMLOOP(i) F.mom[i] += T(0.5) * (L.p + R.p) * n[i];
        F.energy += T(0.5) * (L.p * uL + R.p * uR);
    }
    if (P.useIGR) {
        DIMLOOP(i) F.mom[i] += T(0.5) * (L.sigma + R.sigma) * n[i];
        F.energy += T(0.5) * (L.sigma * uL + R.sigma * uR);
    }
    F.fvel = T(0.5) * (uL + uR);
    F.pflux = T(0.5) * (L.p * uL + R.p * uR) - T(0.5) * C * (R.p - L.p);
#pragma unroll
    for (int ph = 0; ph < NPH; ++ph)
        F.alpha[ph] = T(0.5) * (L.alpha[ph] * uL + R.alpha[ph] * uR) - T(0.5) * C * (R.alpha[ph] - L.alpha[ph]);
}

}  // namespace sifv
