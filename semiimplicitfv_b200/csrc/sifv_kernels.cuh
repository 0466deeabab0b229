// sifv_kernels.cuh -- CUDA kernels of the finite-volume step (sm_100a).
//
// One stage of the explicit step (ExplicitSolver::step,
// src/ExplicitSolver.cpp:109-190) is:
//   k_prim_bc      cons -> prim on interior cells, PRIM ghost fill composed
//                  into one pass (every ghost cell computes the primitive of
//                  its interior source itself, so no ordering is needed)
//   k_face<DIR>    per face: reconstruction of both sides + Riemann flux
//                  (+ upwinded partial-density flux), written SoA
//   k_assemble     per cell: flux divergence in the reference's accumulation
//                  order, sources, and the SSP-RK update (or the
//                  semi-implicit star update), fused
// The semi-implicit stage adds k_bc_prim, k_pressure_setup, the Jacobi
// iterations (k_jacobi) and k_correction.  IGR runs k_igr_setup and, per
// sweep, one k_igr_tile launch per tile plane of the lexicographic
// Gauss-Seidel sweep (the dependency order of src/IGR.cpp:110-156).
#pragma once

#include "sifv_common.cuh"

namespace sifv {

// Stage entry: cons -> prim (interior) + PRIM ghost fill, one pass.
template <int NPH>
__global__ void k_prim_bc(Params P, Fields F, const Ctl* __restrict__ ctl, int interiorOnly) {
    if (ctl && ctl->skip) return;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!ext_coords(P, t, i, j, k)) return;
    const int dim = P.dim;
    size_t d = cidx(P, i, j, k);
    if (is_interior(P, i, j, k)) {
        double rho, u[3], p;
        cons_to_prim_cell<NPH>(P, F, d, rho, u, p);
        F.velU[d] = u[0];
        if (dim >= 2) F.velV[d] = u[1];
        if (dim >= 3) F.velW[d] = u[2];
        F.pres[d] = p;
        if (NPH > 0) F.rho[d] = rho;
        return;
    }
    if (interiorOnly) return;
    double sg[3];
    size_t s = prim_source(P, i, j, k, sg);
    double rho, u[3], p;
    cons_to_prim_cell<NPH>(P, F, s, rho, u, p);
    F.rho[d] = rho;
    F.velU[d] = sg[0] * u[0];
    if (dim >= 2) F.velV[d] = sg[1] * u[1];
    if (dim >= 3) F.velW[d] = sg[2] * u[2];
    F.pres[d] = p;
    F.sigma[d] = F.sigma[s];
#pragma unroll
    for (int ph = 0; ph < NPH; ++ph) {
        if (ph < P.nPh) {
            F.alphaRho[ph][d] = F.alphaRho[ph][s];
            F.alpha[ph][d] = F.alpha[ph][s];
        }
    }
}

// PRIM ghost fill from the primitive fields as they stand
// (RectilinearMesh::applyBoundaryConditions(state, PRIM, halo),
// src/RectilinearMesh.cpp:498-524 with SolutionState::copyCell_P).
// One thread per ghost cell (ghost_coords).
template <int NPH>
__global__ void k_bc_prim(Params P, Fields F) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!ghost_coords(P, t, i, j, k)) return;
    const int dim = P.dim;
    size_t d = cidx(P, i, j, k);
    double sg[3];
    size_t s = prim_source(P, i, j, k, sg);
    F.rho[d] = F.rho[s];
    F.velU[d] = sg[0] * F.velU[s];
    if (dim >= 2) F.velV[d] = sg[1] * F.velV[s];
    if (dim >= 3) F.velW[d] = sg[2] * F.velW[s];
    F.pres[d] = F.pres[s];
    F.sigma[d] = F.sigma[s];
#pragma unroll
    for (int ph = 0; ph < NPH; ++ph) {
        if (ph < P.nPh) {
            F.alphaRho[ph][d] = F.alphaRho[ph][s];
            F.alpha[ph][d] = F.alpha[ph][s];
        }
    }
}

// Scalar ghost fill (RectilinearMesh::fillScalarGhosts, src/RectilinearMesh.cpp:424-492),
// one thread per ghost cell (ghost_count threads).
__global__ void k_scalar_ghosts(Params P, double* __restrict__ f) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (t >= ghost_count(P) || !ghost_coords(P, t, i, j, k)) return;
    f[cidx(P, i, j, k)] = f[scalar_idx(P, i, j, k)];
}

// ---------------------------------------------------------------------------
// Face flux: Reconstructor::reconstructX/Y/Z (src/Reconstruction.cpp:204-541)
// then computeFluxDirect (include/RiemannSolver.hpp:91-100) and, for
// multi-phase, the upwinded partial-density flux of computeRHS
// (src/ExplicitSolver.cpp:307-326).
// ---------------------------------------------------------------------------
template <int DIR, int W, int NPH>
__global__ void __launch_bounds__(128) k_face(Params P, Fields F, const Ctl* __restrict__ ctl) {
    if (ctl && ctl->skip) return;
    const int dim = P.dim;
    // face grid: (nx + [DIR==0]) x (ny + [DIR==1]) x (nz + [DIR==2])
    const int fnx = P.nx + (DIR == 0), fny = P.ny + (DIR == 1), fnz = P.nz + (DIR == 2);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long tot = (long long)fnx * fny * fnz;
    if (t >= tot) return;
    int i, j, k;
    split3(t, fnx, fny, i, j, k);
    const size_t base = cidx(P, i, j, k);  // right cell of the face
    const long st = (DIR == 0) ? 1L : (DIR == 1) ? (long)P.nxT : (long)P.nxT * P.nyT;
    const bool weno = (P.reconOrder == SIFV_WENO1 || P.reconOrder == SIFV_WENO3 || P.reconOrder == SIFV_WENO5);
    const double eps = P.wenoEps;

    FaceState<NPH> L, R;
    L.u[0] = L.u[1] = L.u[2] = 0.0;
    R.u[0] = R.u[1] = R.u[2] = 0.0;
    L.sigma = R.sigma = 0.0;
    recon_pair<W>(F.rho, base, st, weno, eps, L.rho, R.rho);
    recon_pair<W>(F.velU, base, st, weno, eps, L.u[0], R.u[0]);
    if (dim >= 2) recon_pair<W>(F.velV, base, st, weno, eps, L.u[1], R.u[1]);
    if (dim >= 3) recon_pair<W>(F.velW, base, st, weno, eps, L.u[2], R.u[2]);
    recon_pair<W>(F.pres, base, st, weno, eps, L.p, R.p);
    if (P.reconSigma) recon_pair<W>(F.sigma, base, st, weno, eps, L.sigma, R.sigma);
#pragma unroll
    for (int ph = 0; ph < NPH; ++ph) {
        L.alpha[ph] = R.alpha[ph] = 0.0;
        if (ph < P.nPh) recon_pair<W>(F.alpha[ph], base, st, weno, eps, L.alpha[ph], R.alpha[ph]);
    }
    if (NPH > 0) {
        eff_gamma_piinf<NPH>(P, L.alpha, L.gEff, L.piEff);
        eff_gamma_piinf<NPH>(P, R.alpha, R.gEff, R.piEff);
    } else {
        L.gEff = R.gEff = P.gamma;
        L.piEff = R.piEff = P.pInf;
    }

    FaceFlux<NPH> Fx;
    switch (P.riemann) {
        case SIFV_HLLC: hllc_flux<DIR, NPH>(P, L, R, Fx); break;
        case SIFV_RUSANOV: rusanov_flux<DIR, NPH>(P, L, R, Fx); break;
        default: lf_flux<DIR, NPH>(P, L, R, Fx); break;
    }

    // reference face index (src/Reconstruction.cpp:71-81) == t
    double* const* out = F.flux[DIR];
    out[FS_MASS][t] = Fx.mass;
    out[FS_MOMX][t] = Fx.mom[0];
    if (dim >= 2) out[FS_MOMY][t] = Fx.mom[1];
    if (dim >= 3) out[FS_MOMZ][t] = Fx.mom[2];
    out[FS_ENERGY][t] = Fx.energy;
    if (!P.includePressure) out[FS_PFLUX][t] = Fx.pflux;
    if (!P.includePressure || NPH > 0) out[FS_FVEL][t] = Fx.fvel;
    if (NPH > 0) {
        size_t upw = (Fx.mass >= 0) ? base - st : base;
        double rhoUpw = smax(F.rho[upw], 1e-14);
#pragma unroll
        for (int ph = 0; ph < NPH; ++ph) {
            if (ph < P.nPh) {
                out[FS_ALPHA + ph][t] = Fx.alpha[ph];
                out[FS_AR + ph][t] = (F.alphaRho[ph][upw] / rhoUpw) * Fx.mass;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Assemble + update.  The flux divergence reproduces the accumulation order
// of computeRHS (src/ExplicitSolver.cpp:294-483, src/SemiImplicitSolver.cpp:
// 263-457): per direction x, y, z, the cell's low face adds coeff*F, its
// high face subtracts it (divU: the opposite signs), starting from 0.
// ---------------------------------------------------------------------------
// divergence of one flux slot: ((0 + c F_lo) - c F_hi) per direction
__device__ __forceinline__ double div_slot(const Params& P, const Fields& F, const CellFaces& cf, int slot) {
    const int dim = P.dim;
    double r = 0.0;
    DIMLOOP(d) {
        const double* f = F.flux[d][slot];
        double c = cf.coeff[d];
        r += c * f[cf.lo[d]];
        r -= c * f[cf.lo[d] + cf.hiOff[d]];
    }
    return r;
}

__device__ __forceinline__ double div_fvel(const Params& P, const Fields& F, const CellFaces& cf) {
    const int dim = P.dim;
    double r = 0.0;
    DIMLOOP(d) {
        const double* f = F.flux[d][FS_FVEL];
        double c = cf.coeff[d];
        r -= c * f[cf.lo[d]];
        r += c * f[cf.lo[d] + cf.hiOff[d]];
    }
    return r;
}

template <int NPH>
__device__ __forceinline__ void mp_post(const Params& P, const Fields& F, size_t c) {
    double rhoSum = 0.0;
#pragma unroll
    for (int ph = 0; ph < NPH; ++ph) {
        if (ph < P.nPh) {
            double v = smax(F.alphaRho[ph][c], 1e-14);
            F.alphaRho[ph][c] = v;
            rhoSum += v;
        }
    }
    F.rho[c] = rhoSum;
    double a[NPH > 0 ? NPH : 1];
    double aSum = 0.0;
#pragma unroll
    for (int ph = 0; ph < NPH; ++ph) {
        if (ph < P.nPh) {
            a[ph] = smax(F.alpha[ph][c], P.alphaMin);
        }
    }
#pragma unroll
    for (int ph = 0; ph < NPH; ++ph)
        if (ph < P.nPh) aSum += a[ph];
#pragma unroll
    for (int ph = 0; ph < NPH; ++ph)
        if (ph < P.nPh) F.alpha[ph][c] = a[ph] / aSum;
}

// MODE 0: explicit SSP-RK update (src/ExplicitSolver.cpp:127-188).
// MODE 1: semi-implicit star update (src/SemiImplicitSolver.cpp:159-223).
// A face stress (viscous or capillary, four face arrays from `slot`: the
// momentum components and the work) added to one cell's rhs: per direction
// the low face (-) then the high face (+), the reference's face-loop order.
__device__ __forceinline__ void add_face_stress(int dim, const Fields& F, const CellFaces& cf, int slot,
                                                double& rU, double& rV, double& rW, double& rE) {
    DIMLOOP(d) {
        const double co = cf.coeff[d];
        const long long lo = cf.lo[d], hi = cf.lo[d] + cf.hiOff[d];
        double* const* fv = F.flux[d] + slot;
        rU -= co * fv[0][lo];
        if (dim >= 2) rV -= co * fv[1][lo];
        if (dim >= 3) rW -= co * fv[2][lo];
        rE -= co * fv[3][lo];
        rU += co * fv[0][hi];
        if (dim >= 2) rV += co * fv[1][hi];
        if (dim >= 3) rW += co * fv[2][hi];
        rE += co * fv[3][hi];
    }
}

template <int NPH, int MODE>
__global__ void __launch_bounds__(256) k_assemble(Params P, Fields F, const Ctl* __restrict__ ctl, StageCoef K) {
    if (ctl->skip) return;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!int_coords(P, t, i, j, k)) return;
    const int dim = P.dim;
    const size_t c = cidx(P, i, j, k);
    if (F.solid && F.solid[c]) return;   // immersed-boundary solid cells are not updated
    CellFaces cf;
    cell_faces(P, F, i, j, k, cf);

    double rR = div_slot(P, F, cf, FS_MASS);
    double rU = div_slot(P, F, cf, FS_MOMX);
    double rV = (dim >= 2) ? div_slot(P, F, cf, FS_MOMY) : 0.0;
    double rW = (dim >= 3) ? div_slot(P, F, cf, FS_MOMZ) : 0.0;
    double rE = div_slot(P, F, cf, FS_ENERGY);
    double rP = 0.0, divU = 0.0;
    if (MODE == 1) rP = div_slot(P, F, cf, FS_PFLUX);
    if (MODE == 1 || NPH > 0) divU = div_fvel(P, F, cf);
    double rAR[NPH > 0 ? NPH : 1], rA[NPH > 0 ? NPH : 1];
#pragma unroll
    for (int ph = 0; ph < NPH; ++ph) {
        if (ph < P.nPh) {
            rAR[ph] = div_slot(P, F, cf, FS_AR + ph);
            rA[ph] = div_slot(P, F, cf, FS_ALPHA + ph);
            rA[ph] += F.alpha[ph][c] * divU;   // alpha div(u) source
        }
    }
    if (MODE == 1) rP += F.pres[c] * divU;     // p div(u) source
    if (K.hasBodyForce) {                      // src/ExplicitSolver.cpp:498-521
        double rho = F.rho[c];
        rU += rho * K.accel[0];
        if (dim >= 2) rV += rho * K.accel[1];
        if (dim >= 3) rW += rho * K.accel[2];
        double work = F.velU[c] * K.accel[0];
        if (dim >= 2) work += F.velV[c] * K.accel[1];
        if (dim >= 3) work += F.velW[c] * K.accel[2];
        rE += rho * work;
    }

    // addViscousFluxes (src/ViscousFlux.cpp:24-303), then addSurfaceTensionFluxes
    // (src/SurfaceTension.cpp:8-254)
    if (P.visc) add_face_stress(dim, F, cf, FS_VISC, rU, rV, rW, rE);
    if (P.cap) add_face_stress(dim, F, cf, FS_CAP, rU, rV, rW, rE);

    const double dt = ctl->dt;
    const double c1 = K.c1, c2 = K.c2, c3 = K.c3, c4 = K.c4;
    const int RK = P.RKOrder;
    if (K.s == 0 && RK > 1) {   // SolutionState::saveConservativeCell, src/SolutionState.cpp:228-240
        F.rho0[c] = F.rho[c];
        F.rhoU0[c] = F.rhoU[c];
        if (dim >= 2) F.rhoV0[c] = F.rhoV[c];
        if (dim >= 3) F.rhoW0[c] = F.rhoW[c];
        F.rhoE0[c] = F.rhoE[c];
        F.pres0[c] = F.pres[c];
#pragma unroll
        for (int ph = 0; ph < NPH; ++ph) {
            if (ph < P.nPh) {
                F.alphaRho0[ph][c] = F.alphaRho[ph][c];
                F.alpha0[ph][c] = F.alpha[ph][c];
            }
        }
    }
    if (MODE == 0) {
        if (RK == 1) {
            F.rho[c] += dt * rR;
            F.rhoU[c] += dt * rU;
            if (dim >= 2) F.rhoV[c] += dt * rV;
            if (dim >= 3) F.rhoW[c] += dt * rW;
            F.rhoE[c] += dt * rE;
#pragma unroll
            for (int ph = 0; ph < NPH; ++ph)
                if (ph < P.nPh) F.alphaRho[ph][c] += dt * rAR[ph];
#pragma unroll
            for (int ph = 0; ph < NPH; ++ph)
                if (ph < P.nPh) F.alpha[ph][c] += dt * rA[ph];
        } else {
            F.rho[c] = (c1 * F.rho[c] + c2 * F.rho0[c] + c3 * dt * rR) / c4;
            F.rhoU[c] = (c1 * F.rhoU[c] + c2 * F.rhoU0[c] + c3 * dt * rU) / c4;
            if (dim >= 2) F.rhoV[c] = (c1 * F.rhoV[c] + c2 * F.rhoV0[c] + c3 * dt * rV) / c4;
            if (dim >= 3) F.rhoW[c] = (c1 * F.rhoW[c] + c2 * F.rhoW0[c] + c3 * dt * rW) / c4;
            F.rhoE[c] = (c1 * F.rhoE[c] + c2 * F.rhoE0[c] + c3 * dt * rE) / c4;
#pragma unroll
            for (int ph = 0; ph < NPH; ++ph)
                if (ph < P.nPh)
                    F.alphaRho[ph][c] = (c1 * F.alphaRho[ph][c] + c2 * F.alphaRho0[ph][c] + c3 * dt * rAR[ph]) / c4;
#pragma unroll
            for (int ph = 0; ph < NPH; ++ph)
                if (ph < P.nPh) F.alpha[ph][c] = (c1 * F.alpha[ph][c] + c2 * F.alpha0[ph][c] + c3 * dt * rA[ph]) / c4;
        }
        if (NPH > 0) mp_post<NPH>(P, F, c);
    } else {
        double pAdv = F.pres[c];
        double r0 = (RK > 1) ? F.rho0[c] : 0.0;
        double ru0 = (RK > 1) ? F.rhoU0[c] : 0.0;
        double re0 = (RK > 1) ? F.rhoE0[c] : 0.0;
        F.rho[c] = (c1 * F.rho[c] + c2 * r0 + c3 * dt * rR) / c4;
        F.rhoUStar[c] = (c1 * F.rhoU[c] + c2 * ru0 + c3 * dt * rU) / c4;
        if (dim >= 2) {
            double rv0 = (RK > 1) ? F.rhoV0[c] : 0.0;
            F.rhoVStar[c] = (c1 * F.rhoV[c] + c2 * rv0 + c3 * dt * rV) / c4;
        }
        if (dim >= 3) {
            double rw0 = (RK > 1) ? F.rhoW0[c] : 0.0;
            F.rhoWStar[c] = (c1 * F.rhoW[c] + c2 * rw0 + c3 * dt * rW) / c4;
        }
        F.rhoEstar[c] = (c1 * F.rhoE[c] + c2 * re0 + c3 * dt * rE) / c4;
        double p0 = (RK > 1) ? F.pres0[c] : 0.0;
        F.pAdvected[c] = (c1 * pAdv + c2 * p0 + c3 * dt * rP) / c4;
        if (NPH > 0) {
            if (RK == 1) {
#pragma unroll
                for (int ph = 0; ph < NPH; ++ph)
                    if (ph < P.nPh) F.alphaRho[ph][c] += dt * rAR[ph];
#pragma unroll
                for (int ph = 0; ph < NPH; ++ph)
                    if (ph < P.nPh) F.alpha[ph][c] += dt * rA[ph];
            } else {
#pragma unroll
                for (int ph = 0; ph < NPH; ++ph)
                    if (ph < P.nPh)
                        F.alphaRho[ph][c] =
                            (c1 * F.alphaRho[ph][c] + c2 * F.alphaRho0[ph][c] + c3 * dt * rAR[ph]) / c4;
#pragma unroll
                for (int ph = 0; ph < NPH; ++ph)
                    if (ph < P.nPh)
                        F.alpha[ph][c] = (c1 * F.alpha[ph][c] + c2 * F.alpha0[ph][c] + c3 * dt * rA[ph]) / c4;
            }
            mp_post<NPH>(P, F, c);
        }
        double rs = smax(F.rho[c], 1e-14);
        F.velU[c] = F.rhoUStar[c] / rs;
        if (dim >= 2) F.velV[c] = F.rhoVStar[c] / rs;
        if (dim >= 3) F.velW[c] = F.rhoWStar[c] / rs;
    }
}

// ---------------------------------------------------------------------------
// Reductions
// ---------------------------------------------------------------------------
// computeAcousticTimeStep (src/RKTimeStepping.cpp:43-123): min over
// interior cells of cfl * min_d d_d / (|u_d| + c).
template <int NPH>
__global__ void __launch_bounds__(256) k_dt_acoustic(Params P, Fields F, Ctl* ctl, double cfl) {
    if (ctl->skip) return;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    double v = __longlong_as_double(0x7ff0000000000000LL);
    if (int_coords(P, t, i, j, k) && !(F.solid && F.solid[cidx(P, i, j, k)])) {   // ibm: solid cells skipped
        const int dim = P.dim;
        size_t c = cidx(P, i, j, k);
        double cs;
        if (NPH > 0) {
            double a[NPH > 0 ? NPH : 1], ar[NPH > 0 ? NPH : 1];
#pragma unroll
            for (int ph = 0; ph < NPH; ++ph) {
                a[ph] = (ph < P.nPh) ? F.alpha[ph][c] : 0.0;
                ar[ph] = (ph < P.nPh) ? F.alphaRho[ph][c] : 0.0;
            }
            cs = mixture_sound_speed<NPH>(P, F.rho[c], F.pres[c], a, ar);
        } else {
            cs = single_sound_speed(P, F.rho[c], F.pres[c]);
        }
        double dtCell = F.dx[i + P.ngx] / (fabs(F.velU[c]) + cs);
        if (dim >= 2) dtCell = smin(dtCell, F.dy[j + P.ngy] / (fabs(F.velV[c]) + cs));
        if (dim >= 3) dtCell = smin(dtCell, F.dz[k + P.ngz] / (fabs(F.velW[c]) + cs));
        v = cfl * dtCell;
    }
    block_min_to(v, &ctl->dtBits);
}

// computeAdvectiveTimeStep (src/RKTimeStepping.cpp:15-41).
__global__ void __launch_bounds__(256) k_dt_advective(Params P, Fields F, Ctl* ctl, double cfl) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    double v = __longlong_as_double(0x7ff0000000000000LL);
    if (int_coords(P, t, i, j, k)) {
        const int dim = P.dim;
        size_t c = cidx(P, i, j, k);
        double dtCell = F.dx[i + P.ngx] / smax(fabs(F.velU[c]), 1e-14);
        if (dim >= 2) dtCell = smin(dtCell, F.dy[j + P.ngy] / smax(fabs(F.velV[c]), 1e-14));
        if (dim >= 3) dtCell = smin(dtCell, F.dz[k + P.ngz] / smax(fabs(F.velW[c]), 1e-14));
        v = cfl * dtCell;
    }
    block_min_to(v, &ctl->dtBits);
}

// computeViscousDt (src/RKTimeStepping.cpp:161-188), folded into the same
// minimum as the acoustic / advective step (std::min of the two).
__global__ void __launch_bounds__(256) k_dt_viscous(Params P, Fields F, Ctl* ctl, double cfl) {
    if (ctl->skip) return;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    double v = __longlong_as_double(0x7ff0000000000000LL);
    if (int_coords(P, t, i, j, k) && !(F.solid && F.solid[cidx(P, i, j, k)])) {   // ibm: solid cells skipped
        const int dim = P.dim;
        size_t c = cidx(P, i, j, k);
        double dxMin = F.dx[i + P.ngx];
        if (dim >= 2) dxMin = smin(dxMin, F.dy[j + P.ngy]);
        if (dim >= 3) dxMin = smin(dxMin, F.dz[k + P.ngz]);
        double nu = P.mu / smax(F.rho[c], 1e-14);
        double dtCell = dxMin * dxMin / (2.0 * dim * nu);
        v = cfl * dtCell;
    }
    block_min_to(v, &ctl->dtBits);
}

// Viscous stress on the faces of direction DIR (src/ViscousFlux.cpp:24-303):
// central normal gradients, transverse gradients averaged over the two
// cells, face viscosity (computeFaceMu, 8-21), face-averaged velocity for the
// work term; stored per face as tau.x, tau.y, tau.z, work.
template <int DIR>
__global__ void __launch_bounds__(256) k_visc_face(Params P, Fields F, const Ctl* __restrict__ ctl) {
    if (ctl && ctl->skip) return;
    const int dim = P.dim;
    const int fnx = P.nx + (DIR == 0), fny = P.ny + (DIR == 1), fnz = P.nz + (DIR == 2);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long tot = (long long)fnx * fny * fnz;
    if (t >= tot) return;
    int i, j, k;
    split3(t, fnx, fny, i, j, k);
    const double* U = F.velU;
    const double* V = F.velV;
    const double* W = F.velW;
    auto at = [&](int a, int b, int c) { return cidx(P, a, b, c); };
    const int li = i - (DIR == 0), lj = j - (DIR == 1), lk = k - (DIR == 2);
    const size_t iL = at(li, lj, lk), iR = at(i, j, k);
    double muF;
    if (!P.perPhaseMu) {
        muF = P.mu;
    } else {
        double muL = 0.0, muR = 0.0;
        for (int ph = 0; ph < P.nPh; ++ph) {
            muL += F.alpha[ph][iL] * P.phaseMu[ph];
            muR += F.alpha[ph][iR] * P.phaseMu[ph];
        }
        muF = 0.5 * (muL + muR);
    }
    double t0, t1, t2, work;
    if (DIR == 0) {
        double dxi = 0.5 * (F.dx[i - 1 + P.ngx] + F.dx[i + P.ngx]);
        double dudx = (U[iR] - U[iL]) / dxi, dvdx = 0.0, dwdx = 0.0;
        if (dim >= 2) dvdx = (V[iR] - V[iL]) / dxi;
        if (dim >= 3) dwdx = (W[iR] - W[iL]) / dxi;
        double dudy = 0.0, dvdy = 0.0;
        if (dim >= 2) {
            double dyj = F.dy[j + P.ngy];
            size_t Ljm = at(i - 1, j - 1, k), Ljp = at(i - 1, j + 1, k), Rjm = at(i, j - 1, k), Rjp = at(i, j + 1, k);
            double dudyL = (U[Ljp] - U[Ljm]) / (2.0 * dyj), dudyR = (U[Rjp] - U[Rjm]) / (2.0 * dyj);
            dudy = 0.5 * (dudyL + dudyR);
            double dvdyL = (V[Ljp] - V[Ljm]) / (2.0 * dyj), dvdyR = (V[Rjp] - V[Rjm]) / (2.0 * dyj);
            dvdy = 0.5 * (dvdyL + dvdyR);
        }
        double dudz = 0.0, dwdz = 0.0;
        if (dim >= 3) {
            double dzk = F.dz[k + P.ngz];
            size_t Lkm = at(i - 1, j, k - 1), Lkp = at(i - 1, j, k + 1), Rkm = at(i, j, k - 1), Rkp = at(i, j, k + 1);
            double dudzL = (U[Lkp] - U[Lkm]) / (2.0 * dzk), dudzR = (U[Rkp] - U[Rkm]) / (2.0 * dzk);
            dudz = 0.5 * (dudzL + dudzR);
            double dwdzL = (W[Lkp] - W[Lkm]) / (2.0 * dzk), dwdzR = (W[Rkp] - W[Rkm]) / (2.0 * dzk);
            dwdz = 0.5 * (dwdzL + dwdzR);
        }
        double divU = dudx + dvdy + dwdz;
        t0 = muF * (2.0 * dudx - (2.0 / 3.0) * divU);
        t1 = muF * (dvdx + dudy);
        t2 = muF * (dwdx + dudz);
        double uF = 0.5 * (U[iL] + U[iR]), vF = 0.0, wF = 0.0;
        if (dim >= 2) vF = 0.5 * (V[iL] + V[iR]);
        if (dim >= 3) wF = 0.5 * (W[iL] + W[iR]);
        work = t0 * uF + t1 * vF + t2 * wF;
    } else if (DIR == 1) {
        double dyj = 0.5 * (F.dy[j - 1 + P.ngy] + F.dy[j + P.ngy]);
        double dudy = (U[iR] - U[iL]) / dyj, dvdy = (V[iR] - V[iL]) / dyj, dwdy = 0.0;
        if (dim >= 3) dwdy = (W[iR] - W[iL]) / dyj;
        double dxi = F.dx[i + P.ngx];
        size_t Lim = at(i - 1, j - 1, k), Lip = at(i + 1, j - 1, k), Rim = at(i - 1, j, k), Rip = at(i + 1, j, k);
        double dudxL = (U[Lip] - U[Lim]) / (2.0 * dxi), dudxR = (U[Rip] - U[Rim]) / (2.0 * dxi);
        double dudx = 0.5 * (dudxL + dudxR);
        double dvdxL = (V[Lip] - V[Lim]) / (2.0 * dxi), dvdxR = (V[Rip] - V[Rim]) / (2.0 * dxi);
        double dvdx = 0.5 * (dvdxL + dvdxR);
        double dvdz = 0.0, dwdz = 0.0;
        if (dim >= 3) {
            double dzk = F.dz[k + P.ngz];
            size_t Lkm = at(i, j - 1, k - 1), Lkp = at(i, j - 1, k + 1), Rkm = at(i, j, k - 1), Rkp = at(i, j, k + 1);
            double dvdzL = (V[Lkp] - V[Lkm]) / (2.0 * dzk), dvdzR = (V[Rkp] - V[Rkm]) / (2.0 * dzk);
            dvdz = 0.5 * (dvdzL + dvdzR);
            double dwdzL = (W[Lkp] - W[Lkm]) / (2.0 * dzk), dwdzR = (W[Rkp] - W[Rkm]) / (2.0 * dzk);
            dwdz = 0.5 * (dwdzL + dwdzR);
        }
        double divU = dudx + dvdy + dwdz;
        t0 = muF * (dudy + dvdx);
        t1 = muF * (2.0 * dvdy - (2.0 / 3.0) * divU);
        t2 = muF * (dwdy + dvdz);
        double uF = 0.5 * (U[iL] + U[iR]), vF = 0.5 * (V[iL] + V[iR]), wF = 0.0;
        if (dim >= 3) wF = 0.5 * (W[iL] + W[iR]);
        work = t0 * uF + t1 * vF + t2 * wF;
    } else {
        double dzk = 0.5 * (F.dz[k - 1 + P.ngz] + F.dz[k + P.ngz]);
        double dudz = (U[iR] - U[iL]) / dzk, dvdz = (V[iR] - V[iL]) / dzk, dwdz = (W[iR] - W[iL]) / dzk;
        double dxi = F.dx[i + P.ngx];
        size_t Lim = at(i - 1, j, k - 1), Lip = at(i + 1, j, k - 1), Rim = at(i - 1, j, k), Rip = at(i + 1, j, k);
        double dudxL = (U[Lip] - U[Lim]) / (2.0 * dxi), dudxR = (U[Rip] - U[Rim]) / (2.0 * dxi);
        double dudx = 0.5 * (dudxL + dudxR);
        double dwdxL = (W[Lip] - W[Lim]) / (2.0 * dxi), dwdxR = (W[Rip] - W[Rim]) / (2.0 * dxi);
        double dwdx = 0.5 * (dwdxL + dwdxR);
        double dyj = F.dy[j + P.ngy];
        size_t Ljm = at(i, j - 1, k - 1), Ljp = at(i, j + 1, k - 1), Rjm = at(i, j - 1, k), Rjp = at(i, j + 1, k);
        double dvdyL = (V[Ljp] - V[Ljm]) / (2.0 * dyj), dvdyR = (V[Rjp] - V[Rjm]) / (2.0 * dyj);
        double dvdy = 0.5 * (dvdyL + dvdyR);
        double dwdyL = (W[Ljp] - W[Ljm]) / (2.0 * dyj), dwdyR = (W[Rjp] - W[Rjm]) / (2.0 * dyj);
        double dwdy = 0.5 * (dwdyL + dwdyR);
        double divU = dudx + dvdy + dwdz;
        t0 = muF * (dudz + dwdx);
        t1 = muF * (dvdz + dwdy);
        t2 = muF * (2.0 * dwdz - (2.0 / 3.0) * divU);
        double uF = 0.5 * (U[iL] + U[iR]), vF = 0.5 * (V[iL] + V[iR]), wF = 0.5 * (W[iL] + W[iR]);
        work = t0 * uF + t1 * vF + t2 * wF;
    }
    double* const* out = F.flux[DIR] + FS_VISC;
    out[0][t] = t0;
    if (dim >= 2) out[1][t] = t1;
    if (dim >= 3) out[2][t] = t2;
    out[3][t] = work;
}

// computeCapillaryDt (src/RKTimeStepping.cpp:201-228), folded into the same
// minimum as the other limits.
__global__ void __launch_bounds__(256) k_dt_capillary(Params P, Fields F, Ctl* ctl, double cfl) {
    if (ctl->skip) return;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    double v = __longlong_as_double(0x7ff0000000000000LL);
    if (int_coords(P, t, i, j, k) && !(F.solid && F.solid[cidx(P, i, j, k)])) {   // ibm: solid cells skipped
        const int dim = P.dim;
        size_t c = cidx(P, i, j, k);
        double dxMin = F.dx[i + P.ngx];
        if (dim >= 2) dxMin = smin(dxMin, F.dy[j + P.ngy]);
        if (dim >= 3) dxMin = smin(dxMin, F.dz[k + P.ngz]);
        double dtCell = sqrt(smax(F.rho[c], 1e-14) * dxMin * dxMin * dxMin / P.stSigma);
        v = cfl * dtCell;
    }
    block_min_to(v, &ctl->dtBits);
}

// Capillary stress T = sigma (|g| I - g g^T / |g|) on the faces of direction
// DIR, g = grad alpha_0 (normal: two-cell difference; transverse: central
// differences averaged over the two cells), |g| floored at epsGradAlpha;
// work T.u with the face-averaged velocity (src/SurfaceTension.cpp:8-254).
// Stored per face as T.x, T.y, T.z, work.
template <int DIR>
__global__ void __launch_bounds__(256) k_cap_face(Params P, Fields F, const Ctl* __restrict__ ctl) {
    if (ctl && ctl->skip) return;
    const int dim = P.dim;
    const int fnx = P.nx + (DIR == 0), fny = P.ny + (DIR == 1), fnz = P.nz + (DIR == 2);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long tot = (long long)fnx * fny * fnz;
    if (t >= tot) return;
    int i, j, k;
    split3(t, fnx, fny, i, j, k);
    const double* a = F.alpha[0];
    auto at = [&](int x, int y, int z) { return a[cidx(P, x, y, z)]; };
    const int li = i - (DIR == 0), lj = j - (DIR == 1), lk = k - (DIR == 2);
    const size_t iL = cidx(P, li, lj, lk), iR = cidx(P, i, j, k);
    const double sigma = P.stSigma;
    double g[3] = {0.0, 0.0, 0.0};
    {   // normal component
        const double* w = (DIR == 0) ? F.dx : (DIR == 1) ? F.dy : F.dz;
        const int q = (DIR == 0) ? i + P.ngx : (DIR == 1) ? j + P.ngy : k + P.ngz;
        g[DIR] = (a[iR] - a[iL]) / (0.5 * (w[q - 1] + w[q]));
    }
    if (DIR != 0) {   // x transverse (dim >= 2 whenever DIR != 0)
        const double d = F.dx[i + P.ngx];
        const double gL = (at(li + 1, lj, lk) - at(li - 1, lj, lk)) / (2.0 * d);
        const double gR = (at(i + 1, j, k) - at(i - 1, j, k)) / (2.0 * d);
        g[0] = 0.5 * (gL + gR);
    }
    if (DIR != 1 && dim >= 2) {
        const double d = F.dy[j + P.ngy];
        const double gL = (at(li, lj + 1, lk) - at(li, lj - 1, lk)) / (2.0 * d);
        const double gR = (at(i, j + 1, k) - at(i, j - 1, k)) / (2.0 * d);
        g[1] = 0.5 * (gL + gR);
    }
    if (DIR != 2 && dim >= 3) {
        const double d = F.dz[k + P.ngz];
        const double gL = (at(li, lj, lk + 1) - at(li, lj, lk - 1)) / (2.0 * d);
        const double gR = (at(i, j, k + 1) - at(i, j, k - 1)) / (2.0 * d);
        g[2] = 0.5 * (gL + gR);
    }
    const double ng = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    const double reg = smax(ng, P.stEps);
    // tangential-plane part on the diagonal, -sigma g_n g_t / |g| off it
    constexpr int T1 = (DIR == 0) ? 1 : 0, T2 = (DIR == 2) ? 1 : 2;
    double T[3];
    T[DIR] = sigma * (g[T1] * g[T1] + g[T2] * g[T2]) / reg;
    T[T1] = -sigma * g[DIR] * g[T1] / reg;
    T[T2] = -sigma * g[DIR] * g[T2] / reg;
    double uF = 0.5 * (F.velU[iL] + F.velU[iR]), vF = 0.0, wF = 0.0;
    if (dim >= 2) vF = 0.5 * (F.velV[iL] + F.velV[iR]);
    if (dim >= 3) wF = 0.5 * (F.velW[iL] + F.velW[iR]);
    const double work = T[0] * uF + T[1] * vF + T[2] * wF;
    double* const* out = F.flux[DIR] + FS_CAP;
    out[0][t] = T[0];
    if (dim >= 2) out[1][t] = T[1];
    if (dim >= 3) out[2][t] = T[2];
    out[3][t] = work;
}

// ImmersedBoundaryMethod::applyGhostCells (src/ImmersedBoundary.cpp:394-470)
// for entry q: stencil-weighted state at the image point, velocity reversed
// (no-slip) or its normal component mirrored (slip), momentum from the
// interpolated density.
template <int NPH>
__device__ void ib_ghost_entry(const Params& P, const Fields& F, const IbDev& G, int q) {
    const int dim = P.dim;
    const int n = G.n[q];
    const long long* cs = G.interp + 8 * (size_t)q;
    const double* ws = G.w + 8 * (size_t)q;
    double r = 0.0, u = 0.0, v = 0.0, w = 0.0, p = 0.0, sg = 0.0, e = 0.0;
    for (int s = 0; s < n; ++s) {
        const size_t c = (size_t)cs[s];
        const double wt = ws[s];
        r += wt * F.rho[c];
        u += wt * F.velU[c];
        if (dim >= 2) v += wt * F.velV[c];
        if (dim >= 3) w += wt * F.velW[c];
        p += wt * F.pres[c];
        sg += wt * F.sigma[c];
        e += wt * F.rhoE[c];
    }
    const size_t idx = (size_t)G.cell[q];
    F.rho[idx] = r;
    F.pres[idx] = p;
    F.sigma[idx] = sg;
    F.rhoE[idx] = e;
    double gu, gv, gw;
    if (G.wall[q] == 0) {
        gu = -u;
        gv = -v;
        gw = -w;
    } else {
        const double* nr = G.normal + 3 * (size_t)q;
        double dot = u * nr[0];
        if (dim >= 2) dot += v * nr[1];
        if (dim >= 3) dot += w * nr[2];
        gu = u - 2.0 * dot * nr[0];
        gv = v - 2.0 * dot * nr[1];
        gw = w - 2.0 * dot * nr[2];
    }
    F.velU[idx] = gu;
    if (dim >= 2) F.velV[idx] = gv;
    if (dim >= 3) F.velW[idx] = gw;
    F.rhoU[idx] = r * gu;
    if (dim >= 2) F.rhoV[idx] = r * gv;
    if (dim >= 3) F.rhoW[idx] = r * gw;
#pragma unroll
    for (int ph = 0; ph < NPH; ++ph) {
        if (ph < P.nPh) {
            double val = 0.0;
            for (int s = 0; s < n; ++s) val += ws[s] * F.alphaRho[ph][cs[s]];
            F.alphaRho[ph][idx] = val;
        }
    }
#pragma unroll
    for (int ph = 0; ph < NPH; ++ph) {
        if (ph < P.nPh) {
            double val = 0.0;
            for (int s = 0; s < n; ++s) val += ws[s] * F.alpha[ph][cs[s]];
            F.alpha[ph][idx] = val;
        }
    }
}

// One thread per ghost entry; one thread for the whole list, in order, when
// a stencil reads another ghost cell (the reference's sequential loop).
template <int NPH>
__global__ void __launch_bounds__(256) k_ib_ghost(Params P, Fields F, IbDev G, const Ctl* __restrict__ ctl) {
    if (ctl && ctl->skip) return;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (G.sequential) {
        if (t == 0)
            for (int q = 0; q < G.count; ++q) ib_ghost_entry<NPH>(P, F, G, q);
        return;
    }
    if (t < G.count) ib_ghost_entry<NPH>(P, F, G, (int)t);
}

// applyScalarGhostCells (src/ImmersedBoundary.cpp:472-482).
__global__ void __launch_bounds__(256) k_ib_scalar(IbDev G, double* __restrict__ f, const Ctl* __restrict__ ctl) {
    if (ctl && ctl->skip) return;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    auto one = [&](int q) {
        const long long* cs = G.interp + 8 * (size_t)q;
        const double* ws = G.w + 8 * (size_t)q;
        double val = 0.0;
        for (int s = 0; s < G.n[q]; ++s) val += ws[s] * f[cs[s]];
        f[G.cell[q]] = val;
    };
    if (G.sequential) {
        if (t == 0)
            for (int q = 0; q < G.count; ++q) one(q);
        return;
    }
    if (t < G.count) one((int)t);
}

// Reset the dt accumulator to maxDt (dt starts at maxDt in the reference).
__global__ void k_dt_init(Ctl* ctl, double maxDt) {
    if (ctl->skip) return;
    ctl->dtBits = d2bits(maxDt);
}

// dt = min(maxDt, reduction); constDt; min with targetDt; semi-implicit
// clamp (src/ExplicitSolver.cpp:72-90, src/SemiImplicitSolver.cpp:110-123).
// useEnd 1: device-resident loop, targetDt = tEnd - time and steps past tEnd
// are skipped.  useEnd 2: runTimeLoop (src/RKTimeStepping.cpp:259-266):
// targetDt also capped at the next output time, and steps after the one
// that reached an output are skipped until the host has handled it.
__global__ void k_dt_finalize(Ctl* ctl, double constDt, double targetDt, int clampSemi, double minDt, double maxDt,
                              int useEnd) {
    if (useEnd) {
        if (ctl->outputDue || !(ctl->time < ctl->tEnd)) {
            ctl->skip = 1;
            return;
        }
        ctl->skip = 0;
        targetDt = ctl->tEnd - ctl->time;
        if (useEnd == 2 && ctl->nextOutput < ctl->tEnd) targetDt = smin(targetDt, ctl->nextOutput - ctl->time);
    }
    double dt = (constDt > 0) ? constDt : bits2d(ctl->dtBits);
    if (targetDt > 0) dt = smin(dt, targetDt);
    if (clampSemi) dt = (dt < minDt) ? minDt : (maxDt < dt) ? maxDt : dt;
    ctl->dt = dt;
}

// time += dt (src/RKTimeStepping.cpp:272-273); with an output interval, the
// output test of runTimeLoop (275-277).  dtLog[slot]: the step's dt, or -1
// for a skipped step.
__global__ void k_time_advance(Ctl* ctl, double* dtLog = nullptr, int slot = 0) {
    if (ctl->skip) {
        if (dtLog) dtLog[slot] = -1.0;
        return;
    }
    ctl->time += ctl->dt;
    ctl->stepsTaken += 1;
    if (dtLog) dtLog[slot] = ctl->dt;
    if (ctl->outInterval > 0.0 && ctl->time >= ctl->nextOutput - 1e-12 * ctl->outInterval) {
        ctl->outputDue = 1;
        ctl->nextOutput += ctl->outInterval;
    }
}

// The host has written the output: steps run again.
__global__ void k_loop_resume(Ctl* ctl) {
    ctl->outputDue = 0;
    ctl->skip = 0;
}

// runTimeLoop's NaN check (src/RKTimeStepping.cpp:280-292): the first
// interior cell in (k, j, i) order with a NaN in rho, rhoU, rhoE, pres, rhoV,
// rhoW (that order within the cell), as min(cell * 8 + field order).
__global__ void __launch_bounds__(256) k_nan_scan(Params P, Fields F, Ctl* ctl) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!int_coords(P, t, i, j, k)) return;
    const size_t c = cidx(P, i, j, k);
    int f = -1;
    if (isnan(F.rho[c])) f = 0;
    else if (isnan(F.rhoU[c])) f = 1;
    else if (isnan(F.rhoE[c])) f = 2;
    else if (isnan(F.pres[c])) f = 3;
    else if (P.dim >= 2 && isnan(F.rhoV[c])) f = 4;
    else if (P.dim >= 3 && isnan(F.rhoW[c])) f = 5;
    if (f < 0) return;
    const unsigned long long lin =
        (unsigned long long)i + (unsigned long long)P.nx * ((unsigned long long)j + (unsigned long long)P.ny * k);
    atomicMin(&ctl->nanCode, lin * 8ull + (unsigned long long)f);
}

// ---------------------------------------------------------------------------
// Semi-implicit pressure: SemiImplicitSolver::solvePressure
// (src/SemiImplicitSolver.cpp:533-588) and computeDivergence (680-717).
// ---------------------------------------------------------------------------
template <int NPH>
__global__ void __launch_bounds__(256) k_pressure_setup(Params P, Fields F, const Ctl* __restrict__ ctl) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!int_coords(P, t, i, j, k)) return;
    const int dim = P.dim;
    size_t c = cidx(P, i, j, k);
    double cs;
    if (NPH > 0) {
        double a[NPH > 0 ? NPH : 1], ar[NPH > 0 ? NPH : 1];
#pragma unroll
        for (int ph = 0; ph < NPH; ++ph) {
            a[ph] = (ph < P.nPh) ? F.alpha[ph][c] : 0.0;
            ar[ph] = (ph < P.nPh) ? F.alphaRho[ph][c] : 0.0;
        }
        cs = mixture_sound_speed<NPH>(P, F.rho[c], F.pres[c], a, ar);
    } else {
        cs = single_sound_speed(P, F.rho[c], F.pres[c]);
    }
    double rhoc2 = F.rho[c] * cs * cs;
    F.rhoc2[c] = rhoc2;
    double div = 0.0;
    {
        size_t xm = c - 1, xp = c + 1;
        double fl = 0.5 * (F.velU[xm] + F.velU[c]);
        double fr = 0.5 * (F.velU[c] + F.velU[xp]);
        div += (fr - fl) / F.dx[i + P.ngx];
    }
    if (dim >= 2) {
        size_t s = (size_t)P.nxT;
        double fl = 0.5 * (F.velV[c - s] + F.velV[c]);
        double fr = 0.5 * (F.velV[c] + F.velV[c + s]);
        div += (fr - fl) / F.dy[j + P.ngy];
    }
    if (dim >= 3) {
        size_t s = (size_t)P.nxT * P.nyT;
        double fl = 0.5 * (F.velW[c - s] + F.velW[c]);
        double fr = 0.5 * (F.velW[c] + F.velW[c + s]);
        div += (fr - fl) / F.dz[k + P.ngz];
    }
    F.divUstar[c] = div;
    F.pRhs[c] = F.pAdvected[c] - rhoc2 * ctl->dt * div;
    F.pA[c] = F.pres[c];
}

// One Jacobi iteration of JacobiPressureSolver::solve
// (src/JacobiPressureSolver.cpp:57-108) with pressureLaplacian
// (src/PressureLaplacian.cpp:6-60).  Ghost pressures are read through the
// scalar ghost map (fillScalarGhosts at the top of every iteration); rho
// ghosts are the stored PRIM ghosts.  Iteration `it` first checks whether
// iteration it-1 converged (max |dp| < tol) and then does nothing, so
// batches of iterations can be queued without a host round trip.
__global__ void __launch_bounds__(256) k_jacobi(Params P, const double* __restrict__ rho,
                                                const double* __restrict__ rhoc2, const double* __restrict__ rhs,
                                                const double* __restrict__ pin, double* __restrict__ pout, Fields F,
                                                Ctl* ctl, int it, double tol) {
    if (ctl->jacobiDone) return;
    if (it > 0 && bits2d(ctl->res[it - 1]) < tol) {
        if (threadIdx.x == 0) ctl->jacobiDone = it;
        return;
    }
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    double res = 0.0;
    if (int_coords(P, t, i, j, k)) {
        const int dim = P.dim;
        const double dt = ctl->dt;
        const double dt2 = dt * dt;
        size_t c = cidx(P, i, j, k);
        double coeff = rhoc2[c] * dt2;
        double od = 0.0, diag = 0.0;
        {
            size_t xm = c - 1, xp = c + 1;
            size_t pxm = scalar_idx(P, i - 1, j, k), pxp = scalar_idx(P, i + 1, j, k);
            double rL = 0.5 * (rho[c] + rho[xm]), rR = 0.5 * (rho[c] + rho[xp]);
            double dm = F.dx[i - 1 + P.ngx], d0 = F.dx[i + P.ngx], dp = F.dx[i + 1 + P.ngx];
            double dL = 0.5 * (dm + d0), dR = 0.5 * (d0 + dp);
            double cL = 1.0 / (smax(rL, 1e-14) * dL * d0);
            double cR = 1.0 / (smax(rR, 1e-14) * dR * d0);
            od += cL * pin[pxm] + cR * pin[pxp];
            diag += cL + cR;
        }
        if (dim >= 2) {
            size_t s = (size_t)P.nxT;
            size_t pym = scalar_idx(P, i, j - 1, k), pyp = scalar_idx(P, i, j + 1, k);
            double rL = 0.5 * (rho[c] + rho[c - s]), rR = 0.5 * (rho[c] + rho[c + s]);
            double dm = F.dy[j - 1 + P.ngy], d0 = F.dy[j + P.ngy], dp = F.dy[j + 1 + P.ngy];
            double dL = 0.5 * (dm + d0), dR = 0.5 * (d0 + dp);
            double cL = 1.0 / (smax(rL, 1e-14) * dL * d0);
            double cR = 1.0 / (smax(rR, 1e-14) * dR * d0);
            od += cL * pin[pym] + cR * pin[pyp];
            diag += cL + cR;
        }
        if (dim >= 3) {
            size_t s = (size_t)P.nxT * P.nyT;
            size_t pzm = scalar_idx(P, i, j, k - 1), pzp = scalar_idx(P, i, j, k + 1);
            double rL = 0.5 * (rho[c] + rho[c - s]), rR = 0.5 * (rho[c] + rho[c + s]);
            double dm = F.dz[k - 1 + P.ngz], d0 = F.dz[k + P.ngz], dp = F.dz[k + 1 + P.ngz];
            double dL = 0.5 * (dm + d0), dR = 0.5 * (d0 + dp);
            double cL = 1.0 / (smax(rL, 1e-14) * dL * d0);
            double cR = 1.0 / (smax(rR, 1e-14) * dR * d0);
            od += cL * pin[pzm] + cR * pin[pzp];
            diag += cL + cR;
        }
        double denom = 1.0 + coeff * diag;
        double pn = (rhs[c] + coeff * od) / denom;
        pout[c] = pn;
        res = fabs(pn - pin[c]);
    }
    block_max_to(res, &ctl->res[it]);
}

// The same Jacobi iteration split in two: k_jacobi_coef evaluates, once per
// solve, every per-cell quantity that does not change between iterations
// (the 2 dim face coefficients c = 1 / (max(rho_f, 1e-14) d_f d_0), the
// scaled coefficient rhoc2 dt^2 and the denominator 1 + coeff * sum c) with
// k_jacobi's expressions; k_jacobi_pre then only gathers the neighbours:
// bit-identical iterates, six divisions less per cell and iteration.
// coef layout: slot q at coef + q * nc, q = 0..2 dim - 1 (x-, x+, y-, y+,
// z-, z+), then coeff, then denom.
__global__ void __launch_bounds__(256) k_jacobi_coef(Params P, const double* __restrict__ rho,
                                                     const double* __restrict__ rhoc2, Fields F, const Ctl* ctl,
                                                     double* __restrict__ coef, size_t nc) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!int_coords(P, t, i, j, k)) return;
    const int dim = P.dim;
    const double dt = ctl->dt;
    const double dt2 = dt * dt;
    size_t c = cidx(P, i, j, k);
    double coeff = rhoc2[c] * dt2;
    double diag = 0.0;
    {
        double rL = 0.5 * (rho[c] + rho[c - 1]), rR = 0.5 * (rho[c] + rho[c + 1]);
        double dm = F.dx[i - 1 + P.ngx], d0 = F.dx[i + P.ngx], dp = F.dx[i + 1 + P.ngx];
        double dL = 0.5 * (dm + d0), dR = 0.5 * (d0 + dp);
        double cL = 1.0 / (smax(rL, 1e-14) * dL * d0);
        double cR = 1.0 / (smax(rR, 1e-14) * dR * d0);
        coef[c] = cL;
        coef[nc + c] = cR;
        diag += cL + cR;
    }
    if (dim >= 2) {
        size_t s = (size_t)P.nxT;
        double rL = 0.5 * (rho[c] + rho[c - s]), rR = 0.5 * (rho[c] + rho[c + s]);
        double dm = F.dy[j - 1 + P.ngy], d0 = F.dy[j + P.ngy], dp = F.dy[j + 1 + P.ngy];
        double dL = 0.5 * (dm + d0), dR = 0.5 * (d0 + dp);
        double cL = 1.0 / (smax(rL, 1e-14) * dL * d0);
        double cR = 1.0 / (smax(rR, 1e-14) * dR * d0);
        coef[2 * nc + c] = cL;
        coef[3 * nc + c] = cR;
        diag += cL + cR;
    }
    if (dim >= 3) {
        size_t s = (size_t)P.nxT * P.nyT;
        double rL = 0.5 * (rho[c] + rho[c - s]), rR = 0.5 * (rho[c] + rho[c + s]);
        double dm = F.dz[k - 1 + P.ngz], d0 = F.dz[k + P.ngz], dp = F.dz[k + 1 + P.ngz];
        double dL = 0.5 * (dm + d0), dR = 0.5 * (d0 + dp);
        double cL = 1.0 / (smax(rL, 1e-14) * dL * d0);
        double cR = 1.0 / (smax(rR, 1e-14) * dR * d0);
        coef[4 * nc + c] = cL;
        coef[5 * nc + c] = cR;
        diag += cL + cR;
    }
    coef[(size_t)(2 * dim) * nc + c] = coeff;
    coef[(size_t)(2 * dim + 1) * nc + c] = 1.0 + coeff * diag;
}

// Neighbour indices of interior cell (i, j, k) for the Jacobi stencil:
// plain strides inside, the scalar ghost map (periodic wrap / zero gradient,
// scalar_src) across the boundary, one axis at a time.
struct JacNb {
    size_t c, xm, xp, ym, yp, zm, zp;
};
__device__ __forceinline__ JacNb jacobi_nb(const Params& P, int i, int j, int k) {
    JacNb n;
    const long long sy = P.nxT, sz = (long long)P.nxT * P.nyT;
    n.c = cidx(P, i, j, k);
    n.xm = n.c + (long long)(scalar_src(i - 1, P.nx, P.bc[0], P.bc[1]) - i);
    n.xp = n.c + (long long)(scalar_src(i + 1, P.nx, P.bc[0], P.bc[1]) - i);
    n.ym = n.yp = n.zm = n.zp = n.c;
    if (P.dim >= 2) {
        n.ym = n.c + (long long)(scalar_src(j - 1, P.ny, P.bc[2], P.bc[3]) - j) * sy;
        n.yp = n.c + (long long)(scalar_src(j + 1, P.ny, P.bc[2], P.bc[3]) - j) * sy;
    }
    if (P.dim >= 3) {
        n.zm = n.c + (long long)(scalar_src(k - 1, P.nz, P.bc[4], P.bc[5]) - k) * sz;
        n.zp = n.c + (long long)(scalar_src(k + 1, P.nz, P.bc[4], P.bc[5]) - k) * sz;
    }
    return n;
}

// One Jacobi update of one interior cell from the per-cell coefficients;
// returns |p_new - p_old|.
__device__ __forceinline__ double jacobi_pre_update(const Params& P, const double* __restrict__ coef, size_t nc,
                                                    const double* __restrict__ rhs, const double* __restrict__ pin,
                                                    double* __restrict__ pout, const JacNb& n) {
    const int dim = P.dim;
    const size_t c = n.c;
    const double* cf = coef + c;
    double od = 0.0;
    od += cf[0] * pin[n.xm] + cf[nc] * pin[n.xp];
    if (dim >= 2) od += cf[2 * nc] * pin[n.ym] + cf[3 * nc] * pin[n.yp];
    if (dim >= 3) od += cf[4 * nc] * pin[n.zm] + cf[5 * nc] * pin[n.zp];
    const double coeff = cf[(size_t)(2 * dim) * nc];
    const double denom = cf[(size_t)(2 * dim + 1) * nc];
    double pn = (rhs[c] + coeff * od) / denom;
    pout[c] = pn;
    return fabs(pn - pin[c]);
}
__device__ __forceinline__ double jacobi_pre_cell(const Params& P, const double* __restrict__ coef, size_t nc,
                                                  const double* __restrict__ rhs, const double* __restrict__ pin,
                                                  double* __restrict__ pout, long long t) {
    int i, j, k;
    split3(t, P.nx, P.ny, i, j, k);
    return jacobi_pre_update(P, coef, nc, rhs, pin, pout, jacobi_nb(P, i, j, k));
}

// Grid-stride Jacobi iteration (a grid of a few blocks per SM, two cells in
// flight per thread): the convergence check, the block reduction and the
// residual atomic run once per block instead of once per 256 cells.  A NaN
// residual counts as 0, as in block_max_to.
__global__ void __launch_bounds__(256) k_jacobi_pre(Params P, const double* __restrict__ coef, size_t nc,
                                                    const double* __restrict__ rhs, const double* __restrict__ pin,
                                                    double* __restrict__ pout, Ctl* ctl, int it, double tol) {
    if (ctl->jacobiDone) return;
    if (it > 0 && bits2d(ctl->res[it - 1]) < tol) {
        if (threadIdx.x == 0) ctl->jacobiDone = it;
        return;
    }
    const long long tot = (long long)P.nx * P.ny * P.nz;
    const long long stride = (long long)gridDim.x * blockDim.x;
    double res = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += 2 * stride) {
        const double r0 = jacobi_pre_cell(P, coef, nc, rhs, pin, pout, t);
        const double r1 = (t + stride < tot) ? jacobi_pre_cell(P, coef, nc, rhs, pin, pout, t + stride) : 0.0;
        res = smax(res, r0);
        res = smax(res, r1);
    }
    block_max_to(res, &ctl->res[it]);
}

// On a mesh whose interior cell widths are equal along an axis, the high-face
// coefficient of a cell equals the low-face coefficient of its neighbour bit
// for bit (the same operands in the same order: 0.5 (rho_i + rho_{i+1}),
// 0.5 (d_i + d_{i+1}), and d_i == d_{i+1}).  k_jacobi_fcoef then stores one
// coefficient per face (the low face of each cell; the high face of the last
// cell at its ghost neighbour's index) and k_jacobi_face rebuilds the
// denominator from them and rho c^2 dt^2 with k_jacobi's expressions: 56
// bytes per cell and iteration instead of 88, bit-identical iterates.
__global__ void __launch_bounds__(256) k_jacobi_fcoef(Params P, const double* __restrict__ rho, Fields F,
                                                      double* __restrict__ fc, size_t nc) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!int_coords(P, t, i, j, k)) return;
    const int dim = P.dim;
    size_t c = cidx(P, i, j, k);
    {
        double rL = 0.5 * (rho[c] + rho[c - 1]);
        double dm = F.dx[i - 1 + P.ngx], d0 = F.dx[i + P.ngx], dp = F.dx[i + 1 + P.ngx];
        double dL = 0.5 * (dm + d0);
        fc[c] = 1.0 / (smax(rL, 1e-14) * dL * d0);
        if (i == P.nx - 1) {
            double rR = 0.5 * (rho[c] + rho[c + 1]);
            double dR = 0.5 * (d0 + dp);
            fc[c + 1] = 1.0 / (smax(rR, 1e-14) * dR * d0);
        }
    }
    if (dim >= 2) {
        size_t s = (size_t)P.nxT;
        double rL = 0.5 * (rho[c] + rho[c - s]);
        double dm = F.dy[j - 1 + P.ngy], d0 = F.dy[j + P.ngy], dp = F.dy[j + 1 + P.ngy];
        double dL = 0.5 * (dm + d0);
        fc[nc + c] = 1.0 / (smax(rL, 1e-14) * dL * d0);
        if (j == P.ny - 1) {
            double rR = 0.5 * (rho[c] + rho[c + s]);
            double dR = 0.5 * (d0 + dp);
            fc[nc + c + s] = 1.0 / (smax(rR, 1e-14) * dR * d0);
        }
    }
    if (dim >= 3) {
        size_t s = (size_t)P.nxT * P.nyT;
        double rL = 0.5 * (rho[c] + rho[c - s]);
        double dm = F.dz[k - 1 + P.ngz], d0 = F.dz[k + P.ngz], dp = F.dz[k + 1 + P.ngz];
        double dL = 0.5 * (dm + d0);
        fc[2 * nc + c] = 1.0 / (smax(rL, 1e-14) * dL * d0);
        if (k == P.nz - 1) {
            double rR = 0.5 * (rho[c] + rho[c + s]);
            double dR = 0.5 * (d0 + dp);
            fc[2 * nc + c + s] = 1.0 / (smax(rR, 1e-14) * dR * d0);
        }
    }
}

__device__ __forceinline__ double jacobi_face_update(const Params& P, const double* __restrict__ fc, size_t nc,
                                                     const double* __restrict__ rhoc2, const double* __restrict__ rhs,
                                                     const double* __restrict__ pin, double* __restrict__ pout,
                                                     double dt2, const JacNb& n) {
    const int dim = P.dim;
    const size_t c = n.c;
    const size_t sy = (size_t)P.nxT, sz = (size_t)P.nxT * P.nyT;
    double coeff = rhoc2[c] * dt2;
    double od = 0.0, diag = 0.0;
    {
        const double cL = fc[c], cR = fc[c + 1];
        od += cL * pin[n.xm] + cR * pin[n.xp];
        diag += cL + cR;
    }
    if (dim >= 2) {
        const double cL = fc[nc + c], cR = fc[nc + c + sy];
        od += cL * pin[n.ym] + cR * pin[n.yp];
        diag += cL + cR;
    }
    if (dim >= 3) {
        const double cL = fc[2 * nc + c], cR = fc[2 * nc + c + sz];
        od += cL * pin[n.zm] + cR * pin[n.zp];
        diag += cL + cR;
    }
    double denom = 1.0 + coeff * diag;
    double pn = (rhs[c] + coeff * od) / denom;
    pout[c] = pn;
    return fabs(pn - pin[c]);
}
__device__ __forceinline__ double jacobi_face_cell(const Params& P, const double* __restrict__ fc, size_t nc,
                                                   const double* __restrict__ rhoc2, const double* __restrict__ rhs,
                                                   const double* __restrict__ pin, double* __restrict__ pout,
                                                   double dt2, long long t) {
    int i, j, k;
    split3(t, P.nx, P.ny, i, j, k);
    return jacobi_face_update(P, fc, nc, rhoc2, rhs, pin, pout, dt2, jacobi_nb(P, i, j, k));
}

// Grid-stride form as k_jacobi_pre.
__global__ void __launch_bounds__(256) k_jacobi_face(Params P, const double* __restrict__ fc, size_t nc,
                                                     const double* __restrict__ rhoc2,
                                                     const double* __restrict__ rhs, const double* __restrict__ pin,
                                                     double* __restrict__ pout, Ctl* ctl, int it, double tol) {
    if (ctl->jacobiDone) return;
    if (it > 0 && bits2d(ctl->res[it - 1]) < tol) {
        if (threadIdx.x == 0) ctl->jacobiDone = it;
        return;
    }
    const double dt = ctl->dt;
    const double dt2 = dt * dt;
    const long long tot = (long long)P.nx * P.ny * P.nz;
    const long long stride = (long long)gridDim.x * blockDim.x;
    double res = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += 2 * stride) {
        const double r0 = jacobi_face_cell(P, fc, nc, rhoc2, rhs, pin, pout, dt2, t);
        const double r1 = (t + stride < tot) ? jacobi_face_cell(P, fc, nc, rhoc2, rhs, pin, pout, dt2, t + stride)
                                             : 0.0;
        res = smax(res, r0);
        res = smax(res, r1);
    }
    block_max_to(res, &ctl->res[it]);
}

// 3D Jacobi iteration: 32 x 8 blocks of (x, y) columns, each thread walking
// kJacZ cells along z (no index division; the ghost remap per axis only
// where a neighbour leaves the domain).  FACE selects the per-face
// (k_jacobi_face) or per-cell (k_jacobi_pre) coefficients, with their update
// expressions in their order.  The inputs of the next cell of the column are
// loaded before the current cell is computed, so that their memory latency
// overlaps the division.
constexpr int kJacZ = 32;   // 16: 1 % slower at 256^3, 64: 11 % slower
struct JacIn {
    double rc, rh, dn, pc, pxm, pxp, pym, pyp, pzm, pzp, c0, c1, c2, c3, c4, c5;
};
template <bool FACE>
__device__ __forceinline__ JacIn jacobi3_load(const Params& P, const double* __restrict__ coef, size_t nc,
                                              const double* __restrict__ rhoc2, const double* __restrict__ rhs,
                                              const double* __restrict__ pin, const JacNb& n) {
    JacIn v;
    const size_t c = n.c;
    const size_t sy = (size_t)P.nxT, sz = (size_t)P.nxT * P.nyT;
    v.rh = rhs[c];
    v.pc = pin[c];
    v.pxm = pin[n.xm];
    v.pxp = pin[n.xp];
    v.pym = pin[n.ym];
    v.pyp = pin[n.yp];
    v.pzm = pin[n.zm];
    v.pzp = pin[n.zp];
    if (FACE) {
        v.rc = rhoc2[c];
        v.dn = 0.0;
        v.c0 = coef[c];
        v.c1 = coef[c + 1];
        v.c2 = coef[nc + c];
        v.c3 = coef[nc + c + sy];
        v.c4 = coef[2 * nc + c];
        v.c5 = coef[2 * nc + c + sz];
    } else {
        const double* cf = coef + c;
        v.c0 = cf[0];
        v.c1 = cf[nc];
        v.c2 = cf[2 * nc];
        v.c3 = cf[3 * nc];
        v.c4 = cf[4 * nc];
        v.c5 = cf[5 * nc];
        v.rc = cf[6 * nc];
        v.dn = cf[7 * nc];
    }
    return v;
}
template <bool FACE>
__device__ __forceinline__ double jacobi3_new(const JacIn& v, double dt2) {
    if (FACE) {   // jacobi_face_update, dim 3
        double coeff = v.rc * dt2;
        double od = 0.0, diag = 0.0;
        od += v.c0 * v.pxm + v.c1 * v.pxp;
        diag += v.c0 + v.c1;
        od += v.c2 * v.pym + v.c3 * v.pyp;
        diag += v.c2 + v.c3;
        od += v.c4 * v.pzm + v.c5 * v.pzp;
        diag += v.c4 + v.c5;
        double denom = 1.0 + coeff * diag;
        return (v.rh + coeff * od) / denom;
    }
    double od = 0.0;   // jacobi_pre_update, dim 3
    od += v.c0 * v.pxm + v.c1 * v.pxp;
    od += v.c2 * v.pym + v.c3 * v.pyp;
    od += v.c4 * v.pzm + v.c5 * v.pzp;
    return (v.rh + v.rc * od) / v.dn;
}
template <bool FACE>
__global__ void __launch_bounds__(256, 3) k_jacobi3(Params P, const double* __restrict__ coef, size_t nc,
                                                 const double* __restrict__ rhoc2, const double* __restrict__ rhs,
                                                 const double* __restrict__ pin, double* __restrict__ pout, Ctl* ctl,
                                                 int it, double tol) {
    if (ctl->jacobiDone) return;
    if (it > 0 && bits2d(ctl->res[it - 1]) < tol) {
        if (threadIdx.x == 0) ctl->jacobiDone = it;
        return;
    }
    const int i = (int)blockIdx.x * 32 + (int)(threadIdx.x & 31);
    const int j = (int)blockIdx.y * 8 + (int)(threadIdx.x >> 5);
    const int k0 = (int)blockIdx.z * kJacZ;
    double res = 0.0;
    if (i < P.nx && j < P.ny) {
        const double dt = ctl->dt;
        const double dt2 = dt * dt;
        const int k1 = min(k0 + kJacZ, P.nz);
        JacNb n = jacobi_nb(P, i, j, k0);
        JacIn v = jacobi3_load<FACE>(P, coef, nc, rhoc2, rhs, pin, n);
        for (int k = k0; k < k1; ++k) {
            const size_t c = n.c;
            const JacIn cur = v;
            if (k + 1 < k1) {
                n = jacobi_nb(P, i, j, k + 1);
                v = jacobi3_load<FACE>(P, coef, nc, rhoc2, rhs, pin, n);
            }
            const double pn = jacobi3_new<FACE>(cur, dt2);
            pout[c] = pn;
            res = smax(res, fabs(pn - cur.pc));
        }
    }
    block_max_to(res, &ctl->res[it]);
}

// Copy the converged Jacobi iterate (in pA or pB by parity) to dst.
__global__ void k_jacobi_finish(Params P, const double* __restrict__ pA, const double* __restrict__ pB,
                                double* __restrict__ dst, const Ctl* __restrict__ ctl, int maxIter) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!int_coords(P, t, i, j, k)) return;
    int n = ctl->jacobiDone ? ctl->jacobiDone : maxIter;
    const double* src = (n & 1) ? pB : pA;
    size_t c = cidx(P, i, j, k);
    dst[c] = src[c];
}

// ---------------------------------------------------------------------------
// Mixed-precision Jacobi (SIFV_PREC_MIXED, semi-implicit): FP32 inner sweeps
// inside FP64 iterative refinement.  m Jacobi iterations from p are
// p + e_m with e_0 = 0, e_{k+1} = delta + J e_k, delta = D^-1 (b - A p) the
// FP64 Jacobi change at p and J = D^-1 (off-diagonal part); the e sweeps run
// in FP32 on FP32 weights, then p += e in FP64 and delta is re-evaluated in
// FP64, which removes the FP32 error each batch.  The change |e_{k+1} - e_k|
// of a sweep is the Jacobi change of that iteration, so the stopping rule
// (max change < tol) and the iteration count are the reference's
// (src/JacobiPressureSolver.cpp:57-108) up to FP32 rounding of the change.
// Compact arrays (interior cells, x fastest); weights w[q * n + t] for the
// faces x-, x+, y-, y+, z-, z+.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_mx_weights(Params P, const double* __restrict__ coef, size_t nc,
                                                    float* __restrict__ w, long long n) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!int_coords(P, t, i, j, k)) return;
    const size_t c = cidx(P, i, j, k);
    const int nq = 2 * P.dim;
    const double coeff = coef[(size_t)nq * nc + c], denom = coef[(size_t)(nq + 1) * nc + c];
    for (int q = 0; q < nq; ++q) w[q * n + t] = (float)(coeff * coef[q * nc + c] / denom);
}

// FP64 Jacobi change at p (k_jacobi_pre's expressions): delta = p_new - p;
// e = delta (the first sweep of the batch), max |delta| -> res[it].
__global__ void __launch_bounds__(256) k_mx_delta(Params P, const double* __restrict__ coef, size_t nc,
                                                  const double* __restrict__ rhs, const double* __restrict__ pin,
                                                  float* __restrict__ d32, float* __restrict__ e, Ctl* ctl, int it) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    double res = 0.0;
    if (int_coords(P, t, i, j, k)) {
        const int dim = P.dim;
        const size_t c = cidx(P, i, j, k);
        const size_t xm = scalar_idx(P, i - 1, j, k), xp = scalar_idx(P, i + 1, j, k);
        const double* cf = coef + c;
        double od = 0.0;
        od += cf[0] * pin[xm] + cf[nc] * pin[xp];
        if (dim >= 2) od += cf[2 * nc] * pin[scalar_idx(P, i, j - 1, k)] + cf[3 * nc] * pin[scalar_idx(P, i, j + 1, k)];
        if (dim >= 3) od += cf[4 * nc] * pin[scalar_idx(P, i, j, k - 1)] + cf[5 * nc] * pin[scalar_idx(P, i, j, k + 1)];
        const double coeff = cf[(size_t)(2 * dim) * nc];
        const double denom = cf[(size_t)(2 * dim + 1) * nc];
        const double dl = (rhs[c] + coeff * od) / denom - pin[c];
        d32[t] = (float)dl;
        e[t] = (float)dl;
        res = fabs(dl);
    }
    block_max_to(res, &ctl->res[it]);
}

// compact neighbour of interior cell (i, j, k) along an axis under the scalar
// ghost map (periodic wrap, else the boundary cell itself)
__device__ __forceinline__ long long mx_nb(const Params& P, int i, int j, int k, int axis, int side) {
    int q[3] = {i, j, k};
    const int n[3] = {P.nx, P.ny, P.nz};
    int v = q[axis] + side;
    if (v < 0) v = (P.bc[2 * axis] == SIFV_BC_PERIODIC) ? n[axis] - 1 : 0;
    else if (v >= n[axis]) v = (P.bc[2 * axis + 1] == SIFV_BC_PERIODIC) ? 0 : n[axis] - 1;
    q[axis] = v;
    return q[0] + (long long)P.nx * (q[1] + (long long)P.ny * q[2]);
}

// One FP32 sweep e_out = delta + J e_in, iteration `it` of the count; a no-op
// once an earlier iteration's change fell below tol (as k_jacobi_pre), and
// grid-stride with two cells in flight per thread as k_jacobi_pre.
__device__ __forceinline__ double mx_sweep_update(const Params& P, const float* __restrict__ w,
                                                  const float* __restrict__ d32, const float* __restrict__ ein,
                                                  float* __restrict__ eout, long long n, long long t, long long xm,
                                                  long long xp, long long ym, long long yp, long long zm,
                                                  long long zp) {
    float od = w[t] * ein[xm] + w[n + t] * ein[xp];
    if (P.dim >= 2) od += w[2 * n + t] * ein[ym] + w[3 * n + t] * ein[yp];
    if (P.dim >= 3) od += w[4 * n + t] * ein[zm] + w[5 * n + t] * ein[zp];
    const float en = d32[t] + od;
    eout[t] = en;
    return (double)fabsf(en - ein[t]);
}
__device__ __forceinline__ double mx_sweep_cell(const Params& P, const float* __restrict__ w,
                                                const float* __restrict__ d32, const float* __restrict__ ein,
                                                float* __restrict__ eout, long long n, long long t) {
    int i, j, k;
    split3(t, P.nx, P.ny, i, j, k);
    return mx_sweep_update(P, w, d32, ein, eout, n, t, mx_nb(P, i, j, k, 0, -1), mx_nb(P, i, j, k, 0, 1),
                           P.dim >= 2 ? mx_nb(P, i, j, k, 1, -1) : t, P.dim >= 2 ? mx_nb(P, i, j, k, 1, 1) : t,
                           P.dim >= 3 ? mx_nb(P, i, j, k, 2, -1) : t, P.dim >= 3 ? mx_nb(P, i, j, k, 2, 1) : t);
}
__global__ void __launch_bounds__(256) k_mx_sweep(Params P, const float* __restrict__ w, const float* __restrict__ d32,
                                                  const float* __restrict__ ein, float* __restrict__ eout, Ctl* ctl,
                                                  int it, double tol) {
    if (ctl->jacobiDone) return;
    if (it > 0 && bits2d(ctl->res[it - 1]) < tol) {
        if (threadIdx.x == 0) ctl->jacobiDone = it;
        return;
    }
    const long long n = (long long)P.nx * P.ny * P.nz;
    const long long stride = (long long)gridDim.x * blockDim.x;
    double res = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += 2 * stride) {
        const double r0 = mx_sweep_cell(P, w, d32, ein, eout, n, t);
        const double r1 = (t + stride < n) ? mx_sweep_cell(P, w, d32, ein, eout, n, t + stride) : 0.0;
        res = smax(res, r0);
        res = smax(res, r1);
    }
    block_max_to(res, &ctl->res[it]);
}

// 3D form of k_mx_sweep: the column walk of k_jacobi3 (interior indexing,
// mx_nb's wrap / clamp per axis only where a neighbour leaves the domain,
// the next cell's inputs in flight while the current one is computed).
__global__ void __launch_bounds__(256) k_mx_sweep3(Params P, const float* __restrict__ w,
                                                   const float* __restrict__ d32, const float* __restrict__ ein,
                                                   float* __restrict__ eout, Ctl* ctl, int it, double tol) {
    if (ctl->jacobiDone) return;
    if (it > 0 && bits2d(ctl->res[it - 1]) < tol) {
        if (threadIdx.x == 0) ctl->jacobiDone = it;
        return;
    }
    const int i = (int)blockIdx.x * 32 + (int)(threadIdx.x & 31);
    const int j = (int)blockIdx.y * 8 + (int)(threadIdx.x >> 5);
    const int k0 = (int)blockIdx.z * kJacZ;
    double res = 0.0;
    if (i < P.nx && j < P.ny) {
        const long long n = (long long)P.nx * P.ny * P.nz;
        const long long sy = P.nx, sz = (long long)P.nx * P.ny;
        const long long dxm = scalar_src(i - 1, P.nx, P.bc[0], P.bc[1]) - i;
        const long long dxp = scalar_src(i + 1, P.nx, P.bc[0], P.bc[1]) - i;
        const long long dym = (scalar_src(j - 1, P.ny, P.bc[2], P.bc[3]) - j) * sy;
        const long long dyp = (scalar_src(j + 1, P.ny, P.bc[2], P.bc[3]) - j) * sy;
        const int k1 = min(k0 + kJacZ, P.nz);
        // inputs of the next cell loaded before the current one is computed;
        // the arithmetic is mx_sweep_update's (dim 3)
        float v[14];
        auto load = [&](int k) {
            const long long t = i + sy * j + sz * k;
            const long long zm = t + (scalar_src(k - 1, P.nz, P.bc[4], P.bc[5]) - k) * sz;
            const long long zp = t + (scalar_src(k + 1, P.nz, P.bc[4], P.bc[5]) - k) * sz;
            v[0] = w[t]; v[1] = ein[t + dxm]; v[2] = w[n + t]; v[3] = ein[t + dxp];
            v[4] = w[2 * n + t]; v[5] = ein[t + dym]; v[6] = w[3 * n + t]; v[7] = ein[t + dyp];
            v[8] = w[4 * n + t]; v[9] = ein[zm]; v[10] = w[5 * n + t]; v[11] = ein[zp];
            v[12] = d32[t]; v[13] = ein[t];
        };
        load(k0);
        for (int k = k0; k < k1; ++k) {
            float u[14];
#pragma unroll
            for (int q = 0; q < 14; ++q) u[q] = v[q];
            if (k + 1 < k1) load(k + 1);
            float od = u[0] * u[1] + u[2] * u[3];
            od += u[4] * u[5] + u[6] * u[7];
            od += u[8] * u[9] + u[10] * u[11];
            const float en = u[12] + od;
            eout[i + sy * j + sz * k] = en;
            res = smax(res, (double)fabsf(en - u[13]));
        }
    }
    block_max_to(res, &ctl->res[it]);
}

// p += e (interior cells of the ghosted FP64 array)
__global__ void __launch_bounds__(256) k_mx_apply(Params P, const float* __restrict__ e, double* __restrict__ p) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!int_coords(P, t, i, j, k)) return;
    p[cidx(P, i, j, k)] += (double)e[t];
}

// SemiImplicitSolver::correctionStep (src/SemiImplicitSolver.cpp:590-678),
// all per-cell parts fused: momentum from the face-averaged gradient of
// p + sigma (scalar-ghost-filled), velocities, pres = p, and total energy
// from the EOS.  The PRIM ghost fill that follows is k_bc_prim.
template <int NPH>
__global__ void __launch_bounds__(256) k_correction(Params P, Fields F, const double* __restrict__ Pn,
                                                    const Ctl* __restrict__ ctl) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!int_coords(P, t, i, j, k)) return;
    const int dim = P.dim;
    const double dt = ctl->dt;
    size_t c = cidx(P, i, j, k);
    const double* S = F.sigma;
    double pc = Pn[c] + S[c];
    {
        size_t m = scalar_idx(P, i - 1, j, k), p = scalar_idx(P, i + 1, j, k);
        double pTotL = 0.5 * ((Pn[m] + S[m]) + pc);
        double pTotR = 0.5 * (pc + (Pn[p] + S[p]));
        F.rhoU[c] = F.rhoUStar[c] - dt * (pTotR - pTotL) / F.dx[i + P.ngx];
    }
    if (dim >= 2) {
        size_t m = scalar_idx(P, i, j - 1, k), p = scalar_idx(P, i, j + 1, k);
        double pTotL = 0.5 * ((Pn[m] + S[m]) + pc);
        double pTotR = 0.5 * (pc + (Pn[p] + S[p]));
        F.rhoV[c] = F.rhoVStar[c] - dt * (pTotR - pTotL) / F.dy[j + P.ngy];
    }
    if (dim >= 3) {
        size_t m = scalar_idx(P, i, j, k - 1), p = scalar_idx(P, i, j, k + 1);
        double pTotL = 0.5 * ((Pn[m] + S[m]) + pc);
        double pTotR = 0.5 * (pc + (Pn[p] + S[p]));
        F.rhoW[c] = F.rhoWStar[c] - dt * (pTotR - pTotL) / F.dz[k + P.ngz];
    }
    double rho = F.rho[c];
    double rs = smax(rho, 1e-14);
    double u = F.rhoU[c] / rs;
    double v = (dim >= 2) ? F.rhoV[c] / rs : 0.0;
    double w = (dim >= 3) ? F.rhoW[c] / rs : 0.0;
    F.velU[c] = u;
    if (dim >= 2) F.velV[c] = v;
    if (dim >= 3) F.velW[c] = w;
    double pn = Pn[c];
    F.pres[c] = pn;
    double ke = 0.5 * rho * u * u;
    if (dim >= 2) ke += 0.5 * rho * v * v;
    if (dim >= 3) ke += 0.5 * rho * w * w;
    if (NPH > 0) {
        double a[NPH > 0 ? NPH : 1];
#pragma unroll
        for (int ph = 0; ph < NPH; ++ph) a[ph] = (ph < P.nPh) ? F.alpha[ph][c] : 0.0;
        F.rhoE[c] = mixture_total_energy<NPH>(P, pn, a, ke);
    } else {
        F.rhoE[c] = (pn + P.gamma * P.pInf) / (P.gamma - 1.0) + ke;
    }
}

// ---------------------------------------------------------------------------
// IGR (src/IGR.cpp)
// ---------------------------------------------------------------------------
// Velocity gradient (IGRSolver::computeVelocityGradient, src/IGR.cpp:160-200),
// RHS alpha (tr(gu gu) + tr(gu)^2) (computeIGRRhs, 18-35) and the diagonal
// 1/rho + sum alpha/d^2 (1/rho_fl + 1/rho_fr) of the sweep (114-142), which
// do not change across sweeps.
__global__ void __launch_bounds__(256) k_igr_setup(Params P, Fields F, double alpha) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!int_coords(P, t, i, j, k)) return;
    const int dim = P.dim;
    size_t c = cidx(P, i, j, k);
    const size_t sy = (size_t)P.nxT, sz = (size_t)P.nxT * P.nyT;
    double g[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) g[q] = 0.0;
    double invDx = 0.5 / F.dx[i + P.ngx];
    double invDy = 0.5 / ((dim >= 2) ? F.dy[j + P.ngy] : 1.0);
    double invDz = 0.5 / ((dim >= 3) ? F.dz[k + P.ngz] : 1.0);
    g[0] = (F.velU[c + 1] - F.velU[c - 1]) * invDx;
    if (dim >= 2) {
        g[3] = (F.velV[c + 1] - F.velV[c - 1]) * invDx;
        g[1] = (F.velU[c + sy] - F.velU[c - sy]) * invDy;
        g[4] = (F.velV[c + sy] - F.velV[c - sy]) * invDy;
        if (dim >= 3) {
            g[7] = (F.velW[c + sy] - F.velW[c - sy]) * invDy;
            g[6] = (F.velW[c + 1] - F.velW[c - 1]) * invDx;
            g[2] = (F.velU[c + sz] - F.velU[c - sz]) * invDz;
            g[5] = (F.velV[c + sz] - F.velV[c - sz]) * invDz;
            g[8] = (F.velW[c + sz] - F.velW[c - sz]) * invDz;
        }
    }
    double trSq = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
            if (a < dim && b < dim) trSq += g[3 * a + b] * g[3 * b + a];
    double tr = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
        if (a < dim) tr += g[4 * a];
    tr *= tr;
    F.igrRhs[c] = alpha * (trSq + tr);

    double rho_i = F.rho[c];
    double diag = 1.0 / rho_i;
    {
        double rfl = 0.5 * (rho_i + F.rho[c - 1]), rfr = 0.5 * (rho_i + F.rho[c + 1]);
        diag += F.adx2[i + P.ngx] * (1.0 / rfl + 1.0 / rfr);
    }
    if (dim >= 2) {
        double rfl = 0.5 * (rho_i + F.rho[c - sy]), rfr = 0.5 * (rho_i + F.rho[c + sy]);
        diag += F.ady2[j + P.ngy] * (1.0 / rfl + 1.0 / rfr);
    }
    if (dim >= 3) {
        double rfl = 0.5 * (rho_i + F.rho[c - sz]), rfr = 0.5 * (rho_i + F.rho[c + sz]);
        diag += F.adz2[k + P.ngz] * (1.0 / rfl + 1.0 / rfr);
    }
    F.igrDiag[c] = diag;
}

__device__ __forceinline__ void igr_cell(const Params& P, const Fields& F, int i, int j, int k) {
    const int dim = P.dim;
    size_t c = cidx(P, i, j, k);
    if (F.solid && F.solid[c]) return;   // solid cells keep sigma (src/IGR.cpp:51)
    const size_t sy = (size_t)P.nxT, sz = (size_t)P.nxT * P.nyT;
    double* S = F.sigma;
    double rho_i = F.rho[c];
    double off = 0.0;
    {
        double rfl = 0.5 * (rho_i + F.rho[c - 1]), rfr = 0.5 * (rho_i + F.rho[c + 1]);
        off += F.adx2[i + P.ngx] * (S[c - 1] / rfl + S[c + 1] / rfr);
    }
    if (dim >= 2) {
        double rfl = 0.5 * (rho_i + F.rho[c - sy]), rfr = 0.5 * (rho_i + F.rho[c + sy]);
        off += F.ady2[j + P.ngy] * (S[c - sy] / rfl + S[c + sy] / rfr);
    }
    if (dim >= 3) {
        double rfl = 0.5 * (rho_i + F.rho[c - sz]), rfr = 0.5 * (rho_i + F.rho[c + sz]);
        off += F.adz2[k + P.ngz] * (S[c - sz] / rfl + S[c + sz] / rfr);
    }
    S[c] = (F.igrRhs[c] + off) / F.igrDiag[c];
}

// 1D sweep: a single thread walks the line in order.
__global__ void k_igr_sweep_1d(Params P, Fields F) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = 0; i < P.nx; ++i) igr_cell(P, F, i, 0, 0);
}

// 8-byte asynchronous global -> shared copy (cp.async, L1-allocating) and
// the wait for all of this thread's outstanding copies.
__device__ __forceinline__ void cp_async8(double* smemDst, const double* gmemSrc) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smemDst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gmemSrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Sweeps of one IGR solve overlapped in one launch sequence (k_igr_tile,
// k_igr_tile_rec): the tile plane of each active sweep, and whether the
// boundary tiles refresh the scalar ghost layer themselves.
struct IgrPlanes {
    int top;      // tile plane of the first active sweep; sweep slot u runs plane top - u lag
    int lag;      // planes between consecutive sweeps
    int n;        // active sweeps (blocks: n x nty x ntz)
    int ghosts;   // boundary tiles refresh the scalar ghosts
};

__device__ __forceinline__ void igr_tile_ghosts(const Params& P, double* sigma, int I, int J, int K, int ntx,
                                                int nty, int ntz, int i0, int j0, int k0, int ex, int ey, int ez) {
    const int nt = (int)blockDim.x;
    const size_t sy = (size_t)P.nxT, sz = (size_t)P.nxT * P.nyT;
    // x faces: the tile's (y, z) rows
    {
        const bool per = P.bc[0] == SIFV_BC_PERIODIC;
        for (int w = (int)threadIdx.x; w < ey * ez; w += nt) {
            const int b = w % ey, c = w / ey;
            const size_t row = cidx(P, 0, j0 + b, k0 + c);
            if (!per && I == 0 && P.bc[0] != SIFV_BC_EXCHANGE) sigma[row - 1] = sigma[row];
            if (!per && I == ntx - 1 && P.bc[1] != SIFV_BC_EXCHANGE) sigma[row + P.nx] = sigma[row + P.nx - 1];
            if (per && I == ntx - 1) {
                sigma[row - 1] = sigma[row + P.nx - 1];
                sigma[row + P.nx] = sigma[row];
            }
        }
    }
    // y faces: the tile's (x, z) columns
    if (P.dim >= 2) {
        const bool per = P.bc[2] == SIFV_BC_PERIODIC;
        const size_t hi = (size_t)P.ny * sy;
        for (int w = (int)threadIdx.x; w < ex * ez; w += nt) {
            const int a = w % ex, c = w / ex;
            const size_t col = cidx(P, i0 + a, 0, k0 + c);
            if (!per && J == 0 && P.bc[2] != SIFV_BC_EXCHANGE) sigma[col - sy] = sigma[col];
            if (!per && J == nty - 1 && P.bc[3] != SIFV_BC_EXCHANGE) sigma[col + hi] = sigma[col + hi - sy];
            if (per && J == nty - 1) {
                sigma[col - sy] = sigma[col + hi - sy];
                sigma[col + hi] = sigma[col];
            }
        }
    }
    // z faces: the tile's (x, y) columns
    if (P.dim >= 3) {
        const bool per = P.bc[4] == SIFV_BC_PERIODIC;
        const size_t hi = (size_t)P.nz * sz;
        for (int w = (int)threadIdx.x; w < ex * ey; w += nt) {
            const int a = w % ex, b = w / ex;
            const size_t col = cidx(P, i0 + a, j0 + b, 0);
            if (!per && K == 0 && P.bc[4] != SIFV_BC_EXCHANGE) sigma[col - sz] = sigma[col];
            if (!per && K == ntz - 1 && P.bc[5] != SIFV_BC_EXCHANGE) sigma[col + hi] = sigma[col + hi - sz];
            if (per && K == ntz - 1) {
                sigma[col - sz] = sigma[col + hi - sz];
                sigma[col + hi] = sigma[col];
            }
        }
    }
}

// Tiled wavefront of the same lexicographic sweep.  The domain is cut into
// TX x TY x TZ tiles; tile (I, J, K) only reads cells of tiles (I-1, J, K),
// (I, J-1, K), (I, J, K-1) (already updated in this sweep) and of
// (I+1, J, K), (I, J+1, K), (I, J, K+1) (not yet updated), so the tiles of
// one tile plane I + J + K = plane are independent and run as the blocks of
// one launch.  Inside a tile the block walks the anti-diagonal cell planes
// a + b + c = q in order (one __syncthreads per plane) on a shared-memory
// copy of sigma and rho with a one-cell halo, and of the rhs and diagonal;
// every cell is updated with igr_cell's arithmetic in igr_cell's order, so
// the result is bit-identical to the lexicographic sweep.
// Dynamic shared memory: (2 (TX+2)(TY+2)(TZ+2 or 1) + 2 TX TY TZ) doubles.
// Several sweeps overlap as in k_igr_tile_rec (IgrPlanes; boundary tiles
// refresh the ghost layer at their end).
template <int TX, int TY, int TZ>
__global__ void __launch_bounds__(TY * TZ) k_igr_tile(Params P, Fields F, IgrPlanes PL, int ntx, int nty, int ntz) {
    extern __shared__ double smem[];
    constexpr int D3 = (TZ > 1) ? 1 : 0;
    constexpr int HX = TX + 2, HY = TY + 2, HZ = D3 ? TZ + 2 : 1;
    constexpr int HN = HX * HY * HZ, TN = TX * TY * TZ;
    double* sS = smem;
    double* sR = smem + HN;
    double* sRhs = smem + 2 * HN;
    double* sDiag = sRhs + TN;
    double* sAx = sDiag + TN;   // alpha / dx^2 of the tile's columns (no global load inside the wavefront)
    const unsigned perSlot = (unsigned)(nty * ntz);
    const int slot = (int)(blockIdx.x / perSlot);
    const unsigned bt = blockIdx.x % perSlot;
    const int J = (int)(bt % (unsigned)nty), K = (int)(bt / (unsigned)nty);
    const int I = PL.top - slot * PL.lag - J - K;
    if (I < 0 || I >= ntx) return;
    const int i0 = I * TX, j0 = J * TY, k0 = K * TZ;
    const int ex = min(TX, P.nx - i0), ey = min(TY, P.ny - j0), ez = D3 ? min(TZ, P.nz - k0) : 1;
    const int hx = ex + 2, hy = ey + 2, hz = D3 ? ez + 2 : 1;
    // Staging: one warp per x-line (lanes along x, coalesced), copied with
    // cp.async so that every line's loads are in flight together.
    const int lane = (int)threadIdx.x & 31, warp = (int)threadIdx.x >> 5, nwarp = (int)blockDim.x >> 5;
    for (int line = warp; line < hy * hz; line += nwarp) {
        const int b = line % hy, c = line / hy;
        for (int a = lane; a < hx; a += 32) {
            const size_t g = cidx(P, i0 + a - 1, j0 + b - 1, D3 ? k0 + c - 1 : k0);
            const int h = (c * HY + b) * HX + a;
            cp_async8(&sS[h], &F.sigma[g]);
            cp_async8(&sR[h], &F.rho[g]);
        }
    }
    for (int line = warp; line < ey * ez; line += nwarp) {
        const int b = line % ey, c = line / ey;
        for (int a = lane; a < ex; a += 32) {
            const size_t g = cidx(P, i0 + a, j0 + b, k0 + c);
            const int l = (c * TY + b) * TX + a;
            cp_async8(&sRhs[l], &F.igrRhs[g]);
            cp_async8(&sDiag[l], &F.igrDiag[g]);
        }
    }
    for (int a = threadIdx.x; a < ex; a += blockDim.x) cp_async8(&sAx[a], &F.adx2[i0 + a + P.ngx]);
    cp_async_wait_all();
    // thread (tb, tc) owns the x-line (., tb, tc) of the tile and updates
    // its cell a = q - tb - tc at cell plane q
    const int tb = (int)threadIdx.x % TY, tc = (int)threadIdx.x / TY;
    const bool act = tb < ey && tc < ez;
    const double ady = act ? F.ady2[j0 + tb + P.ngy] : 0.0;
    const double adz = (act && D3) ? F.adz2[k0 + tc + P.ngz] : 0.0;
    const int hLine = ((tc + D3) * HY + (tb + 1)) * HX + 1;
    const int lLine = (tc * TY + tb) * TX;
    __syncthreads();
    const int nq = ex + ey + ez - 2;
    for (int q = 0; q < nq; ++q) {
        const int a = q - tb - tc;
        if (act && a >= 0 && a < ex && !(F.solid && F.solid[cidx(P, i0 + a, j0 + tb, k0 + tc)])) {
            const int h = hLine + a;
            const int l = lLine + a;
            const double rho_i = sR[h];
            double off = 0.0;
            {
                double rfl = 0.5 * (rho_i + sR[h - 1]), rfr = 0.5 * (rho_i + sR[h + 1]);
                off += sAx[a] * (sS[h - 1] / rfl + sS[h + 1] / rfr);
            }
            {
                double rfl = 0.5 * (rho_i + sR[h - HX]), rfr = 0.5 * (rho_i + sR[h + HX]);
                off += ady * (sS[h - HX] / rfl + sS[h + HX] / rfr);
            }
            if (D3) {
                double rfl = 0.5 * (rho_i + sR[h - HX * HY]), rfr = 0.5 * (rho_i + sR[h + HX * HY]);
                off += adz * (sS[h - HX * HY] / rfl + sS[h + HX * HY] / rfr);
            }
            sS[h] = (sRhs[l] + off) / sDiag[l];
        }
        __syncthreads();
    }
    for (int line = warp; line < ey * ez; line += nwarp) {
        const int b = line % ey, c = line / ey;
        for (int a = lane; a < ex; a += 32)
            F.sigma[cidx(P, i0 + a, j0 + b, k0 + c)] = sS[((c + D3) * HY + (b + 1)) * HX + (a + 1)];
    }
    if (PL.ghosts) {
        __syncthreads();   // the tile's sigma, written by all warps above
        igr_tile_ghosts(P, F.sigma, I, J, K, ntx, nty, ntz, i0, j0, k0, ex, ey, ez);
    }
}

// ---------------------------------------------------------------------------
// IGR sweep with precomputed reciprocals (3D, 16^3 tiles).
//
// The face densities 0.5 (rho_i + rho_nb) and the diagonal are fixed for all
// sweeps of one IGR solve, so their reciprocals are computed once per solve
// (k_igr_records, correctly rounded IEEE divisions) and each division of the
// sweep becomes div_markstein: the same correctly rounded quotient from a
// multiply and four fused multiply-adds instead of a full division on the
// serial path of the wavefront.
// ---------------------------------------------------------------------------

// Correctly rounded a / b given y = RN(1 / b).  q0 = a y is within 1.5 ulp of
// a / b; one residual correction q1 = RN(q0 + RN(a - b q0) y) is faithful
// (within 1 ulp); Markstein's theorem (P. Markstein, "Computation of
// elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
// Dev. 34(1), 1990: for y = RN(1 / b) and a faithful q, r = a - b q is exact
// and RN(q + r y) = RN(a / b)) makes the second correction the correctly
// rounded quotient.  Valid when |y| lies in [2^-450, 2^450] and a is +0 or
// |a| lies in [2^-450, 2^450] (quotient and residual then stay clear of
// overflow and gradual underflow; a = +0 gives +0 or -0 as a / b does).
// Callers check both with igr_fast_operand / igr_fast_recip and take the
// plain division otherwise.
__device__ __forceinline__ double div_markstein(double a, double b, double y) {
    const double q0 = a * y;
    const double q1 = fma(fma(-q0, b, a), y, q0);
    return fma(fma(-q1, b, a), y, q1);
}
// |x| in [2^-450, 2^450] (biased exponent 573..1473)
__device__ __forceinline__ bool igr_fast_recip(double x) {
    return ((unsigned)__double2hiint(x) & 0x7ff00000u) - 0x23d00000u <= 0x38400000u;
}
// the same, or x = +0
__device__ __forceinline__ bool igr_fast_operand(double x) {
    return igr_fast_recip(x) || (((unsigned)__double2hiint(x) | (unsigned)__double2loint(x)) == 0u);
}
// igr_cell's update from staged values with plain divisions; kept out of
// line so that the compiler does not if-convert it into the common path.
__device__ __noinline__ double igr_cell_plain(double sxm, double sxp, double sym, double syp, double szm, double szp,
                                              double rflx, double rfrx, double rfly, double rfry, double rflz,
                                              double rfrz, double ax, double ay, double az, double rhs, double diag) {
    double off = 0.0;
    off += ax * (sxm / rflx + sxp / rfrx);
    off += ay * (sym / rfly + syp / rfry);
    off += az * (szm / rflz + szp / rfrz);
    return (rhs + off) / diag;
}
__device__ __noinline__ double div_rn_plain(double a, double b) { return a / b; }

// Records of the tile sweep.  The x-line (., tb, tc) of a tile has records
// n = 0..16 (n = 16 only carries the left x-face of the cell past the tile,
// i.e. the right x-face of n = 15); a record is 8 doubles in four 16-byte
// chunks: 1 / rho_f of the x-, y-, y+, z-, z+ faces, the rhs, the diagonal
// and 1 / diagonal.  Chunk ch of record n of line (tb, tc) of tile t sits at
// double2 index (((t * 16 + tc) * 17 + (tb + n) % 17) * 4 + ch) * 16 + tb:
// the 16 lines of one tc fetch records with equal tb + n at the same cell
// plane, so each chunk of their fetch is one contiguous 256-byte run.
constexpr int kIgrTile = 16;
constexpr int kIgrRecsPerLine = kIgrTile + 1;
constexpr int kIgrRecDoubles = 8;
#ifndef SIFV_IGR_PREFETCH
#define SIFV_IGR_PREFETCH 2
#endif
constexpr int kIgrPrefetch = SIFV_IGR_PREFETCH;  // records in flight ahead of the cell being updated
constexpr int kIgrMaxSlots = 32;                 // sweeps overlapping in one launch of k_igr_tile(_rec)
constexpr int kIgrRing = kIgrPrefetch + 2;       // ring slots per thread

__host__ __device__ __forceinline__ size_t igr_rec_index(long long tile, int tb, int tc, int n) {
    return ((((size_t)tile * kIgrTile + tc) * kIgrRecsPerLine + (tb + n) % kIgrRecsPerLine) * 4) * kIgrTile + tb;
}
inline size_t igr_record_doubles(int ntiles) {
    return (size_t)ntiles * (kIgrTile * kIgrTile) * kIgrRecsPerLine * kIgrRecDoubles;
}
inline size_t igr_tile_rec_smem() {
    return sizeof(double) * (2 * 20 * 18 * 18 + kIgrRing * kIgrRecDoubles * kIgrTile * kIgrTile + kIgrTile);
}

// One thread per record, in storage order (tile, tc, (tb + n) % 17, tb) so
// that a warp's stores are contiguous.  The face densities use the sweep's expressions
// (0.5 (rho_i + rho_nb) with the cell's own density first) and so the
// reciprocal belongs to exactly the divisor that the sweep forms.  A
// reciprocal outside div_markstein's range sets *slowRecs (cleared before
// the launch): the sweeps of this solve then divide plainly.
__global__ void __launch_bounds__(256) k_igr_records(Params P, Fields F, double* __restrict__ rec, int ntx, int nty,
                                                     long long total, int* __restrict__ slowRecs) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    constexpr int T = kIgrTile;
    const int tb = (int)(idx % T);
    const int sk = (int)((idx / T) % kIgrRecsPerLine);   // (tb + n) % 17
    const int tc = (int)((idx / ((long long)T * kIgrRecsPerLine)) % T);
    const long long tile = idx / ((long long)kIgrRecsPerLine * T * T);
    const int n = (sk - tb + kIgrRecsPerLine) % kIgrRecsPerLine;
    const int I = (int)(tile % ntx), J = (int)((tile / ntx) % nty), K = (int)(tile / ((long long)ntx * nty));
    const int i0 = I * T, j0 = J * T, k0 = K * T;
    const int ex = min(T, P.nx - i0), ey = min(T, P.ny - j0), ez = min(T, P.nz - k0);
    if (tb >= ey || tc >= ez || n > ex) return;
    const size_t c = cidx(P, i0 + n, j0 + tb, k0 + tc);
    const size_t sy = (size_t)P.nxT, sz = (size_t)P.nxT * P.nyT;
    const double rho_i = F.rho[c];
    double2* o = reinterpret_cast<double2*>(rec) + igr_rec_index(tile, tb, tc, n);
    const double rxl = 1.0 / (0.5 * (rho_i + F.rho[c - 1]));
    if (n == ex) {
        o[0] = make_double2(rxl, 0.0);
        if (!igr_fast_recip(rxl)) atomicOr(slowRecs, 1);
        return;
    }
    const double diag = F.igrDiag[c];
    const double ryl = 1.0 / (0.5 * (rho_i + F.rho[c - sy])), ryr = 1.0 / (0.5 * (rho_i + F.rho[c + sy]));
    const double rzl = 1.0 / (0.5 * (rho_i + F.rho[c - sz])), rzr = 1.0 / (0.5 * (rho_i + F.rho[c + sz]));
    const double rd = 1.0 / diag;
    o[0] = make_double2(rxl, ryl);
    o[kIgrTile] = make_double2(ryr, rzl);
    o[2 * kIgrTile] = make_double2(rzr, F.igrRhs[c]);
    o[3 * kIgrTile] = make_double2(diag, rd);
    if (!(igr_fast_recip(rxl) && igr_fast_recip(ryl) && igr_fast_recip(ryr) && igr_fast_recip(rzl) &&
          igr_fast_recip(rzr) && igr_fast_recip(rd)))
        atomicOr(slowRecs, 1);
}

__device__ __forceinline__ void cp_async16(void* smemDst, const void* gmemSrc) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smemDst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmemSrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// The tiled wavefront of k_igr_tile<16, 16, 16> (same tile planes, same cell
// planes inside a tile, igr_cell's arithmetic in igr_cell's order) with
//  - the sigma and rho halos staged in 16-byte copies: each halo row holds
//    20 doubles from the even ghosted column at or below the tile's first
//    halo column (requires an even row length nxT and 16-byte aligned
//    fields), the tile's columns start at offset xoff in {0, 1};
//  - each thread streaming the records of its x-line through a ring of
//    kIgrRing slots, kIgrPrefetch records ahead of the cell it updates;
//  - the divisions done by div_markstein (one operand check per cell);
//  - each updated cell stored to global memory as soon as it is computed;
//  - the tile planes after the first of a sweep launched with programmatic
//    stream serialization (griddepcontrol): a plane's blocks stage the rho
//    halo and their first records while the previous plane still runs, and
//    read sigma only after it has completed.
// Thread (tb, tc) owns the x-line (., tb, tc) of the tile and updates its
// cell a = q - tb - tc at cell plane q.
//
// Consecutive sweeps overlap (IgrPlanes): sweep s + 1 runs its tile plane p
// in the launch that runs sweep s's plane p + lag.  A tile reads its
// upstream face neighbours (plane p - 1, same sweep, earlier launches) and
// its downstream ones (plane p + 1 of the previous sweep: complete, and not
// yet reached by this sweep), as the lexicographic order asks.  The scalar
// ghost fill between sweeps is done by the boundary tiles at their end
// (ghosts = 1): a tile on the low face of a zero-gradient axis copies its
// first layer into the ghost layer, a tile on the high face its last layer;
// on a periodic axis the high tile writes both images (its own last layer
// below the low face, the low tile's first layer above the high face; with
// lag >= tiles along the axis the low tile holds this sweep's final values
// and the next sweep has not reached it).  Only the ghost layer next to the
// face is written (the 7-point stencil reads no other); the full fill runs
// after the last sweep.
__global__ void __launch_bounds__(256, 1)
    k_igr_tile_rec(Params P, Fields F, const double* __restrict__ rec, const int* __restrict__ slowRecs,
                   IgrPlanes PL, int ntx, int nty, int ntz) {
    constexpr int T = kIgrTile, HXP = 20, HY = T + 2, HZ = T + 2, HN = HXP * HY * HZ;
    constexpr int NT = T * T, D = kIgrPrefetch, R = kIgrRing;
    extern __shared__ __align__(16) double smem[];
    double* sS = smem;
    double* sR = smem + HN;
    double2* ring = reinterpret_cast<double2*>(smem + 2 * HN);   // [R][4 chunks][NT threads]
    double* sAx = smem + 2 * HN + R * kIgrRecDoubles * NT;
    const unsigned perSlot = (unsigned)(nty * ntz);
    const int slot = (int)(blockIdx.x / perSlot);
    const unsigned bt = blockIdx.x % perSlot;
    const int J = (int)(bt % (unsigned)nty), K = (int)(bt / (unsigned)nty);
    const int I = PL.top - slot * PL.lag - J - K;
    if (I < 0 || I >= ntx) return;
    const int tid = (int)threadIdx.x;
    const int i0 = I * T, j0 = J * T, k0 = K * T;
    const int ex = min(T, P.nx - i0), ey = min(T, P.ny - j0), ez = min(T, P.nz - k0);
    const int hy = ey + 2, hz = ez + 2;
    const int xg = i0 - 1 + P.ngx;   // ghosted column of the first halo column
    const int xs = xg & ~1;
    const int xoff = xg - xs;
    // Launched with programmatic stream serialization after the previous
    // tile plane: let the next plane's blocks start, and stage everything
    // that no tile plane writes (rho halo, alpha / dx^2, the first records)
    // before waiting for the previous plane to complete.
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
    auto stageHalo = [&](double* dst, const double* src) {
        for (int w = tid; w < hy * hz * (HXP / 2); w += NT) {
            const int m = w % (HXP / 2), row = w / (HXP / 2);
            const int b = row % hy, c = row / hy;
            const int x = xs + 2 * m;
            if (x + 1 < P.nxT) {
                const size_t g = (size_t)x + (size_t)P.nxT * ((size_t)(j0 + b - 1 + P.ngy) +
                                                              (size_t)P.nyT * (size_t)(k0 + c - 1 + P.ngz));
                cp_async16(&dst[(c * HY + b) * HXP + 2 * m], &src[g]);
            }
        }
    };
    stageHalo(sR, F.rho);
    for (int a = tid; a < ex; a += NT) cp_async8(&sAx[a], &F.adx2[i0 + a + P.ngx]);
    cp_async_commit();
    const int tb = tid % T, tc = tid / T;
    const bool act = tb < ey && tc < ez;
    const long long tile = (long long)I + (long long)ntx * (J + (long long)nty * K);
    const double2* lineRec = reinterpret_cast<const double2*>(rec) + igr_rec_index(tile, 0, tc, 0);   // (tile, tc) block
    // record n of this thread's line goes to ring slot n % R; one commit
    // group per (pre-)step: at cell plane q >= D the group of record a + 1
    // is the (D+1)-th most recent one (earlier ones complete before the loop)
    auto issue = [&](int n) {
        if (act && n >= 0 && n <= ex) {
            double2* dst = ring + (size_t)(n % R) * 4 * NT + tid;
            const double2* src = lineRec + (size_t)((tb + n) % kIgrRecsPerLine) * 4 * T + tb;
#pragma unroll
            for (int ch = 0; ch < 4; ++ch) cp_async16(dst + ch * NT, src + ch * T);
        }
        cp_async_commit();
    };
    for (int q = -(D + 1); q < 0; ++q) issue(q - tb - tc + D + 1);
    const double ady = act ? F.ady2[j0 + tb + P.ngy] : 0.0;
    const double adz = act ? F.adz2[k0 + tc + P.ngz] : 0.0;
    const int hLine = ((tc + 1) * HY + (tb + 1)) * HXP + 1 + xoff;
    const size_t gLine = cidx(P, i0, j0 + tb, k0 + tc);
    const bool fastRecs = *slowRecs == 0;
    asm volatile("griddepcontrol.wait;\n" ::: "memory");   // sigma of the previous tile planes
    stageHalo(sS, F.sigma);
    cp_async_commit();
    cp_async_wait_group<0>();
    __syncthreads();
    const int nq = ex + ey + ez - 2;
    for (int q = 0; q < nq; ++q) {
        const int a = q - tb - tc;
        issue(a + D + 1);
        cp_async_wait_group<D>();   // records a and a + 1 of this thread have landed
        if (act && a >= 0 && a < ex && !(F.solid && F.solid[gLine + a])) {
            const double2* ra = ring + (size_t)(a % R) * 4 * NT + tid;
            const double2 c0 = ra[0], c1 = ra[NT], c2 = ra[2 * NT], c3 = ra[3 * NT];
            const double rxr = ring[(size_t)((a + 1) % R) * 4 * NT + tid].x;
            const int h = hLine + a;
            const double rho_i = sR[h];
            const double sxm = sS[h - 1], sxp = sS[h + 1], sym = sS[h - HXP], syp = sS[h + HXP];
            const double szm = sS[h - HXP * HY], szp = sS[h + HXP * HY];
            const double rflx = 0.5 * (rho_i + sR[h - 1]), rfrx = 0.5 * (rho_i + sR[h + 1]);
            const double rfly = 0.5 * (rho_i + sR[h - HXP]), rfry = 0.5 * (rho_i + sR[h + HXP]);
            const double rflz = 0.5 * (rho_i + sR[h - HXP * HY]), rfrz = 0.5 * (rho_i + sR[h + HXP * HY]);
            double v;
            if (fastRecs && igr_fast_operand(sxm) && igr_fast_operand(sxp) && igr_fast_operand(sym) &&
                igr_fast_operand(syp) && igr_fast_operand(szm) && igr_fast_operand(szp)) {
                double off = 0.0;
                off += sAx[a] * (div_markstein(sxm, rflx, c0.x) + div_markstein(sxp, rfrx, rxr));
                off += ady * (div_markstein(sym, rfly, c0.y) + div_markstein(syp, rfry, c1.x));
                off += adz * (div_markstein(szm, rflz, c1.y) + div_markstein(szp, rfrz, c2.x));
                const double num = c2.y + off;
                v = igr_fast_operand(num) ? div_markstein(num, c3.x, c3.y) : div_rn_plain(num, c3.x);
            } else {
                v = igr_cell_plain(sxm, sxp, sym, syp, szm, szp, rflx, rfrx, rfly, rfry, rflz, rfrz, sAx[a], ady, adz,
                                   c2.y, c3.x);
            }
            sS[h] = v;
            F.sigma[gLine + a] = v;
        }
        __syncthreads();
    }
    if (PL.ghosts) igr_tile_ghosts(P, F.sigma, I, J, K, ntx, nty, ntz, i0, j0, k0, ex, ey, ez);
}

// ---------------------------------------------------------------------------
// Gauss-Seidel pressure solve (GaussSeidelPressureSolver::solve,
// src/GaussSeidelPressureSolver.cpp:10-49): per iteration the scalar ghosts of
// p are filled from the current iterate, then one lexicographic in-place sweep
// p <- (rhs + rho c^2 dt^2 offDiag) / (1 + rho c^2 dt^2 diagL) with the
// PressureLaplacian coefficients (src/PressureLaplacian.cpp:6-60, evaluated
// once per solve by k_jacobi_coef), max |p_new - p_old| as the residual.  The
// sweep runs as the same tiled wavefront as the IGR sweep (bit-identical to
// the lexicographic order).  Every kernel of iteration `it` is a no-op once
// iteration it-1 converged (device-side check, as k_jacobi).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool gs_converged(Ctl* ctl, int it, double tol) {
    if (ctl->jacobiDone) return true;
    if (it > 0 && bits2d(ctl->res[it - 1]) < tol) {
        if (threadIdx.x == 0) ctl->jacobiDone = it;
        return true;
    }
    return false;
}

__global__ void k_gs_ghosts(Params P, double* __restrict__ f, Ctl* ctl, int it, double tol) {
    if (gs_converged(ctl, it, tol)) return;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;   // one thread per ghost cell
    int i, j, k;
    if (t >= ghost_count(P) || !ghost_coords(P, t, i, j, k)) return;
    f[cidx(P, i, j, k)] = f[scalar_idx(P, i, j, k)];
}

// one cell: coefficients in k_jacobi_coef's layout (x-, x+, y-, y+, z-, z+,
// coeff, denom) at cf[q * nc]; neighbours pm / pp per axis
__device__ __forceinline__ double gs_cell(int dim, const double* cf, size_t nc, double rhsC, const double* pn) {
    double od = 0.0;
    od += cf[0] * pn[0] + cf[nc] * pn[1];
    if (dim >= 2) od += cf[2 * nc] * pn[2] + cf[3 * nc] * pn[3];
    if (dim >= 3) od += cf[4 * nc] * pn[4] + cf[5 * nc] * pn[5];
    const double coeff = cf[(size_t)(2 * dim) * nc], denom = cf[(size_t)(2 * dim + 1) * nc];
    return (rhsC + coeff * od) / denom;
}

__global__ void k_gs_sweep_1d(Params P, const double* __restrict__ coef, size_t nc, const double* __restrict__ rhs,
                              double* __restrict__ p, Ctl* ctl, int it, double tol) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (gs_converged(ctl, it, tol)) return;
    double maxRes = 0.0;
    for (int i = 0; i < P.nx; ++i) {
        const size_t c = cidx(P, i, 0, 0);
        const double nb[2] = {p[c - 1], p[c + 1]};
        const double pOld = p[c];
        const double pn = gs_cell(1, coef + c, nc, rhs[c], nb);
        p[c] = pn;
        maxRes = smax(maxRes, fabs(pn - pOld));
    }
    atomicMax(&ctl->res[it], d2bits(maxRes));
}

constexpr int kGsMaxBufs = 34;   // S + 2 buffers for S iterations in flight
struct GsBufs {
    double* b[kGsMaxBufs];
    int nb;   // buffers in use
};
struct GsPlanes {
    int top;   // tile plane of the first active iteration (slot 0); slot u runs plane top - u lag
    int lag;
    int n;     // active iterations in this launch
    int it0;   // index of the iteration in slot 0
    int np;    // tile planes of one iteration
};
// The last iteration whose residual is complete when the tile on plane p of
// iteration it starts: iteration j ends with launch j lag + np - 1, before
// this tile's launch it lag + p.
__device__ __forceinline__ int gs_complete_before(const GsPlanes& PL, int it, int p) {
    return it - (PL.np - p + PL.lag - 1) / PL.lag;
}
template <int TX, int TY, int TZ>
__global__ void __launch_bounds__(TY * TZ) k_gs_tile(Params P, const double* __restrict__ coef, size_t nc,
                                                     const double* __restrict__ rhs, double* __restrict__ p, Ctl* ctl,
                                                     int it, double tol, int plane, int ntx, int nty) {
    extern __shared__ double smem[];
    constexpr int D3 = (TZ > 1) ? 1 : 0;
    constexpr int HX = TX + 2, HY = TY + 2;
    if (gs_converged(ctl, it, tol)) return;
    const int J = (int)(blockIdx.x % (unsigned)nty), K = (int)(blockIdx.x / (unsigned)nty);
    const int I = plane - J - K;
    if (I < 0 || I >= ntx) return;
    const int i0 = I * TX, j0 = J * TY, k0 = K * TZ;
    const int ex = min(TX, P.nx - i0), ey = min(TY, P.ny - j0), ez = D3 ? min(TZ, P.nz - k0) : 1;
    const int hx = ex + 2, hy = ey + 2, hz = D3 ? ez + 2 : 1;
    const int lane = (int)threadIdx.x & 31, warp = (int)threadIdx.x >> 5, nwarp = (int)blockDim.x >> 5;
    for (int line = warp; line < hy * hz; line += nwarp) {
        const int b = line % hy, c = line / hy;
        for (int a = lane; a < hx; a += 32)
            cp_async8(&smem[(c * HY + b) * HX + a], &p[cidx(P, i0 + a - 1, j0 + b - 1, D3 ? k0 + c - 1 : k0)]);
    }
    cp_async_wait_all();
    const int tb = (int)threadIdx.x % TY, tc = (int)threadIdx.x / TY;
    const bool act = tb < ey && tc < ez;
    const int hLine = ((tc + D3) * HY + (tb + 1)) * HX + 1;
    constexpr int DIM = D3 ? 3 : 2;
    constexpr int NCO = 2 * DIM + 2;   // k_jacobi_coef's per-cell coefficients
    double maxRes = 0.0;
    __syncthreads();
    const int nq = ex + ey + ez - 2;
    // The coefficients and rhs of a thread's cells stream from global memory:
    // those of cell a + 2 are loaded at cell plane q (cell a), into the
    // register set that cell plane q + 2 computes with, so that their latency
    // overlaps two cell planes.  The three sets rotate roles every plane
    // (X computes, Z receives), with no copies between them.
    double sA[NCO + 1], sB[NCO + 1], sC[NCO + 1];
    auto step = [&](int q, double (&X)[NCO + 1], double (&Z)[NCO + 1]) {
        const int a = q - tb - tc;
        if (act && a + 2 >= 0 && a + 2 < ex) {
            const size_t c = cidx(P, i0 + a + 2, j0 + tb, k0 + tc);
#pragma unroll
            for (int k = 0; k < NCO; ++k) Z[k] = coef[c + (size_t)k * nc];
            Z[NCO] = rhs[c];
        }
        if (q < 0 || q >= nq) return;
        if (act && a >= 0 && a < ex) {
            const int h = hLine + a;
            const double nb[6] = {smem[h - 1], smem[h + 1], smem[h - HX], smem[h + HX],
                                  D3 ? smem[h - HX * HY] : 0.0, D3 ? smem[h + HX * HY] : 0.0};
            const double pOld = smem[h];
            const double pn = gs_cell(DIM, X, 1, X[NCO], nb);
            smem[h] = pn;
            maxRes = smax(maxRes, fabs(pn - pOld));
        }
        __syncthreads();
    };
    for (int q = -2; q < nq; q += 3) {
        step(q, sA, sC);
        step(q + 1, sB, sA);
        step(q + 2, sC, sB);
    }
    for (int line = warp; line < ey * ez; line += nwarp) {
        const int b = line % ey, c = line / ey;
        for (int a = lane; a < ex; a += 32)
            p[cidx(P, i0 + a, j0 + b, k0 + c)] = smem[((c + D3) * HY + (b + 1)) * HX + (a + 1)];
    }
    block_max_to(maxRes, &ctl->res[it]);
}

// Ghost images of a finished tile of an overlapped Gauss-Seidel iteration
// (any tile shape): the low-side ghost layer into the next iteration's
// buffer, the high-side one into this iteration's (k_gs_tile_rec_ov).
__device__ __forceinline__ void gs_tile_ghosts(const Params& P, double* pNew, double* pNext, int I, int J, int K,
                                               int ntx, int nty, int ntz, int i0, int j0, int k0, int ex, int ey,
                                               int ez) {
    const int nt = (int)blockDim.x;
    const size_t sy = (size_t)P.nxT, sz = (size_t)P.nxT * P.nyT;
    {
        const bool per = P.bc[0] == SIFV_BC_PERIODIC;
        for (int w = (int)threadIdx.x; w < ey * ez; w += nt) {
            const int b = w % ey, c = w / ey;
            const size_t row = cidx(P, 0, j0 + b, k0 + c);
            if (!per && I == 0) pNext[row - 1] = pNew[row];
            if (!per && I == ntx - 1) pNew[row + P.nx] = pNew[row + P.nx - 1];
            if (per && I == ntx - 1) {
                pNext[row - 1] = pNew[row + P.nx - 1];
                pNew[row + P.nx] = pNew[row];
            }
        }
    }
    if (P.dim >= 2) {
        const bool per = P.bc[2] == SIFV_BC_PERIODIC;
        const size_t hi = (size_t)P.ny * sy;
        for (int w = (int)threadIdx.x; w < ex * ez; w += nt) {
            const int a = w % ex, c = w / ex;
            const size_t col = cidx(P, i0 + a, 0, k0 + c);
            if (!per && J == 0) pNext[col - sy] = pNew[col];
            if (!per && J == nty - 1) pNew[col + hi] = pNew[col + hi - sy];
            if (per && J == nty - 1) {
                pNext[col - sy] = pNew[col + hi - sy];
                pNew[col + hi] = pNew[col];
            }
        }
    }
    if (P.dim >= 3) {
        const bool per = P.bc[4] == SIFV_BC_PERIODIC;
        const size_t hi = (size_t)P.nz * sz;
        for (int w = (int)threadIdx.x; w < ex * ey; w += nt) {
            const int a = w % ex, b = w / ex;
            const size_t col = cidx(P, i0 + a, j0 + b, 0);
            if (!per && K == 0) pNext[col - sz] = pNew[col];
            if (!per && K == ntz - 1) pNew[col + hi] = pNew[col + hi - sz];
            if (per && K == ntz - 1) {
                pNext[col - sz] = pNew[col + hi - sz];
                pNew[col + hi] = pNew[col];
            }
        }
    }
}

// Overlapped iterations of the plain tile sweep (2D 32 x 64 tiles, 3D rows
// of odd length): k_gs_tile's arithmetic and order with the buffers,
// staging, skip rule and ghost images of k_gs_tile_rec_ov.
template <int TX, int TY, int TZ>
__global__ void __launch_bounds__(TY * TZ) k_gs_tile_ov(Params P, const double* __restrict__ coef, size_t nc,
                                                        const double* __restrict__ rhs, GsBufs B, Ctl* ctl,
                                                        double tol, GsPlanes PL, int ntx, int nty, int ntz) {
    extern __shared__ double smem[];
    constexpr int D3 = (TZ > 1) ? 1 : 0;
    constexpr int HX = TX + 2, HY = TY + 2;
    __shared__ int skip;
    const unsigned perSlot = (unsigned)(nty * ntz);
    const int slot = (int)(blockIdx.x / perSlot);
    const unsigned bt = blockIdx.x % perSlot;
    const int J = (int)(bt % (unsigned)nty), K = (int)(bt / (unsigned)nty);
    const int I = PL.top - slot * PL.lag - J - K;
    if (I < 0 || I >= ntx) return;
    const int it = PL.it0 + slot;
    if (threadIdx.x == 0) {
        int s = 0;
        const int last = gs_complete_before(PL, it, PL.top - slot * PL.lag);
        for (int j = 0; j <= last; ++j)
            if (bits2d(ctl->res[j]) < tol) { s = 1; break; }
        skip = s;
    }
    __syncthreads();
    if (skip) return;
    const double* __restrict__ pOld = B.b[it % B.nb];
    double* __restrict__ pNew = B.b[(it + 1) % B.nb];
    const int i0 = I * TX, j0 = J * TY, k0 = K * TZ;
    const int ex = min(TX, P.nx - i0), ey = min(TY, P.ny - j0), ez = D3 ? min(TZ, P.nz - k0) : 1;
    const int hx = ex + 2, hy = ey + 2, hz = D3 ? ez + 2 : 1;
    const int lane = (int)threadIdx.x & 31, warp = (int)threadIdx.x >> 5, nwarp = (int)blockDim.x >> 5;
    for (int line = warp; line < hy * hz; line += nwarp) {   // tile + downstream halos: iterate it
        const int b = line % hy, c = line / hy;
        for (int a = lane; a < hx; a += 32)
            cp_async8(&smem[(c * HY + b) * HX + a], &pOld[cidx(P, i0 + a - 1, j0 + b - 1, D3 ? k0 + c - 1 : k0)]);
    }
    cp_async_wait_all();
    __syncthreads();
    {   // upstream face halos: iterate it + 1 (this iteration's upstream tiles / ghost images)
        const int nt = (int)blockDim.x;
        for (int w = (int)threadIdx.x; w < ey * ez; w += nt) {
            const int b = w % ey, c = w / ey;
            smem[((c + D3) * HY + (b + 1)) * HX] = pNew[cidx(P, i0 - 1, j0 + b, k0 + c)];
        }
        for (int w = (int)threadIdx.x; w < ex * ez; w += nt) {
            const int a = w % ex, c = w / ex;
            smem[((c + D3) * HY) * HX + a + 1] = pNew[cidx(P, i0 + a, j0 - 1, k0 + c)];
        }
        if (D3)
            for (int w = (int)threadIdx.x; w < ex * ey; w += nt) {
                const int a = w % ex, b = w / ex;
                smem[(b + 1) * HX + a + 1] = pNew[cidx(P, i0 + a, j0 + b, k0 - 1)];
            }
    }
    const int tb = (int)threadIdx.x % TY, tc = (int)threadIdx.x / TY;
    const bool act = tb < ey && tc < ez;
    const int hLine = ((tc + D3) * HY + (tb + 1)) * HX + 1;
    constexpr int DIM = D3 ? 3 : 2;
    constexpr int NCO = 2 * DIM + 2;
    double maxRes = 0.0;
    __syncthreads();
    const int nq = ex + ey + ez - 2;
    double sA[NCO + 1], sB[NCO + 1], sC[NCO + 1];
    auto step = [&](int q, double (&X)[NCO + 1], double (&Z)[NCO + 1]) {
        const int a = q - tb - tc;
        if (act && a + 2 >= 0 && a + 2 < ex) {
            const size_t c = cidx(P, i0 + a + 2, j0 + tb, k0 + tc);
#pragma unroll
            for (int k = 0; k < NCO; ++k) Z[k] = coef[c + (size_t)k * nc];
            Z[NCO] = rhs[c];
        }
        if (q < 0 || q >= nq) return;
        if (act && a >= 0 && a < ex) {
            const int h = hLine + a;
            const double nb[6] = {smem[h - 1], smem[h + 1], smem[h - HX], smem[h + HX],
                                  D3 ? smem[h - HX * HY] : 0.0, D3 ? smem[h + HX * HY] : 0.0};
            const double po = smem[h];
            const double pn = gs_cell(DIM, X, 1, X[NCO], nb);
            smem[h] = pn;
            maxRes = smax(maxRes, fabs(pn - po));
        }
        __syncthreads();
    };
    for (int q = -2; q < nq; q += 3) {
        step(q, sA, sC);
        step(q + 1, sB, sA);
        step(q + 2, sC, sB);
    }
    for (int line = warp; line < ey * ez; line += nwarp) {
        const int b = line % ey, c = line / ey;
        for (int a = lane; a < ex; a += 32)
            pNew[cidx(P, i0 + a, j0 + b, k0 + c)] = smem[((c + D3) * HY + (b + 1)) * HX + (a + 1)];
    }
    __syncthreads();   // the tile's new values, written by all warps above
    gs_tile_ghosts(P, pNew, B.b[(it + 2) % B.nb], I, J, K, ntx, nty, ntz, i0, j0, k0, ex, ey, ez);
    block_max_to(maxRes, &ctl->res[it]);
}

// ---------------------------------------------------------------------------
// Gauss-Seidel sweep with precomputed records (3D, 16^3 tiles): the tiled
// wavefront of k_gs_tile<16, 16, 16> with the treatment of the IGR record
// sweep.  The coefficients, coeff, denominator and rhs of a cell are fixed
// for the whole solve, so they are laid out once per solve as records that
// the 16 lines of one tile row fetch as contiguous runs (k_gs_records), with
// the reciprocal of the denominator: the division (rhs + coeff od) / denom
// becomes div_markstein's correctly rounded quotient (a plain division where
// its operand check fails, or for the whole solve when a reciprocal is out
// of range).  Each thread streams its line's records through a shared-memory
// ring, each new p is stored as it is computed, and tile planes after the
// first are launched with programmatic stream serialization (their records
// arrive while the previous plane runs; p is read after it completes).
// Record: 10 doubles in five 16-byte chunks (x-, x+, y-, y+, z-, z+
// coefficients, coeff, denom, 1 / denom, rhs); chunk ch of cell n of line
// (tb, tc) of tile t at double2 index (((t 16 + tc) 16 + (tb + n) % 16) 5 + ch) 16 + tb.
// ---------------------------------------------------------------------------
constexpr int kGsRecChunks = 5;

__host__ __device__ __forceinline__ size_t gs_rec_index(long long tile, int tb, int tc, int n) {
    return ((((size_t)tile * kIgrTile + tc) * kIgrTile + (tb + n) % kIgrTile) * kGsRecChunks) * kIgrTile + tb;
}
inline size_t gs_record_doubles(long long ntiles) {
    return (size_t)ntiles * kIgrTile * kIgrTile * kIgrTile * 2 * kGsRecChunks;
}
inline size_t gs_tile_rec_smem() {
    return sizeof(double) * (20 * 18 * 18 + kIgrRing * 2 * kGsRecChunks * kIgrTile * kIgrTile);
}

// Records of the solve from k_jacobi_coef's per-cell coefficients (layout
// coef[q * nc + c], q = 0..7 in 3D) and the rhs; one thread per record.
__global__ void __launch_bounds__(256) k_gs_records(Params P, const double* __restrict__ coef, size_t nc,
                                                    const double* __restrict__ rhs, double* __restrict__ rec,
                                                    int ntx, int nty, long long total, int* __restrict__ slowRecs) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    constexpr int T = kIgrTile;
    const int tb = (int)(idx % T);
    const int sk = (int)((idx / T) % T);
    const int tc = (int)((idx / ((long long)T * T)) % T);
    const long long tile = idx / ((long long)T * T * T);
    const int n = (sk - tb + T) % T;
    const int I = (int)(tile % ntx), J = (int)((tile / ntx) % nty), K = (int)(tile / ((long long)ntx * nty));
    const int i0 = I * T, j0 = J * T, k0 = K * T;
    const int ex = min(T, P.nx - i0), ey = min(T, P.ny - j0), ez = min(T, P.nz - k0);
    if (tb >= ey || tc >= ez || n >= ex) return;
    const size_t c = cidx(P, i0 + n, j0 + tb, k0 + tc);
    double2* o = reinterpret_cast<double2*>(rec) + gs_rec_index(tile, tb, tc, n);
    const double denom = coef[7 * nc + c];
    const double rd = 1.0 / denom;
    o[0] = make_double2(coef[c], coef[nc + c]);
    o[T] = make_double2(coef[2 * nc + c], coef[3 * nc + c]);
    o[2 * T] = make_double2(coef[4 * nc + c], coef[5 * nc + c]);
    o[3 * T] = make_double2(coef[6 * nc + c], denom);
    o[4 * T] = make_double2(rd, rhs[c]);
    if (!igr_fast_recip(rd)) atomicOr(slowRecs, 1);
}

// One tile plane of Gauss-Seidel iteration `it` (a no-op once iteration
// it-1 converged); the residual max goes to ctl->res[it].  Requires an even
// row length nxT and a 16-byte aligned iterate.
__global__ void __launch_bounds__(256, 1) k_gs_tile_rec(Params P, const double* __restrict__ rec,
                                                        const int* __restrict__ slowRecs, double* __restrict__ p,
                                                        Ctl* ctl, int it, double tol, int plane, int ntx, int nty) {
    constexpr int T = kIgrTile, HXP = 20, HY = T + 2, HN = HXP * HY * (T + 2);
    constexpr int NT = T * T, D = kIgrPrefetch, R = kIgrRing, CH = kGsRecChunks;
    extern __shared__ __align__(16) double smem[];
    double* sP = smem;
    double2* ring = reinterpret_cast<double2*>(smem + HN);   // [R][CH chunks][NT threads]
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
    const int J = (int)(blockIdx.x % (unsigned)nty), K = (int)(blockIdx.x / (unsigned)nty);
    const int I = plane - J - K;
    if (I < 0 || I >= ntx) return;
    const int tid = (int)threadIdx.x;
    const int i0 = I * T, j0 = J * T, k0 = K * T;
    const int ex = min(T, P.nx - i0), ey = min(T, P.ny - j0), ez = min(T, P.nz - k0);
    const int hy = ey + 2, hz = ez + 2;
    const int xg = i0 - 1 + P.ngx;
    const int xs = xg & ~1;
    const int xoff = xg - xs;
    const int tb = tid % T, tc = tid / T;
    const bool act = tb < ey && tc < ez;
    const long long tile = (long long)I + (long long)ntx * (J + (long long)nty * K);
    const double2* lineRec = reinterpret_cast<const double2*>(rec) + gs_rec_index(tile, 0, tc, 0);
    auto issue = [&](int n) {
        if (act && n >= 0 && n < ex) {
            double2* dst = ring + (size_t)(n % R) * CH * NT + tid;
            const double2* src = lineRec + (size_t)((tb + n) % T) * CH * T + tb;
#pragma unroll
            for (int ch = 0; ch < CH; ++ch) cp_async16(dst + ch * NT, src + ch * T);
        }
        cp_async_commit();
    };
    // the first records (fixed for the solve) arrive while the previous plane runs
    for (int q = -D; q < 0; ++q) issue(q - tb - tc + D);
    const int hLine = ((tc + 1) * HY + (tb + 1)) * HXP + 1 + xoff;
    const size_t gLine = cidx(P, i0, j0 + tb, k0 + tc);
    asm volatile("griddepcontrol.wait;\n" ::: "memory");   // p of the previous tile planes
    if (gs_converged(ctl, it, tol)) {
        cp_async_wait_group<0>();
        return;
    }
    const bool fastRecs = *slowRecs == 0;
    for (int w = tid; w < hy * hz * (HXP / 2); w += NT) {
        const int m = w % (HXP / 2), row = w / (HXP / 2);
        const int b = row % hy, c = row / hy;
        const int x = xs + 2 * m;
        if (x + 1 < P.nxT) {
            const size_t g = (size_t)x + (size_t)P.nxT * ((size_t)(j0 + b - 1 + P.ngy) +
                                                          (size_t)P.nyT * (size_t)(k0 + c - 1 + P.ngz));
            cp_async16(&sP[(c * HY + b) * HXP + 2 * m], &p[g]);
        }
    }
    cp_async_commit();
    cp_async_wait_group<0>();
    __syncthreads();
    double maxRes = 0.0;
    const int nq = ex + ey + ez - 2;
    for (int q = 0; q < nq; ++q) {
        const int a = q - tb - tc;
        issue(a + D);
        cp_async_wait_group<D>();   // record a of this thread has landed
        if (act && a >= 0 && a < ex) {
            const double2* ra = ring + (size_t)(a % R) * CH * NT + tid;
            const double2 c0 = ra[0], c1 = ra[NT], c2 = ra[2 * NT], c3 = ra[3 * NT], c4 = ra[4 * NT];
            const int h = hLine + a;
            // gs_cell's order: od = cf0 p(x-) + cf1 p(x+), then y, then z
            double od = 0.0;
            od += c0.x * sP[h - 1] + c0.y * sP[h + 1];
            od += c1.x * sP[h - HXP] + c1.y * sP[h + HXP];
            od += c2.x * sP[h - HXP * HY] + c2.y * sP[h + HXP * HY];
            const double num = c4.y + c3.x * od;
            const double pn = (fastRecs && igr_fast_operand(num)) ? div_markstein(num, c3.y, c4.x)
                                                                  : div_rn_plain(num, c3.y);
            const double pOld = sP[h];
            sP[h] = pn;
            p[gLine + a] = pn;
            maxRes = smax(maxRes, fabs(pn - pOld));
        }
        __syncthreads();
    }
    block_max_to(maxRes, &ctl->res[it]);
}

// Gauss-Seidel iterations overlapped (3D record sweep, no halo exchange):
// several iterations in one launch sequence, iteration m + 1 trailing
// iteration m by `lag` tile planes, as the IGR sweeps (k_igr_tile_rec).  A
// Gauss-Seidel iteration stops on its residual, so the iterations after
// the current one run speculatively and must not destroy an iterate that
// turns out to be the answer: iterate n (n = 0 the initial guess) lives in
// buf[n % B.nb], and the iteration producing iterate n + 1 stages its
// tile and its downstream face halos (x+, y+, z+) from iterate n and its
// upstream face halos (x-, y-, z-: upstream tiles of the same iteration,
// earlier launches) from its own buffer -- in-place Gauss-Seidel's operands
// bit for bit.  Ghost layers (the reference fills them from iterate n
// before the sweep): boundary tiles write, at their end, the images of
// their new values -- the low-side ghost layer into the next iteration's
// buffer, the high-side one into their own (read as downstream halo by the
// next iteration); periodic images need lag >= tiles along the axis, as
// for IGR.  With at most S iterations in flight (S = ceil(planes / lag)),
// the residuals of iterations m - S and earlier are complete when iteration
// m starts, and more of them by its later planes; a tile skips when one of
// the complete residuals is below tol, so at most S - 1 iterations run past
// the converged one and never reach its buffer or its predecessor's
// (S + 2 buffers).
__global__ void __launch_bounds__(256, 1) k_gs_tile_rec_ov(Params P, const double* __restrict__ rec,
                                                           const int* __restrict__ slowRecs, GsBufs B, Ctl* ctl,
                                                           double tol, GsPlanes PL, int ntx, int nty, int ntz) {
    constexpr int T = kIgrTile, HXP = 20, HY = T + 2, HN = HXP * HY * (T + 2);
    constexpr int NT = T * T, D = kIgrPrefetch, R = kIgrRing, CH = kGsRecChunks;
    extern __shared__ __align__(16) double smem[];
    double* sP = smem;
    double2* ring = reinterpret_cast<double2*>(smem + HN);   // [R][CH chunks][NT threads]
    __shared__ int skip;
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
    const unsigned perSlot = (unsigned)(nty * ntz);
    const int slot = (int)(blockIdx.x / perSlot);
    const unsigned bt = blockIdx.x % perSlot;
    const int J = (int)(bt % (unsigned)nty), K = (int)(bt / (unsigned)nty);
    const int I = PL.top - slot * PL.lag - J - K;
    if (I < 0 || I >= ntx) return;
    const int it = PL.it0 + slot;                    // this tile's iteration: iterate it -> it + 1
    const double* __restrict__ pOld = B.b[it % B.nb];
    double* __restrict__ pNew = B.b[(it + 1) % B.nb];
    const int tid = (int)threadIdx.x;
    const int i0 = I * T, j0 = J * T, k0 = K * T;
    const int ex = min(T, P.nx - i0), ey = min(T, P.ny - j0), ez = min(T, P.nz - k0);
    const int hy = ey + 2, hz = ez + 2;
    const int xg = i0 - 1 + P.ngx;
    const int xs = xg & ~1;
    const int xoff = xg - xs;
    const int tb = tid % T, tc = tid / T;
    const bool act = tb < ey && tc < ez;
    const long long tile = (long long)I + (long long)ntx * (J + (long long)nty * K);
    const double2* lineRec = reinterpret_cast<const double2*>(rec) + gs_rec_index(tile, 0, tc, 0);
    auto issue = [&](int n) {
        if (act && n >= 0 && n < ex) {
            double2* dst = ring + (size_t)(n % R) * CH * NT + tid;
            const double2* src = lineRec + (size_t)((tb + n) % T) * CH * T + tb;
#pragma unroll
            for (int ch = 0; ch < CH; ++ch) cp_async16(dst + ch * NT, src + ch * T);
        }
        cp_async_commit();
    };
    for (int q = -D; q < 0; ++q) issue(q - tb - tc + D);
    const int hLine = ((tc + 1) * HY + (tb + 1)) * HXP + 1 + xoff;
    const size_t gLine = cidx(P, i0, j0 + tb, k0 + tc);
    asm volatile("griddepcontrol.wait;\n" ::: "memory");   // the previous tile planes
    if (tid == 0) {   // a converged iteration among those complete before this tile started
        int s = 0;
        const int last = gs_complete_before(PL, it, PL.top - slot * PL.lag);
        for (int j = 0; j <= last; ++j)
            if (bits2d(ctl->res[j]) < tol) { s = 1; break; }
        skip = s;
    }
    __syncthreads();
    if (skip) {
        cp_async_wait_group<0>();
        return;
    }
    const bool fastRecs = *slowRecs == 0;
    // tile and downstream halos from iterate it (the whole box; the upstream faces are replaced below)
    for (int w = tid; w < hy * hz * (HXP / 2); w += NT) {
        const int m = w % (HXP / 2), row = w / (HXP / 2);
        const int b = row % hy, c = row / hy;
        const int x = xs + 2 * m;
        if (x + 1 < P.nxT) {
            const size_t g = (size_t)x + (size_t)P.nxT * ((size_t)(j0 + b - 1 + P.ngy) +
                                                          (size_t)P.nyT * (size_t)(k0 + c - 1 + P.ngz));
            cp_async16(&sP[(c * HY + b) * HXP + 2 * m], &pOld[g]);
        }
    }
    cp_async_commit();
    cp_async_wait_group<0>();
    __syncthreads();
    {   // upstream face halos from iterate it + 1 (this iteration's upstream tiles / ghost images)
        const size_t sy = (size_t)P.nxT, sz = (size_t)P.nxT * P.nyT;
        if (act) {   // x- face: (i0 - 1, j0 + tb, k0 + tc)
            sP[((tc + 1) * HY + (tb + 1)) * HXP + xoff] = pNew[gLine - 1];
        }
        {   // y- face: (i0 + a, j0 - 1, k0 + c)
            const int a = tid % T, c = tid / T;
            if (a < ex && c < ez)
                sP[((c + 1) * HY + 0) * HXP + 1 + xoff + a] = pNew[cidx(P, i0 + a, j0, k0 + c) - sy];
        }
        {   // z- face: (i0 + a, j0 + b, k0 - 1)
            const int a = tid % T, b = tid / T;
            if (a < ex && b < ey)
                sP[(0 * HY + (b + 1)) * HXP + 1 + xoff + a] = pNew[cidx(P, i0 + a, j0 + b, k0) - sz];
        }
    }
    __syncthreads();
    double maxRes = 0.0;
    const int nq = ex + ey + ez - 2;
    for (int q = 0; q < nq; ++q) {
        const int a = q - tb - tc;
        issue(a + D);
        cp_async_wait_group<D>();
        if (act && a >= 0 && a < ex) {
            const double2* ra = ring + (size_t)(a % R) * CH * NT + tid;
            const double2 c0 = ra[0], c1 = ra[NT], c2 = ra[2 * NT], c3 = ra[3 * NT], c4 = ra[4 * NT];
            const int h = hLine + a;
            double od = 0.0;
            od += c0.x * sP[h - 1] + c0.y * sP[h + 1];
            od += c1.x * sP[h - HXP] + c1.y * sP[h + HXP];
            od += c2.x * sP[h - HXP * HY] + c2.y * sP[h + HXP * HY];
            const double num = c4.y + c3.x * od;
            const double pn = (fastRecs && igr_fast_operand(num)) ? div_markstein(num, c3.y, c4.x)
                                                                  : div_rn_plain(num, c3.y);
            const double po = sP[h];
            sP[h] = pn;
            pNew[gLine + a] = pn;
            maxRes = smax(maxRes, fabs(pn - po));
        }
        __syncthreads();
    }
    // ghost images of the new values: low side into the next iteration's buffer, high side into this one
    {
        double* __restrict__ pNext = B.b[(it + 2) % B.nb];
        const size_t sy = (size_t)P.nxT, sz = (size_t)P.nxT * P.nyT;
        {
            const int b = tid % T, c = tid / T;
            if (b < ey && c < ez) {
                const size_t row = cidx(P, 0, j0 + b, k0 + c);
                const bool per = P.bc[0] == SIFV_BC_PERIODIC;
                if (!per && I == 0) pNext[row - 1] = pNew[row];
                if (!per && I == ntx - 1) pNew[row + P.nx] = pNew[row + P.nx - 1];
                if (per && I == ntx - 1) {
                    pNext[row - 1] = pNew[row + P.nx - 1];
                    pNew[row + P.nx] = pNew[row];
                }
            }
        }
        {
            const int a = tid % T, c = tid / T;
            if (a < ex && c < ez) {
                const size_t col = cidx(P, i0 + a, 0, k0 + c);
                const size_t hi = (size_t)P.ny * sy;
                const bool per = P.bc[2] == SIFV_BC_PERIODIC;
                if (!per && J == 0) pNext[col - sy] = pNew[col];
                if (!per && J == nty - 1) pNew[col + hi] = pNew[col + hi - sy];
                if (per && J == nty - 1) {
                    pNext[col - sy] = pNew[col + hi - sy];
                    pNew[col + hi] = pNew[col];
                }
            }
        }
        {
            const int a = tid % T, b = tid / T;
            if (a < ex && b < ey) {
                const size_t col = cidx(P, i0 + a, j0 + b, 0);
                const size_t hi = (size_t)P.nz * sz;
                const bool per = P.bc[4] == SIFV_BC_PERIODIC;
                if (!per && K == 0) pNext[col - sz] = pNew[col];
                if (!per && K == ntz - 1) pNew[col + hi] = pNew[col + hi - sz];
                if (per && K == ntz - 1) {
                    pNext[col - sz] = pNew[col + hi - sz];
                    pNew[col + hi] = pNew[col];
                }
            }
        }
    }
    block_max_to(maxRes, &ctl->res[it]);
}

// The ghost cells of `dst` from the scalar ghost map applied to `src`
// (fillScalarGhosts of `src`'s interior into `dst`'s ghost layers).
__global__ void k_scalar_ghosts_from(Params P, const double* __restrict__ src, double* __restrict__ dst) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (t >= ghost_count(P) || !ghost_coords(P, t, i, j, k)) return;
    dst[cidx(P, i, j, k)] = src[scalar_idx(P, i, j, k)];
}

template <int TX, int TY, int TZ>
constexpr size_t gs_tile_smem() {
    return sizeof(double) * (size_t)(TX + 2) * (TY + 2) * (TZ > 1 ? TZ + 2 : 1);
}

template <int TX, int TY, int TZ>
constexpr size_t igr_tile_smem() {
    return sizeof(double) * (2 * (size_t)(TX + 2) * (TY + 2) * (TZ > 1 ? TZ + 2 : 1) + 2 * (size_t)TX * TY * TZ + TX);
}

}  // namespace sifv
