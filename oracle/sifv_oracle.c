/*
 * sifv_oracle.c -- TEST INFRASTRUCTURE ONLY (the CPU oracle).
 *
 * A plain-C restatement of SemiImplicitFV's explicit and semi-implicit
 * finite-volume time step, used by the tests as the parity checker and by
 * the bench as the "port" CPU baseline.  It exports the ABI of
 * include/sifv.h under the prefix sifvo_.  It is never linked into, called
 * by or shipped with the CUDA library.
 *
 * Every function follows the reference file:line cited above it (paths
 * relative to the SemiImplicitFV repository), evaluating each expression in
 * the same order so that, compiled as ISO C without FMA contraction, the
 * results are bit-identical to the reference compiled with
 * -ffp-contract=off.  The oracle is pinned against that reference build
 * (tests/test_oracle_vs_reference.py) and against the reference's golden
 * error tables (examples/1D_advection/*.csv, tests/test_golden.py).
 *
 * Periodic axes: the reference's single-rank periodic self-exchange
 * (src/HaloExchange.cpp:387-465 with MPI_Cart_shift returning self) copies
 * ghost -g <- n-g and n-1+g <- g-1, which is exactly the Periodic branch of
 * fillGhostX/Y/Z; the oracle implements it as that branch.
 */
#include "sifv.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAXPH SIFV_MAX_PHASES

/* std::max / std::min / std::clamp semantics (return the first argument
 * unless the comparison says otherwise; NaN handling follows from that). */
static inline double smax(double a, double b) { return (a < b) ? b : a; }
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline double sclamp(double v, double lo, double hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

/* PrimitiveState (include/State.hpp:18-29) */
typedef struct {
    double rho, u[3], p, T, sigma, gammaEff, piInfEff, alpha[MAXPH];
} Prim;

/* RiemannFlux (include/RiemannSolver.hpp:26-36) */
typedef struct {
    double massFlux, momentumFlux[3], energyFlux, alphaFlux[MAXPH], pressureFlux, faceVelocity;
} Flux;

typedef struct sifvo_ctx {
    sifv_config_t c;
    int dim, nx, ny, nz, ngx, ngy, ngz, nxT, nyT, nzT;
    size_t n;
    double *xExt, *yExt, *zExt;
    int bc[6];
    /* SolutionState (include/SolutionState.hpp:73-113) */
    double *rho, *rhoU, *rhoV, *rhoW, *rhoE, *velU, *velV, *velW, *pres, *sigma;
    double *alphaRho[MAXPH], *alpha[MAXPH];
    double *rho0, *rhoU0, *rhoV0, *rhoW0, *rhoE0, *pres0, *alphaRho0[MAXPH], *alpha0[MAXPH];
    double *rhoUStar, *rhoVStar, *rhoWStar, *rhoEstar, *pAdvected, *rhoc2;
    /* solver scratch */
    double *rhsRho, *rhsRhoU, *rhsRhoV, *rhsRhoW, *rhsRhoE, *rhsP, *divU;
    double *rhsAlphaRho[MAXPH], *rhsAlpha[MAXPH];
    double *gradU; /* 9 per cell */
    double *pressureRhs, *pressure, *divUstar, *pNew;
    Prim *xL, *xR, *yL, *yR, *zL, *zR;
    int lastIters;
    int pressureSolverKind; /* 0 Jacobi, 1 Gauss-Seidel */
    double time;            /* SimulationConfig::time of the current step */
    /* ImmersedBoundaryMethod (include/ImmersedBoundary.hpp:107-135) */
    unsigned char* cellType; /* NULL: no immersed boundary */
    struct IbGhost* ibGhost;
    int ibCount;
    sifv_ib_body_t* ibBodies;
    int ibNBodies;
    /* domain decomposition: faces with SIFV_BC_EXCHANGE, and the caller's
     * halo exchange / dt reduction (sifv_comm_t) */
    int exchangeFaces;
    sifv_comm_t comm;
    int commFailed; /* a hook failed (or was missing) during the current step */
    char err[256];
} ctx_t;

/* GhostCellInfo (include/ImmersedBoundary.hpp:96-103) */
typedef struct IbGhost {
    size_t cell;
    int body;
    double normal[3];
    int n;
    size_t interp[8];
    double w[8];
} IbGhost;

#define SOLID(m, idx) ((m)->cellType && (m)->cellType[idx] != SIFV_CELL_FLUID)

static char g_err[256];

/* ---- mesh (include/RectilinearMesh.hpp:70-105, src/RectilinearMesh.cpp) ---- */
static inline size_t IDX(const ctx_t* m, int i, int j, int k) {
    return (size_t)((i + m->ngx) + m->nxT * ((j + m->ngy) + m->nyT * (k + m->ngz)));
}
static inline double DX(const ctx_t* m, int i) { return m->xExt[i + m->ngx + 1] - m->xExt[i + m->ngx]; }
static inline double DY(const ctx_t* m, int j) { return m->yExt[j + m->ngy + 1] - m->yExt[j + m->ngy]; }
static inline double DZ(const ctx_t* m, int k) { return m->zExt[k + m->ngz + 1] - m->zExt[k + m->ngz]; }
static inline double VOL(const ctx_t* m, int i, int j, int k) { return DX(m, i) * DY(m, j) * DZ(m, k); }

/* RectilinearMesh::buildExtendedNodes, src/RectilinearMesh.cpp:91-114 */
static double* build_ext(const double* phys, int nCells, int ng) {
    int nExt = nCells + 2 * ng + 1;
    double* ext = (double*)calloc((size_t)nExt, sizeof(double));
    for (int i = 0; i <= nCells; ++i) ext[ng + i] = phys[i];
    for (int g = 1; g <= ng; ++g) {
        int mirror = (g - 1 < nCells - 1) ? g - 1 : nCells - 1;
        double width = phys[mirror + 1] - phys[mirror];
        ext[ng - g] = ext[ng - g + 1] - width;
    }
    for (int g = 1; g <= ng; ++g) {
        int mirror = (nCells - g > 0) ? nCells - g : 0;
        double width = phys[mirror + 1] - phys[mirror];
        ext[ng + nCells + g] = ext[ng + nCells + g - 1] + width;
    }
    return ext;
}

/* ---- ghost fill ---- */
/* SolutionState::copyCell_P, src/SolutionState.cpp:79-99 */
static void copy_cell_p(ctx_t* m, size_t dst, size_t src, double sU, double sV, double sW) {
    m->rho[dst] = m->rho[src];
    m->velU[dst] = sU * m->velU[src];
    if (m->dim >= 2) m->velV[dst] = sV * m->velV[src];
    if (m->dim >= 3) m->velW[dst] = sW * m->velW[src];
    m->pres[dst] = m->pres[src];
    m->sigma[dst] = m->sigma[src];
    for (int p = 0; p < m->c.nPhases; ++p) m->alphaRho[p][dst] = m->alphaRho[p][src];
    for (int p = 0; p < m->c.nPhases; ++p) m->alpha[p][dst] = m->alpha[p][src];
}

/* source index and velocity signs of one ghost layer g on one face
 * (the switch statements of src/RectilinearMesh.cpp:147-166,188-207) */
static int ghost_src(int bc, int high, int g, int n, double* s_norm, double* s_all) {
    *s_norm = 1.0;
    *s_all = 1.0;
    switch (bc) {
        case SIFV_BC_SYMMETRY: return high ? n - g : g - 1;
        case SIFV_BC_PERIODIC: return high ? g - 1 : n - g;
        case SIFV_BC_SLIPWALL: *s_norm = -1.0; return high ? n - g : g - 1;
        case SIFV_BC_NOSLIPWALL: *s_all = -1.0; return high ? n - g : g - 1;
        case SIFV_BC_OUTFLOW:
        default: return high ? n - 1 : 0;
    }
}

/* RectilinearMesh::applyBoundaryConditions (PRIM), src/RectilinearMesh.cpp:127-418;
 * with exchange faces (src/RectilinearMesh.cpp:498-524) the exchanged ghost
 * layers stay as converted, and the fills of the faster axes also cover
 * them (the reference's exchanged slabs carry the neighbour's already
 * filled ghosts of those axes). */
static void apply_bc_prim(ctx_t* m) {
    double sn, sa;
    const int EX = SIFV_BC_EXCHANGE;
    const int jlo = (m->dim >= 2 && m->bc[2] == EX) ? -m->ngy : 0, jhi = m->ny + ((m->dim >= 2 && m->bc[3] == EX) ? m->ngy : 0);
    const int klo = (m->dim >= 3 && m->bc[4] == EX) ? -m->ngz : 0, khi = m->nz + ((m->dim >= 3 && m->bc[5] == EX) ? m->ngz : 0);
    /* fillGhostX, src/RectilinearMesh.cpp:137-224 */
    for (int k = klo; k < khi; ++k)
        for (int j = jlo; j < jhi; ++j) {
            if (m->bc[0] != EX)
                for (int g = 1; g <= m->ngx; ++g) {
                    int si = ghost_src(m->bc[0], 0, g, m->nx, &sn, &sa);
                    copy_cell_p(m, IDX(m, -g, j, k), IDX(m, si, j, k), sn * sa, sa, sa);
                }
            if (m->bc[1] != EX)
                for (int g = 1; g <= m->ngx; ++g) {
                    int si = ghost_src(m->bc[1], 1, g, m->nx, &sn, &sa);
                    copy_cell_p(m, IDX(m, m->nx - 1 + g, j, k), IDX(m, si, j, k), sn * sa, sa, sa);
                }
        }
    /* fillGhostY, src/RectilinearMesh.cpp:230-320 */
    if (m->dim >= 2)
        for (int k = klo; k < khi; ++k)
            for (int i = -m->ngx; i < m->nx + m->ngx; ++i) {
                if (m->bc[2] != EX)
                    for (int g = 1; g <= m->ngy; ++g) {
                        int sj = ghost_src(m->bc[2], 0, g, m->ny, &sn, &sa);
                        copy_cell_p(m, IDX(m, i, -g, k), IDX(m, i, sj, k), sa, sn * sa, sa);
                    }
                if (m->bc[3] != EX)
                    for (int g = 1; g <= m->ngy; ++g) {
                        int sj = ghost_src(m->bc[3], 1, g, m->ny, &sn, &sa);
                        copy_cell_p(m, IDX(m, i, m->ny - 1 + g, k), IDX(m, i, sj, k), sa, sn * sa, sa);
                    }
            }
    /* fillGhostZ, src/RectilinearMesh.cpp:326-418 */
    if (m->dim >= 3)
        for (int j = -m->ngy; j < m->ny + m->ngy; ++j)
            for (int i = -m->ngx; i < m->nx + m->ngx; ++i) {
                if (m->bc[4] != EX)
                    for (int g = 1; g <= m->ngz; ++g) {
                        int sk = ghost_src(m->bc[4], 0, g, m->nz, &sn, &sa);
                        copy_cell_p(m, IDX(m, i, j, -g), IDX(m, i, j, sk), sa, sa, sn * sa);
                    }
                if (m->bc[5] != EX)
                    for (int g = 1; g <= m->ngz; ++g) {
                        int sk = ghost_src(m->bc[5], 1, g, m->nz, &sn, &sa);
                        copy_cell_p(m, IDX(m, i, j, m->nz - 1 + g), IDX(m, i, j, sk), sa, sa, sn * sa);
                    }
            }
}

/* Halo exchange of n fields through the caller's hook (HaloExchange,
 * src/HaloExchange.cpp:387-465): the nGhost layers next to every exchange
 * face to the neighbour, the neighbour's into the ghost layers.  A failure
 * is kept in commFailed and ends the step. */
static void exchange_n(ctx_t* m, double* const* f, int n) {
    if (!m->exchangeFaces) return;
    if (!m->comm.exchange || m->comm.exchange(m->comm.user, f, n, NULL) != 0) m->commFailed = 1;
}

/* Maximum over the ranks (the residual MPI_Allreduce of the pressure solvers,
 * src/JacobiPressureSolver.cpp:99-100, src/GaussSeidelPressureSolver.cpp:92-93). */
static void allreduce_max(ctx_t* m, double* v) {
    if (!m->exchangeFaces) return;
    if (!m->comm.allreduce_max || m->comm.allreduce_max(m->comm.user, v, NULL) != 0) m->commFailed = 1;
}

/* RectilinearMesh::fillScalarGhosts, src/RectilinearMesh.cpp:424-492, and
 * the halo variant 526-624: periodic wrap, otherwise zero gradient.  On a
 * decomposed mesh the exchange comes first and the faces it fills are
 * skipped; the faster axes' fills then also cover the exchanged ghost layers
 * of the slower axes, which reproduces the values the reference's
 * onion-peel order (fill x, exchange y including x ghosts, ...) gives there:
 * a ghost's source lies in its own line along the filled axis. */
static void fill_scalar_ghosts(ctx_t* m, double* f) {
    const int EX = SIFV_BC_EXCHANGE;
    exchange_n(m, &f, 1);
    const int jlo = (m->dim >= 2 && m->bc[2] == EX) ? -m->ngy : 0, jhi = m->ny + ((m->dim >= 2 && m->bc[3] == EX) ? m->ngy : 0);
    const int klo = (m->dim >= 3 && m->bc[4] == EX) ? -m->ngz : 0, khi = m->nz + ((m->dim >= 3 && m->bc[5] == EX) ? m->ngz : 0);
    for (int k = klo; k < khi; ++k)
        for (int j = jlo; j < jhi; ++j)
            for (int g = 1; g <= m->ngx; ++g) {
                if (m->bc[0] != EX)
                    f[IDX(m, -g, j, k)] = (m->bc[0] == SIFV_BC_PERIODIC) ? f[IDX(m, m->nx - g, j, k)] : f[IDX(m, 0, j, k)];
                if (m->bc[1] != EX)
                    f[IDX(m, m->nx - 1 + g, j, k)] =
                        (m->bc[1] == SIFV_BC_PERIODIC) ? f[IDX(m, g - 1, j, k)] : f[IDX(m, m->nx - 1, j, k)];
            }
    if (m->dim >= 2)
        for (int k = klo; k < khi; ++k)
            for (int i = -m->ngx; i < m->nx + m->ngx; ++i)
                for (int g = 1; g <= m->ngy; ++g) {
                    if (m->bc[2] != EX)
                        f[IDX(m, i, -g, k)] =
                            (m->bc[2] == SIFV_BC_PERIODIC) ? f[IDX(m, i, m->ny - g, k)] : f[IDX(m, i, 0, k)];
                    if (m->bc[3] != EX)
                        f[IDX(m, i, m->ny - 1 + g, k)] =
                            (m->bc[3] == SIFV_BC_PERIODIC) ? f[IDX(m, i, g - 1, k)] : f[IDX(m, i, m->ny - 1, k)];
                }
    if (m->dim >= 3)
        for (int j = -m->ngy; j < m->ny + m->ngy; ++j)
            for (int i = -m->ngx; i < m->nx + m->ngx; ++i)
                for (int g = 1; g <= m->ngz; ++g) {
                    if (m->bc[4] != EX)
                        f[IDX(m, i, j, -g)] =
                            (m->bc[4] == SIFV_BC_PERIODIC) ? f[IDX(m, i, j, m->nz - g)] : f[IDX(m, i, j, 0)];
                    if (m->bc[5] != EX)
                        f[IDX(m, i, j, m->nz - 1 + g)] =
                            (m->bc[5] == SIFV_BC_PERIODIC) ? f[IDX(m, i, j, g - 1)] : f[IDX(m, i, j, m->nz - 1)];
                }
}

/* ---- EOS ---- */
/* MixtureEOS::effectiveGammaAndPiInf, src/MixtureEOS.cpp:18-31 */
static void eff_gamma_piinf(const ctx_t* m, const double* alphas, double* gEff, double* piEff) {
    double sumInvGm1 = 0.0, sumPiInfTerm = 0.0;
    for (int ph = 0; ph < m->c.nPhases; ++ph) {
        double gk = m->c.phaseGamma[ph];
        double gm1 = gk - 1.0;
        sumInvGm1 += alphas[ph] / gm1;
        sumPiInfTerm += alphas[ph] * gk * m->c.phasePInf[ph] / gm1;
    }
    *gEff = 1.0 + 1.0 / sumInvGm1;
    *piEff = (*gEff - 1.0) / *gEff * sumPiInfTerm;
}

/* MixtureEOS::mixturePressure, src/MixtureEOS.cpp:35-46 */
static double mixture_pressure(const ctx_t* m, double rhoE_internal, const double* alphas) {
    double sumInvGm1 = 0.0, sumPInfTerm = 0.0;
    for (int ph = 0; ph < m->c.nPhases; ++ph) {
        double gm1 = m->c.phaseGamma[ph] - 1.0;
        sumInvGm1 += alphas[ph] / gm1;
        sumPInfTerm += alphas[ph] * m->c.phaseGamma[ph] * m->c.phasePInf[ph] / gm1;
    }
    return (rhoE_internal - sumPInfTerm) / sumInvGm1;
}

/* MixtureEOS::mixtureSoundSpeed (Wood), src/MixtureEOS.cpp:48-63 */
static double mixture_sound_speed(const ctx_t* m, double rho, double p, const double* alphas,
                                  const double* alphaRhos) {
    double sumInvRhoc2 = 0.0;
    for (int ph = 0; ph < m->c.nPhases; ++ph) {
        double a = alphas[ph];
        double rho_k = smax(alphaRhos[ph], 1e-14) / smax(a, 1e-14);
        double gk = m->c.phaseGamma[ph];
        double pInfk = m->c.phasePInf[ph];
        double ck2 = gk * (p + pInfk) / rho_k;
        sumInvRhoc2 += a / (rho_k * smax(ck2, 1e-14));
    }
    double c2 = 1.0 / (rho * smax(sumInvRhoc2, 1e-30));
    return sqrt(smax(c2, 0.0));
}

/* MixtureEOS::mixtureTotalEnergy, src/MixtureEOS.cpp:65-76 */
static double mixture_total_energy(const ctx_t* m, double p, const double* alphas, double ke) {
    double result = ke;
    for (int ph = 0; ph < m->c.nPhases; ++ph) {
        double gm1 = m->c.phaseGamma[ph] - 1.0;
        result += alphas[ph] * (p + m->c.phaseGamma[ph] * m->c.phasePInf[ph]) / gm1;
    }
    return result;
}

/* SolutionState::convertConservativeToPrimitiveVariables, src/SolutionState.cpp:187-205,
 * with IdealGasEOS::toPrimitive (src/IdealGasEOS.cpp:46-64) or
 * StiffenedGasEOS::toPrimitive (src/StiffenedGasEOS.cpp:47-64): one cell. */
static void cons_to_prim_single_cell(ctx_t* m, size_t idx) {
    const double g = m->c.gamma, pinf = m->c.pInf;
    const int stiff = (m->c.eosKind == SIFV_EOS_STIFFENED);
    double U[3] = {m->rhoU[idx], (m->dim >= 2) ? m->rhoV[idx] : 0.0, (m->dim >= 3) ? m->rhoW[idx] : 0.0};
    double rho = smax(m->rho[idx], 1e-14);
    double u[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < m->dim; ++d) u[d] = U[d] / rho;
    double ke = 0.0;
    for (int d = 0; d < m->dim; ++d) ke += u[d] * u[d];
    ke *= 0.5 * rho;
    double e = m->rhoE[idx] - ke;
    double p = stiff ? (g - 1.0) * e - g * pinf : smax((g - 1.0) * e, 1e-14);
    m->velU[idx] = u[0];
    if (m->dim >= 2) m->velV[idx] = u[1];
    if (m->dim >= 3) m->velW[idx] = u[2];
    m->pres[idx] = p;
}

/* MixtureEOS::convertConservativeToPrimitive, src/MixtureEOS.cpp:99-143: one cell */
static void cons_to_prim_mixture_cell(ctx_t* m, size_t idx) {
    double alphas[MAXPH];
    double rho = 0.0;
    for (int ph = 0; ph < m->c.nPhases; ++ph) rho += m->alphaRho[ph][idx];
    m->rho[idx] = smax(rho, 1e-14);
    double rs = m->rho[idx];
    m->velU[idx] = m->rhoU[idx] / rs;
    if (m->dim >= 2) m->velV[idx] = m->rhoV[idx] / rs;
    if (m->dim >= 3) m->velW[idx] = m->rhoW[idx] / rs;
    double ke = 0.5 * rs * m->velU[idx] * m->velU[idx];
    if (m->dim >= 2) ke += 0.5 * rs * m->velV[idx] * m->velV[idx];
    if (m->dim >= 3) ke += 0.5 * rs * m->velW[idx] * m->velW[idx];
    for (int ph = 0; ph < m->c.nPhases; ++ph) alphas[ph] = m->alpha[ph][idx];
    double rhoE_internal = m->rhoE[idx] - ke;
    m->pres[idx] = mixture_pressure(m, rhoE_internal, alphas);
}

static void cons_to_prim_box(ctx_t* m, int i0, int i1, int j0, int j1, int k0, int k1) {
    for (int k = k0; k < k1; ++k)
        for (int j = j0; j < j1; ++j)
            for (int i = i0; i < i1; ++i) {
                size_t idx = IDX(m, i, j, k);
                if (m->c.nPhases > 0) cons_to_prim_mixture_cell(m, idx);
                else cons_to_prim_single_cell(m, idx);
            }
}

/* Interior cells; on a decomposed mesh also the ghost layers of the
 * exchange faces, which hold the neighbour's conservative cells (the
 * reference exchanges the neighbour's primitives instead, the same values:
 * the conversion is per cell). */
static void cons_to_prim(ctx_t* m) {
    cons_to_prim_box(m, 0, m->nx, 0, m->ny, 0, m->nz);
    if (!m->exchangeFaces) return;
    if (m->bc[0] == SIFV_BC_EXCHANGE) cons_to_prim_box(m, -m->ngx, 0, 0, m->ny, 0, m->nz);
    if (m->bc[1] == SIFV_BC_EXCHANGE) cons_to_prim_box(m, m->nx, m->nx + m->ngx, 0, m->ny, 0, m->nz);
    if (m->dim >= 2 && m->bc[2] == SIFV_BC_EXCHANGE) cons_to_prim_box(m, 0, m->nx, -m->ngy, 0, 0, m->nz);
    if (m->dim >= 2 && m->bc[3] == SIFV_BC_EXCHANGE) cons_to_prim_box(m, 0, m->nx, m->ny, m->ny + m->ngy, 0, m->nz);
    if (m->dim >= 3 && m->bc[4] == SIFV_BC_EXCHANGE) cons_to_prim_box(m, 0, m->nx, 0, m->ny, -m->ngz, 0);
    if (m->dim >= 3 && m->bc[5] == SIFV_BC_EXCHANGE) cons_to_prim_box(m, 0, m->nx, 0, m->ny, m->nz, m->nz + m->ngz);
}

/* HaloExchange (src/HaloExchange.cpp:387-465) through the caller's hook:
 * the conservative cells next to every exchange face to the neighbour, the
 * neighbour's into the ghost layers. */
static int exchange_cons(ctx_t* m) {
    if (!m->exchangeFaces) return SIFV_OK;
    if (!m->comm.exchange) return SIFV_ERR_BAD_ARG;
    double* f[6 + 2 * MAXPH];
    int n = 0;
    f[n++] = m->rho;
    f[n++] = m->rhoU;
    if (m->dim >= 2) f[n++] = m->rhoV;
    if (m->dim >= 3) f[n++] = m->rhoW;
    f[n++] = m->rhoE;
    for (int ph = 0; ph < m->c.nPhases; ++ph) f[n++] = m->alphaRho[ph];
    for (int ph = 0; ph < m->c.nPhases; ++ph) f[n++] = m->alpha[ph];
    /* sigma travels with the reference's PRIM set; it matters with IGR and in
     * the semi-implicit correction */
    if (m->c.useIGR || m->c.semiImplicit) f[n++] = m->sigma;
    return m->comm.exchange(m->comm.user, f, n, NULL) == 0 ? SIFV_OK : SIFV_ERR_CUDA;
}

/* The reference's PRIM exchange (HaloExchange::packState, VarSet::PRIM,
 * src/HaloExchange.cpp:204-212) where the primitives are not functions of
 * the conservative cells: after the semi-implicit star update and after the
 * correction. */
static void exchange_prim(ctx_t* m) {
    if (!m->exchangeFaces) return;
    double* f[6 + 2 * MAXPH];
    int n = 0;
    f[n++] = m->rho;
    f[n++] = m->velU;
    if (m->dim >= 2) f[n++] = m->velV;
    if (m->dim >= 3) f[n++] = m->velW;
    f[n++] = m->pres;
    f[n++] = m->sigma;
    for (int ph = 0; ph < m->c.nPhases; ++ph) f[n++] = m->alphaRho[ph];
    for (int ph = 0; ph < m->c.nPhases; ++ph) f[n++] = m->alpha[ph];
    exchange_n(m, f, n);
}

/* ---- time steps ---- */
/* computeAcousticTimeStep, src/RKTimeStepping.cpp:43-123 */
static double acoustic_dt(const ctx_t* m, double cfl, double maxDt, int skipSolid) {
    double dt = maxDt;
    double alphas[MAXPH], alphaRhos[MAXPH];
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i < m->nx; ++i) {
                size_t idx = IDX(m, i, j, k);
                if (skipSolid && SOLID(m, idx)) continue;
                double c;
                if (m->c.nPhases > 0) {
                    for (int ph = 0; ph < m->c.nPhases; ++ph) alphas[ph] = m->alpha[ph][idx];
                    for (int ph = 0; ph < m->c.nPhases; ++ph) alphaRhos[ph] = m->alphaRho[ph][idx];
                    c = mixture_sound_speed(m, m->rho[idx], m->pres[idx], alphas, alphaRhos);
                } else {
                    c = sqrt(m->c.gamma * smax(m->pres[idx] + m->c.pInf, 1e-14) / smax(m->rho[idx], 1e-14));
                }
                double dtCell = DX(m, i) / (fabs(m->velU[idx]) + c);
                if (m->dim >= 2) dtCell = smin(dtCell, DY(m, j) / (fabs(m->velV[idx]) + c));
                if (m->dim >= 3) dtCell = smin(dtCell, DZ(m, k) / (fabs(m->velW[idx]) + c));
                dt = smin(dt, cfl * dtCell);
            }
    return dt;
}

/* computeAdvectiveTimeStep, src/RKTimeStepping.cpp:15-41 */
static double advective_dt(const ctx_t* m, double cfl, double maxDt) {
    double dt = maxDt;
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i < m->nx; ++i) {
                size_t idx = IDX(m, i, j, k);
                double dtCell = DX(m, i) / smax(fabs(m->velU[idx]), 1e-14);
                if (m->dim >= 2) dtCell = smin(dtCell, DY(m, j) / smax(fabs(m->velV[idx]), 1e-14));
                if (m->dim >= 3) dtCell = smin(dtCell, DZ(m, k) / smax(fabs(m->velW[idx]), 1e-14));
                dt = smin(dt, cfl * dtCell);
            }
    return dt;
}

/* ---- reconstruction, src/Reconstruction.cpp:83-200 ---- */
static double weno3L(const double* v, double eps) {
    double p0 = -0.5 * v[0] + 1.5 * v[1];
    double p1 = 0.5 * v[1] + 0.5 * v[2];
    double b0 = (v[1] - v[0]) * (v[1] - v[0]);
    double b1 = (v[2] - v[1]) * (v[2] - v[1]);
    const double d0 = 1.0 / 3.0, d1 = 2.0 / 3.0;
    double a0 = d0 / ((eps + b0) * (eps + b0));
    double a1 = d1 / ((eps + b1) * (eps + b1));
    double aSum = a0 + a1;
    return (a0 * p0 + a1 * p1) / aSum;
}
static double weno3R(const double* v, double eps) {
    double p0 = 0.5 * v[0] + 0.5 * v[1];
    double p1 = 1.5 * v[1] - 0.5 * v[2];
    double b0 = (v[1] - v[0]) * (v[1] - v[0]);
    double b1 = (v[2] - v[1]) * (v[2] - v[1]);
    const double d0 = 2.0 / 3.0, d1 = 1.0 / 3.0;
    double a0 = d0 / ((eps + b0) * (eps + b0));
    double a1 = d1 / ((eps + b1) * (eps + b1));
    double aSum = a0 + a1;
    return (a0 * p0 + a1 * p1) / aSum;
}
static double weno5L(const double* v, double eps) {
    double p0 = (1.0 / 3.0) * v[0] - (7.0 / 6.0) * v[1] + (11.0 / 6.0) * v[2];
    double p1 = -(1.0 / 6.0) * v[1] + (5.0 / 6.0) * v[2] + (1.0 / 3.0) * v[3];
    double p2 = (1.0 / 3.0) * v[2] + (5.0 / 6.0) * v[3] - (1.0 / 6.0) * v[4];
    double t0 = v[0] - 2.0 * v[1] + v[2], s0 = v[0] - 4.0 * v[1] + 3.0 * v[2];
    double t1 = v[1] - 2.0 * v[2] + v[3], s1 = v[1] - v[3];
    double t2 = v[2] - 2.0 * v[3] + v[4], s2 = 3.0 * v[2] - 4.0 * v[3] + v[4];
    double b0 = (13.0 / 12.0) * t0 * t0 + (1.0 / 4.0) * s0 * s0;
    double b1 = (13.0 / 12.0) * t1 * t1 + (1.0 / 4.0) * s1 * s1;
    double b2 = (13.0 / 12.0) * t2 * t2 + (1.0 / 4.0) * s2 * s2;
    const double d0 = 1.0 / 10.0, d1 = 6.0 / 10.0, d2 = 3.0 / 10.0;
    double a0 = d0 / ((eps + b0) * (eps + b0));
    double a1 = d1 / ((eps + b1) * (eps + b1));
    double a2 = d2 / ((eps + b2) * (eps + b2));
    double aSum = a0 + a1 + a2;
    return (a0 * p0 + a1 * p1 + a2 * p2) / aSum;
}
static double weno5R(const double* v, double eps) {
    double p0 = (1.0 / 3.0) * v[4] - (7.0 / 6.0) * v[3] + (11.0 / 6.0) * v[2];
    double p1 = -(1.0 / 6.0) * v[3] + (5.0 / 6.0) * v[2] + (1.0 / 3.0) * v[1];
    double p2 = (1.0 / 3.0) * v[2] + (5.0 / 6.0) * v[1] - (1.0 / 6.0) * v[0];
    double t0 = v[4] - 2.0 * v[3] + v[2], s0 = v[4] - 4.0 * v[3] + 3.0 * v[2];
    double t1 = v[3] - 2.0 * v[2] + v[1], s1 = v[3] - v[1];
    double t2 = v[2] - 2.0 * v[1] + v[0], s2 = 3.0 * v[2] - 4.0 * v[1] + v[0];
    double b0 = (13.0 / 12.0) * t0 * t0 + (1.0 / 4.0) * s0 * s0;
    double b1 = (13.0 / 12.0) * t1 * t1 + (1.0 / 4.0) * s1 * s1;
    double b2 = (13.0 / 12.0) * t2 * t2 + (1.0 / 4.0) * s2 * s2;
    const double d0 = 1.0 / 10.0, d1 = 6.0 / 10.0, d2 = 3.0 / 10.0;
    double a0 = d0 / ((eps + b0) * (eps + b0));
    double a1 = d1 / ((eps + b1) * (eps + b1));
    double a2 = d2 / ((eps + b2) * (eps + b2));
    double aSum = a0 + a1 + a2;
    return (a0 * p0 + a1 * p1 + a2 * p2) / aSum;
}
static double upwind3L(const double* v, double eps) {
    (void)eps;
    double p0 = -0.5 * v[0] + 1.5 * v[1];
    double p1 = 0.5 * v[1] + 0.5 * v[2];
    return (1.0 / 3.0) * p0 + (2.0 / 3.0) * p1;
}
static double upwind3R(const double* v, double eps) {
    (void)eps;
    double p0 = 0.5 * v[0] + 0.5 * v[1];
    double p1 = 1.5 * v[1] - 0.5 * v[2];
    return (2.0 / 3.0) * p0 + (1.0 / 3.0) * p1;
}
static double upwind5L(const double* v, double eps) {
    (void)eps;
    double p0 = (1.0 / 3.0) * v[0] - (7.0 / 6.0) * v[1] + (11.0 / 6.0) * v[2];
    double p1 = -(1.0 / 6.0) * v[1] + (5.0 / 6.0) * v[2] + (1.0 / 3.0) * v[3];
    double p2 = (1.0 / 3.0) * v[2] + (5.0 / 6.0) * v[3] - (1.0 / 6.0) * v[4];
    return (1.0 / 10.0) * p0 + (6.0 / 10.0) * p1 + (3.0 / 10.0) * p2;
}
static double upwind5R(const double* v, double eps) {
    (void)eps;
    double p0 = (1.0 / 3.0) * v[4] - (7.0 / 6.0) * v[3] + (11.0 / 6.0) * v[2];
    double p1 = -(1.0 / 6.0) * v[3] + (5.0 / 6.0) * v[2] + (1.0 / 3.0) * v[1];
    double p2 = (1.0 / 3.0) * v[2] + (5.0 / 6.0) * v[1] - (1.0 / 6.0) * v[0];
    return (1.0 / 10.0) * p0 + (6.0 / 10.0) * p1 + (3.0 / 10.0) * p2;
}

typedef double (*ReconFn)(const double*, double);

/* reconstructScalar, src/Reconstruction.cpp:11-28 */
static void recon_scalar(const double* f, const size_t* cells, int w, ReconFn lf, ReconFn rf, double eps,
                         double* outL, double* outR) {
    double vL[5], vR[5];
    for (int s = 0; s < w; ++s) {
        vL[s] = f[cells[s]];
        vR[s] = f[cells[s + 1]];
    }
    *outL = lf(vL, eps);
    *outR = rf(vR, eps);
}

static void zero_prim(Prim* p) { memset(p, 0, sizeof(Prim)); }

/* One face of Reconstructor::reconstructX/Y/Z (src/Reconstruction.cpp:204-541).
 * `cellAt(o)` is the flat index of the cell at offset o along the sweep
 * direction from the face's right cell (o = -3..2). */
static void recon_face(ctx_t* m, const size_t* off, Prim* L, Prim* R) {
    const int order = m->c.reconOrder;
    const double eps = m->c.wenoEps;
    const int nPh = m->c.nPhases;
    zero_prim(L);
    zero_prim(R);
    if (order == SIFV_WENO1 || order == SIFV_UPWIND1) {
        size_t iL = off[2], iR = off[3];
        L->rho = m->rho[iL]; L->u[0] = m->velU[iL]; L->p = m->pres[iL]; L->sigma = m->sigma[iL];
        R->rho = m->rho[iR]; R->u[0] = m->velU[iR]; R->p = m->pres[iR]; R->sigma = m->sigma[iR];
        if (m->dim >= 2) { L->u[1] = m->velV[iL]; R->u[1] = m->velV[iR]; }
        if (m->dim >= 3) { L->u[2] = m->velW[iL]; R->u[2] = m->velW[iR]; }
        for (int ph = 0; ph < nPh; ++ph) { L->alpha[ph] = m->alpha[ph][iL]; R->alpha[ph] = m->alpha[ph][iR]; }
    } else {
        int w;
        const size_t* c;
        ReconFn lf, rf;
        if (order == SIFV_WENO3 || order == SIFV_UPWIND3) {
            w = 3;
            c = off + 1; /* i-2 .. i+1 */
            lf = (order == SIFV_WENO3) ? weno3L : upwind3L;
            rf = (order == SIFV_WENO3) ? weno3R : upwind3R;
        } else {
            w = 5;
            c = off; /* i-3 .. i+2 */
            lf = (order == SIFV_WENO5) ? weno5L : upwind5L;
            rf = (order == SIFV_WENO5) ? weno5R : upwind5R;
        }
        recon_scalar(m->rho, c, w, lf, rf, eps, &L->rho, &R->rho);
        recon_scalar(m->velU, c, w, lf, rf, eps, &L->u[0], &R->u[0]);
        if (m->dim >= 2) recon_scalar(m->velV, c, w, lf, rf, eps, &L->u[1], &R->u[1]);
        if (m->dim >= 3) recon_scalar(m->velW, c, w, lf, rf, eps, &L->u[2], &R->u[2]);
        recon_scalar(m->pres, c, w, lf, rf, eps, &L->p, &R->p);
        recon_scalar(m->sigma, c, w, lf, rf, eps, &L->sigma, &R->sigma);
        for (int ph = 0; ph < nPh; ++ph)
            recon_scalar(m->alpha[ph], c, w, lf, rf, eps, &L->alpha[ph], &R->alpha[ph]);
    }
    if (nPh > 0) {
        eff_gamma_piinf(m, L->alpha, &L->gammaEff, &L->piInfEff);
        eff_gamma_piinf(m, R->alpha, &R->gammaEff, &R->piInfEff);
    } else {
        L->gammaEff = m->c.gamma; L->piInfEff = m->c.pInf;
        R->gammaEff = m->c.gamma; R->piInfEff = m->c.pInf;
    }
}

/* Reconstructor::reconstruct, src/Reconstruction.cpp:543-552 */
static void reconstruct(ctx_t* m) {
    size_t off[6];
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i <= m->nx; ++i) {
                for (int o = 0; o < 6; ++o) off[o] = IDX(m, i - 3 + o, j, k);
                size_t f = (size_t)(i + (m->nx + 1) * (j + m->ny * k));
                recon_face(m, off, &m->xL[f], &m->xR[f]);
            }
    if (m->dim >= 2)
        for (int k = 0; k < m->nz; ++k)
            for (int j = 0; j <= m->ny; ++j)
                for (int i = 0; i < m->nx; ++i) {
                    for (int o = 0; o < 6; ++o) off[o] = IDX(m, i, j - 3 + o, k);
                    size_t f = (size_t)(i + m->nx * (j + (m->ny + 1) * k));
                    recon_face(m, off, &m->yL[f], &m->yR[f]);
                }
    if (m->dim >= 3)
        for (int k = 0; k <= m->nz; ++k)
            for (int j = 0; j < m->ny; ++j)
                for (int i = 0; i < m->nx; ++i) {
                    for (int o = 0; o < 6; ++o) off[o] = IDX(m, i, j, k - 3 + o);
                    size_t f = (size_t)(i + m->nx * (j + m->ny * k));
                    recon_face(m, off, &m->zL[f], &m->zR[f]);
                }
}

/* ---- Riemann solvers ---- */
/* normalVelocity, include/RiemannSolver.hpp:59-64 */
static double normal_velocity(const Prim* W, const double* n, int dim) {
    double vn = 0.0;
    for (int d = 0; d < dim; ++d) vn += W->u[d] * n[d];
    return vn;
}
/* soundSpeedDirect / rhoEFromState, include/RiemannSolver.hpp:70-78 */
static double sound_speed_direct(const Prim* W) {
    return sqrt(W->gammaEff * smax(W->p + W->piInfEff, 1e-14) / smax(W->rho, 1e-14));
}
static double rhoE_from_state(const Prim* W) {
    double ke = 0.5 * W->rho * (W->u[0] * W->u[0] + W->u[1] * W->u[1] + W->u[2] * W->u[2]);
    return (W->p + W->gammaEff * W->piInfEff) / (W->gammaEff - 1.0) + ke;
}

/* computeHLLCFlux, src/HLLCSolver.cpp:7-161 */
static void hllc_flux(const Prim* L, const Prim* R, const double* n, int dim, int incP, int nPh, Flux* F) {
    memset(F, 0, sizeof(Flux));
    double uL = normal_velocity(L, n, dim), uR = normal_velocity(R, n, dim);
    double rhoEL = rhoE_from_state(L), rhoER = rhoE_from_state(R);
    double sL, sR, sStar;
    if (incP) {
        double cL = sound_speed_direct(L), cR = sound_speed_direct(R);
        sL = smin(uL - cL, uR - cR);
        sR = smax(uL + cL, uR + cR);
        sStar = (R->p - L->p + L->rho * uL * (sL - uL) - R->rho * uR * (sR - uR)) /
                (L->rho * (sL - uL) - R->rho * (sR - uR));
    } else {
        sL = smin(uL, uR);
        sR = smax(uL, uR);
        sStar = 0.5 * (uL + uR);
    }
    if (sL >= 0) {
        F->massFlux = L->rho * uL;
        for (int i = 0; i < dim; ++i) F->momentumFlux[i] = L->rho * L->u[i] * uL;
        F->energyFlux = rhoEL * uL;
        if (incP) {
            for (int i = 0; i < dim; ++i) F->momentumFlux[i] += L->p * n[i];
            F->energyFlux += L->p * uL;
        }
    } else if (sR <= 0) {
        F->massFlux = R->rho * uR;
        for (int i = 0; i < dim; ++i) F->momentumFlux[i] = R->rho * R->u[i] * uR;
        F->energyFlux = rhoER * uR;
        if (incP) {
            for (int i = 0; i < dim; ++i) F->momentumFlux[i] += R->p * n[i];
            F->energyFlux += R->p * uR;
        }
    } else if (sStar >= 0) {
        double rhoStarL = L->rho * (sL - uL) / (sL - sStar);
        F->massFlux = L->rho * uL + sL * (rhoStarL - L->rho);
        if (incP) {
            for (int i = 0; i < dim; ++i) {
                double rhoUStarL = rhoStarL * (L->u[i] + (sStar - uL) * n[i]);
                F->momentumFlux[i] = L->rho * L->u[i] * uL + L->p * n[i] + sL * (rhoUStarL - L->rho * L->u[i]);
            }
            double eL = rhoEL / L->rho;
            double EStarL = rhoStarL * (eL + (sStar - uL) * (sStar + L->p / (L->rho * (sL - uL))));
            F->energyFlux = (rhoEL + L->p) * uL + sL * (EStarL - rhoEL);
        } else {
            for (int i = 0; i < dim; ++i) {
                double rhoUStarL = rhoStarL * (L->u[i] + (sStar - uL) * n[i]);
                F->momentumFlux[i] = L->rho * L->u[i] * uL + sL * (rhoUStarL - L->rho * L->u[i]);
            }
            double eL = rhoEL / L->rho;
            double EStarL = rhoStarL * (eL + (sStar - uL) * sStar);
            F->energyFlux = rhoEL * uL + sL * (EStarL - rhoEL);
        }
    } else {
        double rhoStarR = R->rho * (sR - uR) / (sR - sStar);
        F->massFlux = R->rho * uR + sR * (rhoStarR - R->rho);
        if (incP) {
            for (int i = 0; i < dim; ++i) {
                double rhoUStarR = rhoStarR * (R->u[i] + (sStar - uR) * n[i]);
                F->momentumFlux[i] = R->rho * R->u[i] * uR + R->p * n[i] + sR * (rhoUStarR - R->rho * R->u[i]);
            }
            double eR = rhoER / R->rho;
            double EStarR = rhoStarR * (eR + (sStar - uR) * (sStar + R->p / (R->rho * (sR - uR))));
            F->energyFlux = (rhoER + R->p) * uR + sR * (EStarR - rhoER);
        } else {
            for (int i = 0; i < dim; ++i) {
                double rhoUStarR = rhoStarR * (R->u[i] + (sStar - uR) * n[i]);
                F->momentumFlux[i] = R->rho * R->u[i] * uR + sR * (rhoUStarR - R->rho * R->u[i]);
            }
            double eR = rhoER / R->rho;
            double EStarR = rhoStarR * (eR + (sStar - uR) * sStar);
            F->energyFlux = rhoER * uR + sR * (EStarR - rhoER);
        }
    }
    if (sL >= 0) {
        F->faceVelocity = uL;
        F->pressureFlux = L->p * uL;
        for (int ph = 0; ph < nPh; ++ph) F->alphaFlux[ph] = L->alpha[ph] * uL;
    } else if (sR <= 0) {
        F->faceVelocity = uR;
        F->pressureFlux = R->p * uR;
        for (int ph = 0; ph < nPh; ++ph) F->alphaFlux[ph] = R->alpha[ph] * uR;
    } else {
        F->faceVelocity = sStar;
        if (sStar >= 0) {
            F->pressureFlux = L->p * sStar;
            for (int ph = 0; ph < nPh; ++ph) F->alphaFlux[ph] = L->alpha[ph] * sStar;
        } else {
            F->pressureFlux = R->p * sStar;
            for (int ph = 0; ph < nPh; ++ph) F->alphaFlux[ph] = R->alpha[ph] * sStar;
        }
    }
}

/* computeRusanovFlux, src/RusanovSolver.cpp:7-83 */
static void rusanov_flux(const Prim* L, const Prim* R, const double* n, int dim, int incP, int nPh, Flux* F) {
    memset(F, 0, sizeof(Flux));
    double uL = normal_velocity(L, n, dim), uR = normal_velocity(R, n, dim);
    double absUL = fabs(normal_velocity(L, n, dim)), absUR = fabs(normal_velocity(R, n, dim));
    double sMax;
    if (incP) {
        double cL = sound_speed_direct(L), cR = sound_speed_direct(R);
        sMax = smax(absUL + cL, absUR + cR);
    } else {
        sMax = smax(absUL, absUR);
    }
    double rhoEL = rhoE_from_state(L), rhoER = rhoE_from_state(R);
    double massFluxL = L->rho * uL, momFluxL[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < dim; ++i) momFluxL[i] = L->rho * L->u[i] * uL;
    double energyFluxL = rhoEL * uL;
    double massFluxR = R->rho * uR, momFluxR[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < dim; ++i) momFluxR[i] = R->rho * R->u[i] * uR;
    double energyFluxR = rhoER * uR;
    if (incP) {
        for (int i = 0; i < dim; ++i) {
            momFluxL[i] += L->p * n[i];
            momFluxR[i] += R->p * n[i];
        }
        energyFluxL += L->p * uL;
        energyFluxR += R->p * uR;
    }
    F->massFlux = 0.5 * (massFluxL + massFluxR) - 0.5 * sMax * (R->rho - L->rho);
    for (int i = 0; i < dim; ++i)
        F->momentumFlux[i] = 0.5 * (momFluxL[i] + momFluxR[i]) - 0.5 * sMax * (R->rho * R->u[i] - L->rho * L->u[i]);
    F->energyFlux = 0.5 * (energyFluxL + energyFluxR) - 0.5 * sMax * (rhoER - rhoEL);
    F->faceVelocity = 0.5 * (uL + uR);
    F->pressureFlux = 0.5 * (L->p * uL + R->p * uR) - 0.5 * sMax * (R->p - L->p);
    for (int ph = 0; ph < nPh; ++ph)
        F->alphaFlux[ph] = 0.5 * (L->alpha[ph] * uL + R->alpha[ph] * uR) - 0.5 * sMax * (R->alpha[ph] - L->alpha[ph]);
}

/* computeLFFlux, src/LFSolver.cpp:8-75 */
static void lf_flux(const Prim* L, const Prim* R, const double* n, int dim, int incP, int useIGR, int nPh, Flux* F) {
    memset(F, 0, sizeof(Flux));
    double uL = normal_velocity(L, n, dim), uR = normal_velocity(R, n, dim);
    double uLS = 0.0, uRS = 0.0;
    for (int i = 0; i < dim; ++i) {
        uLS += L->u[i] * L->u[i];
        uRS += R->u[i] * R->u[i];
    }
    uLS = sqrt(uLS);
    uRS = sqrt(uRS);
    double Cc;
    if (incP) {
        double cL = sound_speed_direct(L), cR = sound_speed_direct(R);
        Cc = smax(uLS, uRS) + smax(cL, cR);
    } else {
        Cc = smax(uLS, uRS);
    }
    F->massFlux = 0.5 * (L->rho * uL + R->rho * uR) - 0.5 * Cc * (R->rho - L->rho);
    for (int i = 0; i < dim; ++i)
        F->momentumFlux[i] = 0.5 * (L->rho * L->u[i] * uL + R->rho * R->u[i] * uR) -
                             0.5 * Cc * (R->rho * R->u[i] - L->rho * L->u[i]);
    double rhoEL = rhoE_from_state(L), rhoER = rhoE_from_state(R);
    F->energyFlux = 0.5 * (rhoEL * uL + rhoER * uR) - 0.5 * Cc * (rhoER - rhoEL);
    if (incP) {
        for (int i = 0; i < dim; ++i) F->momentumFlux[i] += 0.5 * (L->p + R->p) * n[i];
        F->energyFlux += 0.5 * (L->p * uL + R->p * uR);
    }
    if (useIGR) {
        for (int i = 0; i < dim; ++i) F->momentumFlux[i] += 0.5 * (L->sigma + R->sigma) * n[i];
        F->energyFlux += 0.5 * (L->sigma * uL + R->sigma * uR);
    }
    F->faceVelocity = 0.5 * (uL + uR);
    F->pressureFlux = 0.5 * (L->p * uL + R->p * uR) - 0.5 * Cc * (R->p - L->p);
    for (int ph = 0; ph < nPh; ++ph)
        F->alphaFlux[ph] = 0.5 * (L->alpha[ph] * uL + R->alpha[ph] * uR) - 0.5 * Cc * (R->alpha[ph] - L->alpha[ph]);
}

/* computeFluxDirect, include/RiemannSolver.hpp:91-100 */
static void flux_direct(const ctx_t* m, const Prim* L, const Prim* R, const double* n, Flux* F) {
    int incP = !m->c.semiImplicit;
    switch (m->c.riemannSolver) {
        case SIFV_HLLC: hllc_flux(L, R, n, m->dim, incP, m->c.nPhases, F); break;
        case SIFV_RUSANOV: rusanov_flux(L, R, n, m->dim, incP, m->c.nPhases, F); break;
        default: lf_flux(L, R, n, m->dim, incP, m->c.useIGR, m->c.nPhases, F); break;
    }
}

/* ---- flux divergence ---- */
/* The face loops of ExplicitSolver::computeRHS (src/ExplicitSolver.cpp:294-483)
 * and SemiImplicitSolver::computeRHS (src/SemiImplicitSolver.cpp:263-457):
 * scatter -coeff*F into the left cell and +coeff*F into the right cell, in
 * face order. */
static void scatter_face(ctx_t* m, const Flux* F, int hasL, size_t iL, double coeffL, int hasR, size_t iR,
                         double coeffR, size_t upw) {
    const int nPh = m->c.nPhases;
    const int semi = m->c.semiImplicit;
    if (hasL) {
        double coeff = coeffL;
        m->rhsRho[iL] -= coeff * F->massFlux;
        m->rhsRhoU[iL] -= coeff * F->momentumFlux[0];
        if (m->dim >= 2) m->rhsRhoV[iL] -= coeff * F->momentumFlux[1];
        if (m->dim >= 3) m->rhsRhoW[iL] -= coeff * F->momentumFlux[2];
        m->rhsRhoE[iL] -= coeff * F->energyFlux;
        if (semi) {
            m->rhsP[iL] -= coeff * F->pressureFlux;
            m->divU[iL] += coeff * F->faceVelocity;
        }
        if (nPh > 0) {
            double rhoUpw = smax(m->rho[upw], 1e-14);
            for (int ph = 0; ph < nPh; ++ph) {
                double arf = (m->alphaRho[ph][upw] / rhoUpw) * F->massFlux;
                m->rhsAlphaRho[ph][iL] -= coeff * arf;
            }
            for (int ph = 0; ph < nPh; ++ph) m->rhsAlpha[ph][iL] -= coeff * F->alphaFlux[ph];
            if (!semi) m->divU[iL] += coeff * F->faceVelocity;
        }
    }
    if (hasR) {
        double coeff = coeffR;
        m->rhsRho[iR] += coeff * F->massFlux;
        m->rhsRhoU[iR] += coeff * F->momentumFlux[0];
        if (m->dim >= 2) m->rhsRhoV[iR] += coeff * F->momentumFlux[1];
        if (m->dim >= 3) m->rhsRhoW[iR] += coeff * F->momentumFlux[2];
        m->rhsRhoE[iR] += coeff * F->energyFlux;
        if (semi) {
            m->rhsP[iR] += coeff * F->pressureFlux;
            m->divU[iR] -= coeff * F->faceVelocity;
        }
        if (nPh > 0) {
            double rhoUpw = smax(m->rho[upw], 1e-14);
            for (int ph = 0; ph < nPh; ++ph) {
                double arf = (m->alphaRho[ph][upw] / rhoUpw) * F->massFlux;
                m->rhsAlphaRho[ph][iR] += coeff * arf;
            }
            for (int ph = 0; ph < nPh; ++ph) m->rhsAlpha[ph][iR] += coeff * F->alphaFlux[ph];
            if (!semi) m->divU[iR] -= coeff * F->faceVelocity;
        }
    }
}

static int has_viscosity(const sifv_config_t* c);
static void add_viscous_fluxes(ctx_t* m);
static void ib_apply_ghosts(ctx_t* m);
static void ib_apply_scalar(ctx_t* m, double* f);
static void add_surface_tension_fluxes(ctx_t* m);

static void compute_rhs(ctx_t* m) {
    const int nPh = m->c.nPhases;
    const int semi = m->c.semiImplicit;
    const size_t n = m->n;
    Flux F;
    reconstruct(m);
    memset(m->rhsRho, 0, n * sizeof(double));
    memset(m->rhsRhoU, 0, n * sizeof(double));
    if (m->dim >= 2) memset(m->rhsRhoV, 0, n * sizeof(double));
    if (m->dim >= 3) memset(m->rhsRhoW, 0, n * sizeof(double));
    memset(m->rhsRhoE, 0, n * sizeof(double));
    if (semi) memset(m->rhsP, 0, n * sizeof(double));
    if (semi || nPh > 0) memset(m->divU, 0, n * sizeof(double));
    for (int ph = 0; ph < nPh; ++ph) {
        memset(m->rhsAlphaRho[ph], 0, n * sizeof(double));
        memset(m->rhsAlpha[ph], 0, n * sizeof(double));
    }
    const double nx_[3] = {1.0, 0.0, 0.0}, ny_[3] = {0.0, 1.0, 0.0}, nz_[3] = {0.0, 0.0, 1.0};
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i <= m->nx; ++i) {
                size_t f = (size_t)(i + (m->nx + 1) * (j + m->ny * k));
                flux_direct(m, &m->xL[f], &m->xR[f], nx_, &F);
                double area = DY(m, j) * DZ(m, k);
                size_t upw = 0;
                if (nPh > 0) upw = (F.massFlux >= 0) ? IDX(m, i - 1, j, k) : IDX(m, i, j, k);
                scatter_face(m, &F, i >= 1, IDX(m, i - 1, j, k), (i >= 1) ? area / VOL(m, i - 1, j, k) : 0.0,
                             i < m->nx, IDX(m, i, j, k), (i < m->nx) ? area / VOL(m, i, j, k) : 0.0, upw);
            }
    if (m->dim >= 2)
        for (int k = 0; k < m->nz; ++k)
            for (int j = 0; j <= m->ny; ++j)
                for (int i = 0; i < m->nx; ++i) {
                    size_t f = (size_t)(i + m->nx * (j + (m->ny + 1) * k));
                    flux_direct(m, &m->yL[f], &m->yR[f], ny_, &F);
                    double area = DX(m, i) * DZ(m, k);
                    size_t upw = 0;
                    if (nPh > 0) upw = (F.massFlux >= 0) ? IDX(m, i, j - 1, k) : IDX(m, i, j, k);
                    scatter_face(m, &F, j >= 1, IDX(m, i, j - 1, k), (j >= 1) ? area / VOL(m, i, j - 1, k) : 0.0,
                                 j < m->ny, IDX(m, i, j, k), (j < m->ny) ? area / VOL(m, i, j, k) : 0.0, upw);
                }
    if (m->dim >= 3)
        for (int k = 0; k <= m->nz; ++k)
            for (int j = 0; j < m->ny; ++j)
                for (int i = 0; i < m->nx; ++i) {
                    size_t f = (size_t)(i + m->nx * (j + m->ny * k));
                    flux_direct(m, &m->zL[f], &m->zR[f], nz_, &F);
                    double area = DX(m, i) * DY(m, j);
                    size_t upw = 0;
                    if (nPh > 0) upw = (F.massFlux >= 0) ? IDX(m, i, j, k - 1) : IDX(m, i, j, k);
                    scatter_face(m, &F, k >= 1, IDX(m, i, j, k - 1), (k >= 1) ? area / VOL(m, i, j, k - 1) : 0.0,
                                 k < m->nz, IDX(m, i, j, k), (k < m->nz) ? area / VOL(m, i, j, k) : 0.0, upw);
                }
    /* alpha source alpha div(u): src/ExplicitSolver.cpp:485-496, src/SemiImplicitSolver.cpp:459-470 */
    if (nPh > 0)
        for (int k = 0; k < m->nz; ++k)
            for (int j = 0; j < m->ny; ++j)
                for (int i = 0; i < m->nx; ++i) {
                    size_t idx = IDX(m, i, j, k);
                    for (int ph = 0; ph < nPh; ++ph) m->rhsAlpha[ph][idx] += m->alpha[ph][idx] * m->divU[idx];
                }
    /* p div(u) source: src/SemiImplicitSolver.cpp:472-482 */
    if (semi)
        for (int k = 0; k < m->nz; ++k)
            for (int j = 0; j < m->ny; ++j)
                for (int i = 0; i < m->nx; ++i) {
                    size_t idx = IDX(m, i, j, k);
                    m->rhsP[idx] += m->pres[idx] * m->divU[idx];
                }
    /* body force: src/ExplicitSolver.cpp:498-521, src/SemiImplicitSolver.cpp:484-507 */
    int hasBF = 0;
    for (int d = 0; d < 3; ++d)
        if (m->c.bfA[d] != 0.0 || m->c.bfB[d] != 0.0) hasBF = 1;
    if (hasBF) {
        double t = m->time;
        double ax = m->c.bfA[0] + m->c.bfB[0] * cos(m->c.bfC[0] * t + m->c.bfD[0]);
        double ay = m->c.bfA[1] + m->c.bfB[1] * cos(m->c.bfC[1] * t + m->c.bfD[1]);
        double az = m->c.bfA[2] + m->c.bfB[2] * cos(m->c.bfC[2] * t + m->c.bfD[2]);
        for (int k = 0; k < m->nz; ++k)
            for (int j = 0; j < m->ny; ++j)
                for (int i = 0; i < m->nx; ++i) {
                    size_t idx = IDX(m, i, j, k);
                    m->rhsRhoU[idx] += m->rho[idx] * ax;
                    if (m->dim >= 2) m->rhsRhoV[idx] += m->rho[idx] * ay;
                    if (m->dim >= 3) m->rhsRhoW[idx] += m->rho[idx] * az;
                    double work = m->velU[idx] * ax;
                    if (m->dim >= 2) work += m->velV[idx] * ay;
                    if (m->dim >= 3) work += m->velW[idx] * az;
                    m->rhsRhoE[idx] += m->rho[idx] * work;
                }
    }
    /* viscous stress: src/ExplicitSolver.cpp:523-527, src/SemiImplicitSolver.cpp:509-513 */
    if (has_viscosity(&m->c)) add_viscous_fluxes(m);
    /* capillary stress: src/ExplicitSolver.cpp:529-534, src/SemiImplicitSolver.cpp:515-520 */
    if (m->c.stSigma > 0.0) add_surface_tension_fluxes(m);
}

/* ---- viscous stress: addViscousFluxes, src/ViscousFlux.cpp:24-303 ---- */
static int has_viscosity(const sifv_config_t* c) { return c->mu > 0.0 || c->nPhaseMu > 0; }

/* computeFaceMu (src/ViscousFlux.cpp:8-21): mixture rule per cell, face average */
static double face_mu(const ctx_t* m, size_t iL, size_t iR) {
    if (m->c.nPhaseMu == 0) return m->c.mu;
    double muL = 0.0, muR = 0.0;
    for (int ph = 0; ph < m->c.nPhases; ++ph) {
        muL += m->alpha[ph][iL] * m->c.phaseMu[ph];
        muR += m->alpha[ph][iR] * m->c.phaseMu[ph];
    }
    return 0.5 * (muL + muR);
}

/* accumulate one face's stress into its two cells (L: +, R: -) */
static void visc_scatter(ctx_t* m, int hasL, size_t iL, double cL, int hasR, size_t iR, double cR, double t0,
                         double t1, double t2, double work) {
    const int dim = m->dim;
    if (hasL) {
        m->rhsRhoU[iL] += cL * t0;
        if (dim >= 2) m->rhsRhoV[iL] += cL * t1;
        if (dim >= 3) m->rhsRhoW[iL] += cL * t2;
        m->rhsRhoE[iL] += cL * work;
    }
    if (hasR) {
        m->rhsRhoU[iR] -= cR * t0;
        if (dim >= 2) m->rhsRhoV[iR] -= cR * t1;
        if (dim >= 3) m->rhsRhoW[iR] -= cR * t2;
        m->rhsRhoE[iR] -= cR * work;
    }
}

static void add_viscous_fluxes(ctx_t* m) {
    const int dim = m->dim;
    const double* U = m->velU;
    const double* V = m->velV;
    const double* W = m->velW;
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i <= m->nx; ++i) {
                size_t iL = IDX(m, i - 1, j, k), iR = IDX(m, i, j, k);
                double dxi = 0.5 * (DX(m, i - 1) + DX(m, i));
                double dudx = (U[iR] - U[iL]) / dxi, dvdx = 0.0, dwdx = 0.0;
                if (dim >= 2) dvdx = (V[iR] - V[iL]) / dxi;
                if (dim >= 3) dwdx = (W[iR] - W[iL]) / dxi;
                double dudy = 0.0, dvdy = 0.0;
                if (dim >= 2) {
                    double dyj = DY(m, j);
                    size_t Ljm = IDX(m, i - 1, j - 1, k), Ljp = IDX(m, i - 1, j + 1, k);
                    size_t Rjm = IDX(m, i, j - 1, k), Rjp = IDX(m, i, j + 1, k);
                    double dudyL = (U[Ljp] - U[Ljm]) / (2.0 * dyj), dudyR = (U[Rjp] - U[Rjm]) / (2.0 * dyj);
                    dudy = 0.5 * (dudyL + dudyR);
                    double dvdyL = (V[Ljp] - V[Ljm]) / (2.0 * dyj), dvdyR = (V[Rjp] - V[Rjm]) / (2.0 * dyj);
                    dvdy = 0.5 * (dvdyL + dvdyR);
                }
                double dudz = 0.0, dwdz = 0.0;
                if (dim >= 3) {
                    double dzk = DZ(m, k);
                    size_t Lkm = IDX(m, i - 1, j, k - 1), Lkp = IDX(m, i - 1, j, k + 1);
                    size_t Rkm = IDX(m, i, j, k - 1), Rkp = IDX(m, i, j, k + 1);
                    double dudzL = (U[Lkp] - U[Lkm]) / (2.0 * dzk), dudzR = (U[Rkp] - U[Rkm]) / (2.0 * dzk);
                    dudz = 0.5 * (dudzL + dudzR);
                    double dwdzL = (W[Lkp] - W[Lkm]) / (2.0 * dzk), dwdzR = (W[Rkp] - W[Rkm]) / (2.0 * dzk);
                    dwdz = 0.5 * (dwdzL + dwdzR);
                }
                double divU = dudx + dvdy + dwdz;
                double muF = face_mu(m, iL, iR);
                double txx = muF * (2.0 * dudx - (2.0 / 3.0) * divU);
                double txy = muF * (dvdx + dudy);
                double txz = muF * (dwdx + dudz);
                double uF = 0.5 * (U[iL] + U[iR]), vF = 0.0, wF = 0.0;
                if (dim >= 2) vF = 0.5 * (V[iL] + V[iR]);
                if (dim >= 3) wF = 0.5 * (W[iL] + W[iR]);
                double work = txx * uF + txy * vF + txz * wF;
                double area = DY(m, j) * DZ(m, k);
                visc_scatter(m, i >= 1, iL, (i >= 1) ? area / VOL(m, i - 1, j, k) : 0.0, i < m->nx, iR,
                             (i < m->nx) ? area / VOL(m, i, j, k) : 0.0, txx, txy, txz, work);
            }
    if (dim >= 2)
        for (int k = 0; k < m->nz; ++k)
            for (int j = 0; j <= m->ny; ++j)
                for (int i = 0; i < m->nx; ++i) {
                    size_t iL = IDX(m, i, j - 1, k), iR = IDX(m, i, j, k);
                    double dyj = 0.5 * (DY(m, j - 1) + DY(m, j));
                    double dudy = (U[iR] - U[iL]) / dyj, dvdy = (V[iR] - V[iL]) / dyj, dwdy = 0.0;
                    if (dim >= 3) dwdy = (W[iR] - W[iL]) / dyj;
                    double dxi = DX(m, i);
                    size_t Lim = IDX(m, i - 1, j - 1, k), Lip = IDX(m, i + 1, j - 1, k);
                    size_t Rim = IDX(m, i - 1, j, k), Rip = IDX(m, i + 1, j, k);
                    double dudxL = (U[Lip] - U[Lim]) / (2.0 * dxi), dudxR = (U[Rip] - U[Rim]) / (2.0 * dxi);
                    double dudx = 0.5 * (dudxL + dudxR);
                    double dvdxL = (V[Lip] - V[Lim]) / (2.0 * dxi), dvdxR = (V[Rip] - V[Rim]) / (2.0 * dxi);
                    double dvdx = 0.5 * (dvdxL + dvdxR);
                    double dvdz = 0.0, dwdz = 0.0;
                    if (dim >= 3) {
                        double dzk = DZ(m, k);
                        size_t Lkm = IDX(m, i, j - 1, k - 1), Lkp = IDX(m, i, j - 1, k + 1);
                        size_t Rkm = IDX(m, i, j, k - 1), Rkp = IDX(m, i, j, k + 1);
                        double dvdzL = (V[Lkp] - V[Lkm]) / (2.0 * dzk), dvdzR = (V[Rkp] - V[Rkm]) / (2.0 * dzk);
                        dvdz = 0.5 * (dvdzL + dvdzR);
                        double dwdzL = (W[Lkp] - W[Lkm]) / (2.0 * dzk), dwdzR = (W[Rkp] - W[Rkm]) / (2.0 * dzk);
                        dwdz = 0.5 * (dwdzL + dwdzR);
                    }
                    double divU = dudx + dvdy + dwdz;
                    double muF = face_mu(m, iL, iR);
                    double tyx = muF * (dudy + dvdx);
                    double tyy = muF * (2.0 * dvdy - (2.0 / 3.0) * divU);
                    double tyz = muF * (dwdy + dvdz);
                    double uF = 0.5 * (U[iL] + U[iR]), vF = 0.5 * (V[iL] + V[iR]), wF = 0.0;
                    if (dim >= 3) wF = 0.5 * (W[iL] + W[iR]);
                    double work = tyx * uF + tyy * vF + tyz * wF;
                    double area = DX(m, i) * DZ(m, k);
                    visc_scatter(m, j >= 1, iL, (j >= 1) ? area / VOL(m, i, j - 1, k) : 0.0, j < m->ny, iR,
                                 (j < m->ny) ? area / VOL(m, i, j, k) : 0.0, tyx, tyy, tyz, work);
                }
    if (dim >= 3)
        for (int k = 0; k <= m->nz; ++k)
            for (int j = 0; j < m->ny; ++j)
                for (int i = 0; i < m->nx; ++i) {
                    size_t iL = IDX(m, i, j, k - 1), iR = IDX(m, i, j, k);
                    double dzk = 0.5 * (DZ(m, k - 1) + DZ(m, k));
                    double dudz = (U[iR] - U[iL]) / dzk, dvdz = (V[iR] - V[iL]) / dzk, dwdz = (W[iR] - W[iL]) / dzk;
                    double dxi = DX(m, i);
                    size_t Lim = IDX(m, i - 1, j, k - 1), Lip = IDX(m, i + 1, j, k - 1);
                    size_t Rim = IDX(m, i - 1, j, k), Rip = IDX(m, i + 1, j, k);
                    double dudxL = (U[Lip] - U[Lim]) / (2.0 * dxi), dudxR = (U[Rip] - U[Rim]) / (2.0 * dxi);
                    double dudx = 0.5 * (dudxL + dudxR);
                    double dwdxL = (W[Lip] - W[Lim]) / (2.0 * dxi), dwdxR = (W[Rip] - W[Rim]) / (2.0 * dxi);
                    double dwdx = 0.5 * (dwdxL + dwdxR);
                    double dyj = DY(m, j);
                    size_t Ljm = IDX(m, i, j - 1, k - 1), Ljp = IDX(m, i, j + 1, k - 1);
                    size_t Rjm = IDX(m, i, j - 1, k), Rjp = IDX(m, i, j + 1, k);
                    double dvdyL = (V[Ljp] - V[Ljm]) / (2.0 * dyj), dvdyR = (V[Rjp] - V[Rjm]) / (2.0 * dyj);
                    double dvdy = 0.5 * (dvdyL + dvdyR);
                    double dwdyL = (W[Ljp] - W[Ljm]) / (2.0 * dyj), dwdyR = (W[Rjp] - W[Rjm]) / (2.0 * dyj);
                    double dwdy = 0.5 * (dwdyL + dwdyR);
                    double divU = dudx + dvdy + dwdz;
                    double muF = face_mu(m, iL, iR);
                    double tzx = muF * (dudz + dwdx);
                    double tzy = muF * (dvdz + dwdy);
                    double tzz = muF * (2.0 * dwdz - (2.0 / 3.0) * divU);
                    double uF = 0.5 * (U[iL] + U[iR]), vF = 0.5 * (V[iL] + V[iR]), wF = 0.5 * (W[iL] + W[iR]);
                    double work = tzx * uF + tzy * vF + tzz * wF;
                    double area = DX(m, i) * DY(m, j);
                    visc_scatter(m, k >= 1, iL, (k >= 1) ? area / VOL(m, i, j, k - 1) : 0.0, k < m->nz, iR,
                                 (k < m->nz) ? area / VOL(m, i, j, k) : 0.0, tzx, tzy, tzz, work);
                }
}

/* computeViscousDt, src/RKTimeStepping.cpp:161-188 */
static double viscous_dt(const ctx_t* m, double mu, double cfl, double maxDt, int skipSolid) {
    double dt = maxDt;
    const int dim = m->dim;
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i < m->nx; ++i) {
                size_t idx = IDX(m, i, j, k);
                if (skipSolid && SOLID(m, idx)) continue;
                double dxMin = DX(m, i);
                if (dim >= 2) dxMin = smin(dxMin, DY(m, j));
                if (dim >= 3) dxMin = smin(dxMin, DZ(m, k));
                double nu = mu / smax(m->rho[idx], 1e-14);
                double dtCell = dxMin * dxMin / (2.0 * dim * nu);
                dt = smin(dt, cfl * dtCell);
            }
    return dt;
}

/* ---- capillary stress: addSurfaceTensionFluxes, src/SurfaceTension.cpp:8-254 ---- */
/* T = sigma (|g| I - g g^T / |g|) of g = grad alpha_0 at the face (normal:
 * two-cell difference; transverse: central differences averaged over the
 * two cells), |g| regularised by epsGradAlpha; work T.u_face.  Same
 * accumulation as the viscous stress. */
static void add_surface_tension_fluxes(ctx_t* m) {
    const int dim = m->dim;
    const double sigma = m->c.stSigma, eps = m->c.stEpsGradAlpha;
    const double* a = m->alpha[0];
    const double* U = m->velU;
    const double* V = m->velV;
    const double* W = m->velW;
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i <= m->nx; ++i) {
                size_t iL = IDX(m, i - 1, j, k), iR = IDX(m, i, j, k);
                double dxi = 0.5 * (DX(m, i - 1) + DX(m, i));
                double gx = (a[iR] - a[iL]) / dxi, gy = 0.0, gz = 0.0;
                if (dim >= 2) {
                    double dyj = DY(m, j);
                    double gL = (a[IDX(m, i - 1, j + 1, k)] - a[IDX(m, i - 1, j - 1, k)]) / (2.0 * dyj);
                    double gR = (a[IDX(m, i, j + 1, k)] - a[IDX(m, i, j - 1, k)]) / (2.0 * dyj);
                    gy = 0.5 * (gL + gR);
                }
                if (dim >= 3) {
                    double dzk = DZ(m, k);
                    double gL = (a[IDX(m, i - 1, j, k + 1)] - a[IDX(m, i - 1, j, k - 1)]) / (2.0 * dzk);
                    double gR = (a[IDX(m, i, j, k + 1)] - a[IDX(m, i, j, k - 1)]) / (2.0 * dzk);
                    gz = 0.5 * (gL + gR);
                }
                double ng = sqrt(gx * gx + gy * gy + gz * gz);
                double reg = smax(ng, eps);
                double txx = sigma * (gy * gy + gz * gz) / reg;
                double txy = -sigma * gx * gy / reg;
                double txz = -sigma * gx * gz / reg;
                double uF = 0.5 * (U[iL] + U[iR]), vF = 0.0, wF = 0.0;
                if (dim >= 2) vF = 0.5 * (V[iL] + V[iR]);
                if (dim >= 3) wF = 0.5 * (W[iL] + W[iR]);
                double work = txx * uF + txy * vF + txz * wF;
                double area = DY(m, j) * DZ(m, k);
                visc_scatter(m, i >= 1, iL, (i >= 1) ? area / VOL(m, i - 1, j, k) : 0.0, i < m->nx, iR,
                             (i < m->nx) ? area / VOL(m, i, j, k) : 0.0, txx, txy, txz, work);
            }
    if (dim >= 2)
        for (int k = 0; k < m->nz; ++k)
            for (int j = 0; j <= m->ny; ++j)
                for (int i = 0; i < m->nx; ++i) {
                    size_t iL = IDX(m, i, j - 1, k), iR = IDX(m, i, j, k);
                    double dyj = 0.5 * (DY(m, j - 1) + DY(m, j));
                    double gy = (a[iR] - a[iL]) / dyj, gz = 0.0;
                    double dxi = DX(m, i);
                    double gxL = (a[IDX(m, i + 1, j - 1, k)] - a[IDX(m, i - 1, j - 1, k)]) / (2.0 * dxi);
                    double gxR = (a[IDX(m, i + 1, j, k)] - a[IDX(m, i - 1, j, k)]) / (2.0 * dxi);
                    double gx = 0.5 * (gxL + gxR);
                    if (dim >= 3) {
                        double dzk = DZ(m, k);
                        double gL = (a[IDX(m, i, j - 1, k + 1)] - a[IDX(m, i, j - 1, k - 1)]) / (2.0 * dzk);
                        double gR = (a[IDX(m, i, j, k + 1)] - a[IDX(m, i, j, k - 1)]) / (2.0 * dzk);
                        gz = 0.5 * (gL + gR);
                    }
                    double ng = sqrt(gx * gx + gy * gy + gz * gz);
                    double reg = smax(ng, eps);
                    double tyx = -sigma * gy * gx / reg;
                    double tyy = sigma * (gx * gx + gz * gz) / reg;
                    double tyz = -sigma * gy * gz / reg;
                    double uF = 0.5 * (U[iL] + U[iR]), vF = 0.5 * (V[iL] + V[iR]), wF = 0.0;
                    if (dim >= 3) wF = 0.5 * (W[iL] + W[iR]);
                    double work = tyx * uF + tyy * vF + tyz * wF;
                    double area = DX(m, i) * DZ(m, k);
                    visc_scatter(m, j >= 1, iL, (j >= 1) ? area / VOL(m, i, j - 1, k) : 0.0, j < m->ny, iR,
                                 (j < m->ny) ? area / VOL(m, i, j, k) : 0.0, tyx, tyy, tyz, work);
                }
    if (dim >= 3)
        for (int k = 0; k <= m->nz; ++k)
            for (int j = 0; j < m->ny; ++j)
                for (int i = 0; i < m->nx; ++i) {
                    size_t iL = IDX(m, i, j, k - 1), iR = IDX(m, i, j, k);
                    double dzk = 0.5 * (DZ(m, k - 1) + DZ(m, k));
                    double gz = (a[iR] - a[iL]) / dzk;
                    double dxi = DX(m, i);
                    double gxL = (a[IDX(m, i + 1, j, k - 1)] - a[IDX(m, i - 1, j, k - 1)]) / (2.0 * dxi);
                    double gxR = (a[IDX(m, i + 1, j, k)] - a[IDX(m, i - 1, j, k)]) / (2.0 * dxi);
                    double gx = 0.5 * (gxL + gxR);
                    double dyj = DY(m, j);
                    double gyL = (a[IDX(m, i, j + 1, k - 1)] - a[IDX(m, i, j - 1, k - 1)]) / (2.0 * dyj);
                    double gyR = (a[IDX(m, i, j + 1, k)] - a[IDX(m, i, j - 1, k)]) / (2.0 * dyj);
                    double gy = 0.5 * (gyL + gyR);
                    double ng = sqrt(gx * gx + gy * gy + gz * gz);
                    double reg = smax(ng, eps);
                    double tzx = -sigma * gz * gx / reg;
                    double tzy = -sigma * gz * gy / reg;
                    double tzz = sigma * (gx * gx + gy * gy) / reg;
                    double uF = 0.5 * (U[iL] + U[iR]), vF = 0.5 * (V[iL] + V[iR]), wF = 0.5 * (W[iL] + W[iR]);
                    double work = tzx * uF + tzy * vF + tzz * wF;
                    double area = DX(m, i) * DY(m, j);
                    visc_scatter(m, k >= 1, iL, (k >= 1) ? area / VOL(m, i, j, k - 1) : 0.0, k < m->nz, iR,
                                 (k < m->nz) ? area / VOL(m, i, j, k) : 0.0, tzx, tzy, tzz, work);
                }
}

/* computeCapillaryDt, src/RKTimeStepping.cpp:201-228 */
static double capillary_dt(const ctx_t* m, double sigma, double cfl, double maxDt, int skipSolid) {
    double dt = maxDt;
    const int dim = m->dim;
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i < m->nx; ++i) {
                size_t idx = IDX(m, i, j, k);
                if (skipSolid && SOLID(m, idx)) continue;
                double dxMin = DX(m, i);
                if (dim >= 2) dxMin = smin(dxMin, DY(m, j));
                if (dim >= 3) dxMin = smin(dxMin, DZ(m, k));
                double dtCell = sqrt(smax(m->rho[idx], 1e-14) * dxMin * dxMin * dxMin / sigma);
                dt = smin(dt, cfl * dtCell);
            }
    return dt;
}

/* ---- IGR ---- */
/* IGRSolver::computeVelocityGradient, src/IGR.cpp:160-200, assembled as in
 * ExplicitSolver::computeVelocityGradients (src/ExplicitSolver.cpp:215-267)
 * and SemiImplicitSolver::computeVelocityGradients (src/SemiImplicitSolver.cpp:719-771). */
static void velocity_gradients(ctx_t* m) {
    const int dim = m->dim;
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i < m->nx; ++i) {
                size_t idx = IDX(m, i, j, k);
                size_t xm = IDX(m, i - 1, j, k), xp = IDX(m, i + 1, j, k);
                double uxm[3] = {m->velU[xm], (dim >= 2) ? m->velV[xm] : 0.0, (dim >= 3) ? m->velW[xm] : 0.0};
                double uxp[3] = {m->velU[xp], (dim >= 2) ? m->velV[xp] : 0.0, (dim >= 3) ? m->velW[xp] : 0.0};
                double uym[3], uyp[3], uzm[3], uzp[3], dyj, dzk;
                if (dim >= 2) {
                    size_t ym = IDX(m, i, j - 1, k), yp = IDX(m, i, j + 1, k);
                    uym[0] = m->velU[ym]; uym[1] = m->velV[ym]; uym[2] = (dim >= 3) ? m->velW[ym] : 0.0;
                    uyp[0] = m->velU[yp]; uyp[1] = m->velV[yp]; uyp[2] = (dim >= 3) ? m->velW[yp] : 0.0;
                    dyj = DY(m, j);
                } else {
                    uym[0] = uyp[0] = m->velU[idx]; uym[1] = uyp[1] = 0.0; uym[2] = uyp[2] = 0.0;
                    dyj = 1.0;
                }
                if (dim >= 3) {
                    size_t zm = IDX(m, i, j, k - 1), zp = IDX(m, i, j, k + 1);
                    uzm[0] = m->velU[zm]; uzm[1] = m->velV[zm]; uzm[2] = m->velW[zm];
                    uzp[0] = m->velU[zp]; uzp[1] = m->velV[zp]; uzp[2] = m->velW[zp];
                    dzk = DZ(m, k);
                } else {
                    uzm[0] = uzp[0] = m->velU[idx];
                    uzm[1] = uzp[1] = (dim >= 2) ? m->velV[idx] : 0.0;
                    uzm[2] = uzp[2] = 0.0;
                    dzk = 1.0;
                }
                double* g = m->gradU + 9 * idx; /* g[3*a + b] = du_a/dx_b */
                for (int q = 0; q < 9; ++q) g[q] = 0.0;
                double invDx = 0.5 / DX(m, i), invDy = 0.5 / dyj, invDz = 0.5 / dzk;
                g[0] = (uxp[0] - uxm[0]) * invDx;
                if (dim >= 2) {
                    g[3] = (uxp[1] - uxm[1]) * invDx;
                    g[1] = (uyp[0] - uym[0]) * invDy;
                    g[4] = (uyp[1] - uym[1]) * invDy;
                    if (dim >= 3) {
                        g[7] = (uyp[2] - uym[2]) * invDy;
                        g[6] = (uxp[2] - uxm[2]) * invDx;
                        g[2] = (uzp[0] - uzm[0]) * invDz;
                        g[5] = (uzp[1] - uzm[1]) * invDz;
                        g[8] = (uzp[2] - uzm[2]) * invDz;
                    }
                }
            }
}

/* IGRSolver::computeIGRRhs, src/IGR.cpp:18-35 */
static double igr_rhs(const ctx_t* m, const double* g, double alpha) {
    double trSq = 0.0;
    for (int a = 0; a < m->dim; ++a)
        for (int b = 0; b < m->dim; ++b) trSq += g[3 * a + b] * g[3 * b + a];
    double trSquared = 0.0;
    for (int a = 0; a < m->dim; ++a) trSquared += g[3 * a + a];
    trSquared *= trSquared;
    return alpha * (trSq + trSquared);
}

/* IGRSolver::solveEntropicPressure, src/IGR.cpp:102-158 (lexicographic,
 * in-place Gauss-Seidel; scalar ghost refresh after every sweep). */
static void igr_solve(ctx_t* m, int step) {
    int maxIters = (step == 0) ? m->c.IGRWarmStartIters : m->c.IGRIters;
    double alpha = m->c.alphaCoeff * DX(m, 0) * DX(m, 0);
    for (int it = 0; it < maxIters; ++it) {
        for (int k = 0; k < m->nz; ++k)
            for (int j = 0; j < m->ny; ++j)
                for (int i = 0; i < m->nx; ++i) {
                    size_t idx = IDX(m, i, j, k);
                    if (SOLID(m, idx)) continue;
                    double rhs = igr_rhs(m, m->gradU + 9 * idx, alpha);
                    double diag = 1.0 / m->rho[idx];
                    double offdiag = 0.0;
                    size_t ixl = IDX(m, i - 1, j, k), ixr = IDX(m, i + 1, j, k);
                    double rho_i = m->rho[idx];
                    double rfl = 0.5 * (rho_i + m->rho[ixl]);
                    double rfr = 0.5 * (rho_i + m->rho[ixr]);
                    double dx2 = 1.0 / (DX(m, i) * DX(m, i));
                    diag += alpha * dx2 * (1.0 / rfl + 1.0 / rfr);
                    offdiag += alpha * dx2 * (m->sigma[ixl] / rfl + m->sigma[ixr] / rfr);
                    if (m->dim >= 2) {
                        size_t iyl = IDX(m, i, j - 1, k), iyr = IDX(m, i, j + 1, k);
                        double ryl = 0.5 * (rho_i + m->rho[iyl]);
                        double ryr = 0.5 * (rho_i + m->rho[iyr]);
                        double dy2 = 1.0 / (DY(m, j) * DY(m, j));
                        diag += alpha * dy2 * (1.0 / ryl + 1.0 / ryr);
                        offdiag += alpha * dy2 * (m->sigma[iyl] / ryl + m->sigma[iyr] / ryr);
                    }
                    if (m->dim >= 3) {
                        size_t izl = IDX(m, i, j, k - 1), izr = IDX(m, i, j, k + 1);
                        double rzl = 0.5 * (rho_i + m->rho[izl]);
                        double rzr = 0.5 * (rho_i + m->rho[izr]);
                        double dz2 = 1.0 / (DZ(m, k) * DZ(m, k));
                        diag += alpha * dz2 * (1.0 / rzl + 1.0 / rzr);
                        offdiag += alpha * dz2 * (m->sigma[izl] / rzl + m->sigma[izr] / rzr);
                    }
                    m->sigma[idx] = (rhs + offdiag) / diag;
                }
        fill_scalar_ghosts(m, m->sigma);
        if (m->cellType) ib_apply_scalar(m, m->sigma);
    }
}

/* ---- pressure solve ---- */
/* pressureLaplacian, src/PressureLaplacian.cpp:6-60 */
static double pressure_laplacian(const ctx_t* m, const double* rho, const double* p, int i, int j, int k,
                                 double* offDiag) {
    double od = 0.0, diag = 0.0;
    size_t idx = IDX(m, i, j, k);
    {
        size_t xm = IDX(m, i - 1, j, k), xp = IDX(m, i + 1, j, k);
        double rhoL = 0.5 * (rho[idx] + rho[xm]), rhoR = 0.5 * (rho[idx] + rho[xp]);
        double dL = 0.5 * (DX(m, i - 1) + DX(m, i)), dR = 0.5 * (DX(m, i) + DX(m, i + 1));
        double cL = 1.0 / (smax(rhoL, 1e-14) * dL * DX(m, i));
        double cR = 1.0 / (smax(rhoR, 1e-14) * dR * DX(m, i));
        od += cL * p[xm] + cR * p[xp];
        diag += cL + cR;
    }
    if (m->dim >= 2) {
        size_t ym = IDX(m, i, j - 1, k), yp = IDX(m, i, j + 1, k);
        double rhoL = 0.5 * (rho[idx] + rho[ym]), rhoR = 0.5 * (rho[idx] + rho[yp]);
        double dL = 0.5 * (DY(m, j - 1) + DY(m, j)), dR = 0.5 * (DY(m, j) + DY(m, j + 1));
        double cL = 1.0 / (smax(rhoL, 1e-14) * dL * DY(m, j));
        double cR = 1.0 / (smax(rhoR, 1e-14) * dR * DY(m, j));
        od += cL * p[ym] + cR * p[yp];
        diag += cL + cR;
    }
    if (m->dim >= 3) {
        size_t zm = IDX(m, i, j, k - 1), zp = IDX(m, i, j, k + 1);
        double rhoL = 0.5 * (rho[idx] + rho[zm]), rhoR = 0.5 * (rho[idx] + rho[zp]);
        double dL = 0.5 * (DZ(m, k - 1) + DZ(m, k)), dR = 0.5 * (DZ(m, k) + DZ(m, k + 1));
        double cL = 1.0 / (smax(rhoL, 1e-14) * dL * DZ(m, k));
        double cR = 1.0 / (smax(rhoR, 1e-14) * dR * DZ(m, k));
        od += cL * p[zm] + cR * p[zp];
        diag += cL + cR;
    }
    *offDiag = od;
    return diag;
}

/* JacobiPressureSolver::solve, src/JacobiPressureSolver.cpp:57-108 */
static int jacobi_solve(ctx_t* m, const double* rho, const double* rhoc2, const double* rhs, double* p, double dt,
                        double tol, int maxIter) {
    double* pNew = m->pNew;
    memset(pNew, 0, m->n * sizeof(double));
    double dt2 = dt * dt;
    for (int it = 0; it < maxIter; ++it) {
        fill_scalar_ghosts(m, p);
        double maxRes = 0.0;
        for (int k = 0; k < m->nz; ++k)
            for (int j = 0; j < m->ny; ++j)
                for (int i = 0; i < m->nx; ++i) {
                    size_t idx = IDX(m, i, j, k);
                    double coeff = rhoc2[idx] * dt2;
                    double od;
                    double diagL = pressure_laplacian(m, rho, p, i, j, k, &od);
                    double denom = 1.0 + coeff * diagL;
                    pNew[idx] = (rhs[idx] + coeff * od) / denom;
                    double res = fabs(pNew[idx] - p[idx]);
                    maxRes = smax(maxRes, res);
                }
        for (int k = 0; k < m->nz; ++k)
            for (int j = 0; j < m->ny; ++j)
                for (int i = 0; i < m->nx; ++i) p[IDX(m, i, j, k)] = pNew[IDX(m, i, j, k)];
        allreduce_max(m, &maxRes);
        if (maxRes < tol) return it + 1;
    }
    return maxIter;
}

/* GaussSeidelPressureSolver::solve, src/GaussSeidelPressureSolver.cpp:54-103
 * (outside the CUDA scope; here to pin the semi-implicit golden table). */
static int gs_solve(ctx_t* m, const double* rho, const double* rhoc2, const double* rhs, double* p, double dt,
                    double tol, int maxIter) {
    double dt2 = dt * dt;
    for (int it = 0; it < maxIter; ++it) {
        fill_scalar_ghosts(m, p);
        double maxRes = 0.0;
        for (int k = 0; k < m->nz; ++k)
            for (int j = 0; j < m->ny; ++j)
                for (int i = 0; i < m->nx; ++i) {
                    size_t idx = IDX(m, i, j, k);
                    double coeff = rhoc2[idx] * dt2;
                    double od;
                    double diagL = pressure_laplacian(m, rho, p, i, j, k, &od);
                    double denom = 1.0 + coeff * diagL;
                    double pOld = p[idx];
                    p[idx] = (rhs[idx] + coeff * od) / denom;
                    double res = fabs(p[idx] - pOld);
                    maxRes = smax(maxRes, res);
                }
        allreduce_max(m, &maxRes);
        if (maxRes < tol) return it + 1;
    }
    return maxIter;
}

static int pressure_solve(ctx_t* m, const double* rho, const double* rhoc2, const double* rhs, double* p, double dt,
                          double tol, int maxIter) {
    if (m->pressureSolverKind == 1) return gs_solve(m, rho, rhoc2, rhs, p, dt, tol, maxIter);
    return jacobi_solve(m, rho, rhoc2, rhs, p, dt, tol, maxIter);
}

/* ---- steps ---- */
static void rk_coefs(int order, double rk[3][4]) {
    /* src/ExplicitSolver.cpp:92-103 */
    static const double c1[3][4] = {{1.0, 0.0, 1.0, 1.0}, {0, 0, 0, 0}, {0, 0, 0, 0}};
    static const double c2[3][4] = {{1.0, 0.0, 1.0, 1.0}, {1.0, 1.0, 1.0, 2.0}, {0, 0, 0, 0}};
    static const double c3[3][4] = {{1.0, 0.0, 1.0, 1.0}, {1.0, 3.0, 1.0, 4.0}, {2.0, 1.0, 2.0, 3.0}};
    memcpy(rk, order == 1 ? c1 : order == 2 ? c2 : c3, sizeof(double) * 12);
}

/* SolutionState::saveConservativeCell, src/SolutionState.cpp:228-240 */
static void save_cell(ctx_t* m, size_t idx) {
    m->rho0[idx] = m->rho[idx];
    m->rhoU0[idx] = m->rhoU[idx];
    if (m->dim >= 2) m->rhoV0[idx] = m->rhoV[idx];
    if (m->dim >= 3) m->rhoW0[idx] = m->rhoW[idx];
    m->rhoE0[idx] = m->rhoE[idx];
    m->pres0[idx] = m->pres[idx];
    for (int ph = 0; ph < m->c.nPhases; ++ph) {
        m->alphaRho0[ph][idx] = m->alphaRho[ph][idx];
        m->alpha0[ph][idx] = m->alpha[ph][idx];
    }
}

/* multi-phase post-update, src/ExplicitSolver.cpp:169-185 */
static void mp_post(ctx_t* m, size_t idx) {
    const int nPh = m->c.nPhases;
    double rhoSum = 0.0;
    for (int ph = 0; ph < nPh; ++ph) {
        m->alphaRho[ph][idx] = smax(m->alphaRho[ph][idx], 1e-14);
        rhoSum += m->alphaRho[ph][idx];
    }
    m->rho[idx] = rhoSum;
    for (int ph = 0; ph < nPh; ++ph) m->alpha[ph][idx] = smax(m->alpha[ph][idx], m->c.alphaMin);
    double alphaSum = 0.0;
    for (int ph = 0; ph < nPh; ++ph) alphaSum += m->alpha[ph][idx];
    for (int ph = 0; ph < nPh; ++ph) m->alpha[ph][idx] /= alphaSum;
}

/* ExplicitSolver::step, src/ExplicitSolver.cpp:68-203 */
static double explicit_step(ctx_t* m, int step, double targetDt) {
    const sifv_config_t* c = &m->c;
    double dt;
    if (c->constDt > 0) {
        dt = c->constDt;
    } else {
        dt = acoustic_dt(m, c->cfl, c->maxDt, 1);
        if (has_viscosity(c)) dt = smin(dt, viscous_dt(m, c->mu, c->cfl, c->maxDt, 1));
        if (c->stSigma > 0.0) dt = smin(dt, capillary_dt(m, c->stSigma, c->cfl, c->maxDt, 1));
        /* decomposed run: MPI_Allreduce(MIN), src/RKTimeStepping.cpp:148-159 */
        if (m->comm.allreduce_min) m->comm.allreduce_min(m->comm.user, &dt, NULL);
    }
    if (targetDt > 0) dt = smin(dt, targetDt);
    double rk[3][4];
    rk_coefs(c->RKOrder, rk);
    const int nPh = c->nPhases;
    m->commFailed = 0;
    for (int s = 0; s < c->RKOrder; ++s) {
        if (exchange_cons(m) != SIFV_OK) return -1.0;
        cons_to_prim(m);
        apply_bc_prim(m);
        if (m->cellType) ib_apply_ghosts(m);
        if (c->useIGR) {
            velocity_gradients(m);
            igr_solve(m, step);
        }
        compute_rhs(m);
        double c1 = rk[s][0], c2 = rk[s][1], c3 = rk[s][2], c4 = rk[s][3];
        for (int k = 0; k < m->nz; ++k)
            for (int j = 0; j < m->ny; ++j)
                for (int i = 0; i < m->nx; ++i) {
                    size_t idx = IDX(m, i, j, k);
                    if (SOLID(m, idx)) continue;
                    if (s == 0 && c->RKOrder > 1) save_cell(m, idx);
                    if (c->RKOrder == 1) {
                        m->rho[idx] += dt * m->rhsRho[idx];
                        m->rhoU[idx] += dt * m->rhsRhoU[idx];
                        if (m->dim >= 2) m->rhoV[idx] += dt * m->rhsRhoV[idx];
                        if (m->dim >= 3) m->rhoW[idx] += dt * m->rhsRhoW[idx];
                        m->rhoE[idx] += dt * m->rhsRhoE[idx];
                        for (int ph = 0; ph < nPh; ++ph) m->alphaRho[ph][idx] += dt * m->rhsAlphaRho[ph][idx];
                        for (int ph = 0; ph < nPh; ++ph) m->alpha[ph][idx] += dt * m->rhsAlpha[ph][idx];
                    } else {
                        m->rho[idx] = (c1 * m->rho[idx] + c2 * m->rho0[idx] + c3 * dt * m->rhsRho[idx]) / c4;
                        m->rhoU[idx] = (c1 * m->rhoU[idx] + c2 * m->rhoU0[idx] + c3 * dt * m->rhsRhoU[idx]) / c4;
                        if (m->dim >= 2)
                            m->rhoV[idx] = (c1 * m->rhoV[idx] + c2 * m->rhoV0[idx] + c3 * dt * m->rhsRhoV[idx]) / c4;
                        if (m->dim >= 3)
                            m->rhoW[idx] = (c1 * m->rhoW[idx] + c2 * m->rhoW0[idx] + c3 * dt * m->rhsRhoW[idx]) / c4;
                        m->rhoE[idx] = (c1 * m->rhoE[idx] + c2 * m->rhoE0[idx] + c3 * dt * m->rhsRhoE[idx]) / c4;
                        for (int ph = 0; ph < nPh; ++ph)
                            m->alphaRho[ph][idx] = (c1 * m->alphaRho[ph][idx] + c2 * m->alphaRho0[ph][idx] +
                                                    c3 * dt * m->rhsAlphaRho[ph][idx]) / c4;
                        for (int ph = 0; ph < nPh; ++ph)
                            m->alpha[ph][idx] =
                                (c1 * m->alpha[ph][idx] + c2 * m->alpha0[ph][idx] + c3 * dt * m->rhsAlpha[ph][idx]) / c4;
                    }
                    if (nPh > 0) mp_post(m, idx);
                }
    }
    if (exchange_cons(m) != SIFV_OK || m->commFailed) return -1.0;
    cons_to_prim(m);
    apply_bc_prim(m);
    if (m->cellType) ib_apply_ghosts(m);
    return dt;
}

/* SemiImplicitSolver::computeDivergence, src/SemiImplicitSolver.cpp:680-717 */
static void compute_divergence(ctx_t* m, double* divOut) {
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i < m->nx; ++i) {
                size_t idx = IDX(m, i, j, k);
                double div = 0.0;
                {
                    size_t xm = IDX(m, i - 1, j, k), xp = IDX(m, i + 1, j, k);
                    double uFaceL = 0.5 * (m->velU[xm] + m->velU[idx]);
                    double uFaceR = 0.5 * (m->velU[idx] + m->velU[xp]);
                    div += (uFaceR - uFaceL) / DX(m, i);
                }
                if (m->dim >= 2) {
                    size_t ym = IDX(m, i, j - 1, k), yp = IDX(m, i, j + 1, k);
                    double vFaceL = 0.5 * (m->velV[ym] + m->velV[idx]);
                    double vFaceR = 0.5 * (m->velV[idx] + m->velV[yp]);
                    div += (vFaceR - vFaceL) / DY(m, j);
                }
                if (m->dim >= 3) {
                    size_t zm = IDX(m, i, j, k - 1), zp = IDX(m, i, j, k + 1);
                    double wFaceL = 0.5 * (m->velW[zm] + m->velW[idx]);
                    double wFaceR = 0.5 * (m->velW[idx] + m->velW[zp]);
                    div += (wFaceR - wFaceL) / DZ(m, k);
                }
                divOut[idx] = div;
            }
}

/* SemiImplicitSolver::solvePressure, src/SemiImplicitSolver.cpp:533-588 */
static int solve_pressure(ctx_t* m, double dt) {
    const int nPh = m->c.nPhases;
    double alphas[MAXPH], alphaRhos[MAXPH];
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i < m->nx; ++i) {
                size_t idx = IDX(m, i, j, k);
                double cc;
                if (nPh > 0) {
                    for (int ph = 0; ph < nPh; ++ph) alphas[ph] = m->alpha[ph][idx];
                    for (int ph = 0; ph < nPh; ++ph) alphaRhos[ph] = m->alphaRho[ph][idx];
                    cc = mixture_sound_speed(m, m->rho[idx], m->pres[idx], alphas, alphaRhos);
                } else {
                    cc = sqrt(m->c.gamma * smax(m->pres[idx] + m->c.pInf, 1e-14) / smax(m->rho[idx], 1e-14));
                }
                m->rhoc2[idx] = m->rho[idx] * cc * cc;
            }
    compute_divergence(m, m->divUstar);
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i < m->nx; ++i) {
                size_t idx = IDX(m, i, j, k);
                m->pressureRhs[idx] = m->pAdvected[idx] - m->rhoc2[idx] * dt * m->divUstar[idx];
            }
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i < m->nx; ++i) m->pressure[IDX(m, i, j, k)] = m->pres[IDX(m, i, j, k)];
    int iters = pressure_solve(m, m->rho, m->rhoc2, m->pressureRhs, m->pressure, dt, m->c.pressureTol,
                               m->c.maxPressureIters);
    fill_scalar_ghosts(m, m->pressure);
    fill_scalar_ghosts(m, m->sigma);
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i < m->nx; ++i) m->pres[IDX(m, i, j, k)] = m->pressure[IDX(m, i, j, k)];
    return iters;
}

/* SemiImplicitSolver::correctionStep, src/SemiImplicitSolver.cpp:590-678 */
static void correction_step(ctx_t* m, double dt) {
    const double* P = m->pressure;
    const double* S = m->sigma;
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i < m->nx; ++i) {
                size_t idx = IDX(m, i, j, k);
                {
                    size_t xm = IDX(m, i - 1, j, k), xp = IDX(m, i + 1, j, k);
                    double pTotL = 0.5 * ((P[xm] + S[xm]) + (P[idx] + S[idx]));
                    double pTotR = 0.5 * ((P[idx] + S[idx]) + (P[xp] + S[xp]));
                    m->rhoU[idx] = m->rhoUStar[idx] - dt * (pTotR - pTotL) / DX(m, i);
                }
                if (m->dim >= 2) {
                    size_t ym = IDX(m, i, j - 1, k), yp = IDX(m, i, j + 1, k);
                    double pTotL = 0.5 * ((P[ym] + S[ym]) + (P[idx] + S[idx]));
                    double pTotR = 0.5 * ((P[idx] + S[idx]) + (P[yp] + S[yp]));
                    m->rhoV[idx] = m->rhoVStar[idx] - dt * (pTotR - pTotL) / DY(m, j);
                }
                if (m->dim >= 3) {
                    size_t zm = IDX(m, i, j, k - 1), zp = IDX(m, i, j, k + 1);
                    double pTotL = 0.5 * ((P[zm] + S[zm]) + (P[idx] + S[idx]));
                    double pTotR = 0.5 * ((P[idx] + S[idx]) + (P[zp] + S[zp]));
                    m->rhoW[idx] = m->rhoWStar[idx] - dt * (pTotR - pTotL) / DZ(m, k);
                }
            }
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i < m->nx; ++i) {
                size_t idx = IDX(m, i, j, k);
                double rs = smax(m->rho[idx], 1e-14);
                m->velU[idx] = m->rhoU[idx] / rs;
                if (m->dim >= 2) m->velV[idx] = m->rhoV[idx] / rs;
                if (m->dim >= 3) m->velW[idx] = m->rhoW[idx] / rs;
            }
    exchange_prim(m);
    apply_bc_prim(m);
    double alphas[MAXPH];
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i < m->nx; ++i) {
                size_t idx = IDX(m, i, j, k);
                double rho = m->rho[idx];
                double ke = 0.5 * rho * m->velU[idx] * m->velU[idx];
                if (m->dim >= 2) ke += 0.5 * rho * m->velV[idx] * m->velV[idx];
                if (m->dim >= 3) ke += 0.5 * rho * m->velW[idx] * m->velW[idx];
                if (m->c.nPhases > 0) {
                    for (int ph = 0; ph < m->c.nPhases; ++ph) alphas[ph] = m->alpha[ph][idx];
                    m->rhoE[idx] = mixture_total_energy(m, P[idx], alphas, ke);
                } else {
                    m->rhoE[idx] = (P[idx] + m->c.gamma * m->c.pInf) / (m->c.gamma - 1.0) + ke;
                }
            }
}

/* SemiImplicitSolver::step, src/SemiImplicitSolver.cpp:106-236 */
static double semi_step(ctx_t* m, int step, double targetDt) {
    const sifv_config_t* c = &m->c;
    double dt = advective_dt(m, c->siCfl, c->siMaxDt);
    if (has_viscosity(c)) dt = smin(dt, viscous_dt(m, c->mu, c->siCfl, c->siMaxDt, 0));
    if (c->stSigma > 0.0) dt = smin(dt, capillary_dt(m, c->stSigma, c->siCfl, c->siMaxDt, 0));
    /* decomposed run: MPI_Allreduce(MIN) of each local dt, src/RKTimeStepping.cpp:125-133 */
    if (m->exchangeFaces && m->comm.allreduce_min && m->comm.allreduce_min(m->comm.user, &dt, NULL) != 0)
        return -1.0;
    if (targetDt > 0) dt = smin(dt, targetDt);
    dt = sclamp(dt, c->siMinDt, c->siMaxDt);
    double rk[3][4];
    rk_coefs(c->RKOrder, rk);
    const int nPh = c->nPhases;
    const int RK = c->RKOrder;
    m->commFailed = 0;
    for (int s = 0; s < RK; ++s) {
        if (exchange_cons(m) != SIFV_OK) return -1.0;
        cons_to_prim(m);
        apply_bc_prim(m);
        if (c->useIGR) {
            velocity_gradients(m);
            igr_solve(m, step);
        }
        compute_rhs(m);
        double c1 = rk[s][0], c2 = rk[s][1], c3 = rk[s][2], c4 = rk[s][3];
        for (int k = 0; k < m->nz; ++k)
            for (int j = 0; j < m->ny; ++j)
                for (int i = 0; i < m->nx; ++i) {
                    size_t idx = IDX(m, i, j, k);
                    if (s == 0 && RK > 1) save_cell(m, idx);
                    m->pAdvected[idx] = m->pres[idx];
                    double r0 = (RK > 1) ? m->rho0[idx] : 0.0;
                    double ru0 = (RK > 1) ? m->rhoU0[idx] : 0.0;
                    double re0 = (RK > 1) ? m->rhoE0[idx] : 0.0;
                    m->rho[idx] = (c1 * m->rho[idx] + c2 * r0 + c3 * dt * m->rhsRho[idx]) / c4;
                    m->rhoUStar[idx] = (c1 * m->rhoU[idx] + c2 * ru0 + c3 * dt * m->rhsRhoU[idx]) / c4;
                    if (m->dim >= 2) {
                        double rv0 = (RK > 1) ? m->rhoV0[idx] : 0.0;
                        m->rhoVStar[idx] = (c1 * m->rhoV[idx] + c2 * rv0 + c3 * dt * m->rhsRhoV[idx]) / c4;
                    }
                    if (m->dim >= 3) {
                        double rw0 = (RK > 1) ? m->rhoW0[idx] : 0.0;
                        m->rhoWStar[idx] = (c1 * m->rhoW[idx] + c2 * rw0 + c3 * dt * m->rhsRhoW[idx]) / c4;
                    }
                    m->rhoEstar[idx] = (c1 * m->rhoE[idx] + c2 * re0 + c3 * dt * m->rhsRhoE[idx]) / c4;
                    double p0 = (RK > 1) ? m->pres0[idx] : 0.0;
                    m->pAdvected[idx] = (c1 * m->pAdvected[idx] + c2 * p0 + c3 * dt * m->rhsP[idx]) / c4;
                    if (nPh > 0) {
                        if (RK == 1) {
                            for (int ph = 0; ph < nPh; ++ph) m->alphaRho[ph][idx] += dt * m->rhsAlphaRho[ph][idx];
                            for (int ph = 0; ph < nPh; ++ph) m->alpha[ph][idx] += dt * m->rhsAlpha[ph][idx];
                        } else {
                            for (int ph = 0; ph < nPh; ++ph)
                                m->alphaRho[ph][idx] = (c1 * m->alphaRho[ph][idx] + c2 * m->alphaRho0[ph][idx] +
                                                        c3 * dt * m->rhsAlphaRho[ph][idx]) / c4;
                            for (int ph = 0; ph < nPh; ++ph)
                                m->alpha[ph][idx] =
                                    (c1 * m->alpha[ph][idx] + c2 * m->alpha0[ph][idx] + c3 * dt * m->rhsAlpha[ph][idx]) / c4;
                        }
                        mp_post(m, idx);
                    }
                    double rs = smax(m->rho[idx], 1e-14);
                    m->velU[idx] = m->rhoUStar[idx] / rs;
                    if (m->dim >= 2) m->velV[idx] = m->rhoVStar[idx] / rs;
                    if (m->dim >= 3) m->velW[idx] = m->rhoWStar[idx] / rs;
                }
        exchange_prim(m);   /* density + star velocity, src/SemiImplicitSolver.cpp:228-229 */
        apply_bc_prim(m);
        m->lastIters = solve_pressure(m, dt);
        correction_step(m, dt);
        if (m->commFailed) return -1.0;
    }
    return dt;
}

/* ---------------------------------------------------------------------- */
/* exported ABI (prefix sifvo_)                                             */
/* ---------------------------------------------------------------------- */

static double* dalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

/* SimulationConfig::validate (include/SimulationConfig.hpp:123-209) */
static int validate(const sifv_config_t* c, char* err) {
#define FAIL(msg) do { snprintf(err, 256, "%s", msg); return SIFV_ERR_BAD_CONFIG; } while (0)
    if (c->dim < 1 || c->dim > 3) FAIL("dim must be 1, 2, or 3");
    if (c->RKOrder < 1 || c->RKOrder > 3) FAIL("RKOrder must be 1, 2, or 3");
    int req = (c->reconOrder == SIFV_WENO1 || c->reconOrder == SIFV_UPWIND1) ? 1
            : (c->reconOrder == SIFV_WENO3 || c->reconOrder == SIFV_UPWIND3) ? 2 : 3;
    if (c->nGhost < req) FAIL("nGhost is too small for chosen reconOrder");
    if (c->semiImplicit) {
        if (c->siCfl <= 0) FAIL("semiImplicitParams.cfl must be > 0");
        if (c->siMinDt <= 0) FAIL("semiImplicitParams.minDt must be > 0");
        if (c->siMaxDt <= c->siMinDt) FAIL("semiImplicitParams.maxDt must be > minDt");
        if (c->pressureTol <= 0) FAIL("semiImplicitParams.pressureTol must be > 0");
        if (c->maxPressureIters <= 0) FAIL("semiImplicitParams.maxPressureIters must be > 0");
    } else {
        if (c->cfl <= 0) FAIL("explicitParams.cfl must be > 0");
        if (c->minDt <= 0) FAIL("explicitParams.minDt must be > 0");
        if (c->maxDt <= c->minDt) FAIL("explicitParams.maxDt must be > minDt");
    }
    if (c->useIGR) {
        if (c->alphaCoeff <= 0) FAIL("igrParams.alphaCoeff must be > 0");
        if (c->IGRIters <= 0) FAIL("igrParams.IGRIters must be > 0");
        if (c->IGRWarmStartIters < 0) FAIL("igrParams.IGRWarmStartIters must be >= 0");
    }
    if (c->nPhases < 0 || c->nPhases > MAXPH) FAIL("nPhases out of range");
    for (int p = 0; p < c->nPhases; ++p) {
        if (c->phaseGamma[p] <= 1.0) FAIL("multiPhaseParams.phases[].gamma must be > 1");
        if (c->phasePInf[p] < 0.0) FAIL("multiPhaseParams.phases[].pInf must be >= 0");
    }
    if (c->nPhases > 0 && c->alphaMin <= 0.0) FAIL("multiPhaseParams.alphaMin must be > 0");
    if (c->mu < 0.0) FAIL("viscousParams.mu must be >= 0");
    if (c->nPhaseMu > 0) {
        if (c->nPhases <= 0) FAIL("viscousParams.phaseMu requires multi-phase (nPhases >= 2)");
        if (c->nPhaseMu != c->nPhases) FAIL("viscousParams.phaseMu.size() must equal nPhases");
        for (int p = 0; p < c->nPhaseMu; ++p)
            if (c->phaseMu[p] < 0.0) FAIL("viscousParams.phaseMu[] must be >= 0");
    }
    if (c->stSigma < 0.0) FAIL("surfaceTensionParams.sigma must be >= 0");
    if (c->stEpsGradAlpha <= 0.0) FAIL("surfaceTensionParams.epsGradAlpha must be > 0");
    if (c->stSigma > 0.0 && c->nPhases <= 0) FAIL("surfaceTensionParams.sigma requires multi-phase (nPhases >= 2)");
    return SIFV_OK;
#undef FAIL
}

const char* sifvo_last_error(const ctx_t* m) { return m ? m->err : g_err; }

int sifvo_config_validate(const sifv_config_t* c) { return validate(c, g_err); }

int sifvo_create(const sifv_config_t* cfg, const sifv_mesh_t* mesh, int device, ctx_t** out) {
    (void)device;
    *out = NULL;
    int st = validate(cfg, g_err);
    if (st != SIFV_OK) return st;
    ctx_t* m = (ctx_t*)calloc(1, sizeof(ctx_t));
    m->c = *cfg;
    m->dim = cfg->dim;
    m->nx = mesh->nx;
    m->ny = (cfg->dim >= 2) ? mesh->ny : 1;
    m->nz = (cfg->dim >= 3) ? mesh->nz : 1;
    m->ngx = cfg->nGhost;
    m->ngy = (cfg->dim >= 2) ? cfg->nGhost : 0;
    m->ngz = (cfg->dim >= 3) ? cfg->nGhost : 0;
    m->nxT = m->nx + 2 * m->ngx;
    m->nyT = m->ny + 2 * m->ngy;
    m->nzT = m->nz + 2 * m->ngz;
    m->n = (size_t)m->nxT * m->nyT * m->nzT;
    static const double unit[2] = {0.0, 1.0};
    m->xExt = build_ext(mesh->xNodes ? mesh->xNodes : unit, m->nx, m->ngx);
    m->yExt = build_ext((cfg->dim >= 2 && mesh->yNodes) ? mesh->yNodes : unit, m->ny, m->ngy);
    m->zExt = build_ext((cfg->dim >= 3 && mesh->zNodes) ? mesh->zNodes : unit, m->nz, m->ngz);
    for (int f = 0; f < 6; ++f) {
        m->bc[f] = mesh->bc[f];
        if (f < 2 * cfg->dim && mesh->bc[f] == SIFV_BC_EXCHANGE) m->exchangeFaces = 1;
    }
    if (m->exchangeFaces && (has_viscosity(cfg) || cfg->stSigma > 0.0)) {
        snprintf(g_err, sizeof(g_err), "SIFV_BC_EXCHANGE faces are not supported with viscosity or surface tension");
        free(m->xExt); free(m->yExt); free(m->zExt); free(m);
        return SIFV_ERR_UNSUPPORTED;
    }
    size_t n = m->n;
    double** all[] = {&m->rho, &m->rhoU, &m->rhoV, &m->rhoW, &m->rhoE, &m->velU, &m->velV, &m->velW, &m->pres,
                      &m->sigma, &m->rho0, &m->rhoU0, &m->rhoV0, &m->rhoW0, &m->rhoE0, &m->pres0, &m->rhoUStar,
                      &m->rhoVStar, &m->rhoWStar, &m->rhoEstar, &m->pAdvected, &m->rhoc2, &m->rhsRho, &m->rhsRhoU,
                      &m->rhsRhoV, &m->rhsRhoW, &m->rhsRhoE, &m->rhsP, &m->divU, &m->pressureRhs, &m->pressure,
                      &m->divUstar, &m->pNew};
    for (size_t q = 0; q < sizeof(all) / sizeof(all[0]); ++q) *all[q] = dalloc(n);
    for (int p = 0; p < cfg->nPhases; ++p) {
        m->alphaRho[p] = dalloc(n); m->alpha[p] = dalloc(n);
        m->alphaRho0[p] = dalloc(n); m->alpha0[p] = dalloc(n);
        m->rhsAlphaRho[p] = dalloc(n); m->rhsAlpha[p] = dalloc(n);
    }
    m->gradU = dalloc(9 * n);
    size_t nxf = (size_t)(m->nx + 1) * m->ny * m->nz, nyf = (size_t)m->nx * (m->ny + 1) * m->nz,
           nzf = (size_t)m->nx * m->ny * (m->nz + 1);
    m->xL = (Prim*)calloc(nxf, sizeof(Prim)); m->xR = (Prim*)calloc(nxf, sizeof(Prim));
    m->yL = (Prim*)calloc(nyf, sizeof(Prim)); m->yR = (Prim*)calloc(nyf, sizeof(Prim));
    m->zL = (Prim*)calloc(nzf, sizeof(Prim)); m->zR = (Prim*)calloc(nzf, sizeof(Prim));
    *out = m;
    return SIFV_OK;
}

int sifvo_set_comm(ctx_t* m, const sifv_comm_t* comm) {
    if (comm) m->comm = *comm;
    else memset(&m->comm, 0, sizeof(m->comm));
    return SIFV_OK;
}

int sifvo_destroy(ctx_t* m) {
    if (!m) return SIFV_OK;
    double* all[] = {m->rho, m->rhoU, m->rhoV, m->rhoW, m->rhoE, m->velU, m->velV, m->velW, m->pres, m->sigma,
                     m->rho0, m->rhoU0, m->rhoV0, m->rhoW0, m->rhoE0, m->pres0, m->rhoUStar, m->rhoVStar,
                     m->rhoWStar, m->rhoEstar, m->pAdvected, m->rhoc2, m->rhsRho, m->rhsRhoU, m->rhsRhoV,
                     m->rhsRhoW, m->rhsRhoE, m->rhsP, m->divU, m->pressureRhs, m->pressure, m->divUstar,
                     m->pNew, m->gradU, m->xExt, m->yExt, m->zExt};
    for (size_t q = 0; q < sizeof(all) / sizeof(all[0]); ++q) free(all[q]);
    for (int p = 0; p < m->c.nPhases; ++p) {
        free(m->alphaRho[p]); free(m->alpha[p]); free(m->alphaRho0[p]);
        free(m->alpha0[p]); free(m->rhsAlphaRho[p]); free(m->rhsAlpha[p]);
    }
    free(m->xL); free(m->xR); free(m->yL); free(m->yR); free(m->zL); free(m->zR);
    free(m->cellType); free(m->ibGhost); free(m->ibBodies);
    free(m);
    return SIFV_OK;
}

int sifvo_extents(const ctx_t* m, int* nx, int* ny, int* nz) {
    *nx = m->nxT; *ny = m->nyT; *nz = m->nzT;
    return SIFV_OK;
}

size_t sifvo_total_cells(const ctx_t* m) { return m->n; }

static double* field_ptr(ctx_t* m, int f) {
    switch (f) {
        case SIFV_F_RHO: return m->rho;
        case SIFV_F_RHOU: return m->rhoU;
        case SIFV_F_RHOV: return m->dim >= 2 ? m->rhoV : NULL;
        case SIFV_F_RHOW: return m->dim >= 3 ? m->rhoW : NULL;
        case SIFV_F_RHOE: return m->rhoE;
        case SIFV_F_VELU: return m->velU;
        case SIFV_F_VELV: return m->dim >= 2 ? m->velV : NULL;
        case SIFV_F_VELW: return m->dim >= 3 ? m->velW : NULL;
        case SIFV_F_PRES: return m->pres;
        case SIFV_F_SIGMA: return m->sigma;
        default: break;
    }
    if (f >= 16 && f < 16 + m->c.nPhases) return m->alphaRho[f - 16];
    if (f >= 32 && f < 32 + m->c.nPhases) return m->alpha[f - 32];
    return NULL;
}

int sifvo_set_field(ctx_t* m, int f, const double* src, int onDevice) {
    (void)onDevice;
    double* p = field_ptr(m, f);
    if (!p) { snprintf(m->err, sizeof m->err, "field %d not allocated", f); return SIFV_ERR_BAD_ARG; }
    memcpy(p, src, m->n * sizeof(double));
    return SIFV_OK;
}

int sifvo_get_field(ctx_t* m, int f, double* dst, int onDevice) {
    (void)onDevice;
    double* p = field_ptr(m, f);
    if (!p) { snprintf(m->err, sizeof m->err, "field %d not allocated", f); return SIFV_ERR_BAD_ARG; }
    memcpy(dst, p, m->n * sizeof(double));
    return SIFV_OK;
}

int sifvo_step(ctx_t* m, int step, double time, double targetDt, double* dtOut) {
    m->time = time;
    double dt = m->c.semiImplicit ? semi_step(m, step, targetDt) : explicit_step(m, step, targetDt);
    if (dtOut) *dtOut = dt;
    if (dt < 0.0) {
        snprintf(m->err, sizeof(m->err), "halo exchange failed (or not set: sifvo_set_comm)");
        return SIFV_ERR_CUDA;
    }
    return SIFV_OK;
}

int sifvo_last_pressure_iterations(const ctx_t* m, int* iters) {
    *iters = m->lastIters;
    return SIFV_OK;
}

int sifvo_set_pressure_solver(ctx_t* m, int kind) {
    m->pressureSolverKind = kind;
    return SIFV_OK;
}

int sifvo_pressure_solve(ctx_t* m, const double* rho, const double* rhoc2, const double* rhs, double* p, double dt,
                         double tol, int maxIter, int onDevice, int* iters) {
    (void)onDevice;
    *iters = pressure_solve(m, rho, rhoc2, rhs, p, dt, tol, maxIter);
    return (*iters >= maxIter) ? SIFV_NOT_CONVERGED : SIFV_OK;
}

int sifvo_igr_solve(ctx_t* m, int step) {
    velocity_gradients(m);
    igr_solve(m, step);
    return SIFV_OK;
}

int sifvo_acoustic_dt(ctx_t* m, double cfl, double maxDt, double* dt) {
    *dt = acoustic_dt(m, cfl, maxDt, 0);
    return SIFV_OK;
}

int sifvo_advective_dt(ctx_t* m, double cfl, double maxDt, double* dt) {
    *dt = advective_dt(m, cfl, maxDt);
    return SIFV_OK;
}

int sifvo_convert_cons_to_prim(ctx_t* m) {
    cons_to_prim(m);
    return SIFV_OK;
}

int sifvo_apply_bc(ctx_t* m) {
    apply_bc_prim(m);
    return SIFV_OK;
}

/* runTimeLoop's NaN check (src/RKTimeStepping.cpp:280-292): the first
 * interior cell in (k, j, i) order with a NaN in rho, rhoU, rhoE, pres,
 * rhoV (dim >= 2), rhoW (dim >= 3), tested in that order. */
int sifvo_check_nan(ctx_t* m, int* field, long long* cell) {
    *field = -1;
    *cell = -1;
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i < m->nx; ++i) {
                size_t idx = IDX(m, i, j, k);
                int f = -1;
                if (isnan(m->rho[idx])) f = SIFV_F_RHO;
                else if (isnan(m->rhoU[idx])) f = SIFV_F_RHOU;
                else if (isnan(m->rhoE[idx])) f = SIFV_F_RHOE;
                else if (isnan(m->pres[idx])) f = SIFV_F_PRES;
                else if (m->dim >= 2 && isnan(m->rhoV[idx])) f = SIFV_F_RHOV;
                else if (m->dim >= 3 && isnan(m->rhoW[idx])) f = SIFV_F_RHOW;
                if (f >= 0) {
                    *field = f;
                    *cell = (long long)i + (long long)m->nx * ((long long)j + (long long)m->ny * k);
                    return SIFV_OK;
                }
            }
    return SIFV_OK;
}

/* ---- immersed boundaries: src/ImmersedBoundary.cpp ---- */
static inline double CX(const ctx_t* m, int i) { return 0.5 * (m->xExt[i + m->ngx] + m->xExt[i + m->ngx + 1]); }
static inline double CY(const ctx_t* m, int j) { return 0.5 * (m->yExt[j + m->ngy] + m->yExt[j + m->ngy + 1]); }
static inline double CZ(const ctx_t* m, int k) { return 0.5 * (m->zExt[k + m->ngz] + m->zExt[k + m->ngz + 1]); }
static inline double sgn1(double v) { return (v >= 0) ? 1.0 : -1.0; }

/* cross-section coordinates of a cylinder (src/ImmersedBoundary.cpp:84-96) */
static void cyl_plane(const sifv_ib_body_t* b, double x, double y, double z, double* p0, double* p1) {
    if (b->axis == 0) { *p0 = y; *p1 = z; }
    else if (b->axis == 1) { *p0 = x; *p1 = z; }
    else { *p0 = x; *p1 = y; }
}

/* IBCircle / IBRectangle / IBCylinder / IBRectangularPrism::signedDistance
 * (src/ImmersedBoundary.cpp:11-16, 42-52, 84-96, 127-140) */
static double ib_sdf(const sifv_ib_body_t* b, double x, double y, double z) {
    const double* p = b->p;
    switch (b->shape) {
        case SIFV_IB_CIRCLE: {
            double dx = x - p[0], dy = y - p[1];
            return sqrt(dx * dx + dy * dy) - p[2];
        }
        case SIFV_IB_RECTANGLE: {
            double qx = fabs(x - p[0]) - p[2], qy = fabs(y - p[1]) - p[3];
            double out = sqrt(smax(qx, 0.0) * smax(qx, 0.0) + smax(qy, 0.0) * smax(qy, 0.0));
            return out + smin(smax(qx, qy), 0.0);
        }
        case SIFV_IB_CYLINDER: {
            double p0, p1;
            cyl_plane(b, x, y, z, &p0, &p1);
            double d0 = p0 - p[0], d1 = p1 - p[1];
            return sqrt(d0 * d0 + d1 * d1) - p[2];
        }
        default: {
            double qx = fabs(x - p[0]) - p[3], qy = fabs(y - p[1]) - p[4], qz = fabs(z - p[2]) - p[5];
            double out = sqrt(smax(qx, 0.0) * smax(qx, 0.0) + smax(qy, 0.0) * smax(qy, 0.0) +
                              smax(qz, 0.0) * smax(qz, 0.0));
            return out + smin(smax(smax(qx, qy), qz), 0.0);
        }
    }
}

/* closestPoint (src/ImmersedBoundary.cpp:18-28, 54-70, 98-119, 142-165) */
static void ib_closest(const sifv_ib_body_t* b, double x, double y, double z, double o[3]) {
    const double* p = b->p;
    switch (b->shape) {
        case SIFV_IB_CIRCLE: {
            double dx = x - p[0], dy = y - p[1];
            double dist = sqrt(dx * dx + dy * dy);
            if (dist < 1e-14) { o[0] = p[0] + p[2]; o[1] = p[1]; o[2] = 0.0; return; }
            double s = p[2] / dist;
            o[0] = p[0] + dx * s; o[1] = p[1] + dy * s; o[2] = 0.0;
            return;
        }
        case SIFV_IB_RECTANGLE: {
            double dx = x - p[0], dy = y - p[1];
            double cxl = sclamp(dx, -p[2], p[2]), cyl = sclamp(dy, -p[3], p[3]);
            if (fabs(dx) <= p[2] && fabs(dy) <= p[3]) {
                double tx = p[2] - fabs(dx), ty = p[3] - fabs(dy);
                if (tx < ty) cxl = (dx >= 0) ? p[2] : -p[2];
                else cyl = (dy >= 0) ? p[3] : -p[3];
            }
            o[0] = p[0] + cxl; o[1] = p[1] + cyl; o[2] = 0.0;
            return;
        }
        case SIFV_IB_CYLINDER: {
            double p0, p1;
            cyl_plane(b, x, y, z, &p0, &p1);
            double d0 = p0 - p[0], d1 = p1 - p[1];
            double dist = sqrt(d0 * d0 + d1 * d1);
            double q0, q1;
            if (dist < 1e-14) { q0 = p[0] + p[2]; q1 = p[1]; }
            else { double s = p[2] / dist; q0 = p[0] + d0 * s; q1 = p[1] + d1 * s; }
            if (b->axis == 0) { o[0] = x; o[1] = q0; o[2] = q1; }
            else if (b->axis == 1) { o[0] = q0; o[1] = y; o[2] = q1; }
            else { o[0] = q0; o[1] = q1; o[2] = z; }
            return;
        }
        default: {
            double dx = x - p[0], dy = y - p[1], dz = z - p[2];
            double cxl = sclamp(dx, -p[3], p[3]), cyl = sclamp(dy, -p[4], p[4]), czl = sclamp(dz, -p[5], p[5]);
            if (fabs(dx) <= p[3] && fabs(dy) <= p[4] && fabs(dz) <= p[5]) {
                double tx = p[3] - fabs(dx), ty = p[4] - fabs(dy), tz = p[5] - fabs(dz);
                if (tx <= ty && tx <= tz) cxl = (dx >= 0) ? p[3] : -p[3];
                else if (ty <= tx && ty <= tz) cyl = (dy >= 0) ? p[4] : -p[4];
                else czl = (dz >= 0) ? p[5] : -p[5];
            }
            o[0] = p[0] + cxl; o[1] = p[1] + cyl; o[2] = p[2] + czl;
            return;
        }
    }
}

/* outwardNormal (src/ImmersedBoundary.cpp:30-40, 72-82, 121-140, 167-180) */
static void ib_normal(const sifv_ib_body_t* b, double x, double y, double z, double o[3]) {
    const double* p = b->p;
    switch (b->shape) {
        case SIFV_IB_CIRCLE: {
            double dx = x - p[0], dy = y - p[1];
            double dist = sqrt(dx * dx + dy * dy);
            if (dist < 1e-14) { o[0] = 1.0; o[1] = 0.0; o[2] = 0.0; return; }
            o[0] = dx / dist; o[1] = dy / dist; o[2] = 0.0;
            return;
        }
        case SIFV_IB_RECTANGLE: {
            double cp[3];
            ib_closest(b, x, y, z, cp);
            double dx = cp[0] - p[0], dy = cp[1] - p[1];
            int onX = fabs(fabs(dx) - p[2]) < 1e-12, onY = fabs(fabs(dy) - p[3]) < 1e-12;
            if (onX && !onY) { o[0] = sgn1(dx); o[1] = 0.0; o[2] = 0.0; }
            else if (onY && !onX) { o[0] = 0.0; o[1] = sgn1(dy); o[2] = 0.0; }
            else { double len = sqrt(2.0); o[0] = sgn1(dx) / len; o[1] = sgn1(dy) / len; o[2] = 0.0; }
            return;
        }
        case SIFV_IB_CYLINDER: {
            double p0, p1;
            cyl_plane(b, x, y, z, &p0, &p1);
            double d0 = p0 - p[0], d1 = p1 - p[1];
            double dist = sqrt(d0 * d0 + d1 * d1);
            double n0 = 1.0, n1 = 0.0;
            if (!(dist < 1e-14)) { n0 = d0 / dist; n1 = d1 / dist; }
            if (b->axis == 0) { o[0] = 0.0; o[1] = n0; o[2] = n1; }
            else if (b->axis == 1) { o[0] = n0; o[1] = 0.0; o[2] = n1; }
            else { o[0] = n0; o[1] = n1; o[2] = 0.0; }
            return;
        }
        default: {
            double cp[3];
            ib_closest(b, x, y, z, cp);
            double dx = cp[0] - p[0], dy = cp[1] - p[1], dz = cp[2] - p[2];
            double nx = 0.0, ny = 0.0, nz = 0.0;
            if (fabs(fabs(dx) - p[3]) < 1e-12) nx = sgn1(dx);
            if (fabs(fabs(dy) - p[4]) < 1e-12) ny = sgn1(dy);
            if (fabs(fabs(dz) - p[5]) < 1e-12) nz = sgn1(dz);
            double len = sqrt(nx * nx + ny * ny + nz * nz);
            if (len < 1e-14) { o[0] = 1.0; o[1] = 0.0; o[2] = 0.0; return; }
            o[0] = nx / len; o[1] = ny / len; o[2] = nz / len;
            return;
        }
    }
}

/* ImmersedBoundaryMethod::findCell (src/ImmersedBoundary.cpp:190-214) */
static int ib_find_cell(const ctx_t* m, double coord, int dir) {
    int n = (dir == 0) ? m->nx : (dir == 1) ? m->ny : m->nz;
    if (n <= 1) return 0;
    double (*cen)(const ctx_t*, int) = (dir == 0) ? CX : (dir == 1) ? CY : CZ;
    if (coord <= cen(m, 0)) return 0;
    if (coord >= cen(m, n - 1)) return (n - 2 > 0) ? n - 2 : 0;
    for (int i = 0; i < n - 1; ++i)
        if (coord >= cen(m, i) && coord < cen(m, i + 1)) return i;
    return (n - 2 > 0) ? n - 2 : 0;
}

static double ib_t(double v, double c0, double c1) {
    double d = c1 - c0;
    return (d > 1e-14) ? sclamp((v - c0) / d, 0.0, 1.0) : 0.0;
}

/* ImmersedBoundaryMethod::buildInterpStencil (src/ImmersedBoundary.cpp:216-300) */
static void ib_stencil(const ctx_t* m, double x, double y, double z, IbGhost* g) {
    const int dim = m->dim;
    int i0 = ib_find_cell(m, x, 0);
    int j0 = (dim >= 2) ? ib_find_cell(m, y, 1) : 0;
    int k0 = (dim >= 3) ? ib_find_cell(m, z, 2) : 0;
    int i1 = (i0 + 1 < m->nx - 1) ? i0 + 1 : m->nx - 1;
    double tx = ib_t(x, CX(m, i0), CX(m, i1));
    if (dim == 1) {
        g->n = 2;
        g->interp[0] = IDX(m, i0, 0, 0); g->interp[1] = IDX(m, i1, 0, 0);
        g->w[0] = 1.0 - tx; g->w[1] = tx;
    } else {
        int j1 = (j0 + 1 < m->ny - 1) ? j0 + 1 : m->ny - 1;
        double ty = ib_t(y, CY(m, j0), CY(m, j1));
        if (dim == 2) {
            g->n = 4;
            g->interp[0] = IDX(m, i0, j0, 0); g->interp[1] = IDX(m, i1, j0, 0);
            g->interp[2] = IDX(m, i0, j1, 0); g->interp[3] = IDX(m, i1, j1, 0);
            g->w[0] = (1.0 - tx) * (1.0 - ty); g->w[1] = tx * (1.0 - ty);
            g->w[2] = (1.0 - tx) * ty; g->w[3] = tx * ty;
        } else {
            int k1 = (k0 + 1 < m->nz - 1) ? k0 + 1 : m->nz - 1;
            double tz = ib_t(z, CZ(m, k0), CZ(m, k1));
            g->n = 8;
            g->interp[0] = IDX(m, i0, j0, k0); g->interp[1] = IDX(m, i1, j0, k0);
            g->interp[2] = IDX(m, i0, j1, k0); g->interp[3] = IDX(m, i1, j1, k0);
            g->interp[4] = IDX(m, i0, j0, k1); g->interp[5] = IDX(m, i1, j0, k1);
            g->interp[6] = IDX(m, i0, j1, k1); g->interp[7] = IDX(m, i1, j1, k1);
            g->w[0] = (1.0 - tx) * (1.0 - ty) * (1.0 - tz); g->w[1] = tx * (1.0 - ty) * (1.0 - tz);
            g->w[2] = (1.0 - tx) * ty * (1.0 - tz); g->w[3] = tx * ty * (1.0 - tz);
            g->w[4] = (1.0 - tx) * (1.0 - ty) * tz; g->w[5] = tx * (1.0 - ty) * tz;
            g->w[6] = (1.0 - tx) * ty * tz; g->w[7] = tx * ty * tz;
        }
    }
    int allFluid = 1;
    for (int s = 0; s < g->n; ++s)
        if (m->cellType[g->interp[s]] != SIFV_CELL_FLUID) { allFluid = 0; break; }
    if (!allFluid) {
        size_t f = g->interp[0];
        for (int s = 0; s < g->n; ++s)
            if (m->cellType[g->interp[s]] == SIFV_CELL_FLUID) { f = g->interp[s]; break; }
        g->n = 1;
        g->interp[0] = f;
        g->w[0] = 1.0;
    }
}

/* ImmersedBoundaryMethod::classifyCells (src/ImmersedBoundary.cpp:302-392) */
static void ib_classify(ctx_t* m) {
    const int dim = m->dim;
    free(m->cellType); free(m->ibGhost);
    m->cellType = (unsigned char*)calloc(m->n, 1);
    int* owner = (int*)malloc(m->n * sizeof(int));
    for (size_t q = 0; q < m->n; ++q) owner[q] = -1;
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i < m->nx; ++i) {
                size_t idx = IDX(m, i, j, k);
                for (int b = 0; b < m->ibNBodies; ++b)
                    if (ib_sdf(&m->ibBodies[b], CX(m, i), CY(m, j), CZ(m, k)) < 0) {
                        m->cellType[idx] = SIFV_CELL_DEAD;
                        owner[idx] = b;
                        break;
                    }
            }
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i < m->nx; ++i) {
                size_t idx = IDX(m, i, j, k);
                if (m->cellType[idx] != SIFV_CELL_DEAD) continue;
                int fl = 0;
                if (i > 0 && m->cellType[IDX(m, i - 1, j, k)] == SIFV_CELL_FLUID) fl = 1;
                if (i < m->nx - 1 && m->cellType[IDX(m, i + 1, j, k)] == SIFV_CELL_FLUID) fl = 1;
                if (dim >= 2) {
                    if (j > 0 && m->cellType[IDX(m, i, j - 1, k)] == SIFV_CELL_FLUID) fl = 1;
                    if (j < m->ny - 1 && m->cellType[IDX(m, i, j + 1, k)] == SIFV_CELL_FLUID) fl = 1;
                }
                if (dim >= 3) {
                    if (k > 0 && m->cellType[IDX(m, i, j, k - 1)] == SIFV_CELL_FLUID) fl = 1;
                    if (k < m->nz - 1 && m->cellType[IDX(m, i, j, k + 1)] == SIFV_CELL_FLUID) fl = 1;
                }
                if (fl) m->cellType[idx] = SIFV_CELL_GHOST;
            }
    int cap = 0;
    for (size_t q = 0; q < m->n; ++q) cap += m->cellType[q] == SIFV_CELL_GHOST;
    m->ibGhost = (IbGhost*)calloc(cap > 0 ? (size_t)cap : 1, sizeof(IbGhost));
    m->ibCount = 0;
    for (int k = 0; k < m->nz; ++k)
        for (int j = 0; j < m->ny; ++j)
            for (int i = 0; i < m->nx; ++i) {
                size_t idx = IDX(m, i, j, k);
                if (m->cellType[idx] != SIFV_CELL_GHOST) continue;
                IbGhost* g = &m->ibGhost[m->ibCount++];
                const sifv_ib_body_t* b = &m->ibBodies[owner[idx]];
                double xG = CX(m, i), yG = CY(m, j), zG = CZ(m, k), cp[3];
                ib_closest(b, xG, yG, zG, cp);
                ib_normal(b, xG, yG, zG, g->normal);
                g->cell = idx;
                g->body = owner[idx];
                ib_stencil(m, 2.0 * cp[0] - xG, 2.0 * cp[1] - yG, 2.0 * cp[2] - zG, g);
            }
    free(owner);
}

/* ImmersedBoundaryMethod::applyGhostCells (src/ImmersedBoundary.cpp:394-470) */
static void ib_apply_ghosts(ctx_t* m) {
    const int dim = m->dim, nPh = m->c.nPhases;
    for (int q = 0; q < m->ibCount; ++q) {
        const IbGhost* g = &m->ibGhost[q];
        double r = 0.0, u = 0.0, v = 0.0, w = 0.0, p = 0.0, sg = 0.0, e = 0.0;
        for (int s = 0; s < g->n; ++s) {
            size_t c = g->interp[s];
            double ws = g->w[s];
            r += ws * m->rho[c];
            u += ws * m->velU[c];
            if (dim >= 2) v += ws * m->velV[c];
            if (dim >= 3) w += ws * m->velW[c];
            p += ws * m->pres[c];
            sg += ws * m->sigma[c];
            e += ws * m->rhoE[c];
        }
        size_t idx = g->cell;
        m->rho[idx] = r;
        m->pres[idx] = p;
        m->sigma[idx] = sg;
        m->rhoE[idx] = e;
        double gu, gv, gw;
        if (m->ibBodies[g->body].wall == SIFV_IB_NOSLIP) {
            gu = -u; gv = -v; gw = -w;
        } else {
            double dot = u * g->normal[0];
            if (dim >= 2) dot += v * g->normal[1];
            if (dim >= 3) dot += w * g->normal[2];
            gu = u - 2.0 * dot * g->normal[0];
            gv = v - 2.0 * dot * g->normal[1];
            gw = w - 2.0 * dot * g->normal[2];
        }
        m->velU[idx] = gu;
        if (dim >= 2) m->velV[idx] = gv;
        if (dim >= 3) m->velW[idx] = gw;
        m->rhoU[idx] = r * gu;
        if (dim >= 2) m->rhoV[idx] = r * gv;
        if (dim >= 3) m->rhoW[idx] = r * gw;
        for (int ph = 0; ph < nPh; ++ph) {
            double val = 0.0;
            for (int s = 0; s < g->n; ++s) val += g->w[s] * m->alphaRho[ph][g->interp[s]];
            m->alphaRho[ph][idx] = val;
        }
        for (int ph = 0; ph < nPh; ++ph) {
            double val = 0.0;
            for (int s = 0; s < g->n; ++s) val += g->w[s] * m->alpha[ph][g->interp[s]];
            m->alpha[ph][idx] = val;
        }
    }
}

/* ImmersedBoundaryMethod::applyScalarGhostCells (src/ImmersedBoundary.cpp:472-482) */
static void ib_apply_scalar(ctx_t* m, double* f) {
    for (int q = 0; q < m->ibCount; ++q) {
        const IbGhost* g = &m->ibGhost[q];
        double val = 0.0;
        for (int s = 0; s < g->n; ++s) val += g->w[s] * f[g->interp[s]];
        f[g->cell] = val;
    }
}

int sifvo_set_immersed_bodies(ctx_t* m, const sifv_ib_body_t* bodies, int nBodies) {
    if (!m || nBodies < 0 || (nBodies > 0 && !bodies)) return SIFV_ERR_BAD_ARG;
    if (nBodies > 0 && m->c.semiImplicit) {
        snprintf(m->err, sizeof(m->err), "the semi-implicit step has no immersed boundary");
        return SIFV_ERR_UNSUPPORTED;
    }
    if (nBodies > 0 && m->exchangeFaces) {
        snprintf(m->err, sizeof(m->err), "immersed boundaries are not supported with SIFV_BC_EXCHANGE faces");
        return SIFV_ERR_UNSUPPORTED;
    }
    free(m->ibBodies); free(m->cellType); free(m->ibGhost);
    m->ibBodies = NULL; m->cellType = NULL; m->ibGhost = NULL;
    m->ibCount = 0;
    m->ibNBodies = nBodies;
    if (nBodies == 0) return SIFV_OK;
    m->ibBodies = (sifv_ib_body_t*)malloc((size_t)nBodies * sizeof(sifv_ib_body_t));
    memcpy(m->ibBodies, bodies, (size_t)nBodies * sizeof(sifv_ib_body_t));
    ib_classify(m);
    return SIFV_OK;
}

int sifvo_ib_cell_types(ctx_t* m, unsigned char* types) {
    for (size_t q = 0; q < m->n; ++q) types[q] = m->cellType ? m->cellType[q] : SIFV_CELL_FLUID;
    return SIFV_OK;
}

int sifvo_apply_ib_ghost_cells(ctx_t* m) {
    if (m->cellType) ib_apply_ghosts(m);
    return SIFV_OK;
}
