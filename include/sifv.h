/*
 * sifv.h -- C ABI of the B200 (sm_100a) finite-volume time step.
 *
 * This is the drop-in boundary between a host code written against the
 * SemiImplicitFV interfaces (SimulationConfig, RiemannSolverType,
 * PressureSolver, IGRSolver) and the CUDA kernels of this library.  Every
 * entry point takes plain pointers, sizes and PODs; no C++ or torch types
 * cross it.  All calls return an int status (SIFV_OK == 0, >0 warning,
 * <0 error); sifv_last_error() gives the message.  A context is not
 * thread safe: use one host thread per context.  Distinct contexts are
 * independent.
 *
 * Reference interfaces replaced (paths relative to the SemiImplicitFV
 * repository):
 *   sifv_config_t      <- SimulationConfig         include/SimulationConfig.hpp:72-210
 *   sifv_mesh_t        <- RectilinearMesh ctor     include/RectilinearMesh.hpp:35-38
 *                         + setBoundaryCondition   include/RectilinearMesh.hpp:117
 *   sifv_set/get_field <- SolutionState SoA        include/SolutionState.hpp:73-113
 *   sifv_step          <- ExplicitSolver::step     include/ExplicitSolver.hpp:33-36
 *                         SemiImplicitSolver::step include/SemiImplicitSolver.hpp:36
 *   sifv_pressure_solve<- PressureSolver::solve    include/PressureSolver.hpp:17-38
 *                         (JacobiPressureSolver     src/JacobiPressureSolver.cpp:57-108)
 *   sifv_igr_solve     <- IGRSolver::solveEntropicPressure include/IGR.hpp:42-51
 *   sifv_acoustic_dt   <- computeAcousticTimeStep  src/RKTimeStepping.cpp:43-123,148-159
 *   sifv_advective_dt  <- computeAdvectiveTimeStep src/RKTimeStepping.cpp:15-41,125-134
 *   sifv_convert_cons_to_prim
 *                      <- SolutionState::convertConservativeToPrimitiveVariables
 *                         src/SolutionState.cpp:187-205 and
 *                         MixtureEOS::convertConservativeToPrimitive src/MixtureEOS.cpp:99-143
 *   sifv_apply_bc      <- RectilinearMesh::applyBoundaryConditions(state, PRIM, halo)
 *                         src/RectilinearMesh.cpp:498-524
 */
#ifndef SIFV_H
#define SIFV_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SIFV_ABI_VERSION 1
#define SIFV_MAX_PHASES 8

/* ---- status codes ---------------------------------------------------- */
#define SIFV_OK                 0
#define SIFV_NOT_CONVERGED      1   /* pressure solve reached maxIter (the reference returns maxIter silently) */
#define SIFV_ERR_BAD_CONFIG    -1   /* SimulationConfig::validate() would throw std::invalid_argument */
#define SIFV_ERR_BAD_ARG       -2
#define SIFV_ERR_CUDA          -3
#define SIFV_ERR_NAN           -4
#define SIFV_ERR_UNSUPPORTED   -5
#define SIFV_ERR_TIMEOUT       -6   /* a bounded device wait ran out; the context stays usable */
#define SIFV_ERR_NO_DEVICE     -7

/* ---- enums mirrored from the reference -------------------------------- */
/* ReconstructionOrder, include/SimulationConfig.hpp:13-20 */
#define SIFV_WENO1   0
#define SIFV_WENO3   1
#define SIFV_WENO5   2
#define SIFV_UPWIND1 3
#define SIFV_UPWIND3 4
#define SIFV_UPWIND5 5
/* RiemannSolverType, include/RiemannSolver.hpp:16 */
#define SIFV_LF      0
#define SIFV_RUSANOV 1
#define SIFV_HLLC    2
/* BoundaryCondition, include/RectilinearMesh.hpp:14-20 */
#define SIFV_BC_SYMMETRY   0
#define SIFV_BC_OUTFLOW    1
#define SIFV_BC_PERIODIC   2
#define SIFV_BC_SLIPWALL   3
#define SIFV_BC_NOSLIPWALL 4
/* A face shared with a neighbouring rank of a domain decomposition (the
 * reference's non-physical MPI faces, src/MPIContext.cpp:80-170): its ghost
 * layers hold the neighbour's cells, filled by the context's halo exchange
 * (sifv_set_comm), instead of a boundary condition. */
#define SIFV_BC_EXCHANGE   16
/* single-phase EOS: IdealGasEOS (src/IdealGasEOS.cpp) or StiffenedGasEOS (src/StiffenedGasEOS.cpp) */
#define SIFV_EOS_IDEAL     0
#define SIFV_EOS_STIFFENED 1
/* arithmetic of the reconstruction/flux bulk */
#define SIFV_PREC_FP64      0   /* FP64 in the reference's operation order: bit-identical results */
#define SIFV_PREC_MIXED     1   /* FP32 reconstruction/flux bulk; FP64 state, primitive recovery, divergence, RK update */
#define SIFV_PREC_FP64_FAST 2   /* FP64, fused sweeps with reassociated arithmetic (FMA, shared WENO indicators) */
/* SIFV_PREC_MIXED and SIFV_PREC_FP64_FAST run the explicit single-phase
 * WENO5 step (any dim, any Riemann solver, no IGR, no body force); other
 * configurations are rejected by sifv_create with SIFV_ERR_UNSUPPORTED. */

/* ---- field identifiers (SolutionState members) ------------------------ */
#define SIFV_F_RHO    0
#define SIFV_F_RHOU   1
#define SIFV_F_RHOV   2
#define SIFV_F_RHOW   3
#define SIFV_F_RHOE   4
#define SIFV_F_VELU   5
#define SIFV_F_VELV   6
#define SIFV_F_VELW   7
#define SIFV_F_PRES   8
#define SIFV_F_SIGMA  9
#define SIFV_F_ALPHARHO(ph) (16 + (ph))   /* alphaRho[ph] */
#define SIFV_F_ALPHA(ph)    (32 + (ph))   /* alpha[ph]    */

/* Flat mirror of SimulationConfig (include/SimulationConfig.hpp:72-210) plus
 * the EOS / Riemann-solver choice that the reference passes as objects. */
typedef struct sifv_config {
    int    dim;                 /* 1, 2 or 3 */
    int    nGhost;
    int    RKOrder;             /* 1, 2 or 3 (Shu-Osher SSP) */
    int    useIGR;
    int    semiImplicit;
    int    reconOrder;          /* SIFV_WENO* / SIFV_UPWIND* */
    double wenoEps;
    int    riemannSolver;       /* SIFV_LF / SIFV_RUSANOV / SIFV_HLLC */
    int    eosKind;             /* SIFV_EOS_IDEAL / SIFV_EOS_STIFFENED */
    double gamma;
    double pInf;
    /* ExplicitParams */
    double cfl, constDt, maxDt, minDt;
    /* SemiImplicitParams */
    double siCfl, siMaxDt, siMinDt;
    int    maxPressureIters;
    double pressureTol;
    /* IGRParams */
    double alphaCoeff;
    int    IGRIters;
    int    IGRWarmStartIters;
    /* MultiPhaseParams (nPhases == 0: single phase) */
    int    nPhases;
    double phaseGamma[SIFV_MAX_PHASES];
    double phasePInf[SIFV_MAX_PHASES];
    double alphaMin;
    /* BodyForceParams: accel_d(t) = a_d + b_d cos(c_d t + d_d) */
    double bfA[3], bfB[3], bfC[3], bfD[3];
    /* SIFV_PREC_* */
    int    precision;
    /* ViscousParams (include/SimulationConfig.hpp:62-65): dynamic viscosity
     * mu, or per-phase viscosities phaseMu[0 .. nPhaseMu-1] (nPhaseMu ==
     * nPhases; 0 = the scalar mu).  Viscous when mu > 0 or nPhaseMu > 0
     * (SimulationConfig::hasViscosity). */
    double mu;
    double phaseMu[SIFV_MAX_PHASES];
    int    nPhaseMu;
    /* SurfaceTensionParams (include/SimulationConfig.hpp:67-70): capillary
     * coefficient sigma (0 = off; needs nPhases >= 2, the interface is
     * phase 0's volume fraction) and the |grad alpha| regularisation. */
    double stSigma;
    double stEpsGradAlpha;
} sifv_config_t;

/* Mesh: physical node coordinates per axis (n+1 entries; NULL for an
 * inactive axis means {0, 1}) and the six face boundary conditions
 * (XLow, XHigh, YLow, YHigh, ZLow, ZHigh).  Periodic axes must be periodic
 * on both faces. */
typedef struct sifv_mesh {
    int nx, ny, nz;
    const double* xNodes;
    const double* yNodes;
    const double* zNodes;
    int bc[6];
} sifv_mesh_t;

typedef struct sifv_ctx sifv_ctx_t;

/* Fill a config with the reference's defaults (SimulationConfig members'
 * initialisers, include/SimulationConfig.hpp:22-92). */
void sifv_config_defaults(sifv_config_t* cfg);

/* Validate exactly as SimulationConfig::validate()
 * (include/SimulationConfig.hpp:123-209); message via sifv_last_error(NULL). */
int sifv_config_validate(const sifv_config_t* cfg);

/* Create a context on CUDA device `device`: allocates the device SoA state
 * (totalCells doubles per field, ghosts included) and scratch. */
int sifv_create(const sifv_config_t* cfg, const sifv_mesh_t* mesh, int device,
                sifv_ctx_t** out);
int sifv_destroy(sifv_ctx_t* ctx);

/* Message of the last error on this context (ctx == NULL: last
 * context-free error of the calling thread). */
const char* sifv_last_error(const sifv_ctx_t* ctx);

/* Extents including ghosts (RectilinearMesh::nxTotal/nyTotal/nzTotal). */
int sifv_extents(const sifv_ctx_t* ctx, int* nxTot, int* nyTot, int* nzTot);
size_t sifv_total_cells(const sifv_ctx_t* ctx);

/* Copy a whole field (totalCells doubles, x fastest, ghosts included) in or
 * out.  onDevice != 0: the pointer is device memory on the context's
 * device.  Copies are ordered on the context's stream and complete before
 * return. */
int sifv_set_field(sifv_ctx_t* ctx, int field, const double* src, int onDevice);
int sifv_get_field(sifv_ctx_t* ctx, int field, double* dst, int onDevice);
/* Device address of a field (zero-copy access for device-resident callers). */
int sifv_field_device_ptr(sifv_ctx_t* ctx, int field, double** dptr);

/* Use a caller-owned cudaStream_t (NULL: the context's own stream). */
int sifv_set_stream(sifv_ctx_t* ctx, void* stream);
int sifv_synchronize(sifv_ctx_t* ctx);

/* One time step, ExplicitSolver::step or SemiImplicitSolver::step by
 * cfg->semiImplicit.  `step` and `time` are SimulationConfig::step/time
 * (IGR warm start on step 0; body-force phase).  targetDt > 0 caps dt as
 * in the reference.  *dtOut receives the dt taken.  Returns
 * SIFV_NOT_CONVERGED (still a completed step) when any pressure solve of
 * the step reached maxPressureIters. */
int sifv_step(sifv_ctx_t* ctx, int step, double time, double targetDt, double* dtOut);

/* nSteps steps back to back with no host round trip between them: dt is
 * reduced and applied on the device, and each step's dt is capped by
 * tEnd - t (tEnd <= 0: no cap).  Explicit path only.  On return
 * *timeOut = time after the last step.  Steps after t reaches tEnd are
 * skipped on the device. */
int sifv_advance(sifv_ctx_t* ctx, int step0, double time0, double tEnd, int nSteps,
                 double* timeOut, int* stepsTaken);

/* Jacobi iterations of the last pressure solve (SemiImplicitSolver::
 * lastPressureIterations, include/SemiImplicitSolver.hpp:46). */
int sifv_last_pressure_iterations(const sifv_ctx_t* ctx, int* iters);

/* PressureSolver::solve (include/PressureSolver.hpp:17-38) for the Jacobi
 * solver: (1 + rhoc2 dt^2 L) p = rhs + rhoc2 dt^2 offdiag(p), iterated
 * until max|p_new - p| < tol or maxIter.  All arrays are totalCells long;
 * `pressure` is the initial guess on entry and the solution on return
 * (interior cells; ghosts are not written).  onDevice != 0: device
 * pointers.  *iters as the reference's return value. */
int sifv_pressure_solve(sifv_ctx_t* ctx, const double* rho, const double* rhoc2,
                        const double* rhs, double* pressure, double dt, double tol,
                        int maxIter, int onDevice, int* iters);

/* IGRSolver::solveEntropicPressure on the context's state: velocity
 * gradients from the current primitive fields (ghosts must be filled, see
 * sifv_apply_bc), then the lexicographic Gauss-Seidel sweeps of the
 * reference (IGRWarmStartIters on step 0, else IGRIters) updating sigma. */
int sifv_igr_solve(sifv_ctx_t* ctx, int step);

/* Time-step reductions on the context's state (interior cells). */
int sifv_acoustic_dt(sifv_ctx_t* ctx, double cfl, double maxDt, double* dt);
int sifv_advective_dt(sifv_ctx_t* ctx, double cfl, double maxDt, double* dt);

/* Conservative -> primitive on interior cells, and the PRIM ghost fill. */
int sifv_convert_cons_to_prim(sifv_ctx_t* ctx);
int sifv_apply_bc(sifv_ctx_t* ctx);

/* One step as sifv_step, with a CUDA event after every kernel family:
 * per family (in launch order of first appearance) the summed device
 * milliseconds and the number of launches.  `names` receives the family
 * names separated by newlines (truncated to namesCap bytes). */
int sifv_profile_step(sifv_ctx_t* ctx, int step, double time, double targetDt, char* names, int namesCap,
                      double* ms, int* counts, int maxFamilies, int* nFamilies);

/* Device time of the kernels launched by the last sifv_step / sifv_advance
 * call, and the number of kernel launches it made. */
int sifv_last_step_stats(const sifv_ctx_t* ctx, double* deviceMs, int* launches);

/* ---- pressure solver selection ----------------------------------------- */
/* The PressureSolver plugin the semi-implicit step and sifv_pressure_solve
 * use: JacobiPressureSolver (src/JacobiPressureSolver.cpp:57-108, default)
 * or GaussSeidelPressureSolver (src/GaussSeidelPressureSolver.cpp:10-49,
 * lexicographic in-place sweeps run as a tiled wavefront, bit-identical). */
#define SIFV_PRESSURE_JACOBI 0
#define SIFV_PRESSURE_GAUSS_SEIDEL 1
/* HyprePressureSolver (src/HyprePressureSolver.cpp, built with Hypre only):
 * conjugate gradients preconditioned by one multigrid V-cycle (weighted
 * Jacobi relaxation, Galerkin coarse levels), stopping when the residual's
 * two-norm falls to tol times the right-hand side's; Neumann faces on
 * physical boundaries.  The same linear system and stopping rule as the
 * reference's Hypre PCG+PFMG, not its bits: the multigrid hierarchy is this
 * library's own.  Iteration counts stay nearly flat as the mesh grows. */
#define SIFV_PRESSURE_PCG_MG 2
int sifv_set_pressure_solver(sifv_ctx_t* ctx, int kind);

/* ---- immersed boundaries ---------------------------------------------------- */
/* ImmersedBoundaryMethod (include/ImmersedBoundary.hpp, src/ImmersedBoundary.cpp)
 * on the explicit step: classifyCells at set-up (cells inside a body are
 * dead, dead cells with a fluid face neighbour are ghost cells; each ghost
 * cell gets the mirror image point of its centroid through the body surface
 * and a bi/trilinear stencil of fluid cells), then per stage and after the
 * step applyGhostCells (interpolated state, velocity reflected: reversed for
 * no-slip, normal component mirrored for slip), solid cells skipped in the
 * update, the dt limits and the IGR sweeps (with the scalar ghost fill of
 * sigma after each sweep).  Explicit SIFV_PREC_FP64 steps only, as in the
 * reference (the semi-implicit solver has no immersed boundary). */
#define SIFV_IB_CIRCLE     0   /* IBCircle(p = cx, cy, r) */
#define SIFV_IB_RECTANGLE  1   /* IBRectangle(p = cx, cy, hw, hh) */
#define SIFV_IB_CYLINDER   2   /* IBCylinder(p = c0, c1, r; axis) */
#define SIFV_IB_PRISM      3   /* IBRectangularPrism(p = cx, cy, cz, hw, hh, hd) */
#define SIFV_IB_NOSLIP     0   /* IBBody::WallType::NoSlip (the default) */
#define SIFV_IB_SLIP       1
#define SIFV_CELL_FLUID    0   /* CellType */
#define SIFV_CELL_GHOST    1
#define SIFV_CELL_DEAD     2
typedef struct sifv_ib_body {
    int shape;        /* SIFV_IB_CIRCLE .. SIFV_IB_PRISM */
    int wall;         /* SIFV_IB_NOSLIP / SIFV_IB_SLIP */
    int axis;         /* cylinder axis (0 x, 1 y, 2 z) */
    double p[6];
} sifv_ib_body_t;
/* Bodies of any shape, through the three queries of IBBody (signed
 * distance, negative inside; closest surface point; outward normal there),
 * called on the host during set-up only. */
typedef struct sifv_ib_shapes {
    void* user;
    double (*signedDistance)(void* user, int body, double x, double y, double z);
    void (*closestPoint)(void* user, int body, double x, double y, double z, double out[3]);
    void (*outwardNormal)(void* user, int body, double x, double y, double z, double out[3]);
} sifv_ib_shapes_t;
/* addBody for each body + classifyCells; nBodies = 0 removes the boundary. */
int sifv_set_immersed_bodies(sifv_ctx_t* ctx, const sifv_ib_body_t* bodies, int nBodies);
int sifv_set_immersed_shapes(sifv_ctx_t* ctx, int nBodies, const int* wall, const sifv_ib_shapes_t* shapes);
/* CellType of every cell (totalCells bytes, SIFV_CELL_*; cells outside the
 * interior are fluid). */
int sifv_ib_cell_types(sifv_ctx_t* ctx, unsigned char* types);
/* applyGhostCells on the context's current primitive state. */
int sifv_apply_ib_ghost_cells(sifv_ctx_t* ctx);

/* ---- output path: NaN check, VTK, time loop ------------------------------- */
/* runTimeLoop's NaN check (src/RKTimeStepping.cpp:280-311) on the device:
 * the first interior cell in (k, j, i) order holding a NaN in rho, rhoU,
 * rhoE, pres, rhoV (dim >= 2) or rhoW (dim >= 3), tested in that order.
 * *field = the SIFV_F_* id of that field, or -1 when there is none;
 * *cell = its interior index i + nx (j + ny k) (-1 when none). */
int sifv_check_nan(sifv_ctx_t* ctx, int* field, long long* cell);

/* VTK XML output with the files and bytes of VTKSession / VTKWriter
 * (src/VTKSession.cpp, src/VTKWriter.cpp) for one rank:
 *   <dir>/<base>.pvd                                 time series
 *   <dir>/snapshot_<n>/<base>_<n>_r0.vtr             the piece (RectilinearGrid, ASCII)
 *   <dir>/snapshot_<n>/<base>_<n>.pvtr               its parallel meta-file
 * The session is host-side: sifv_vtk_open writes the .pvd header.
 * nThreads <= 0: one formatting thread per hardware thread. */
typedef struct sifv_vtk sifv_vtk_t;
int sifv_vtk_open(const char* dir, const char* baseName, const sifv_config_t* cfg, const sifv_mesh_t* mesh,
                  int nThreads, sifv_vtk_t** out);
/* Host fields in the context layout (totalCells doubles, ghosts included):
 * every pointer the written arrays need (pres, sigma when useIGR, rhoE,
 * vel and mom of the active dims, rho single-phase or alphaRho[] / alpha[]
 * of each phase). */
typedef struct sifv_vtk_fields {
    const double* pres;
    const double* sigma;
    const double* rhoE;
    const double* vel[3];
    const double* mom[3];
    const double* rho;
    const double* alphaRho[SIFV_MAX_PHASES];
    const double* alpha[SIFV_MAX_PHASES];
} sifv_vtk_fields_t;
/* VTKSession::write(state, time) from host arrays; synchronous. */
int sifv_vtk_write_host(sifv_vtk_t* vtk, double time, const sifv_vtk_fields_t* fields);
/* VTKSession::write from a context's device state: the fields are copied
 * to a device staging slot on the context's stream (the next step may run
 * at once), brought to pinned host memory on a copy stream and written by
 * the session's writer thread while the context keeps stepping.  Two
 * staging slots; a third write waits for the oldest. */
int sifv_vtk_write(sifv_vtk_t* vtk, sifv_ctx_t* ctx, double time);
/* Wait for every queued write; returns the first write error. */
int sifv_vtk_flush(sifv_vtk_t* vtk);
/* Flush, then release the session (VTKSession::finalize). */
int sifv_vtk_close(sifv_vtk_t* vtk);
const char* sifv_vtk_last_error(const sifv_vtk_t* vtk);

/* runTimeLoop (src/RKTimeStepping.cpp:241-356, TimeLoopParams
 * include/RKTimeStepping.hpp:91-99) on a context: output at t = 0 and
 * whenever t >= nextOutput - 1e-12 outputInterval, dt capped to hit every
 * output time and endTime, NaN check at each output.  Explicit steps
 * without body force run device-resident (dt, time and the output
 * condition live on the device; the host looks in every `batch` steps);
 * semi-implicit and body-force steps run one step per host round trip.
 * progress (may be NULL) is called for step 1 and every printInterval-th
 * step with the step's dt.  vtk may be NULL (no files).  Returns SIFV_OK,
 * or SIFV_ERR_NAN with *result naming the field and cell (the snapshot of
 * that output is still written, as in the reference). */
typedef struct sifv_time_loop {
    double endTime;
    double outputInterval;
    int printInterval;
    int checkNaN;
    int step0;        /* SimulationConfig::step at entry */
    int batch;        /* device-resident steps between host checks (<= 0: 64) */
} sifv_time_loop_t;
typedef struct sifv_loop_result {
    double time;
    int steps;        /* SimulationConfig::step at exit */
    int outputs;      /* outputs reached, t = 0 included */
    int nanField;     /* SIFV_F_* of the NaN, -1 = none */
    long long nanCell;
    double nanTime;
    int nanStep;
} sifv_loop_result_t;
typedef void (*sifv_progress_fn)(void* user, int step, double time, double dt);
int sifv_run_time_loop(sifv_ctx_t* ctx, const sifv_time_loop_t* params, sifv_vtk_t* vtk,
                       sifv_progress_fn progress, void* user, sifv_loop_result_t* result);

/* ---- diagnostics ----------------------------------------------------------- */
/* Maximum relative error of the fast paths' reciprocal, square root and
 * reciprocal square root against IEEE 1/x, sqrt(x) and 1/sqrt(x) (the last
 * rounded twice) over n arguments spread across [2^-60, 2^60)
 * (SIFV_PREC_FP64_FAST / SIFV_PREC_MIXED use them; SIFV_PREC_FP64 does not).
 * maxRelRsqrt may be NULL.  Returns 0 or SIFV_ERR_CUDA. */
int sifv_fastmath_selftest(long long n, double* maxRelRcp, double* maxRelSqrt, double* maxRelRsqrt);

/* ---- discrete adjoint and tangent of the explicit step ------------------ */
/* Reverse- and forward-mode derivatives of the map U(t0) -> U(tEnd) that
 * sifv_step iterates (ExplicitSolver::step, src/ExplicitSolver.cpp:68-203:
 * cons -> prim, PRIM ghost fill, WENO5 / UPWIND5 reconstruction, Riemann
 * flux, flux divergence, SSP-RK stages), single-phase, SIFV_PREC_FP64, no
 * IGR or body force.  The time-step sequence is held fixed (the CFL minimum
 * is not differentiable); every branch (HLLC wave pattern, wave-speed
 * estimates, clamps) is the one the forward pass took.
 *
 * sifv_adjoint_forward runs the forward from the context's state, with the
 * CFL dt and targetDt = tEnd - t (as the reference's time loop) or with the
 * given dt sequence, records the sequence and a checkpoint of the
 * conservative state every checkpointEvery steps.  sifv_adjoint_set_seed
 * sets dJ/dU(tEnd) (interior cells; ghosts ignored); sifv_adjoint_backward
 * recomputes each checkpoint segment (storing its stage states) and sweeps
 * it in reverse; sifv_adjoint_get_gradient then returns dJ/dU(t0) (ghost
 * entries zero) and the context's state is the forward end state again.
 * sifv_tangent_forward advances the state and the direction set by
 * sifv_tangent_set_direction together (dU(tEnd) by sifv_tangent_get). */
int sifv_adjoint_forward(sifv_ctx_t* ctx, int step0, double time0, double tEnd, int maxSteps, int checkpointEvery,
                         const double* dtSchedule, int nSchedule, double* timeOut, int* stepsOut);
int sifv_adjoint_schedule(const sifv_ctx_t* ctx, double* dts, int cap, int* n);
int sifv_adjoint_set_seed(sifv_ctx_t* ctx, int field, const double* seed, int onDevice);
int sifv_adjoint_backward(sifv_ctx_t* ctx, double* deviceMs);
int sifv_adjoint_get_gradient(sifv_ctx_t* ctx, int field, double* grad, int onDevice);
int sifv_tangent_set_direction(sifv_ctx_t* ctx, int field, const double* dir, int onDevice);
int sifv_tangent_forward(sifv_ctx_t* ctx, int step0, double time0, double tEnd, int maxSteps,
                         const double* dtSchedule, int nSchedule, double* timeOut, int* stepsOut);
int sifv_tangent_get(sifv_ctx_t* ctx, int field, double* out, int onDevice);
/* Arithmetic of the reverse sweep's local Jacobians (the flux and
 * reconstruction derivatives of every face): SIFV_PREC_FP64 (default) or
 * SIFV_PREC_MIXED (FP32; the forward trajectory, the adjoint state and the
 * accumulation of the face shares stay FP64). */
int sifv_adjoint_set_precision(sifv_ctx_t* ctx, int precision);

/* ---- batched ensembles -------------------------------------------------- */
/* Many independent 1D problems of different sizes (same configuration and
 * boundary conditions, own mesh [xLo[k], xHi[k]] with nCells[k] cells)
 * advanced to a common end time by ONE kernel launch: one CTA per instance
 * runs the instance's whole time loop (own dt, targetDt = tEnd - t as the
 * reference's time loop caps it, src/RKTimeStepping.cpp:258-266).  Explicit
 * 1D WENO5 / UPWIND5, single- or multi-phase, any Riemann solver;
 * SIFV_PREC_FP64 (bit-identical to running each instance alone) or
 * SIFV_PREC_MIXED (FP32 reconstruction / Riemann bulk; the primitive
 * recovery, including the mixture pressure from total energy, the carried
 * state and the update stay FP64).  Fields are packed instance after instance, each
 * with its ghosts, x fastest (sifv_ensemble_layout gives the nInst + 1
 * offsets). */
typedef struct sifv_ensemble sifv_ensemble_t;
int sifv_ensemble_create(const sifv_config_t* cfg, int nInst, const int* nCells, const double* xLo,
                         const double* xHi, const int bc[2], int device, sifv_ensemble_t** out);
int sifv_ensemble_destroy(sifv_ensemble_t* e);
const char* sifv_ensemble_last_error(const sifv_ensemble_t* e);
int sifv_ensemble_layout(const sifv_ensemble_t* e, long long* offsets);
int sifv_ensemble_set_field(sifv_ensemble_t* e, int field, const double* packed, int onDevice);
int sifv_ensemble_get_field(sifv_ensemble_t* e, int field, double* packed, int onDevice);
/* Advance every instance until its time reaches tEnd or it has taken
 * maxSteps steps in total (<= 0: no step limit).  blockSize 0: the
 * autotuned (or default 256) threads per instance.  timesOut / stepsOut
 * (nInst entries each, may be NULL) receive each instance's time and step
 * count; *deviceMs the launch's device time.  An instance whose time step
 * comes out non-positive (a blown-up state) stops there and the call
 * returns SIFV_ERR_NAN; tEnd must be finite unless maxSteps > 0. */
int sifv_ensemble_run(sifv_ensemble_t* e, double tEnd, int maxSteps, int blockSize, double* timesOut,
                      int* stepsOut, double* deviceMs);
/* Time a probe at 128 / 256 / 512 (and, mixed, 1024) threads per instance
 * in which each instance takes steps in proportion to its cell count (as in
 * a run to a common end time), the largest probeSteps; keep the fastest
 * block size for later runs and restore the state. */
int sifv_ensemble_autotune(sifv_ensemble_t* e, int probeSteps, int* blockSizeOut);

/* Work-unit shape of the 2D fused stage kernel (fast FP64 / mixed):
 * times `reps` launches of a step's first stage (from the current state into
 * scratch, so the state is not changed) for 1-4 work units per resident
 * warp and keeps the fastest for later steps of this context; *choice = the
 * units per warp chosen (0: the configuration has no fused 2D stage).  No
 * counterpart in the reference. */
int sifv_autotune(sifv_ctx_t* ctx, int reps, int* choice);
/* Set the work units per resident warp of the 2D fused stage kernel (1-4)
 * without timing; SIFV_ERR_BAD_ARG outside 1-4.  Every choice computes each
 * cell with the same arithmetic. */
int sifv_set_work_units(sifv_ctx_t* ctx, int unitsPerWarp);

/* ---- domain decomposition (one rank per GPU) -------------------------- */
/* The halo exchange and reductions of a context whose mesh has
 * SIFV_BC_EXCHANGE faces: HaloExchange (src/HaloExchange.cpp:387-465), the
 * MPI_Allreduce of the time step (src/RKTimeStepping.cpp:125-159) and of the
 * pressure solvers' residual (src/JacobiPressureSolver.cpp:99-100,
 * src/GaussSeidelPressureSolver.cpp:92-93), supplied by the caller (NCCL,
 * MPI, or host copies).  The library calls them while it queues a step on
 * its stream:
 *   exchange(user, fields, nfields, stream): fields are nfields arrays of
 *     the context's extended grid (device arrays; host arrays for a CPU
 *     backend).  For every SIFV_BC_EXCHANGE face, send the nGhost layers of
 *     cells next to the face to the neighbour across it and receive the
 *     neighbour's into this context's nGhost ghost layers of that face,
 *     ordered after the work already on `stream` and before the work queued
 *     after the call.  Every rank asks for the same fields in the same order:
 *     at each stage start the conservative state (rho, rhoU, [rhoV], [rhoW],
 *     rhoE, alphaRho and alpha of each phase, then sigma with IGR or in the
 *     semi-implicit step); in the semi-implicit step the primitives after the
 *     star update and after the correction (rho, velU, [velV], [velW], pres,
 *     sigma, alphaRho, alpha); one scalar (sigma after every IGR sweep, the
 *     pressure iterate before every Jacobi / Gauss-Seidel iteration and the
 *     solution after the solve).
 *   allreduce_min(user, value, stream): replace the non-negative double at
 *     `value` (device address; host for a CPU backend) by its minimum over
 *     all ranks, ordered the same way (the time step).
 *   allreduce_max(user, value, stream): the same with the maximum (the
 *     pressure solvers' residual, once per iteration).
 * Each returns 0 on success; a non-zero return ends the step with
 * SIFV_ERR_CUDA.  Supported on a decomposed mesh: the explicit step
 * (reference order in 1-3D, with or without IGR; the fast / mixed 2D step)
 * and the reference-ordered semi-implicit step (with or without IGR; Jacobi
 * or Gauss-Seidel pressure solve, each rank sweeping its own cells in the
 * reference's order as its MPI ranks do).  Viscous / capillary terms,
 * immersed boundaries, the mixed-precision semi-implicit step and the PCG
 * solver are rejected with SIFV_ERR_UNSUPPORTED.  A NULL comm clears the
 * hooks.  allreduce_max may be NULL for an explicit step. */
typedef struct sifv_comm {
    int (*exchange)(void* user, double* const* fields, int nfields, void* stream);
    int (*allreduce_min)(void* user, double* value, void* stream);
    void* user;
    int (*allreduce_max)(void* user, double* value, void* stream);
} sifv_comm_t;
int sifv_set_comm(sifv_ctx_t* ctx, const sifv_comm_t* comm);

/* Measured FP64 fused multiply-add throughput of the current device (TFLOP/s,
 * 2 flops per FMA, best of `reps` timed launches of a resident grid): the
 * FP64 co-bound the benchmark reports beside the HBM roofline of the fused
 * stage kernels.  No counterpart in the reference. */
int sifv_fp64_peak_probe(int reps, double* tflops);

/* ---- allocation-free pressure solve ----------------------------------- */
/* Sizes of the static device scratch behind sifv_pressure_solve_noalloc
 * (reserved on every GPU that loads the library, about 32 MB). */
#define SIFV_NOALLOC_MAX_CELLS 2097152   /* cells per solve, ghosts included */
#define SIFV_NOALLOC_MAX_ITERS 4096      /* maxIter */
#define SIFV_NOALLOC_MAX_AXIS  8192      /* cells along one axis, ghosts included */

/* The Jacobi pressure solve of sifv_pressure_solve for callers that cannot
 * allocate device memory -- hosts whose GPU memory belongs to their own
 * pool allocator, or code that must not call cudaMalloc/cudaFree between
 * stream operations because those calls can synchronise the device.  It
 * needs no context and allocates nothing: the two Jacobi iterates, the
 * residual slots and the cell widths live in one file-scope static device
 * array (the sizes above).  This entry point has no counterpart in the
 * reference.
 *
 * rho, rhoc2, rhs and pressure are DEVICE arrays of the mesh's totalCells
 * (ghosts included, x fastest) on the current device; pressure holds the
 * initial guess and receives the solution in its interior cells (ghosts
 * untouched).  Work is queued on `stream` (NULL: the legacy default
 * stream).  Meshes or maxIter above the SIFV_NOALLOC_* limits are rejected
 * with SIFV_ERR_BAD_ARG.  The first call on a device (and the first after
 * a device reset, or under another context on that device) looks up the
 * static array's device address (cudaGetSymbolAddress) with that device
 * current and keeps it for later calls.  Each call waits on `stream` (cudaStreamSynchronize)
 * while it runs: it reads the convergence flag back to the host between
 * batches of iterations, and it returns once the solution is in `pressure`.
 * All calls on a device share the one array and find the previous call's
 * contents there (the call clears what must start at zero): calls that
 * overlap on the GPU race and must be serialised by the caller.
 * Errors: sifv_noalloc_last_error(). */
int sifv_pressure_solve_noalloc(const sifv_mesh_t* mesh, int dim, int nGhost, const double* rho,
                                const double* rhoc2, const double* rhs, double* pressure, double dt,
                                double tol, int maxIter, void* stream, int* iters);
const char* sifv_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* SIFV_H */
