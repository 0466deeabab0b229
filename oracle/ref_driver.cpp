// ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C API (prefix sifvr_) over the UNMODIFIED SemiImplicitFV reference
// classes, compiled in place from the reference's src/ against the
// single-rank MPI shim (oracle/mpi_shim).  It mirrors include/sifv.h so that
// the tests can drive the reference, the C restatement (sifvo_) and the CUDA
// library (sifv_) with the same calls.  Nothing here is part of the product.
//
// The set-up follows the reference's own drivers: Runtime::createUniformMesh
// (src/Runtime.cpp:39-119) builds an MPIContext with `periods` and a
// RectilinearMesh from the local node arrays; Runtime::setBoundaryCondition
// (src/Runtime.cpp:123-127) sets a face BC only on physical boundaries;
// Runtime::attachSolver (src/Runtime.cpp:131-139) attaches a HaloExchange.
#include <mpi.h>

#include "ExplicitSolver.hpp"
#include "GaussSeidelPressureSolver.hpp"
#include "HLLCSolver.hpp"
#include "HaloExchange.hpp"
#include "IGR.hpp"
#include "IdealGasEOS.hpp"
#include "JacobiPressureSolver.hpp"
#include "LFSolver.hpp"
#include "MPIContext.hpp"
#include "MixtureEOS.hpp"
#include "RKTimeStepping.hpp"
#include "RectilinearMesh.hpp"
#include "RusanovSolver.hpp"
#include "SemiImplicitSolver.hpp"
#include "SimulationConfig.hpp"
#include "SolutionState.hpp"
#include "StiffenedGasEOS.hpp"
#include "ImmersedBoundary.hpp"
#include "Runtime.hpp"
#include "VTKSession.hpp"

#include "sifv.h"

#include <array>
#include <chrono>
#include <cstring>
#include <exception>
#include <mutex>
#include <memory>
#include <string>
#include <vector>

using namespace SemiImplicitFV;

struct sifvr_ctx {
    SimulationConfig config;
    std::unique_ptr<MPIContext> mpi;
    std::unique_ptr<RectilinearMesh> mesh;
    std::unique_ptr<HaloExchange> halo;
    SolutionState state;
    std::shared_ptr<EquationOfState> eos;
    std::shared_ptr<RiemannSolver> riemann;
    std::shared_ptr<IGRSolver> igr;
    std::shared_ptr<PressureSolver> psolver;
    std::unique_ptr<ExplicitSolver> expl;
    std::unique_ptr<SemiImplicitSolver> semi;
    std::string err;
    int lastIters = 0;
    std::unique_ptr<ImmersedBoundaryMethod> ibm;
};

static thread_local std::string g_err;

static std::vector<double> nodesOrUnit(const double* p, int n) {
    if (!p) return {0.0, 1.0};
    return std::vector<double>(p, p + n + 1);
}

static SimulationConfig toConfig(const sifv_config_t* c) {
    SimulationConfig s;
    s.dim = c->dim;
    s.nGhost = c->nGhost;
    s.RKOrder = c->RKOrder;
    s.useIGR = c->useIGR != 0;
    s.semiImplicit = c->semiImplicit != 0;
    s.reconOrder = static_cast<ReconstructionOrder>(c->reconOrder);
    s.wenoEps = c->wenoEps;
    s.explicitParams.cfl = c->cfl;
    s.explicitParams.constDt = c->constDt;
    s.explicitParams.maxDt = c->maxDt;
    s.explicitParams.minDt = c->minDt;
    s.semiImplicitParams.cfl = c->siCfl;
    s.semiImplicitParams.maxDt = c->siMaxDt;
    s.semiImplicitParams.minDt = c->siMinDt;
    s.semiImplicitParams.maxPressureIters = c->maxPressureIters;
    s.semiImplicitParams.pressureTol = c->pressureTol;
    s.igrParams.alphaCoeff = c->alphaCoeff;
    s.igrParams.IGRIters = c->IGRIters;
    s.igrParams.IGRWarmStartIters = c->IGRWarmStartIters;
    s.multiPhaseParams.nPhases = c->nPhases;
    s.multiPhaseParams.phases.clear();
    for (int p = 0; p < c->nPhases; ++p)
        s.multiPhaseParams.phases.push_back({c->phaseGamma[p], c->phasePInf[p]});
    s.multiPhaseParams.alphaMin = c->alphaMin;
    for (int d = 0; d < 3; ++d) {
        s.bodyForceParams.a[d] = c->bfA[d];
        s.bodyForceParams.b[d] = c->bfB[d];
        s.bodyForceParams.c[d] = c->bfC[d];
        s.bodyForceParams.d[d] = c->bfD[d];
    }
    s.viscousParams.mu = c->mu;
    s.viscousParams.phaseMu.assign(c->phaseMu, c->phaseMu + c->nPhaseMu);
    s.surfaceTensionParams.sigma = c->stSigma;
    s.surfaceTensionParams.epsGradAlpha = c->stEpsGradAlpha;
    return s;
}

static std::vector<double>* fieldVec(sifvr_ctx* ctx, int field) {
    SolutionState& s = ctx->state;
    switch (field) {
        case SIFV_F_RHO: return &s.rho;
        case SIFV_F_RHOU: return &s.rhoU;
        case SIFV_F_RHOV: return &s.rhoV;
        case SIFV_F_RHOW: return &s.rhoW;
        case SIFV_F_RHOE: return &s.rhoE;
        case SIFV_F_VELU: return &s.velU;
        case SIFV_F_VELV: return &s.velV;
        case SIFV_F_VELW: return &s.velW;
        case SIFV_F_PRES: return &s.pres;
        case SIFV_F_SIGMA: return &s.sigma;
        default: break;
    }
    if (field >= 16 && field < 16 + static_cast<int>(s.alphaRho.size())) return &s.alphaRho[field - 16];
    if (field >= 32 && field < 32 + static_cast<int>(s.alpha.size())) return &s.alpha[field - 32];
    return nullptr;
}

extern "C" {

const char* sifvr_last_error(const sifvr_ctx* ctx) {
    return ctx ? ctx->err.c_str() : g_err.c_str();
}

// A context on a process grid of procsPerDir ranks per axis (0: MPI_Dims_create
// chooses), the third argument of MPIContext::create (src/MPIContext.cpp:80-120).
static int create_on_grid(const sifv_config_t* cfg, const sifv_mesh_t* m, const std::array<int, 3>& procs,
                          sifvr_ctx** out) {
    *out = nullptr;
    try {
        int mpiInit = 0;
        MPI_Initialized(&mpiInit);
        if (!mpiInit) { int argc = 0; char** argv = nullptr; MPI_Init(&argc, &argv); }
        auto ctx = std::make_unique<sifvr_ctx>();
        ctx->config = toConfig(cfg);
        ctx->config.validate();
        const SimulationConfig& config = ctx->config;
        std::vector<double> xn = nodesOrUnit(m->xNodes, m->nx);
        std::vector<double> yn = (config.dim >= 2) ? nodesOrUnit(m->yNodes, m->ny) : std::vector<double>{0.0, 1.0};
        std::vector<double> zn = (config.dim >= 3) ? nodesOrUnit(m->zNodes, m->nz) : std::vector<double>{0.0, 1.0};
        int gnx = static_cast<int>(xn.size()) - 1, gny = static_cast<int>(yn.size()) - 1,
            gnz = static_cast<int>(zn.size()) - 1;
        std::array<int, 3> periods = {0, 0, 0};
        for (int d = 0; d < 3; ++d)
            periods[d] = (m->bc[2 * d] == SIFV_BC_PERIODIC && m->bc[2 * d + 1] == SIFV_BC_PERIODIC) ? 1 : 0;
        ctx->mpi = std::make_unique<MPIContext>(
            MPIContext::create(gnx, gny, gnz, xn, yn, zn, config.dim, periods, procs));
        ctx->mesh = std::make_unique<RectilinearMesh>(config, ctx->mpi->localXNodes(),
                                                      ctx->mpi->localYNodes(), ctx->mpi->localZNodes());
        for (int f = 0; f < 6; ++f)
            if (ctx->mpi->isPhysicalBoundary(f))
                ctx->mesh->setBoundaryCondition(f, static_cast<BoundaryCondition>(m->bc[f]));
        ctx->state.allocate(ctx->mesh->totalCells(), config);
        if (cfg->eosKind == SIFV_EOS_STIFFENED)
            ctx->eos = std::make_shared<StiffenedGasEOS>(cfg->gamma, cfg->pInf, 287.0, config);
        else
            ctx->eos = std::make_shared<IdealGasEOS>(cfg->gamma, 287.0, config);
        switch (cfg->riemannSolver) {
            case SIFV_HLLC: ctx->riemann = std::make_shared<HLLCSolver>(ctx->eos, config); break;
            case SIFV_RUSANOV: ctx->riemann = std::make_shared<RusanovSolver>(ctx->eos, config); break;
            default: ctx->riemann = std::make_shared<LFSolver>(ctx->eos, config); break;
        }
        if (config.useIGR) ctx->igr = std::make_shared<IGRSolver>(config.igrParams);
        ctx->psolver = std::make_shared<JacobiPressureSolver>();
        ctx->halo = std::make_unique<HaloExchange>(*ctx->mpi, *ctx->mesh);
        if (config.semiImplicit) {
            ctx->semi = std::make_unique<SemiImplicitSolver>(*ctx->mesh, ctx->riemann, ctx->psolver,
                                                             ctx->eos, ctx->igr, config);
            ctx->semi->setHaloExchange(ctx->halo.get());
        } else {
            ctx->expl = std::make_unique<ExplicitSolver>(*ctx->mesh, ctx->riemann, ctx->eos, ctx->igr, config);
            ctx->expl->setHaloExchange(ctx->halo.get());
        }
        *out = ctx.release();
        return SIFV_OK;
    } catch (const std::exception& e) {
        g_err = e.what();
        return SIFV_ERR_BAD_CONFIG;
    }
}

int sifvr_create(const sifv_config_t* cfg, const sifv_mesh_t* m, int /*device*/, sifvr_ctx** out) {
    return create_on_grid(cfg, m, {0, 0, 0}, out);
}

// Swap the pressure solver of a semi-implicit context: 0 Jacobi, 1 Gauss-Seidel.
int sifvr_set_pressure_solver(sifvr_ctx* ctx, int kind) {
    if (!ctx->semi) return SIFV_ERR_BAD_ARG;
    if (kind == 1) ctx->psolver = std::make_shared<GaussSeidelPressureSolver>();
    else ctx->psolver = std::make_shared<JacobiPressureSolver>();
    ctx->semi = std::make_unique<SemiImplicitSolver>(*ctx->mesh, ctx->riemann, ctx->psolver, ctx->eos,
                                                     ctx->igr, ctx->config);
    ctx->semi->setHaloExchange(ctx->halo.get());
    return SIFV_OK;
}

int sifvr_destroy(sifvr_ctx* ctx) { delete ctx; return SIFV_OK; }

int sifvr_extents(const sifvr_ctx* ctx, int* nx, int* ny, int* nz) {
    *nx = ctx->mesh->nxTotal(); *ny = ctx->mesh->nyTotal(); *nz = ctx->mesh->nzTotal();
    return SIFV_OK;
}

size_t sifvr_total_cells(const sifvr_ctx* ctx) { return ctx->mesh->totalCells(); }

int sifvr_set_field(sifvr_ctx* ctx, int field, const double* src, int) {
    std::vector<double>* v = fieldVec(ctx, field);
    if (!v || v->empty()) { ctx->err = "field not allocated"; return SIFV_ERR_BAD_ARG; }
    std::memcpy(v->data(), src, v->size() * sizeof(double));
    return SIFV_OK;
}

int sifvr_get_field(sifvr_ctx* ctx, int field, double* dst, int) {
    std::vector<double>* v = fieldVec(ctx, field);
    if (!v || v->empty()) { ctx->err = "field not allocated"; return SIFV_ERR_BAD_ARG; }
    std::memcpy(dst, v->data(), v->size() * sizeof(double));
    return SIFV_OK;
}

int sifvr_step(sifvr_ctx* ctx, int step, double time, double targetDt, double* dtOut) {
    try {
        ctx->config.step = step;
        ctx->config.time = time;
        double dt;
        if (ctx->semi) {
            dt = ctx->semi->step(ctx->config, *ctx->mesh, ctx->state, targetDt);
            ctx->lastIters = ctx->semi->lastPressureIterations();
        } else {
            dt = ctx->expl->step(ctx->config, *ctx->mesh, ctx->state, targetDt);
        }
        if (dtOut) *dtOut = dt;
        return SIFV_OK;
    } catch (const std::exception& e) {
        ctx->err = e.what();
        return SIFV_ERR_BAD_ARG;
    }
}

int sifvr_last_pressure_iterations(const sifvr_ctx* ctx, int* iters) {
    *iters = ctx->lastIters;
    return SIFV_OK;
}

int sifvr_pressure_solve(sifvr_ctx* ctx, const double* rho, const double* rhoc2, const double* rhs,
                         double* pressure, double dt, double tol, int maxIter, int, int* iters) {
    std::size_t n = ctx->mesh->totalCells();
    std::vector<double> vr(rho, rho + n), vc(rhoc2, rhoc2 + n), vh(rhs, rhs + n), vp(pressure, pressure + n);
    *iters = ctx->psolver->solve(*ctx->mesh, vr, vc, vh, vp, dt, tol, maxIter, *ctx->halo);
    std::memcpy(pressure, vp.data(), n * sizeof(double));
    return SIFV_OK;
}

int sifvr_acoustic_dt(sifvr_ctx* ctx, double cfl, double maxDt, double* dt) {
    *dt = computeAcousticTimeStep(*ctx->mesh, ctx->state, *ctx->eos, ctx->config, cfl, maxDt,
                                  ctx->mpi->comm());
    return SIFV_OK;
}

int sifvr_advective_dt(sifvr_ctx* ctx, double cfl, double maxDt, double* dt) {
    *dt = computeAdvectiveTimeStep(*ctx->mesh, ctx->state, cfl, maxDt, ctx->mpi->comm());
    return SIFV_OK;
}

int sifvr_convert_cons_to_prim(sifvr_ctx* ctx) {
    if (ctx->config.isMultiPhase())
        MixtureEOS::convertConservativeToPrimitive(*ctx->mesh, ctx->state, ctx->config.multiPhaseParams);
    else
        ctx->state.convertConservativeToPrimitiveVariables(*ctx->mesh, ctx->eos);
    return SIFV_OK;
}

int sifvr_apply_bc(sifvr_ctx* ctx) {
    ctx->mesh->applyBoundaryConditions(ctx->state, VarSet::PRIM, *ctx->halo);
    return SIFV_OK;
}

// IGRSolver::solveEntropicPressure with the reference's own gradient
// assembly (ExplicitSolver::computeVelocityGradients, src/ExplicitSolver.cpp:215-267).
int sifvr_igr_solve(sifvr_ctx* ctx, int step) {
    if (!ctx->igr) { ctx->err = "useIGR is off"; return SIFV_ERR_BAD_ARG; }
    const RectilinearMesh& mesh = *ctx->mesh;
    const SolutionState& state = ctx->state;
    int dim = mesh.dim();
    std::vector<GradientTensor> gradU(mesh.totalCells());
    for (int k = 0; k < mesh.nz(); ++k)
        for (int j = 0; j < mesh.ny(); ++j)
            for (int i = 0; i < mesh.nx(); ++i) {
                std::size_t idx = mesh.index(i, j, k);
                std::size_t xm = mesh.index(i - 1, j, k), xp = mesh.index(i + 1, j, k);
                std::array<double, 3> u_xm = {state.velU[xm], (dim >= 2) ? state.velV[xm] : 0.0,
                                              (dim >= 3) ? state.velW[xm] : 0.0};
                std::array<double, 3> u_xp = {state.velU[xp], (dim >= 2) ? state.velV[xp] : 0.0,
                                              (dim >= 3) ? state.velW[xp] : 0.0};
                std::array<double, 3> u_ym, u_yp, u_zm, u_zp;
                double dyj, dzk;
                if (dim >= 2) {
                    std::size_t ym = mesh.index(i, j - 1, k), yp = mesh.index(i, j + 1, k);
                    u_ym = {state.velU[ym], state.velV[ym], (dim >= 3) ? state.velW[ym] : 0.0};
                    u_yp = {state.velU[yp], state.velV[yp], (dim >= 3) ? state.velW[yp] : 0.0};
                    dyj = mesh.dy(j);
                } else {
                    u_ym = u_yp = {state.velU[idx], 0.0, 0.0};
                    dyj = 1.0;
                }
                if (dim >= 3) {
                    std::size_t zm = mesh.index(i, j, k - 1), zp = mesh.index(i, j, k + 1);
                    u_zm = {state.velU[zm], state.velV[zm], state.velW[zm]};
                    u_zp = {state.velU[zp], state.velV[zp], state.velW[zp]};
                    dzk = mesh.dz(k);
                } else {
                    u_zm = u_zp = {state.velU[idx], (dim >= 2) ? state.velV[idx] : 0.0, 0.0};
                    dzk = 1.0;
                }
                gradU[idx] = IGRSolver::computeVelocityGradient(u_xm, u_xp, u_ym, u_yp, u_zm, u_zp,
                                                                mesh.dx(i), dyj, dzk, dim);
            }
    SimulationConfig cfg = ctx->config;
    cfg.step = step;
    ctx->igr->solveEntropicPressure(cfg, mesh, ctx->state, gradU, *ctx->halo);
    return SIFV_OK;
}

// The reference's own runTimeLoop (src/RKTimeStepping.cpp:241-356) with its
// VTKSession (src/VTKSession.cpp) over this context's solver, starting at
// t = 0, step 0.  The Runtime only provides the MPI context VTKSession
// reads (global sizes, this rank's extent); the mesh written is the
// context's own.  *stepsOut = SimulationConfig::step at exit.
int sifvr_reference_time_loop(sifvr_ctx* ctx, const char* dir, const char* base, double endTime, double outputInterval,
                        int printInterval, int* stepsOut) {
    try {
        int argc = 0;
        char** argv = nullptr;
        Runtime rt(argc, argv);
        const RectilinearMesh& m = *ctx->mesh;
        if (ctx->config.dim == 1) rt.createUniformMesh(ctx->config, m.nx(), 0.0, 1.0);
        else if (ctx->config.dim == 2) rt.createUniformMesh(ctx->config, m.nx(), 0.0, 1.0, m.ny(), 0.0, 1.0);
        else rt.createUniformMesh(ctx->config, m.nx(), 0.0, 1.0, m.ny(), 0.0, 1.0, m.nz(), 0.0, 1.0);
        VTKSession vtk(rt, base, m, ctx->config, dir);
        TimeLoopParams p;
        p.endTime = endTime;
        p.outputInterval = outputInterval;
        p.printInterval = printInterval;
        p.checkNaN = true;
        ctx->config.step = 0;
        ctx->config.time = 0.0;
        auto stepFn = [ctx](double targetDt) {
            if (ctx->semi) return ctx->semi->step(ctx->config, *ctx->mesh, ctx->state, targetDt);
            return ctx->expl->step(ctx->config, *ctx->mesh, ctx->state, targetDt);
        };
        runTimeLoop(rt, ctx->config, m, ctx->state, vtk, stepFn, p);
        if (stepsOut) *stepsOut = ctx->config.step;
        return SIFV_OK;
    } catch (const std::exception& e) {
        ctx->err = e.what();
        return SIFV_ERR_BAD_ARG;
    }
}

// ImmersedBoundaryMethod with the reference's own body classes, attached to
// the explicit solver as Runtime::attachIBM does (src/Runtime.cpp:143-146).
int sifvr_set_immersed_bodies(sifvr_ctx* ctx, const sifv_ib_body_t* b, int n) {
    try {
        if (n > 0 && !ctx->expl) {
            ctx->err = "the semi-implicit step has no immersed boundary";
            return SIFV_ERR_UNSUPPORTED;
        }
        if (ctx->expl) ctx->expl->setIBM(nullptr);
        ctx->ibm.reset();
        if (n == 0) return SIFV_OK;
        ctx->ibm = std::make_unique<ImmersedBoundaryMethod>();
        for (int q = 0; q < n; ++q) {
            const double* p = b[q].p;
            std::shared_ptr<IBBody> body;
            if (b[q].shape == SIFV_IB_CIRCLE) body = std::make_shared<IBCircle>(p[0], p[1], p[2]);
            else if (b[q].shape == SIFV_IB_RECTANGLE) body = std::make_shared<IBRectangle>(p[0], p[1], p[2], p[3]);
            else if (b[q].shape == SIFV_IB_CYLINDER) body = std::make_shared<IBCylinder>(p[0], p[1], p[2], b[q].axis);
            else body = std::make_shared<IBRectangularPrism>(p[0], p[1], p[2], p[3], p[4], p[5]);
            body->setWallType(b[q].wall == SIFV_IB_SLIP ? IBBody::WallType::Slip : IBBody::WallType::NoSlip);
            ctx->ibm->addBody(body);
        }
        ctx->ibm->classifyCells(*ctx->mesh);
        ctx->expl->setIBM(ctx->ibm.get());
        return SIFV_OK;
    } catch (const std::exception& e) {
        ctx->err = e.what();
        return SIFV_ERR_BAD_ARG;
    }
}

int sifvr_ib_cell_types(sifvr_ctx* ctx, unsigned char* types) {
    const std::size_t n = ctx->mesh->totalCells();
    for (std::size_t q = 0; q < n; ++q)
        types[q] = ctx->ibm ? static_cast<unsigned char>(ctx->ibm->cellType(q)) : 0;
    return SIFV_OK;
}

int sifvr_apply_ib_ghost_cells(sifvr_ctx* ctx) {
    if (ctx->ibm) ctx->ibm->applyGhostCells(*ctx->mesh, ctx->state, ctx->config.dim);
    return SIFV_OK;
}

// The reference's own solver decomposed over nranks MPI ranks (threads of
// this process through the MPI shim's sifv_mpi_shim_run), as an MPI launch
// of the reference's drivers would run it: MPIContext::create splits the
// global mesh (src/MPIContext.cpp:80-170), HaloExchange moves the ghost
// layers (src/HaloExchange.cpp:387-465) and dt / residuals are reduced over
// the ranks.  procsPerDir (may be null: MPI_Dims_create chooses) fixes the
// process grid, e.g. {1, 1, n} for slabs along z; pressureKind picks the
// semi-implicit pressure solver (0 Jacobi, 1 Gauss-Seidel).  Every rank copies the interior block of the global initial
// fields init[f] (ghosts included, x fastest; its own ghosts start at
// zero, as in the reference's drivers), takes `warmup` steps, then `steps`
// steps between two barriers, and copies its interior block back into
// out[f] (global arrays; may be null).  secondsOut = the timed steps' wall
// time, maximum over the ranks; dtsOut (warmup + steps values, may be
// null) = the time steps; itersOut (the same length, may be null) = the
// pressure iterations of each step's last stage; dimsOut = the process grid.
struct MpiRunArgs {
    const sifv_config_t* cfg;
    const sifv_mesh_t* mesh;
    std::array<int, 3> procs;
    int pressureKind;
    int nfields;
    const int* fieldIds;
    const double* const* init;
    double* const* out;
    int warmup, steps;
    double seconds;
    double* dts;
    int* iters;
    int dims[3];
    int status;
    std::mutex m;
    std::string err;
};

static void mpi_rank_main(void* user, int rank) {
    MpiRunArgs& A = *static_cast<MpiRunArgs*>(user);
    sifvr_ctx* ctx = nullptr;
    int st = create_on_grid(A.cfg, A.mesh, A.procs, &ctx);
    if (st == SIFV_OK && A.pressureKind != 0) st = sifvr_set_pressure_solver(ctx, A.pressureKind);
    if (st != SIFV_OK) {
        std::lock_guard<std::mutex> lock(A.m);
        A.status = st;
        A.err = g_err;
        return;   // every rank fails the same way (same configuration)
    }
    const int dim = ctx->config.dim, ng = ctx->config.nGhost;
    const std::array<int, 6> ext = ctx->mpi->localExtent();
    const int gng[3] = {ng, dim >= 2 ? ng : 0, dim >= 3 ? ng : 0};
    const long long gnx = A.mesh->nx + 2LL * gng[0];
    const long long gny = (dim >= 2 ? A.mesh->ny : 1) + 2LL * gng[1];
    const RectilinearMesh& m = *ctx->mesh;
    auto globalIndex = [&](int i, int j, int k) -> std::size_t {
        return static_cast<std::size_t>(((long long)(k + ext[4] + gng[2]) * gny + (j + ext[2] + gng[1])) * gnx +
                                        (i + ext[0] + gng[0]));
    };
    for (int f = 0; f < A.nfields; ++f) {
        std::vector<double>* v = fieldVec(ctx, A.fieldIds[f]);
        if (!v || v->empty() || !A.init || !A.init[f]) continue;
        std::fill(v->begin(), v->end(), 0.0);
        for (int k = 0; k < m.nz(); ++k)
            for (int j = 0; j < m.ny(); ++j)
                for (int i = 0; i < m.nx(); ++i) (*v)[m.index(i, j, k)] = A.init[f][globalIndex(i, j, k)];
    }
    double t = 0.0;
    int step = 0;
    auto one = [&]() {
        double dt = 0.0;
        if (sifvr_step(ctx, step, t, -1.0, &dt) != SIFV_OK) {
            std::lock_guard<std::mutex> lock(A.m);
            A.status = SIFV_ERR_BAD_ARG;
            A.err = ctx->err;
        }
        if (rank == 0 && A.dts) A.dts[step] = dt;
        if (rank == 0 && A.iters) A.iters[step] = ctx->lastIters;
        t += dt;
        ++step;
    };
    for (int q = 0; q < A.warmup; ++q) one();
    double token = 0.0;
    MPI_Allreduce(MPI_IN_PLACE, &token, 1, MPI_DOUBLE, MPI_MAX, MPI_COMM_WORLD);
    auto t0 = std::chrono::steady_clock::now();
    for (int q = 0; q < A.steps; ++q) one();
    MPI_Allreduce(MPI_IN_PLACE, &token, 1, MPI_DOUBLE, MPI_MAX, MPI_COMM_WORLD);
    double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    MPI_Allreduce(MPI_IN_PLACE, &sec, 1, MPI_DOUBLE, MPI_MAX, MPI_COMM_WORLD);
    for (int f = 0; f < A.nfields && A.out; ++f) {
        std::vector<double>* v = fieldVec(ctx, A.fieldIds[f]);
        if (!v || v->empty() || !A.out[f]) continue;
        for (int k = 0; k < m.nz(); ++k)
            for (int j = 0; j < m.ny(); ++j)
                for (int i = 0; i < m.nx(); ++i) A.out[f][globalIndex(i, j, k)] = (*v)[m.index(i, j, k)];
    }
    if (rank == 0) {
        A.seconds = sec;
        for (int d = 0; d < 3; ++d) A.dims[d] = ctx->mpi->dims()[d];
    }
    sifvr_destroy(ctx);
}

int sifvr_mpi_run(const sifv_config_t* cfg, const sifv_mesh_t* mesh, int nranks, const int* procsPerDir,
                  int pressureKind, int nfields, const int* fieldIds, const double* const* init, double* const* out,
                  int warmup, int steps, double* secondsOut, double* dtsOut, int* itersOut, int* dimsOut) {
    if (!cfg || !mesh || nranks < 1 || warmup < 0 || steps < 0) return SIFV_ERR_BAD_ARG;
    MpiRunArgs A;
    A.cfg = cfg;
    A.mesh = mesh;
    A.procs = {0, 0, 0};
    if (procsPerDir)
        for (int d = 0; d < 3; ++d) A.procs[d] = procsPerDir[d];
    A.pressureKind = pressureKind;
    A.nfields = nfields;
    A.fieldIds = fieldIds;
    A.init = init;
    A.out = out;
    A.warmup = warmup;
    A.steps = steps;
    A.seconds = 0.0;
    A.dts = dtsOut;
    A.iters = itersOut;
    A.dims[0] = A.dims[1] = A.dims[2] = 0;
    A.status = SIFV_OK;
    if (sifv_mpi_shim_run(nranks, mpi_rank_main, &A) != 0) return SIFV_ERR_BAD_ARG;
    if (A.status != SIFV_OK) {
        g_err = A.err;
        return A.status;
    }
    if (secondsOut) *secondsOut = A.seconds;
    if (dimsOut)
        for (int d = 0; d < 3; ++d) dimsOut[d] = A.dims[d];
    return SIFV_OK;
}

}  // extern "C"

