// SifvCudaSolvers.hpp -- drop-in C++ adapters that put the CUDA time step
// behind the SemiImplicitFV host interfaces.
//
// Header-only; compile it together with the SemiImplicitFV headers
// (include/*.hpp of that project) and link libsifv_b200.so.  The classes
// keep the reference's constructor and step() signatures so a driver
// switches by changing one type:
//
//   ExplicitSolver      (include/ExplicitSolver.hpp:21-36)      -> CudaExplicitSolver
//   SemiImplicitSolver  (include/SemiImplicitSolver.hpp:22-46)  -> CudaSemiImplicitSolver
//   PressureSolver      (include/PressureSolver.hpp:13-41)      -> CudaJacobiPressureSolver,
//                                                                  CudaGaussSeidelPressureSolver
//
// Errors of the C ABI are rethrown as the reference's exception types
// (std::invalid_argument for configuration errors, std::runtime_error
// otherwise).  The CUDA path runs one rank on one GPU: a periodic axis is
// recognised from the halo (a single rank is its own neighbour on a
// periodic axis, src/MPIContext.cpp:138-140), and multi-rank halos are
// rejected.
#pragma once

#include <array>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "EquationOfState.hpp"
#include "HaloExchange.hpp"
#include "IGR.hpp"
#include "ImmersedBoundary.hpp"
#include "PressureSolver.hpp"
#include "RectilinearMesh.hpp"
#include "RiemannSolver.hpp"
#include "SimulationConfig.hpp"
#include "SolutionState.hpp"
#include "sifv.h"

namespace SemiImplicitFV {
namespace b200 {

// When the host's SolutionState is read and written.
enum class SyncPolicy {
    EveryStep,  // upload before and download after every step: exact drop-in semantics
    OnDemand    // state stays on the GPU between steps; call syncToHost / syncToDevice
};

inline void throwStatus(int st, const char* what) {
    if (st >= 0) return;
    std::string msg = std::string(what) + ": " + sifv_last_error(nullptr);
    if (st == SIFV_ERR_BAD_CONFIG) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

inline void throwStatus(int st, const sifv_ctx_t* ctx, const char* what) {
    if (st >= 0) return;
    std::string msg = std::string(what) + ": " + sifv_last_error(ctx);
    if (st == SIFV_ERR_BAD_CONFIG) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

// SimulationConfig + EOS + Riemann solver choice -> sifv_config_t.
inline sifv_config_t toSifvConfig(const SimulationConfig& c, const EquationOfState& eos,
                                  const RiemannSolver& riemann, int precision) {
    sifv_config_t s;
    sifv_config_defaults(&s);
    s.dim = c.dim;
    s.nGhost = c.nGhost;
    s.RKOrder = c.RKOrder;
    s.useIGR = c.useIGR ? 1 : 0;
    s.semiImplicit = c.semiImplicit ? 1 : 0;
    s.reconOrder = static_cast<int>(c.reconOrder);
    s.wenoEps = c.wenoEps;
    // the reference maps the solver by name (src/ExplicitSolver.cpp:31-34)
    const std::string name = riemann.name();
    s.riemannSolver = (name == "HLLC") ? SIFV_HLLC : (name == "Rusanov") ? SIFV_RUSANOV : SIFV_LF;
    // IdealGasEOS clamps p >= 1e-14 in toPrimitive, StiffenedGasEOS does not
    s.eosKind = (eos.name() == "IdealGas") ? SIFV_EOS_IDEAL : SIFV_EOS_STIFFENED;
    s.gamma = eos.gamma();
    s.pInf = eos.pInf();
    s.cfl = c.explicitParams.cfl;
    s.constDt = c.explicitParams.constDt;
    s.maxDt = c.explicitParams.maxDt;
    s.minDt = c.explicitParams.minDt;
    s.siCfl = c.semiImplicitParams.cfl;
    s.siMaxDt = c.semiImplicitParams.maxDt;
    s.siMinDt = c.semiImplicitParams.minDt;
    s.maxPressureIters = c.semiImplicitParams.maxPressureIters;
    s.pressureTol = c.semiImplicitParams.pressureTol;
    s.alphaCoeff = c.igrParams.alphaCoeff;
    s.IGRIters = c.igrParams.IGRIters;
    s.IGRWarmStartIters = c.igrParams.IGRWarmStartIters;
    s.nPhases = c.multiPhaseParams.nPhases;
    for (int p = 0; p < c.multiPhaseParams.nPhases && p < SIFV_MAX_PHASES; ++p) {
        s.phaseGamma[p] = c.multiPhaseParams.phases[p].gamma;
        s.phasePInf[p] = c.multiPhaseParams.phases[p].pInf;
    }
    s.alphaMin = c.multiPhaseParams.alphaMin;
    for (int d = 0; d < 3; ++d) {
        s.bfA[d] = c.bodyForceParams.a[d];
        s.bfB[d] = c.bodyForceParams.b[d];
        s.bfC[d] = c.bodyForceParams.c[d];
        s.bfD[d] = c.bodyForceParams.d[d];
    }
    s.precision = precision;
    s.mu = c.viscousParams.mu;
    if (c.viscousParams.phaseMu.size() > (size_t)SIFV_MAX_PHASES)
        throw std::invalid_argument("viscousParams.phaseMu has more than SIFV_MAX_PHASES entries");
    s.nPhaseMu = (int)c.viscousParams.phaseMu.size();
    for (int p = 0; p < s.nPhaseMu; ++p) s.phaseMu[p] = c.viscousParams.phaseMu[p];
    s.stSigma = c.surfaceTensionParams.sigma;
    s.stEpsGradAlpha = c.surfaceTensionParams.epsGradAlpha;
    return s;
}

// Node arrays + BCs of a RectilinearMesh (single rank).  A face whose
// halo neighbour is this rank itself is periodic.
struct MeshNodes {
    std::vector<double> x, y, z;
    sifv_mesh_t m{};
    MeshNodes(const RectilinearMesh& mesh, const HaloExchange* halo) {
        for (int i = 0; i <= mesh.nx(); ++i) x.push_back(mesh.nodeX(i));
        for (int j = 0; j <= mesh.ny(); ++j) y.push_back(mesh.nodeY(j));
        for (int k = 0; k <= mesh.nz(); ++k) z.push_back(mesh.nodeZ(k));
        m.nx = mesh.nx();
        m.ny = mesh.ny();
        m.nz = mesh.nz();
        m.xNodes = x.data();
        m.yNodes = y.data();
        m.zNodes = z.data();
        for (int f = 0; f < 6; ++f) {
            int bc = static_cast<int>(mesh.boundaryCondition(f));
            if (halo) {
                if (halo->mpi().size() > 1)
                    throw std::runtime_error("the CUDA step runs one rank per mesh (no multi-rank halos)");
                if (!halo->mpi().isPhysicalBoundary(f)) bc = SIFV_BC_PERIODIC;   // self-neighbour
            }
            m.bc[f] = bc;
        }
    }
};

// Field bundle of a SolutionState <-> device context.
inline void uploadState(sifv_ctx_t* ctx, const SolutionState& s, int dim, int nPhases) {
    auto put = [&](int id, const std::vector<double>& v) {
        if (!v.empty()) throwStatus(sifv_set_field(ctx, id, v.data(), 0), ctx, "sifv_set_field");
    };
    put(SIFV_F_RHO, s.rho); put(SIFV_F_RHOU, s.rhoU); put(SIFV_F_RHOE, s.rhoE);
    put(SIFV_F_VELU, s.velU); put(SIFV_F_PRES, s.pres); put(SIFV_F_SIGMA, s.sigma);
    if (dim >= 2) { put(SIFV_F_RHOV, s.rhoV); put(SIFV_F_VELV, s.velV); }
    if (dim >= 3) { put(SIFV_F_RHOW, s.rhoW); put(SIFV_F_VELW, s.velW); }
    for (int p = 0; p < nPhases; ++p) { put(SIFV_F_ALPHARHO(p), s.alphaRho[p]); put(SIFV_F_ALPHA(p), s.alpha[p]); }
}

inline void downloadState(sifv_ctx_t* ctx, SolutionState& s, int dim, int nPhases) {
    auto get = [&](int id, std::vector<double>& v) {
        if (!v.empty()) throwStatus(sifv_get_field(ctx, id, v.data(), 0), ctx, "sifv_get_field");
    };
    get(SIFV_F_RHO, s.rho); get(SIFV_F_RHOU, s.rhoU); get(SIFV_F_RHOE, s.rhoE);
    get(SIFV_F_VELU, s.velU); get(SIFV_F_PRES, s.pres); get(SIFV_F_SIGMA, s.sigma);
    if (dim >= 2) { get(SIFV_F_RHOV, s.rhoV); get(SIFV_F_VELV, s.velV); }
    if (dim >= 3) { get(SIFV_F_RHOW, s.rhoW); get(SIFV_F_VELW, s.velW); }
    for (int p = 0; p < nPhases; ++p) { get(SIFV_F_ALPHARHO(p), s.alphaRho[p]); get(SIFV_F_ALPHA(p), s.alpha[p]); }
}

// Common machinery of the two steppers: lazy context creation (the halo is
// attached after construction in the reference's drivers), sync policy.
class CudaStepperBase {
public:
    CudaStepperBase(std::shared_ptr<RiemannSolver> riemann, std::shared_ptr<EquationOfState> eos,
                    const SimulationConfig& config, int device, int precision, SyncPolicy sync)
        : riemann_(std::move(riemann)), eos_(std::move(eos)), device_(device), precision_(precision), sync_(sync) {
        config.validate();
    }
    virtual ~CudaStepperBase() { if (ctx_) sifv_destroy(ctx_); }
    CudaStepperBase(const CudaStepperBase&) = delete;
    CudaStepperBase& operator=(const CudaStepperBase&) = delete;

    void setHaloExchange(HaloExchange* halo) { halo_ = halo; }

    // OnDemand policy: move the state explicitly.
    void syncToHost(SolutionState& state) { downloadState(ctx_, state, dim_, nPhases_); }
    void syncToDevice(const SolutionState& state) { uploadState(ctx_, state, dim_, nPhases_); }

    RiemannSolver& riemannSolver() { return *riemann_; }
    const EquationOfState& eos() const { return *eos_; }
    sifv_ctx_t* context() { return ctx_; }

protected:
    double stepImpl(const SimulationConfig& config, const RectilinearMesh& mesh, SolutionState& state,
                    double targetDt) {
        if (!ctx_) {
            sifv_config_t c = toSifvConfig(config, *eos_, *riemann_, precision_);
            MeshNodes nodes(mesh, halo_);
            throwStatus(sifv_create(&c, &nodes.m, device_, &ctx_), "sifv_create");
            throwStatus(sifv_set_pressure_solver(ctx_, pressureKind_), ctx_, "sifv_set_pressure_solver");
            afterCreate();
            dim_ = config.dim;
            nPhases_ = config.multiPhaseParams.nPhases;
            uploadState(ctx_, state, dim_, nPhases_);
        } else if (sync_ == SyncPolicy::EveryStep) {
            uploadState(ctx_, state, dim_, nPhases_);
        }
        double dt = 0.0;
        int st = sifv_step(ctx_, config.step, config.time, targetDt, &dt);
        throwStatus(st, ctx_, "sifv_step");
        if (sync_ == SyncPolicy::EveryStep) downloadState(ctx_, state, dim_, nPhases_);
        return dt;
    }

    // set-up that needs the context (called once, right after it exists)
    virtual void afterCreate() {}

    std::shared_ptr<RiemannSolver> riemann_;
    std::shared_ptr<EquationOfState> eos_;
    HaloExchange* halo_ = nullptr;
    sifv_ctx_t* ctx_ = nullptr;
    int device_, precision_;
    int pressureKind_ = SIFV_PRESSURE_JACOBI;
    SyncPolicy sync_;
    int dim_ = 0, nPhases_ = 0;
};

// Drop-in for ImmersedBoundaryMethod (include/ImmersedBoundary.hpp:107-135)
// that also keeps its bodies: CudaExplicitSolver::setIBM classifies the same
// cells on the GPU side through the bodies' own IBBody queries, so bodies of
// any shape carry over.  Use it where the driver declares its
// ImmersedBoundaryMethod; addBody / classifyCells / cellType work unchanged.
class CudaImmersedBoundary : public ImmersedBoundaryMethod {
public:
    void addBody(std::shared_ptr<IBBody> body) {
        ImmersedBoundaryMethod::addBody(body);
        cudaBodies_.push_back(std::move(body));
    }
    const std::vector<std::shared_ptr<IBBody>>& bodies() const { return cudaBodies_; }

private:
    std::vector<std::shared_ptr<IBBody>> cudaBodies_;
};

// Drop-in for ExplicitSolver (include/ExplicitSolver.hpp:21-36).
class CudaExplicitSolver : public CudaStepperBase {
public:
    CudaExplicitSolver(const RectilinearMesh& /*mesh*/, std::shared_ptr<RiemannSolver> riemannSolver,
                       std::shared_ptr<EquationOfState> eos, std::shared_ptr<IGRSolver> /*igrSolver*/,
                       const SimulationConfig& config, int device = 0, int precision = SIFV_PREC_FP64,
                       SyncPolicy sync = SyncPolicy::EveryStep)
        : CudaStepperBase(std::move(riemannSolver), std::move(eos), config, device, precision, sync) {
        if (config.semiImplicit) throw std::invalid_argument("CudaExplicitSolver needs semiImplicit == false");
    }

    double step(const SimulationConfig& config, const RectilinearMesh& mesh, SolutionState& state,
                double targetDt = -1.0) {
        return stepImpl(config, mesh, state, targetDt);
    }

    // ExplicitSolver::setIBM (include/ExplicitSolver.hpp:39-42); nullptr detaches.
    void setIBM(CudaImmersedBoundary* ibm) {
        ibm_ = ibm;
        if (ctx_) attachIBM();
    }

protected:
    void afterCreate() override {
        if (ibm_) attachIBM();
    }

private:
    void attachIBM() {
        if (!ibm_) {
            throwStatus(sifv_set_immersed_shapes(ctx_, 0, nullptr, nullptr), ctx_, "sifv_set_immersed_shapes");
            return;
        }
        const auto& bodies = ibm_->bodies();
        std::vector<int> wall;
        for (const auto& b : bodies)
            wall.push_back(b->wallType() == IBBody::WallType::Slip ? SIFV_IB_SLIP : SIFV_IB_NOSLIP);
        sifv_ib_shapes_t s{};
        s.user = ibm_;
        s.signedDistance = [](void* u, int b, double x, double y, double z) {
            return static_cast<CudaImmersedBoundary*>(u)->bodies()[b]->signedDistance(x, y, z);
        };
        s.closestPoint = [](void* u, int b, double x, double y, double z, double o[3]) {
            auto p = static_cast<CudaImmersedBoundary*>(u)->bodies()[b]->closestPoint(x, y, z);
            o[0] = p[0]; o[1] = p[1]; o[2] = p[2];
        };
        s.outwardNormal = [](void* u, int b, double x, double y, double z, double o[3]) {
            auto p = static_cast<CudaImmersedBoundary*>(u)->bodies()[b]->outwardNormal(x, y, z);
            o[0] = p[0]; o[1] = p[1]; o[2] = p[2];
        };
        throwStatus(sifv_set_immersed_shapes(ctx_, (int)bodies.size(), wall.data(), &s), ctx_,
                    "sifv_set_immersed_shapes");
    }

    CudaImmersedBoundary* ibm_ = nullptr;
};

// Drop-in for SemiImplicitSolver (include/SemiImplicitSolver.hpp:22-46) with
// the pressure solve on the GPU: Jacobi or Gauss-Seidel, whichever
// PressureSolver the constructor receives (by its name()).
class CudaSemiImplicitSolver : public CudaStepperBase {
public:
    CudaSemiImplicitSolver(const RectilinearMesh& /*mesh*/, std::shared_ptr<RiemannSolver> riemannSolver,
                           std::shared_ptr<PressureSolver> pressureSolver, std::shared_ptr<EquationOfState> eos,
                           std::shared_ptr<IGRSolver> /*igrSolver*/, const SimulationConfig& config, int device = 0,
                           SyncPolicy sync = SyncPolicy::EveryStep)
        : CudaStepperBase(std::move(riemannSolver), std::move(eos), config, device, SIFV_PREC_FP64, sync),
          pressure_(std::move(pressureSolver)) {
        if (!config.semiImplicit) throw std::invalid_argument("CudaSemiImplicitSolver needs semiImplicit == true");
        const std::string kind = pressure_ ? pressure_->name() : std::string("Jacobi");
        if (kind == "GaussSeidel") pressureKind_ = SIFV_PRESSURE_GAUSS_SEIDEL;
        else if (kind == "PCG+MG" || kind == "HyprePCG+PFMG") pressureKind_ = SIFV_PRESSURE_PCG_MG;
        else if (kind != "Jacobi")
            throw std::invalid_argument(
                "the CUDA semi-implicit step solves the pressure with Jacobi, GaussSeidel or PCG+MG");
    }

    double step(const SimulationConfig& config, const RectilinearMesh& mesh, SolutionState& state,
                double targetDt = -1.0) {
        double dt = stepImpl(config, mesh, state, targetDt);
        sifv_last_pressure_iterations(ctx_, &lastIters_);
        return dt;
    }

    int lastPressureIterations() const { return lastIters_; }
    PressureSolver& pressureSolver() { return *pressure_; }

private:
    std::shared_ptr<PressureSolver> pressure_;
    int lastIters_ = 0;
};

// Drop-in PressureSolver (include/PressureSolver.hpp:13-41) on the GPU: the
// Jacobi iteration of src/JacobiPressureSolver.cpp, the Gauss-Seidel sweeps
// of src/GaussSeidelPressureSolver.cpp, or conjugate gradients with a
// multigrid V-cycle in place of HyprePressureSolver (PCG+PFMG).  Host arrays in, host arrays out; the
// device context is cached per mesh.
class CudaPressureSolverPlugin : public PressureSolver {
public:
    CudaPressureSolverPlugin(int kind, int device) : kind_(kind), device_(device) {}
    ~CudaPressureSolverPlugin() override { if (ctx_) sifv_destroy(ctx_); }
    CudaPressureSolverPlugin(const CudaPressureSolverPlugin&) = delete;
    CudaPressureSolverPlugin& operator=(const CudaPressureSolverPlugin&) = delete;

    int solve(const RectilinearMesh& mesh, const std::vector<double>& rho, const std::vector<double>& rhoc2,
              const std::vector<double>& rhs, std::vector<double>& pressure, double dt, double tolerance,
              int maxIter) override {
        return run(mesh, nullptr, rho, rhoc2, rhs, pressure, dt, tolerance, maxIter);
    }

    int solve(const RectilinearMesh& mesh, const std::vector<double>& rho, const std::vector<double>& rhoc2,
              const std::vector<double>& rhs, std::vector<double>& pressure, double dt, double tolerance,
              int maxIter, HaloExchange& halo) override {
        return run(mesh, &halo, rho, rhoc2, rhs, pressure, dt, tolerance, maxIter);
    }

    std::string name() const override {
        return kind_ == SIFV_PRESSURE_GAUSS_SEIDEL ? "GaussSeidel" : kind_ == SIFV_PRESSURE_PCG_MG ? "PCG+MG" : "Jacobi";
    }

private:
    int run(const RectilinearMesh& mesh, const HaloExchange* halo, const std::vector<double>& rho,
            const std::vector<double>& rhoc2, const std::vector<double>& rhs, std::vector<double>& pressure,
            double dt, double tolerance, int maxIter) {
        const int key[4] = {mesh.nx(), mesh.ny(), mesh.nz(), mesh.nGhost()};
        if (!ctx_ || key[0] != key_[0] || key[1] != key_[1] || key[2] != key_[2] || key[3] != key_[3]) {
            if (ctx_) sifv_destroy(ctx_);
            ctx_ = nullptr;
            sifv_config_t c;
            sifv_config_defaults(&c);
            c.dim = mesh.dim();
            c.nGhost = mesh.nGhost();
            c.reconOrder = (mesh.nGhost() >= 3) ? SIFV_WENO5 : (mesh.nGhost() == 2) ? SIFV_WENO3 : SIFV_WENO1;
            c.semiImplicit = 1;
            c.maxPressureIters = maxIter;
            MeshNodes nodes(mesh, halo);
            throwStatus(sifv_create(&c, &nodes.m, device_, &ctx_), "sifv_create");
            throwStatus(sifv_set_pressure_solver(ctx_, kind_), ctx_, "sifv_set_pressure_solver");
            for (int q = 0; q < 4; ++q) key_[q] = key[q];
        }
        int iters = 0;
        int st = sifv_pressure_solve(ctx_, rho.data(), rhoc2.data(), rhs.data(), pressure.data(), dt, tolerance,
                                     maxIter, 0, &iters);
        throwStatus(st, ctx_, "sifv_pressure_solve");
        return iters;
    }

    int kind_, device_;
    sifv_ctx_t* ctx_ = nullptr;
    int key_[4] = {-1, -1, -1, -1};
};

class CudaJacobiPressureSolver : public CudaPressureSolverPlugin {
public:
    explicit CudaJacobiPressureSolver(int device = 0) : CudaPressureSolverPlugin(SIFV_PRESSURE_JACOBI, device) {}
};

class CudaGaussSeidelPressureSolver : public CudaPressureSolverPlugin {
public:
    explicit CudaGaussSeidelPressureSolver(int device = 0)
        : CudaPressureSolverPlugin(SIFV_PRESSURE_GAUSS_SEIDEL, device) {}
};

// In place of HyprePressureSolver (include/HyprePressureSolver.hpp), which
// needs Hypre: the same system, Neumann faces on physical boundaries, the
// same two-norm relative-residual stopping rule; returns the CG iterations.
class CudaPcgMgPressureSolver : public CudaPressureSolverPlugin {
public:
    explicit CudaPcgMgPressureSolver(int device = 0) : CudaPressureSolverPlugin(SIFV_PRESSURE_PCG_MG, device) {}
};

}  // namespace b200
}  // namespace SemiImplicitFV
