// adapter_selftest.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Drives the reference's own solver classes and the drop-in CUDA adapters
// (semiimplicitfv_b200/host/SifvCudaSolvers.hpp) side by side on the same
// problem, set up the way the reference's example drivers do, and reports
// the largest relative difference of the conserved fields.  Built against
// the reference headers by oracle/Makefile (target `adapter`); loaded by
// tests/test_gpu_adapter.py.
#include <mpi.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "ExplicitSolver.hpp"
#include "HLLCSolver.hpp"
#include "HaloExchange.hpp"
#include "IGR.hpp"
#include "ImmersedBoundary.hpp"
#include "IdealGasEOS.hpp"
#include "JacobiPressureSolver.hpp"
#include "GaussSeidelPressureSolver.hpp"
#include "MPIContext.hpp"
#include "RectilinearMesh.hpp"
#include "SemiImplicitSolver.hpp"
#include "SifvCudaSolvers.hpp"

using namespace SemiImplicitFV;

namespace {

std::vector<double> linspace(double a, double b, int n) {   // n cells -> n+1 nodes (src/Runtime.cpp:12-17)
    std::vector<double> v(n + 1);
    for (int i = 0; i <= n; ++i) v[i] = a + (b - a) * i / n;
    return v;
}

struct Setup {
    std::unique_ptr<MPIContext> mpi;
    std::unique_ptr<RectilinearMesh> mesh;
    std::unique_ptr<HaloExchange> halo;
};

Setup makeMesh(const SimulationConfig& cfg, int nx, int ny, int nz, std::array<int, 3> periods, BoundaryCondition bc) {
    int init = 0;
    MPI_Initialized(&init);
    if (!init) { int argc = 0; char** argv = nullptr; MPI_Init(&argc, &argv); }
    Setup s;
    std::vector<double> xn = linspace(0, 1, nx), yn = linspace(0, 1, ny), zn = linspace(0, 1, nz);
    if (cfg.dim < 2) yn = {0.0, 1.0};
    if (cfg.dim < 3) zn = {0.0, 1.0};
    s.mpi = std::make_unique<MPIContext>(MPIContext::create(nx, cfg.dim >= 2 ? ny : 1, cfg.dim >= 3 ? nz : 1, xn,
                                                            yn, zn, cfg.dim, periods));
    s.mesh = std::make_unique<RectilinearMesh>(cfg, s.mpi->localXNodes(), s.mpi->localYNodes(), s.mpi->localZNodes());
    for (int f = 0; f < 6; ++f)
        if (s.mpi->isPhysicalBoundary(f)) s.mesh->setBoundaryCondition(f, bc);
    s.halo = std::make_unique<HaloExchange>(*s.mpi, *s.mesh);
    return s;
}

double maxRel(const std::vector<double>& a, const std::vector<double>& b, const RectilinearMesh& m) {
    double d = 0.0, scale = 0.0;
    for (int k = 0; k < m.nz(); ++k)
        for (int j = 0; j < m.ny(); ++j)
            for (int i = 0; i < m.nx(); ++i) {
                std::size_t c = m.index(i, j, k);
                d = std::max(d, std::fabs(a[c] - b[c]));
                scale = std::max(scale, std::fabs(b[c]));
            }
    return scale > 0 ? d / scale : d;
}

// 2D four-quadrant Riemann IC (examples/2D_riemann/2D_riemann.cpp:24-76, 0.5323 states).
void riemannIC(const RectilinearMesh& mesh, SolutionState& st, const IdealGasEOS& eos) {
    for (int j = 0; j < mesh.ny(); ++j)
        for (int i = 0; i < mesh.nx(); ++i) {
            double x = mesh.cellCentroidX(i), y = mesh.cellCentroidY(j);
            PrimitiveState W;
            if (x >= 0.8 && y >= 0.8) { W.rho = 1.5; W.u = {0, 0, 0}; W.p = 1.5; }
            else if (x < 0.8 && y >= 0.8) { W.rho = 0.5323; W.u = {1.206, 0, 0}; W.p = 0.3; }
            else if (x < 0.8 && y < 0.8) { W.rho = 0.138; W.u = {1.206, 1.206, 0}; W.p = 0.029; }
            else { W.rho = 0.5323; W.u = {0, 1.206, 0}; W.p = 0.3; }
            std::size_t idx = mesh.index(i, j, 0);
            st.setPrimitiveState(idx, W);
            st.setConservativeState(idx, eos.toConservative(W));
        }
}

// 3D acoustic pulse: rho 1, u (0.1, 0.05, 0), p = 1 + 1e-3 exp(-r^2/0.01).
void pulseIC(const RectilinearMesh& mesh, SolutionState& st, const IdealGasEOS& eos) {
    for (int k = 0; k < mesh.nz(); ++k)
        for (int j = 0; j < mesh.ny(); ++j)
            for (int i = 0; i < mesh.nx(); ++i) {
                double x = mesh.cellCentroidX(i) - 0.5, y = mesh.cellCentroidY(j) - 0.5, z = mesh.cellCentroidZ(k) - 0.5;
                PrimitiveState W;
                W.rho = 1.0;
                W.u = {0.1, 0.05, 0.0};
                W.p = 1.0 + 1e-3 * std::exp(-(x * x + y * y + z * z) / 0.01);
                std::size_t idx = mesh.index(i, j, k);
                st.setPrimitiveState(idx, W);
                st.setConservativeState(idx, eos.toConservative(W));
            }
}

double explicitCase(int n, int nsteps, int precision, int bcCode, double mu) {
    try {
        SimulationConfig cfg;
        cfg.dim = 2; cfg.nGhost = 3; cfg.RKOrder = 3; cfg.reconOrder = ReconstructionOrder::WENO5;
        cfg.explicitParams.cfl = 0.6;
        cfg.viscousParams.mu = mu;
        cfg.validate();
        BoundaryCondition bc = static_cast<BoundaryCondition>(bcCode);
        std::array<int, 3> periods = {0, 0, 0};
        if (bc == BoundaryCondition::Periodic) periods = {1, 1, 0};
        Setup a = makeMesh(cfg, n, n, 1, periods, bc), b = makeMesh(cfg, n, n, 1, periods, bc);
        auto eos = std::make_shared<IdealGasEOS>(1.4, 287.0, cfg);
        auto riemann = std::make_shared<HLLCSolver>(eos, cfg);
        SolutionState sa, sb;
        sa.allocate(a.mesh->totalCells(), cfg);
        sb.allocate(b.mesh->totalCells(), cfg);
        riemannIC(*a.mesh, sa, *eos);
        riemannIC(*b.mesh, sb, *eos);
        ExplicitSolver ref(*a.mesh, riemann, eos, nullptr, cfg);
        ref.setHaloExchange(a.halo.get());
        b200::CudaExplicitSolver gpu(*b.mesh, riemann, eos, nullptr, cfg, 0, precision);
        gpu.setHaloExchange(b.halo.get());
        SimulationConfig ca = cfg, cb = cfg;
        for (int s = 0; s < nsteps; ++s) {
            double da = ref.step(ca, *a.mesh, sa, -1.0);
            double db = gpu.step(cb, *b.mesh, sb, -1.0);
            if (da != db && precision == SIFV_PREC_FP64) return 1.0;
            ca.time += da; ca.step++;
            cb.time += db; cb.step++;
        }
        double w = 0.0;
        w = std::max(w, maxRel(sb.rho, sa.rho, *a.mesh));
        w = std::max(w, maxRel(sb.rhoU, sa.rhoU, *a.mesh));
        w = std::max(w, maxRel(sb.rhoV, sa.rhoV, *a.mesh));
        w = std::max(w, maxRel(sb.rhoE, sa.rhoE, *a.mesh));
        return w;
    } catch (...) {
        return -1.0;
    }
}

}  // namespace

extern "C" {

// Explicit: reference ExplicitSolver vs CudaExplicitSolver on the 2D Riemann
// problem, n x n, nsteps steps.  Returns the worst relative L-inf over
// rho, rhoU, rhoV, rhoE (negative on an exception).
double sifv_adapter_selftest_explicit(int n, int nsteps, int precision, int bcCode) {
    return explicitCase(n, nsteps, precision, bcCode, 0.0);
}

// The same with viscousParams.mu = mu (viscous stress + viscous dt limit).
double sifv_adapter_selftest_explicit_viscous(int n, int nsteps, int bcCode, double mu) {
    return explicitCase(n, nsteps, SIFV_PREC_FP64, bcCode, mu);
}

// Immersed boundary: ExplicitSolver + ImmersedBoundaryMethod vs
// CudaExplicitSolver + CudaImmersedBoundary, uniform Mach 0.2 stream past a
// circle (0.35, 0.5) r 0.12 on the unit square (n x n, outflow), slip or
// no-slip wall, optionally with IGR; bit-identical expected.
double sifv_adapter_selftest_ibm(int n, int nsteps, int slip, int igrOn) {
    try {
        SimulationConfig cfg;
        cfg.dim = 2; cfg.nGhost = 3; cfg.RKOrder = 3; cfg.reconOrder = ReconstructionOrder::WENO5;
        cfg.explicitParams.cfl = 0.5;
        cfg.useIGR = igrOn != 0;
        cfg.igrParams.alphaCoeff = 1.0;
        cfg.validate();
        Setup a = makeMesh(cfg, n, n, 1, {0, 0, 0}, BoundaryCondition::Outflow);
        Setup b = makeMesh(cfg, n, n, 1, {0, 0, 0}, BoundaryCondition::Outflow);
        auto eos = std::make_shared<IdealGasEOS>(1.4, 287.0, cfg);
        auto riemann = std::make_shared<HLLCSolver>(eos, cfg);
        auto igr = igrOn ? std::make_shared<IGRSolver>(cfg.igrParams) : nullptr;
        SolutionState sa, sb;
        sa.allocate(a.mesh->totalCells(), cfg);
        sb.allocate(b.mesh->totalCells(), cfg);
        PrimitiveState W;
        W.rho = 1.0; W.u = {1.0, 0.0, 0.0}; W.p = 1.0 / (1.4 * 0.04);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                std::size_t ia = a.mesh->index(i, j, 0), ib = b.mesh->index(i, j, 0);
                sa.setPrimitiveState(ia, W); sa.setConservativeState(ia, eos->toConservative(W));
                sb.setPrimitiveState(ib, W); sb.setConservativeState(ib, eos->toConservative(W));
            }
        auto circle = std::make_shared<IBCircle>(0.35, 0.5, 0.12);
        circle->setWallType(slip ? IBBody::WallType::Slip : IBBody::WallType::NoSlip);
        ImmersedBoundaryMethod ibmRef;
        ibmRef.addBody(circle);
        ibmRef.classifyCells(*a.mesh);
        b200::CudaImmersedBoundary ibmGpu;
        ibmGpu.addBody(circle);
        ibmGpu.classifyCells(*b.mesh);
        ExplicitSolver ref(*a.mesh, riemann, eos, igr, cfg);
        ref.setHaloExchange(a.halo.get());
        ref.setIBM(&ibmRef);
        b200::CudaExplicitSolver gpu(*b.mesh, riemann, eos, igr, cfg);
        gpu.setHaloExchange(b.halo.get());
        gpu.setIBM(&ibmGpu);
        SimulationConfig ca = cfg, cb = cfg;
        for (int s = 0; s < nsteps; ++s) {
            double da = ref.step(ca, *a.mesh, sa, -1.0);
            double db = gpu.step(cb, *b.mesh, sb, -1.0);
            if (da != db) return 1.0;
            ca.time += da; ca.step++;
            cb.time += db; cb.step++;
        }
        double w = 0.0;
        w = std::max(w, maxRel(sb.rho, sa.rho, *a.mesh));
        w = std::max(w, maxRel(sb.rhoU, sa.rhoU, *a.mesh));
        w = std::max(w, maxRel(sb.rhoV, sa.rhoV, *a.mesh));
        w = std::max(w, maxRel(sb.rhoE, sa.rhoE, *a.mesh));
        w = std::max(w, maxRel(sb.sigma, sa.sigma, *a.mesh));
        return w;
    } catch (...) {
        return -1.0;
    }
}

// Semi-implicit + IGR: reference SemiImplicitSolver vs CudaSemiImplicitSolver
// on the periodic 3D pulse (n^3, RK1).  `plugin` bit 0 instead plugs the
// CUDA PressureSolver into the REFERENCE solver (the PressureSolver plugin
// interface); bit 1 selects Gauss-Seidel instead of Jacobi on both sides.
// *itersOut: last pressure iterations of the CUDA side.
double sifv_adapter_selftest_semi(int n, int nsteps, int plugin, int* itersOut) {
    try {
        SimulationConfig cfg;
        cfg.dim = 3; cfg.nGhost = 3; cfg.RKOrder = 1; cfg.reconOrder = ReconstructionOrder::WENO5;
        cfg.semiImplicit = true; cfg.useIGR = true;
        cfg.semiImplicitParams.cfl = 0.8; cfg.semiImplicitParams.pressureTol = 1e-6;
        cfg.semiImplicitParams.maxPressureIters = 1000;
        cfg.igrParams.alphaCoeff = 10.0; cfg.igrParams.IGRIters = 5;
        cfg.validate();
        Setup a = makeMesh(cfg, n, n, n, {1, 1, 1}, BoundaryCondition::Periodic);
        Setup b = makeMesh(cfg, n, n, n, {1, 1, 1}, BoundaryCondition::Periodic);
        auto eos = std::make_shared<IdealGasEOS>(1.4, 287.0, cfg);
        auto riemann = std::make_shared<HLLCSolver>(eos, cfg);
        auto igr = std::make_shared<IGRSolver>(cfg.igrParams);
        SolutionState sa, sb;
        sa.allocate(a.mesh->totalCells(), cfg);
        sb.allocate(b.mesh->totalCells(), cfg);
        pulseIC(*a.mesh, sa, *eos);
        pulseIC(*b.mesh, sb, *eos);
        const bool gs = (plugin & 2) != 0;
        plugin &= 1;
        auto refSolver = [gs]() -> std::shared_ptr<PressureSolver> {
            if (gs) return std::make_shared<GaussSeidelPressureSolver>();
            return std::make_shared<JacobiPressureSolver>();
        };
        SemiImplicitSolver ref(*a.mesh, riemann, refSolver(), eos, igr, cfg);
        ref.setHaloExchange(a.halo.get());
        std::unique_ptr<SemiImplicitSolver> refPlug;
        std::unique_ptr<b200::CudaSemiImplicitSolver> gpu;
        if (plugin) {
            std::shared_ptr<PressureSolver> cudaPS;
            if (gs) cudaPS = std::make_shared<b200::CudaGaussSeidelPressureSolver>();
            else cudaPS = std::make_shared<b200::CudaJacobiPressureSolver>();
            refPlug = std::make_unique<SemiImplicitSolver>(*b.mesh, riemann, cudaPS, eos, igr, cfg);
            refPlug->setHaloExchange(b.halo.get());
        } else {
            gpu = std::make_unique<b200::CudaSemiImplicitSolver>(*b.mesh, riemann, refSolver(), eos, igr, cfg);
            gpu->setHaloExchange(b.halo.get());
        }
        SimulationConfig ca = cfg, cb = cfg;
        for (int s = 0; s < nsteps; ++s) {
            double da = ref.step(ca, *a.mesh, sa, -1.0);
            double db = plugin ? refPlug->step(cb, *b.mesh, sb, -1.0) : gpu->step(cb, *b.mesh, sb, -1.0);
            if (da != db) return 1.0;
            int ia = ref.lastPressureIterations();
            int ib = plugin ? refPlug->lastPressureIterations() : gpu->lastPressureIterations();
            if (ia != ib) return 2.0;
            if (itersOut) *itersOut = ib;
            ca.time += da; ca.step++;
            cb.time += db; cb.step++;
        }
        double w = 0.0;
        w = std::max(w, maxRel(sb.rho, sa.rho, *a.mesh));
        w = std::max(w, maxRel(sb.rhoU, sa.rhoU, *a.mesh));
        w = std::max(w, maxRel(sb.rhoV, sa.rhoV, *a.mesh));
        w = std::max(w, maxRel(sb.rhoW, sa.rhoW, *a.mesh));
        w = std::max(w, maxRel(sb.rhoE, sa.rhoE, *a.mesh));
        w = std::max(w, maxRel(sb.sigma, sa.sigma, *a.mesh));
        return w;
    } catch (...) {
        return -1.0;
    }
}

}  // extern "C"
