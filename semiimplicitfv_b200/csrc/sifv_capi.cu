// sifv_capi.cu -- the C ABI of include/sifv.h: context, device allocation,
// the step orchestration (ExplicitSolver::step / SemiImplicitSolver::step)
// and the standalone PressureSolver / IGR / dt entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "sifv.h"
#include "sifv_adjoint_api.h"
#include "sifv_kernels.cuh"
#include "sifv_gs_march.cuh"
#include "sifv_mg.cuh"
#include "sifv_sweep_api.h"
#include "sifv_ib_api.h"
#include "sifv_vtk_api.h"

using namespace sifv;

namespace {

thread_local std::string g_err;

constexpr int kCellThreads = 256;
constexpr int kFaceThreads = 128;

}  // namespace

struct sifv_ctx {
    sifv_config_t cfg{};
    Params P{};
    Fields F{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t ownStream = nullptr;
    std::vector<void*> allocs;
    Ctl* ctl = nullptr;        // device control block
    Ctl* ctlHost = nullptr;    // pinned mirror
    int resCap = 0;
    std::string err;
    int lastIters = 0;
    float lastMs = 0.f;
    int lastLaunches = 0;
    int launches = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    size_t ncells = 0, nint = 0;
    double alphaIGR = 0.0;
    int nphT = 0;   // NPH template bucket (0, 2 or 8)
    int W = 5;      // stencil width
    // scratch for the standalone pressure solve with host arrays
    double *sRho = nullptr, *sRhoc2 = nullptr, *sRhs = nullptr, *sP = nullptr;
    // per-kernel-family timing (sifv_profile_step)
    bool profiling = false;
    std::vector<std::pair<std::string, cudaEvent_t>> marks;
    // fused sweep path (SIFV_PREC_MIXED / SIFV_PREC_FP64_FAST)
    bool sweep = false;
    double* rhsBuf[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    double* invW[3] = {nullptr, nullptr, nullptr};
    double* rhoP = nullptr;
    // discrete adjoint / tangent (sifv_adjoint_*, sifv_tangent_*)
    double forcedDt = -1.0;                   // > 0: the steps use this dt (no CFL reduction)
    std::function<int(int, int)> stageHook;   // (stage, phase): 0 before the prim fill, 1 before the update, 2 after
    bool dtReady = false;                     // ctl->dtBits holds the acoustic dt of the current state
                                              // (folded in by the last fast 2D stage of the previous step)
    bool exchangeFaces = false;               // the mesh has SIFV_BC_EXCHANGE faces
    int marchScale = 1;                       // work units per resident warp of the 2D fused stage (sifv_autotune)
    sifv_comm_t comm{};                       // halo exchange / dt reduction of a decomposed run
    int adjEvery = 0;
    std::vector<double> adjDts;               // time-step sequence of the recorded forward run
    std::vector<double*> adjCkpt;             // (dim + 2) arrays per checkpoint, then the final state
    double* adjStage = nullptr;               // stage inputs of one segment
    size_t adjStageCap = 0;
    bool adjReady = false;
    bool igrTileReady = false;
    double* igrRec = nullptr;                 // IGR sweep records (k_igr_records), then one int flag
    double* gsRec = nullptr;                  // Gauss-Seidel sweep records (k_gs_records), then one int flag
    std::vector<double*> gsBuf;               // iterate buffers 2 .. of the overlapped Gauss-Seidel sweeps
    double2* marchQ[kMarchMaxBufs] = {};     // 2D Gauss-Seidel wavefront: iterates (skewed pair layout)
    double* marchRec = nullptr;               // its records (Gauss-Seidel)
    double* marchRecIgr = nullptr;            // its records (IGR)
    int* marchInt = nullptr;                  // progress [G], flags [2], slowRecs [1], done [marchIntCap]
    int marchIntCap = -1;
    int marchOk = -1;                         // -1 unknown, 0 no cooperative launch, 1 usable
    long long marchCtas = 0;                  // co-resident CTAs of k_march_gs
    int marchMode = -1;                       // SIFV_GS_MARCH: -1 (unset) periodic meshes, 0 never, 1 always
    int marchSegs = 0;                        // SIFV_GS_MARCH_SEGMENTS: segments along the march axis (0: chosen)
    int gsPrevIters = 0;                      // iterations of the previous Gauss-Seidel solve (first batch size)
    double* jacCoef = nullptr;                // Jacobi coefficients: per face (dim arrays) or per cell (2 dim + 2)
    bool uniformAxes = false;                 // interior cell widths bitwise equal along every active axis
    int pressureKind = 0;                     // 0 Jacobi (default), 1 Gauss-Seidel
    double* gsCoef = nullptr;                 // per-cell Gauss-Seidel coefficients (2 dim + 2 arrays)
    double* tileB[4] = {nullptr, nullptr, nullptr, nullptr};   // 2D fused-stage scratch states
    double* tileC[4] = {nullptr, nullptr, nullptr, nullptr};                // dynamic shared memory limit of the IGR tile kernel set
    double* lam[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    double* acc0[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    double* share[3] = {nullptr, nullptr, nullptr};
    double* tan[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    double* tan0[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    double* tanW[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    double* tanF[3][5] = {};
    double* loopLog = nullptr;                // per-step dt of a device-resident time-loop batch
    int loopLogCap = 0;
    // immersed boundary (sifv_set_immersed_*)
    std::vector<double> cenX, cenY, cenZ;     // interior cell centroids
    std::vector<unsigned char> ibTypes;       // CellType per cell (host copy), empty when off
    IbDev ib{};
    std::vector<void*> ibAllocs;
    // PCG + multigrid pressure solver (SIFV_PRESSURE_PCG_MG)
    std::vector<MgLevel> mg;
    double* cg[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};   // x r z p q 1/m
    double* cgScal = nullptr;    // 8 device scalars
    double* cgPartial = nullptr; // block partial sums of the fine level
    // mixed-precision Jacobi (semi-implicit SIFV_PREC_MIXED)
    double* mxCoef = nullptr;    // k_jacobi_coef layout, FP64
    float* mxW = nullptr;        // 2 dim FP32 weights per cell
    float* mxD = nullptr;        // FP32 delta
    float* mxE[2] = {nullptr, nullptr};
    int lastInPlace = 0;         // the last pressure solve left its result in F.pA
    int jacPrevIters = 0;        // iterations of the previous Jacobi solve (first batch size)
    unsigned jacGrid = 0;        // resident-grid size of the grid-stride Jacobi kernels
    unsigned mxGrid = 0;         // the same for k_mx_sweep
    int adjFp32 = 0;             // FP32 local Jacobians in the reverse sweep
};

namespace {

int fail(sifv_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    else g_err = msg;
    return code;
}

#define CUDA_TRY(ctx, call)                                                                     \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return fail(ctx, SIFV_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

#define LAUNCH_CHECK(ctx)                                                                                  \
    do {                                                                                                   \
        cudaError_t e_ = cudaGetLastError();                                                               \
        if (e_ != cudaSuccess) return fail(ctx, SIFV_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e_)); \
    } while (0)

unsigned blocks(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// Record an event after a kernel family when profiling.
void mark(sifv_ctx* c, const char* family) {
    if (!c->profiling) return;
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, c->stream);
    c->marks.emplace_back(family, e);
}

void mark_cb(void* user, const char* family) { mark(static_cast<sifv_ctx*>(user), family); }

// RectilinearMesh::buildExtendedNodes, src/RectilinearMesh.cpp:91-114
std::vector<double> build_ext(const double* phys, int nCells, int ng) {
    std::vector<double> ext(nCells + 2 * ng + 1);
    for (int i = 0; i <= nCells; ++i) ext[ng + i] = phys[i];
    for (int g = 1; g <= ng; ++g) {
        int mirror = std::min(g - 1, nCells - 1);
        double width = phys[mirror + 1] - phys[mirror];
        ext[ng - g] = ext[ng - g + 1] - width;
    }
    for (int g = 1; g <= ng; ++g) {
        int mirror = std::max(nCells - g, 0);
        double width = phys[mirror + 1] - phys[mirror];
        ext[ng + nCells + g] = ext[ng + nCells + g - 1] + width;
    }
    return ext;
}

int validate(const sifv_config_t* c, std::string& msg) {
    // SimulationConfig::validate, include/SimulationConfig.hpp:123-209
    auto bad = [&](const char* m) { msg = m; return SIFV_ERR_BAD_CONFIG; };
    if (c->dim < 1 || c->dim > 3) return bad("dim must be 1, 2, or 3");
    if (c->RKOrder < 1 || c->RKOrder > 3) return bad("RKOrder must be 1, 2, or 3");
    if (c->reconOrder < SIFV_WENO1 || c->reconOrder > SIFV_UPWIND5) return bad("unknown reconOrder");
    int req = (c->reconOrder == SIFV_WENO1 || c->reconOrder == SIFV_UPWIND1) ? 1
            : (c->reconOrder == SIFV_WENO3 || c->reconOrder == SIFV_UPWIND3) ? 2 : 3;
    if (c->nGhost < req) return bad("nGhost is too small for chosen reconOrder");
    if (c->semiImplicit) {
        if (c->siCfl <= 0) return bad("semiImplicitParams.cfl must be > 0");
        if (c->siMinDt <= 0) return bad("semiImplicitParams.minDt must be > 0");
        if (c->siMaxDt <= c->siMinDt) return bad("semiImplicitParams.maxDt must be > minDt");
        if (c->pressureTol <= 0) return bad("semiImplicitParams.pressureTol must be > 0");
        if (c->maxPressureIters <= 0) return bad("semiImplicitParams.maxPressureIters must be > 0");
    } else {
        if (c->cfl <= 0) return bad("explicitParams.cfl must be > 0");
        if (c->minDt <= 0) return bad("explicitParams.minDt must be > 0");
        if (c->maxDt <= c->minDt) return bad("explicitParams.maxDt must be > minDt");
    }
    if (c->useIGR) {
        if (c->alphaCoeff <= 0) return bad("igrParams.alphaCoeff must be > 0");
        if (c->IGRIters <= 0) return bad("igrParams.IGRIters must be > 0");
        if (c->IGRWarmStartIters < 0) return bad("igrParams.IGRWarmStartIters must be >= 0");
    }
    if (c->nPhases < 0 || c->nPhases > SIFV_MAX_PHASES) return bad("nPhases must be in [0, 8]");
    for (int p = 0; p < c->nPhases; ++p) {
        if (c->phaseGamma[p] <= 1.0) return bad("multiPhaseParams.phases[].gamma must be > 1");
        if (c->phasePInf[p] < 0.0) return bad("multiPhaseParams.phases[].pInf must be >= 0");
    }
    if (c->nPhases > 0 && c->alphaMin <= 0.0) return bad("multiPhaseParams.alphaMin must be > 0");
    if (c->riemannSolver < SIFV_LF || c->riemannSolver > SIFV_HLLC) return bad("unknown riemannSolver");
    if (c->mu < 0.0) return bad("viscousParams.mu must be >= 0");
    if (c->nPhaseMu < 0 || c->nPhaseMu > SIFV_MAX_PHASES) return bad("viscousParams.phaseMu has too many entries");
    if (c->nPhaseMu > 0) {
        if (c->nPhases <= 0) return bad("viscousParams.phaseMu requires multi-phase (nPhases >= 2)");
        if (c->nPhaseMu != c->nPhases) return bad("viscousParams.phaseMu.size() must equal nPhases");
        for (int p = 0; p < c->nPhaseMu; ++p)
            if (c->phaseMu[p] < 0.0) return bad("viscousParams.phaseMu[] must be >= 0");
    }
    if (c->stSigma < 0.0) return bad("surfaceTensionParams.sigma must be >= 0");
    if (c->stEpsGradAlpha <= 0.0) return bad("surfaceTensionParams.epsGradAlpha must be > 0");
    if (c->stSigma > 0.0 && c->nPhases <= 0)
        return bad("surfaceTensionParams.sigma requires multi-phase (nPhases >= 2)");
    if (c->precision != SIFV_PREC_FP64 && c->precision != SIFV_PREC_MIXED && c->precision != SIFV_PREC_FP64_FAST)
        return bad("unknown precision");
    return SIFV_OK;
}

double* dalloc(sifv_ctx* c, size_t n, int& st) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(double));
    if (e != cudaSuccess) {
        st = fail(c, SIFV_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        return nullptr;
    }
    cudaMemsetAsync(p, 0, std::max<size_t>(n, 1) * sizeof(double), c->stream);
    c->allocs.push_back(p);
    return static_cast<double*>(p);
}

double* field_ptr(sifv_ctx* c, int f) {
    Fields& F = c->F;
    switch (f) {
        case SIFV_F_RHO: return F.rho;
        case SIFV_F_RHOU: return F.rhoU;
        case SIFV_F_RHOV: return F.rhoV;
        case SIFV_F_RHOW: return F.rhoW;
        case SIFV_F_RHOE: return F.rhoE;
        case SIFV_F_VELU: return F.velU;
        case SIFV_F_VELV: return F.velV;
        case SIFV_F_VELW: return F.velW;
        case SIFV_F_PRES: return F.pres;
        case SIFV_F_SIGMA: return F.sigma;
        default: break;
    }
    if (f >= 16 && f < 16 + c->cfg.nPhases) return F.alphaRho[f - 16];
    if (f >= 32 && f < 32 + c->cfg.nPhases) return F.alpha[f - 32];
    return nullptr;
}

// Grow the control block's residual history to n entries; the control
// fields (dt, time, flags) carry over to the new block.
int ensure_res(sifv_ctx* c, int n) {
    if (n <= c->resCap) return SIFV_OK;
    Ctl* old = c->ctl;
    Ctl* oldHost = c->ctlHost;
    Ctl* fresh = nullptr;
    Ctl* freshHost = nullptr;
    size_t bytes = sizeof(Ctl) + sizeof(unsigned long long) * (size_t)(n + 1);
    CUDA_TRY(c, cudaMalloc(&fresh, bytes));
    CUDA_TRY(c, cudaMallocHost(&freshHost, bytes));
    CUDA_TRY(c, cudaMemsetAsync(fresh, 0, bytes, c->stream));
    if (old) CUDA_TRY(c, cudaMemcpyAsync(fresh, old, offsetof(Ctl, res), cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (old) cudaFree(old);
    if (oldHost) cudaFreeHost(oldHost);
    c->ctl = fresh;
    c->ctlHost = freshHost;
    c->resCap = n;
    return SIFV_OK;
}

// ---- launchers ------------------------------------------------------------

template <int NPH>
void launch_face_nph(sifv_ctx* c, int dir) {
    const Params& P = c->P;
    long long nf = (long long)(P.nx + (dir == 0)) * (P.ny + (dir == 1)) * (P.nz + (dir == 2));
    unsigned g = blocks(nf, kFaceThreads);
    cudaStream_t s = c->stream;
#define FACE_CASE(D, Wd) k_face<D, Wd, NPH><<<g, kFaceThreads, 0, s>>>(c->P, c->F, c->ctl)
    if (dir == 0) {
        if (c->W == 1) FACE_CASE(0, 1); else if (c->W == 3) FACE_CASE(0, 3); else FACE_CASE(0, 5);
    } else if (dir == 1) {
        if (c->W == 1) FACE_CASE(1, 1); else if (c->W == 3) FACE_CASE(1, 3); else FACE_CASE(1, 5);
    } else {
        if (c->W == 1) FACE_CASE(2, 1); else if (c->W == 3) FACE_CASE(2, 3); else FACE_CASE(2, 5);
    }
#undef FACE_CASE
    c->launches++;
    mark(c, dir == 0 ? "face_x" : dir == 1 ? "face_y" : "face_z");
}

void launch_face(sifv_ctx* c, int dir) {
    if (c->nphT == 0) launch_face_nph<0>(c, dir);
    else if (c->nphT == 2) launch_face_nph<2>(c, dir);
    else launch_face_nph<8>(c, dir);
}

#define NPH_DISPATCH(c, KERNEL_CALL)                 \
    do {                                             \
        if ((c)->nphT == 0) { constexpr int NPHV = 0; KERNEL_CALL; } \
        else if ((c)->nphT == 2) { constexpr int NPHV = 2; KERNEL_CALL; } \
        else { constexpr int NPHV = 8; KERNEL_CALL; } \
    } while (0)

void launch_prim_bc(sifv_ctx* c, bool interiorOnly = false) {
    long long n = (long long)c->ncells;
    NPH_DISPATCH(c, (k_prim_bc<NPHV><<<blocks(n, kCellThreads), kCellThreads, 0, c->stream>>>(
                         c->P, c->F, c->ctl, interiorOnly ? 1 : 0)));
    c->launches++;
    mark(c, "prim_bc");
}

void launch_bc_prim(sifv_ctx* c) {
    long long n = ghost_count(c->P);
    NPH_DISPATCH(c, (k_bc_prim<NPHV><<<blocks(n, kCellThreads), kCellThreads, 0, c->stream>>>(c->P, c->F)));
    c->launches++;
    mark(c, "bc_prim");
}

void launch_scalar_ghosts(sifv_ctx* c, double* f) {
    k_scalar_ghosts<<<blocks(ghost_count(c->P), kCellThreads), kCellThreads, 0, c->stream>>>(c->P, f);
    c->launches++;
}

// applyGhostCells / applyScalarGhostCells of the immersed boundary, when set.
void launch_ib_ghost(sifv_ctx* c) {
    if (!c->ib.count) return;
    const unsigned g = c->ib.sequential ? 1u : blocks(c->ib.count, kCellThreads);
    NPH_DISPATCH(c, (k_ib_ghost<NPHV><<<g, kCellThreads, 0, c->stream>>>(c->P, c->F, c->ib, c->ctl)));
    c->launches++;
    mark(c, "ib_ghost");
}

void launch_ib_scalar(sifv_ctx* c, double* f) {
    if (!c->ib.count) return;
    const unsigned g = c->ib.sequential ? 1u : blocks(c->ib.count, kCellThreads);
    k_ib_scalar<<<g, kCellThreads, 0, c->stream>>>(c->ib, f, c->ctl);
    c->launches++;
}

// halo exchange / reductions of a decomposed mesh (defined with the step)
int exchange_fields(sifv_ctx* c, double* const* fields, int n);
int exchange_scalar(sifv_ctx* c, const double* f);
int reduce_residual(sifv_ctx* c, unsigned long long* slot);

int march_run(sifv_ctx* c, int kind, const double* rhs, double tol, int maxIter, int& iters,
              const double*& result);

int igr_solve(sifv_ctx* c, int step) {
    const Params& P = c->P;
    k_igr_setup<<<blocks((long long)c->nint, kCellThreads), kCellThreads, 0, c->stream>>>(P, c->F, c->alphaIGR);
    c->launches++;
    int iters = (step == 0) ? c->cfg.IGRWarmStartIters : c->cfg.IGRIters;
    // tiled wavefront: 16^3 tiles in 3D, 32 x 64 tiles in 2D
    constexpr int T3 = 16, T2X = 32, T2Y = 64;
    const bool d3 = P.dim == 3;
    const int tx = d3 ? T3 : T2X, ty = d3 ? T3 : T2Y, tz = d3 ? T3 : 1;
    const int ntx = (P.nx + tx - 1) / tx, nty = (P.ny + ty - 1) / ty, ntz = (P.nz + tz - 1) / tz;
    const int nplanes = ntx + nty + ntz - 2;
    const size_t smem = d3 ? igr_tile_smem<T3, T3, T3>() : igr_tile_smem<T2X, T2Y, 1>();
    if (P.dim >= 2 && !c->igrTileReady) {
        cudaError_t e = d3 ? cudaFuncSetAttribute(k_igr_tile<T3, T3, T3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)smem)
                           : cudaFuncSetAttribute(k_igr_tile<T2X, T2Y, 1>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return fail(c, SIFV_ERR_CUDA, std::string("IGR tile smem: ") + cudaGetErrorString(e));
        c->igrTileReady = true;
    }
    // 3D: the record sweep (k_igr_tile_rec) when its 16-byte halo copies are
    // aligned (even row length, 16-byte aligned sigma and rho)
    const bool rec = d3 && T3 == kIgrTile && P.nxT % 2 == 0 && ((uintptr_t)c->F.sigma % 16) == 0 &&
                     ((uintptr_t)c->F.rho % 16) == 0;
    int* slowRecs = nullptr;
    if (rec) {
        const int ntiles = ntx * nty * ntz;
        const size_t nrec = igr_record_doubles(ntiles);
        if (!c->igrRec) {
            int sa = SIFV_OK;
            c->igrRec = dalloc(c, nrec + 2, sa);
            if (sa != SIFV_OK) return sa;
            cudaError_t e = cudaFuncSetAttribute(k_igr_tile_rec, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)igr_tile_rec_smem());
            if (e != cudaSuccess)
                return fail(c, SIFV_ERR_CUDA, std::string("IGR record tile smem: ") + cudaGetErrorString(e));
        }
        slowRecs = reinterpret_cast<int*>(c->igrRec + nrec);
        CUDA_TRY(c, cudaMemsetAsync(slowRecs, 0, sizeof(int), c->stream));
        const long long total = (long long)ntiles * kIgrTile * kIgrTile * kIgrRecsPerLine;
        k_igr_records<<<blocks(total, 256), 256, 0, c->stream>>>(P, c->F, c->igrRec, ntx, nty, total, slowRecs);
        c->launches++;
    }
    // Sweeps (record or plain tiles, 2D and 3D) overlap when nothing runs between them (no halo exchange,
    // no immersed-boundary fix-up): sweep s + 1 trails sweep s by `lag` tile
    // planes, at least 2 (no face-adjacent tiles in one launch) and, on a
    // periodic axis, the tiles along it (the wrap-around ghost images of
    // sweep s are final before sweep s + 1 reads them).
    const bool periodic2d = P.bc[0] == SIFV_BC_PERIODIC || P.bc[1] == SIFV_BC_PERIODIC ||
                            P.bc[2] == SIFV_BC_PERIODIC || P.bc[3] == SIFV_BC_PERIODIC;
    if (P.dim == 2 && iters > 1 && !c->exchangeFaces && !c->ib.count && !c->F.solid && c->marchMode != 0 &&
        (c->marchMode == 1 || periodic2d || std::max(P.nx, P.ny) >= 1024)) {
        // the persistent wavefront (all sweeps in one launch): on a mesh with a periodic face, and without
        // one from 1024 cells along the longer axis (rows cut into segments); the tiled sweeps below
        // otherwise
        int done = 0;
        const double* res = nullptr;
        const int ms = march_run(c, 1, nullptr, 0.0, iters, done, res);
        if (ms == SIFV_OK) {
            mark(c, "igr");
            return SIFV_OK;
        }
        if (ms != 1) return ms;
    }
    if (P.dim >= 2 && iters > 1 && !c->exchangeFaces && !c->ib.count) {
        int lag = 2;
        if (P.bc[0] == SIFV_BC_PERIODIC) lag = std::max(lag, ntx);
        if (P.bc[2] == SIFV_BC_PERIODIC) lag = std::max(lag, nty);
        if (P.bc[4] == SIFV_BC_PERIODIC) lag = std::max(lag, ntz);
        lag = std::max(lag, (nplanes + kIgrMaxSlots - 1) / kIgrMaxSlots);
        const int total = nplanes + (iters - 1) * lag;
        bool first = true;
        int launched = 0;
        for (int pc = 0; pc < total; ++pc) {
            // active sweeps: s with 0 <= pc - s lag < nplanes, a run s0 .. s0 + n - 1 (none when the
            // lag exceeds the planes of a sweep and pc falls between two sweeps)
            const int s0 = pc >= nplanes ? (pc - nplanes) / lag + 1 : 0, s1 = std::min(iters - 1, pc / lag);
            if (s1 < s0) continue;
            IgrPlanes PL{};
            PL.top = pc - s0 * lag;
            PL.lag = lag;
            PL.n = s1 - s0 + 1;
            PL.ghosts = 1;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            at[0].val.programmaticStreamSerializationAllowed = 1;
            cudaLaunchConfig_t lc = {};
            lc.gridDim = dim3((unsigned)(PL.n * nty * ntz));
            lc.stream = c->stream;
            if (rec) {
                lc.blockDim = dim3(kIgrTile * kIgrTile);
                lc.dynamicSmemBytes = igr_tile_rec_smem();
                lc.attrs = at;
                lc.numAttrs = first ? 0 : 1;   // planes after the first overlap their record prologue
                CUDA_TRY(c, cudaLaunchKernelEx(&lc, k_igr_tile_rec, P, c->F, (const double*)c->igrRec,
                                               (const int*)slowRecs, PL, ntx, nty, ntz));
            } else if (d3) {
                lc.blockDim = dim3(T3 * T3);
                lc.dynamicSmemBytes = smem;
                CUDA_TRY(c, cudaLaunchKernelEx(&lc, k_igr_tile<T3, T3, T3>, P, c->F, PL, ntx, nty, ntz));
            } else {
                lc.blockDim = dim3(T2Y);
                lc.dynamicSmemBytes = smem;
                CUDA_TRY(c, cudaLaunchKernelEx(&lc, k_igr_tile<T2X, T2Y, 1>, P, c->F, PL, ntx, nty, ntz));
            }
            first = false;
            ++launched;
        }
        c->launches += launched;
        launch_scalar_ghosts(c, c->F.sigma);   // the full fill after the last sweep (src/IGR.cpp:155)
        mark(c, "igr");
        LAUNCH_CHECK(c);
        return SIFV_OK;
    }
    for (int it = 0; it < iters; ++it) {
        if (P.dim == 1) {
            k_igr_sweep_1d<<<1, 32, 0, c->stream>>>(P, c->F);
            c->launches++;
        } else {
            for (int pl = 0; pl < nplanes; ++pl) {
                if (rec) {
                    // planes after the first overlap their prologue with the previous plane
                    cudaLaunchAttribute at[1];
                    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
                    at[0].val.programmaticStreamSerializationAllowed = 1;
                    cudaLaunchConfig_t lc = {};
                    lc.gridDim = dim3((unsigned)(nty * ntz));
                    lc.blockDim = dim3(kIgrTile * kIgrTile);
                    lc.dynamicSmemBytes = igr_tile_rec_smem();
                    lc.stream = c->stream;
                    lc.attrs = at;
                    lc.numAttrs = pl > 0 ? 1 : 0;
                    IgrPlanes PL{};
                    PL.top = pl;
                    PL.lag = 0;
                    PL.n = 1;
                    CUDA_TRY(c, cudaLaunchKernelEx(&lc, k_igr_tile_rec, P, c->F, (const double*)c->igrRec,
                                                   (const int*)slowRecs, PL, ntx, nty, ntz));
                } else {
                    IgrPlanes PL{};
                    PL.top = pl;
                    PL.n = 1;
                    if (d3)
                        k_igr_tile<T3, T3, T3><<<(unsigned)(nty * ntz), T3 * T3, smem, c->stream>>>(P, c->F, PL, ntx,
                                                                                                  nty, ntz);
                    else
                        k_igr_tile<T2X, T2Y, 1><<<(unsigned)nty, T2Y, smem, c->stream>>>(P, c->F, PL, ntx, nty, ntz);
                }
            }
            c->launches += nplanes;
        }
        {   // fillScalarGhosts(sigma, halo), src/IGR.cpp:155
            int st = exchange_scalar(c, c->F.sigma);
            if (st != SIFV_OK) return st;
        }
        launch_scalar_ghosts(c, c->F.sigma);
        launch_ib_scalar(c, c->F.sigma);   // src/IGR.cpp:156
    }
    mark(c, "igr");
    LAUNCH_CHECK(c);
    return SIFV_OK;
}

// Jacobi iterations on (rho, rhoc2, rhs) with initial guess in F.pA;
// returns the number of iterations as JacobiPressureSolver::solve does and
// the buffer holding the result.
int jacobi_run(sifv_ctx* c, const double* rho, const double* rhoc2, const double* rhs, double tol, int maxIter,
               int& iters, const double*& result) {
    int st = ensure_res(c, maxIter);
    if (st != SIFV_OK) return st;
    CUDA_TRY(c, cudaMemsetAsync(&c->ctl->jacobiDone, 0, sizeof(int), c->stream));
    CUDA_TRY(c, cudaMemsetAsync(c->ctl->res, 0, sizeof(unsigned long long) * (size_t)maxIter, c->stream));
    unsigned g = blocks((long long)c->nint, kCellThreads);
    const bool faceCoef = c->uniformAxes;
    if (!c->jacCoef) {
        int sa = SIFV_OK;
        c->jacCoef = dalloc(c, c->ncells * (size_t)(faceCoef ? c->P.dim : 2 * c->P.dim + 2), sa);
        if (sa != SIFV_OK) return sa;
    }
    if (faceCoef)
        k_jacobi_fcoef<<<g, kCellThreads, 0, c->stream>>>(c->P, rho, c->F, c->jacCoef, c->ncells);
    else
        k_jacobi_coef<<<g, kCellThreads, 0, c->stream>>>(c->P, rho, rhoc2, c->F, c->ctl, c->jacCoef, c->ncells);
    // Batches between host convergence checks: 4, 8, 16, 32; a solve after an
    // earlier one starts with 3/4 of its iteration count in one batch (the
    // counts change slowly from step to step), which spares most of the
    // launches that only find the solve converged.
    if (!c->jacGrid) {
        int sm = 0, nb1 = 0, nb2 = 0;
        CUDA_TRY(c, cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, c->device));
        CUDA_TRY(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb1, k_jacobi_face, kCellThreads, 0));
        CUDA_TRY(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb2, k_jacobi_pre, kCellThreads, 0));
        c->jacGrid = (unsigned)std::max(1, sm * std::max(1, std::min(nb1, nb2)));
    }
    const unsigned gj = std::min(g, c->jacGrid);
    int it = 0, batch = c->jacPrevIters > 5 ? (3 * c->jacPrevIters) / 4 : 4;
    bool first = true;
    int done = 0;
    while (it < maxIter) {
        int nb = std::min(batch, maxIter - it);
        for (int q = 0; q < nb; ++q, ++it) {
            const double* pin = (it & 1) ? c->F.pB : c->F.pA;
            double* pout = (it & 1) ? c->F.pA : c->F.pB;
            {   // decomposed mesh: the iterate's ghost layers from the neighbours (src/JacobiPressureSolver.cpp:72)
                int st = exchange_scalar(c, pin);
                if (st != SIFV_OK) return st;
            }
            if (c->P.dim == 3) {
                const dim3 g3((unsigned)((c->P.nx + 31) / 32), (unsigned)((c->P.ny + 7) / 8),
                              (unsigned)((c->P.nz + kJacZ - 1) / kJacZ));
                if (faceCoef)
                    k_jacobi3<true><<<g3, 256, 0, c->stream>>>(c->P, c->jacCoef, c->ncells, rhoc2, rhs, pin, pout,
                                                               c->ctl, it, tol);
                else
                    k_jacobi3<false><<<g3, 256, 0, c->stream>>>(c->P, c->jacCoef, c->ncells, rhoc2, rhs, pin, pout,
                                                                c->ctl, it, tol);
            } else if (faceCoef)
                k_jacobi_face<<<gj, kCellThreads, 0, c->stream>>>(c->P, c->jacCoef, c->ncells, rhoc2, rhs, pin, pout,
                                                                 c->ctl, it, tol);
            else
                k_jacobi_pre<<<gj, kCellThreads, 0, c->stream>>>(c->P, c->jacCoef, c->ncells, rhs, pin, pout, c->ctl,
                                                                it, tol);
            {   // the iteration's change, maximum over the ranks, before the next iteration tests it
                int st = reduce_residual(c, &c->ctl->res[it]);
                if (st != SIFV_OK) return st;
            }
        }
        c->launches += nb;
        LAUNCH_CHECK(c);
        CUDA_TRY(c, cudaMemcpyAsync(c->ctlHost, c->ctl, sizeof(Ctl) + sizeof(unsigned long long) * (size_t)it,
                                    cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        if (c->ctlHost->jacobiDone) {
            done = c->ctlHost->jacobiDone;
            break;
        }
        double last;
        unsigned long long b = c->ctlHost->res[it - 1];
        std::memcpy(&last, &b, sizeof(double));
        if (last < tol) {
            done = it;
            break;
        }
        batch = first && batch > 4 ? 4 : std::min(batch * 2, 32);
        first = false;
    }
    iters = done ? done : maxIter;
    c->jacPrevIters = iters;
    result = (iters & 1) ? c->F.pB : c->F.pA;
    mark(c, "jacobi");
    return SIFV_OK;
}

// 2D sweeps as one persistent wavefront (k_march_gs): records and iterate 0,
// one cooperative launch for all sweeps, the result back in the mesh layout.
// kind 0: Gauss-Seidel pressure iterations from c->gsCoef, rhs and F.pA
// (result in F.pA, the iteration count from the per-sweep residuals; the
// ghost layers from the iterate before the last sweep, as the reference's
// last fill leaves them).  kind 1: `maxIter` IGR sweeps on F.sigma (ghost
// layers filled from the result, src/IGR.cpp:155).  The warps walk along a
// periodic axis (free for the wavefront), along the longer one when both are
// periodic.  Returns 1 (nothing done) when the launch does not fit the
// device or the progress counters would overflow.
int march_run(sifv_ctx* c, int kind, const double* rhs, double tol, int maxIter, int& iters,
              const double*& result) {
    const Params& P = c->P;
    const bool px = P.bc[0] == SIFV_BC_PERIODIC || P.bc[1] == SIFV_BC_PERIODIC;
    const bool py = P.bc[2] == SIFV_BC_PERIODIC || P.bc[3] == SIFV_BC_PERIODIC;
    // walk along y when only y is periodic, or both or neither are and y is longer
    const bool tr = (py && !px) || (px == py && P.ny > P.nx);
    const int Nm = tr ? P.ny : P.nx, Nn = tr ? P.nx : P.ny;     // march and row extents
    const int bm0 = tr ? P.bc[2] : P.bc[0], bm1 = tr ? P.bc[3] : P.bc[1];
    const int bn0 = tr ? P.bc[0] : P.bc[2], bn1 = tr ? P.bc[1] : P.bc[3];
    const int NH = (Nm + 1) / 2, SW = NH + 32, NS = NH + 31;
    const int G = Nn / 32 + 1, GA = (Nn + 1) / 32 + 1;
    const int ctasPerSeg = (G + kMarchWarps - 1) / kMarchWarps;
    if ((long long)(maxIter + 2) * NS >= (1LL << 30)) return 1;
    // instances: Gauss-Seidel and IGR cells, batch length 8 or the short one, each walking along x or y
    using MarchFn = void (*)(Params, GsMarch, Ctl*);
    constexpr int DS = kMarchShortD;
    const MarchFn fns[8] = {k_march_gs<kMarchWarps, 8, false, 0>,  k_march_gs<kMarchWarps, 8, true, 0>,
                            k_march_gs<kMarchWarps, DS, false, 0>, k_march_gs<kMarchWarps, DS, true, 0>,
                            k_march_gs<kMarchWarps, 8, false, 1>,  k_march_gs<kMarchWarps, 8, true, 1>,
                            k_march_gs<kMarchWarps, DS, false, 1>, k_march_gs<kMarchWarps, DS, true, 1>};
    const int fnD[8] = {8, 8, DS, DS, 8, 8, DS, DS}, fnKind[8] = {0, 0, 0, 0, 1, 1, 1, 1};
    // D = the short batch when a periodic row axis makes the groups' lags (about 32 + 2 D + 10 steps
    // each) longer than a sweep; otherwise D = 8
    const bool rowPeriodic = bn0 == SIFV_BC_PERIODIC || bn1 == SIFV_BC_PERIODIC;
    const bool short8 = rowPeriodic && (long long)G * (32 + 2 * 8 + 10) > NS;
    const int fi = (kind ? 4 : 0) + (short8 ? 2 : 0) + (tr ? 1 : 0);
    const int D = fnD[fi];
    const MarchFn fn = fns[fi];
    const size_t smem = march_smem(D, kind);
    if (c->marchOk < 0) {
        c->marchOk = 0;
        int coop = 0, sms = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
        long long fit = -1;
        for (int q = 0; q < 8 && coop; ++q) {
            const size_t sq = march_smem(fnD[q], fnKind[q]);
            int perSm = 0;
            if (cudaFuncSetAttribute(fns[q], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sq) != cudaSuccess ||
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, fns[q], 32 * (kMarchWarps + 1), sq) !=
                    cudaSuccess) {
                fit = -1;
                break;
            }
            fit = (fit < 0) ? (long long)perSm * sms : std::min(fit, (long long)perSm * sms);
        }
        if (fit > 0) {
            c->marchOk = 1;
            c->marchCtas = fit;
        }
        cudaGetLastError();
    }
    if (!c->marchOk || ctasPerSeg > c->marchCtas) return 1;
    // Without a periodic face the rows are cut into S segments along the march axis (about 192 pairs each,
    // as many as the co-resident CTAs allow): a segment's sweep k follows the left segment's sweep k and
    // the right one's sweep k - 1, so the segments work on consecutive sweeps at once.
    int S = 1;
    if (!px && !py) {
        const long long fit = c->marchCtas / ctasPerSeg;
        S = (int)std::max<long long>(1, std::min<long long>(fit, (NH + 191) / 192));
        if (c->marchSegs > 0) S = (int)std::min<long long>(fit, c->marchSegs);
    }
    const int L = (NH + S - 1) / S;
    S = (NH + L - 1) / L;
    const int ctas = ctasPerSeg * S, NSs = L + 31;
    const size_t qn = (size_t)GA * SW * 32;   // pairs per iterate
    // buffers: the warps spread over about (G (32 + 2 D + 40) + S NSs) / NSs sweeps, plus the converged
    // iterate, its predecessor and one sweep of slack; at most 1 GiB together, or 8 buffers where 1 GiB
    // holds fewer (as many bytes as the Gauss-Seidel records): at 8192² 1 GiB would leave 3 buffers while
    // the warps spread over about 4 sweeps, and the leading groups would stall on buffers still being read
    int nb = std::min(kMarchMaxBufs, 4 + (G * (32 + 2 * D + 40) + S * NSs + NSs - 1) / NSs);
    const size_t bufBytes = qn * sizeof(double2);
    nb = std::max(3, std::min<int>(nb, (int)(std::max<size_t>(size_t(1) << 30, 8 * bufBytes) / bufBytes)));
    int sa = SIFV_OK;
    double*& recBuf = kind ? c->marchRecIgr : c->marchRec;
    if (!recBuf) {
        recBuf = dalloc(c, qn * 4 * march_chunks(kind), sa);   // 2 cells x chunks double2 per pair
        if (sa != SIFV_OK) return sa;
    }
    for (int q = 0; q < nb; ++q)
        if (!c->marchQ[q]) {
            c->marchQ[q] = reinterpret_cast<double2*>(dalloc(c, qn * 2, sa));
            if (sa != SIFV_OK) return sa;
        }
    if (c->marchIntCap < maxIter) {   // ints in double units
        const int cap = std::max(maxIter, 64);
        c->marchInt = reinterpret_cast<int*>(dalloc(c, ((size_t)G * S + 3 + cap + 1) / 2 + 1, sa));
        if (sa != SIFV_OK) return sa;
        c->marchIntCap = cap;
    }
    int* prog = c->marchInt;   // [S][G]
    int* flags = prog + (size_t)G * S;
    int* slowRecs = flags + 2;
    int* done = slowRecs + 1;
    CUDA_TRY(c, cudaMemsetAsync(c->marchInt, 0, sizeof(int) * ((size_t)G * S + 3 + maxIter), c->stream));
    const long long total = (long long)qn;
    if (kind)
        k_march_igr_setup<<<blocks(total, 256), 256, 0, c->stream>>>(P, c->F, reinterpret_cast<double2*>(recBuf),
                                                                    c->marchQ[0], SW, total, slowRecs, tr ? 1 : 0);
    else
        k_march_gs_setup<<<blocks(total, 256), 256, 0, c->stream>>>(P, c->gsCoef, c->ncells, rhs, c->F.pA,
                                                                   reinterpret_cast<double2*>(recBuf), c->marchQ[0],
                                                                   SW, total, slowRecs, tr ? 1 : 0);
    GsMarch M{};
    M.rec = reinterpret_cast<const double2*>(recBuf);
    for (int q = 0; q < nb; ++q) M.q[q] = c->marchQ[q];
    M.prog = prog;
    M.done = done;
    M.flags = flags;
    M.slowRecs = slowRecs;
    M.nb = nb;
    M.G = G;
    M.GA = GA;
    M.SW = SW;
    M.NS = NS;
    M.S = S;
    M.L = L;
    M.ctasPerSeg = ctasPerSeg;
    M.NH = NH;
    M.maxIter = maxIter;
    M.nx = Nm;
    M.ny = Nn;
    M.xsLo = (bm0 == SIFV_BC_PERIODIC) ? Nm - 1 : 0;
    M.xsHi = (bm1 == SIFV_BC_PERIODIC) ? 0 : Nm - 1;
    M.perLoY = bn0 == SIFV_BC_PERIODIC;
    M.perHiY = bn1 == SIFV_BC_PERIODIC;
    M.tol = tol;
    M.ghost0 = c->F.sigma;
    M.wRow = tr ? c->F.adx2 : c->F.ady2;
    M.wRowOff = tr ? P.ngx : P.ngy;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3((unsigned)ctas);
    lc.blockDim = dim3(32 * (kMarchWarps + 1));
    lc.dynamicSmemBytes = smem;
    lc.stream = c->stream;
    lc.attrs = at;
    lc.numAttrs = 1;
    CUDA_TRY(c, cudaLaunchKernelEx(&lc, fn, P, M, c->ctl));
    c->launches += 2;
    LAUNCH_CHECK(c);
    int hostFlags[2] = {0, 0};
    CUDA_TRY(c, cudaMemcpyAsync(hostFlags, flags, sizeof(hostFlags), cudaMemcpyDeviceToHost, c->stream));
    if (!kind)
        CUDA_TRY(c, cudaMemcpyAsync(c->ctlHost, c->ctl, sizeof(Ctl) + sizeof(unsigned long long) * (size_t)maxIter,
                                    cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (hostFlags[1]) return fail(c, SIFV_ERR_CUDA, "2D sweep wavefront: a wait timed out");
    iters = maxIter;
    for (int j = 0; !kind && j < maxIter; ++j) {
        double r;
        std::memcpy(&r, &c->ctlHost->res[j], sizeof(double));
        if (r < tol) {
            iters = j + 1;
            break;
        }
    }
    double* out = kind ? c->F.sigma : c->F.pA;
    k_march_gs_out<<<blocks((long long)P.nxT * P.nyT, kCellThreads), kCellThreads, 0, c->stream>>>(
        P, c->marchQ[iters % nb], c->marchQ[(kind ? iters : iters - 1) % nb], out, SW, tr ? 1 : 0);
    c->launches++;
    result = out;
    return SIFV_OK;
}

// GaussSeidelPressureSolver::solve on the device: in place on F.pA (the
// initial guess), coefficients once per solve, per iteration a scalar ghost
// fill and one tiled-wavefront sweep; convergence as jacobi_run.
int gs_run(sifv_ctx* c, const double* rho, const double* rhoc2, const double* rhs, double tol, int maxIter,
           int& iters, const double*& result) {
    int st = ensure_res(c, maxIter);
    if (st != SIFV_OK) return st;
    CUDA_TRY(c, cudaMemsetAsync(&c->ctl->jacobiDone, 0, sizeof(int), c->stream));
    CUDA_TRY(c, cudaMemsetAsync(c->ctl->res, 0, sizeof(unsigned long long) * (size_t)maxIter, c->stream));
    const Params& P = c->P;
    unsigned g = blocks((long long)c->nint, kCellThreads);
    if (!c->gsCoef) {
        int sa = SIFV_OK;
        c->gsCoef = dalloc(c, c->ncells * (size_t)(2 * P.dim + 2), sa);
        if (sa != SIFV_OK) return sa;
    }
    k_jacobi_coef<<<g, kCellThreads, 0, c->stream>>>(P, rho, rhoc2, c->F, c->ctl, c->gsCoef, c->ncells);
    constexpr int T3 = 16, T2X = 32, T2Y = 64;
    const bool d3 = P.dim == 3;
    const int tx = d3 ? T3 : T2X, ty = d3 ? T3 : T2Y, tz = d3 ? T3 : 1;
    const int ntx = (P.nx + tx - 1) / tx, nty = (P.ny + ty - 1) / ty, ntz = (P.nz + tz - 1) / tz;
    const int nplanes = ntx + nty + ntz - 2;
    const size_t smem = d3 ? gs_tile_smem<T3, T3, T3>() : gs_tile_smem<T2X, T2Y, 1>();
    if (P.dim >= 2) {
        cudaError_t e = d3 ? cudaFuncSetAttribute(k_gs_tile<T3, T3, T3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)smem)
                           : cudaFuncSetAttribute(k_gs_tile<T2X, T2Y, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)smem);
        if (e != cudaSuccess) return fail(c, SIFV_ERR_CUDA, std::string("GS tile smem: ") + cudaGetErrorString(e));
    }
    double* pp = c->F.pA;
    // 3D: the record sweep (k_gs_tile_rec) when its 16-byte halo copies are
    // aligned (even row length, 16-byte aligned iterate)
    const bool recs = d3 && T3 == kIgrTile && P.nxT % 2 == 0 && ((uintptr_t)pp % 16) == 0;
    int* slowRecs = nullptr;
    if (recs) {
        const long long ntiles = (long long)ntx * nty * ntz;
        const size_t nrec = gs_record_doubles(ntiles);
        if (!c->gsRec) {
            int sa = SIFV_OK;
            c->gsRec = dalloc(c, nrec + 2, sa);
            if (sa != SIFV_OK) return sa;
            CUDA_TRY(c, cudaFuncSetAttribute(k_gs_tile_rec, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)gs_tile_rec_smem()));
        }
        slowRecs = reinterpret_cast<int*>(c->gsRec + nrec);
        CUDA_TRY(c, cudaMemsetAsync(slowRecs, 0, sizeof(int), c->stream));
        const long long total = ntiles * kIgrTile * kIgrTile * kIgrTile;
        k_gs_records<<<blocks(total, 256), 256, 0, c->stream>>>(P, c->gsCoef, c->ncells, rhs, c->gsRec, ntx, nty,
                                                                 total, slowRecs);
        c->launches++;
    }
    const bool periodic2d = P.bc[0] == SIFV_BC_PERIODIC || P.bc[1] == SIFV_BC_PERIODIC ||
                            P.bc[2] == SIFV_BC_PERIODIC || P.bc[3] == SIFV_BC_PERIODIC;
    if (P.dim == 2 && !c->exchangeFaces && maxIter >= 2 && c->marchMode != 0 &&
        (c->marchMode == 1 || periodic2d || std::max(P.nx, P.ny) >= 2048)) {
        // the persistent wavefront: on a mesh with a periodic face, and without one from 2048 cells along
        // the longer axis (rows cut into segments); below that the tiled sweeps, which overlap many
        // iterations there (their iterations lag by 2 tile planes), are as fast
        const int ms = march_run(c, 0, rhs, tol, maxIter, iters, result);
        if (ms == SIFV_OK) {
            c->gsPrevIters = iters;
            mark(c, "gauss_seidel");
        }
        if (ms != 1) return ms;
    }
    if (P.dim >= 2 && !c->exchangeFaces && maxIter >= 2) {
        // overlapped iterations (k_gs_tile_rec_ov, k_gs_tile_ov): iterate n in buf[n % nb], nb = S + 2
        // for S iterations in flight.  The lag is at least 2 planes and, on a periodic axis, the tiles
        // along it; in 3D at most three iterations are in flight (a tile plane already fills the GPU),
        // in 2D as many as the planes allow, within 30 and 1 GiB of extra iterates.
        int lag = 2;
        if (P.bc[0] == SIFV_BC_PERIODIC) lag = std::max(lag, ntx);
        if (P.bc[2] == SIFV_BC_PERIODIC) lag = std::max(lag, nty);
        if (P.bc[4] == SIFV_BC_PERIODIC) lag = std::max(lag, ntz);
        const size_t bufBytes = c->ncells * sizeof(double);
        const int sMax = d3 ? 3 : (int)std::max<size_t>(1, std::min<size_t>(30, (size_t(1) << 30) / bufBytes));
        lag = std::max(lag, (nplanes + sMax - 1) / sMax);
        const int S = (nplanes + lag - 1) / lag;
        const int nb = S + 2;
        while ((int)c->gsBuf.size() < nb - 2) {
            int sa = SIFV_OK;
            double* p = dalloc(c, c->ncells, sa);
            if (sa != SIFV_OK) return sa;
            c->gsBuf.push_back(p);
        }
        if (recs)
            CUDA_TRY(c, cudaFuncSetAttribute(k_gs_tile_rec_ov, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)gs_tile_rec_smem()));
        else if (d3)
            CUDA_TRY(c, cudaFuncSetAttribute(k_gs_tile_ov<T3, T3, T3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem));
        else
            CUDA_TRY(c, cudaFuncSetAttribute(k_gs_tile_ov<T2X, T2Y, 1>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        GsBufs B{};
        B.nb = nb;
        B.b[0] = c->F.pA;
        B.b[1] = c->F.pB;
        for (int q = 0; q < nb - 2; ++q) B.b[q + 2] = c->gsBuf[q];
        // the ghost layers the first iteration reads: iterate 0's images in buf 0 and buf 1
        const unsigned gg = blocks(ghost_count(P), kCellThreads);
        k_scalar_ghosts<<<gg, kCellThreads, 0, c->stream>>>(P, B.b[0]);
        k_scalar_ghosts_from<<<gg, kCellThreads, 0, c->stream>>>(P, B.b[0], B.b[1]);
        c->launches += 2;
        const int total = nplanes + (maxIter - 1) * lag;
        const int guess = std::max(2, c->gsPrevIters > 4 ? (3 * c->gsPrevIters) / 4 : 4);
        int pc = 0, chunk = nplanes + (guess - 1) * lag, done = 0;
        bool first = true;
        while (pc < total && !done) {
            const int end = std::min(total, pc + chunk);
            for (; pc < end; ++pc) {
                const int s0 = pc >= nplanes ? (pc - nplanes) / lag + 1 : 0, s1 = std::min(maxIter - 1, pc / lag);
                if (s1 < s0) continue;
                GsPlanes PL{};
                PL.top = pc - s0 * lag;
                PL.lag = lag;
                PL.n = s1 - s0 + 1;
                PL.it0 = s0;
                PL.np = nplanes;
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
                at[0].val.programmaticStreamSerializationAllowed = 1;
                cudaLaunchConfig_t lc = {};
                lc.gridDim = dim3((unsigned)(PL.n * nty * ntz));
                lc.stream = c->stream;
                if (recs) {
                    lc.blockDim = dim3(kIgrTile * kIgrTile);
                    lc.dynamicSmemBytes = gs_tile_rec_smem();
                    lc.attrs = at;
                    lc.numAttrs = first ? 0 : 1;
                    CUDA_TRY(c, cudaLaunchKernelEx(&lc, k_gs_tile_rec_ov, P, (const double*)c->gsRec,
                                                   (const int*)slowRecs, B, c->ctl, tol, PL, ntx, nty, ntz));
                } else if (d3) {
                    lc.blockDim = dim3(T3 * T3);
                    lc.dynamicSmemBytes = smem;
                    CUDA_TRY(c, cudaLaunchKernelEx(&lc, k_gs_tile_ov<T3, T3, T3>, P, (const double*)c->gsCoef,
                                                   c->ncells, rhs, B, c->ctl, tol, PL, ntx, nty, ntz));
                } else {
                    lc.blockDim = dim3(T2Y);
                    lc.dynamicSmemBytes = smem;
                    CUDA_TRY(c, cudaLaunchKernelEx(&lc, k_gs_tile_ov<T2X, T2Y, 1>, P, (const double*)c->gsCoef,
                                                   c->ncells, rhs, B, c->ctl, tol, PL, ntx, nty, ntz));
                }
                first = false;
                c->launches++;
            }
            LAUNCH_CHECK(c);
            // iterations complete after launch pc - 1: j lag + nplanes - 1 <= pc - 1
            const int complete = std::min(maxIter, pc >= nplanes ? (pc - nplanes) / lag + 1 : 0);
            CUDA_TRY(c, cudaMemcpyAsync(c->ctlHost, c->ctl,
                                        sizeof(Ctl) + sizeof(unsigned long long) * (size_t)std::max(complete, 1),
                                        cudaMemcpyDeviceToHost, c->stream));
            CUDA_TRY(c, cudaStreamSynchronize(c->stream));
            for (int j = 0; j < complete; ++j) {
                double r;
                std::memcpy(&r, &c->ctlHost->res[j], sizeof(double));
                if (r < tol) {
                    done = j + 1;
                    break;
                }
            }
            chunk = std::min(2 * chunk, 16 * lag + nplanes);
        }
        iters = done ? done : maxIter;
        c->gsPrevIters = iters;
        // the result's ghosts as the reference leaves them: filled from the iterate before the last sweep
        k_scalar_ghosts_from<<<gg, kCellThreads, 0, c->stream>>>(P, B.b[(iters - 1) % nb], B.b[iters % nb]);
        c->launches++;
        result = B.b[iters % nb];
        mark(c, "gauss_seidel");
        return SIFV_OK;
    }
    int it = 0, batch = 2, done = 0;
    while (it < maxIter) {
        int nb = std::min(batch, maxIter - it);
        for (int q = 0; q < nb; ++q, ++it) {
            {   // decomposed mesh: fillScalarGhosts(pressure, halo), src/GaussSeidelPressureSolver.cpp:69
                int st = exchange_scalar(c, pp);
                if (st != SIFV_OK) return st;
            }
            k_gs_ghosts<<<blocks(ghost_count(P), kCellThreads), kCellThreads, 0, c->stream>>>(P, pp, c->ctl, it, tol);
            if (recs) {
                for (int pl = 0; pl < nplanes; ++pl) {
                    // planes after the first overlap their record prologue with the previous plane
                    cudaLaunchAttribute at[1];
                    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
                    at[0].val.programmaticStreamSerializationAllowed = 1;
                    cudaLaunchConfig_t lc = {};
                    lc.gridDim = dim3((unsigned)(nty * ntz));
                    lc.blockDim = dim3(kIgrTile * kIgrTile);
                    lc.dynamicSmemBytes = gs_tile_rec_smem();
                    lc.stream = c->stream;
                    lc.attrs = at;
                    lc.numAttrs = pl > 0 ? 1 : 0;
                    CUDA_TRY(c, cudaLaunchKernelEx(&lc, k_gs_tile_rec, P, (const double*)c->gsRec,
                                                   (const int*)slowRecs, pp, c->ctl, it, tol, pl, ntx, nty));
                }
                c->launches += 1 + nplanes;
            } else if (P.dim == 1) {
                k_gs_sweep_1d<<<1, 32, 0, c->stream>>>(P, c->gsCoef, c->ncells, rhs, pp, c->ctl, it, tol);
                c->launches += 2;
            } else {
                for (int pl = 0; pl < nplanes; ++pl) {
                    if (d3)
                        k_gs_tile<T3, T3, T3><<<(unsigned)(nty * ntz), T3 * T3, smem, c->stream>>>(
                            P, c->gsCoef, c->ncells, rhs, pp, c->ctl, it, tol, pl, ntx, nty);
                    else
                        k_gs_tile<T2X, T2Y, 1><<<(unsigned)nty, T2Y, smem, c->stream>>>(P, c->gsCoef, c->ncells, rhs,
                                                                                      pp, c->ctl, it, tol, pl, ntx,
                                                                                      nty);
                }
                c->launches += 1 + nplanes;
            }
            {   // src/GaussSeidelPressureSolver.cpp:92-93
                int st = reduce_residual(c, &c->ctl->res[it]);
                if (st != SIFV_OK) return st;
            }
        }
        LAUNCH_CHECK(c);
        CUDA_TRY(c, cudaMemcpyAsync(c->ctlHost, c->ctl, sizeof(Ctl) + sizeof(unsigned long long) * (size_t)it,
                                    cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        if (c->ctlHost->jacobiDone) {
            done = c->ctlHost->jacobiDone;
            break;
        }
        double last;
        unsigned long long b = c->ctlHost->res[it - 1];
        std::memcpy(&last, &b, sizeof(double));
        if (last < tol) {
            done = it;
            break;
        }
        batch = std::min(batch * 2, 16);
    }
    iters = done ? done : maxIter;
    result = pp;
    mark(c, "gauss_seidel");
    return SIFV_OK;
}

// Multigrid hierarchy for the fine mesh: every axis longer than 1 halves
// (ceil) until a level holds at most 256 cells.
int mg_alloc(sifv_ctx* c) {
    if (!c->mg.empty()) return SIFV_OK;
    int st = SIFV_OK;
    int nx = c->P.nx, ny = c->P.ny, nz = c->P.nz;
    for (int l = 0;; ++l) {
        MgLevel L{};
        L.nx = nx; L.ny = ny; L.nz = nz;
        L.n = (long long)nx * ny * nz;
        L.m = dalloc(c, L.n, st);
        L.tx = dalloc(c, L.n, st);
        L.ty = dalloc(c, L.n, st);
        L.tz = dalloc(c, L.n, st);
        L.diag = dalloc(c, L.n, st);
        L.r = dalloc(c, L.n, st);
        L.t = dalloc(c, L.n, st);
        if (l > 0) {
            L.x = dalloc(c, L.n, st);
            L.b = dalloc(c, L.n, st);
        }
        if (st != SIFV_OK) return st;
        c->mg.push_back(L);
        if (L.n <= 256 || (nx <= 2 && ny <= 2 && nz <= 2)) break;
        nx = (nx > 1) ? (nx + 1) / 2 : 1;
        ny = (ny > 1) ? (ny + 1) / 2 : 1;
        nz = (nz > 1) ? (nz + 1) / 2 : 1;
    }
    const long long n0 = c->mg[0].n;
    for (int q = 0; q < 6; ++q) c->cg[q] = dalloc(c, n0, st);
    c->cgScal = dalloc(c, 8, st);
    c->cgPartial = dalloc(c, blocks(n0, kCellThreads) + 1, st);
    return st;
}

constexpr double kMgOmega = 0.8;       // weighted-Jacobi relaxation
constexpr int kMgCoarsestSweeps = 60;  // relaxation sweeps on the coarsest level

// z = V(r): one V(1,1)-cycle from z = 0 (level 0 reads b = r, writes x = z).
void mg_vcycle(sifv_ctx* c, int l, const double* r0, double* z0) {
    const int dim = c->P.dim;
    MgLevel L = c->mg[l];
    if (l == 0) {
        L.b = const_cast<double*>(r0);
        L.x = z0;
    }
    const unsigned g = blocks(L.n, kCellThreads);
    if (l + 1 == (int)c->mg.size()) {
        k_mg_coarsest<<<1, 1024, 0, c->stream>>>(L, dim, kMgOmega, kMgCoarsestSweeps);
        c->launches++;
        return;
    }
    MgLevel C = c->mg[l + 1];
    k_mg_smooth0<<<g, kCellThreads, 0, c->stream>>>(L, kMgOmega);
    k_mg_residual<<<g, kCellThreads, 0, c->stream>>>(L, dim);
    k_mg_restrict<<<blocks(C.n, kCellThreads), kCellThreads, 0, c->stream>>>(L, C);
    c->launches += 3;
    mg_vcycle(c, l + 1, nullptr, nullptr);
    k_mg_prolong<<<g, kCellThreads, 0, c->stream>>>(L, C);
    k_mg_smooth<<<g, kCellThreads, 0, c->stream>>>(L, dim, L.x, L.t, kMgOmega);
    cudaMemcpyAsync(L.x, L.t, sizeof(double) * L.n, cudaMemcpyDeviceToDevice, c->stream);
    c->launches += 2;
}

// HyprePressureSolver::solve (src/HyprePressureSolver.cpp:333-399): PCG on
// the symmetric scaled system with a multigrid V-cycle as preconditioner,
// stopping when |r|_2 <= tol |rhs|_2 on the unscaled system.  Initial guess
// and result in F.pA (interior; ghosts untouched).
int mg_run(sifv_ctx* c, const double* rho, const double* rhoc2, const double* rhs, double tol, int maxIter,
           int& iters, const double*& result) {
    int st = mg_alloc(c);
    if (st != SIFV_OK) return st;
    st = ensure_res(c, maxIter);
    if (st != SIFV_OK) return st;
    const int dim = c->P.dim;
    MgLevel L0 = c->mg[0];
    const long long n0 = L0.n;
    const unsigned g0 = blocks(n0, kCellThreads);
    double *x = c->cg[0], *r = c->cg[1], *z = c->cg[2], *p = c->cg[3], *q = c->cg[4], *wInv = c->cg[5];
    double* s = c->cgScal;
    double* part = c->cgPartial;
    MgLevel Lf = L0;
    Lf.x = x;
    Lf.b = r;   // the scaled right-hand side lands in r, then r = b - M x in place
    k_mg_fine<<<g0, kCellThreads, 0, c->stream>>>(c->P, c->F, rho, rhoc2, rhs, c->F.pA, c->ctl, Lf, wInv);
    for (size_t l = 0; l + 1 < c->mg.size(); ++l)
        k_mg_coarsen<<<blocks(c->mg[l + 1].n, kCellThreads), kCellThreads, 0, c->stream>>>(c->mg[l], c->mg[l + 1], dim);
    for (const MgLevel& L : c->mg) k_mg_diag<<<blocks(L.n, kCellThreads), kCellThreads, 0, c->stream>>>(L, dim);
    // |rhs|^2 into s[4], then r = b - M x and |r/m|^2 into s[2]
    k_mg_bnorm<<<g0, kCellThreads, 0, c->stream>>>(n0, r, wInv, part);
    k_mg_sum<<<1, 1024, 0, c->stream>>>(part, (int)g0, s, 4);
    Lf.b = r;
    k_mg_residual0<<<g0, kCellThreads, 0, c->stream>>>(Lf, dim, wInv, r, part);
    k_mg_sum<<<1, 1024, 0, c->stream>>>(part, (int)g0, s, 2);
    c->launches += 6 + 2 * (int)c->mg.size();
    LAUNCH_CHECK(c);
    double hs[5];
    CUDA_TRY(c, cudaMemcpyAsync(hs, s, sizeof(hs), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    const double bb = hs[4], eps = tol * tol;
    double rr = hs[2];
    int it = 0;
    if (bb == 0.0) {   // Hypre: zero right-hand side -> zero solution
        CUDA_TRY(c, cudaMemsetAsync(x, 0, sizeof(double) * n0, c->stream));
        rr = 0.0;
    } else if (!(rr <= eps * bb)) {
        mg_vcycle(c, 0, r, z);
        k_mg_dot<<<g0, kCellThreads, 0, c->stream>>>(n0, r, z, part);
        k_mg_sum<<<1, 1024, 0, c->stream>>>(part, (int)g0, s, 0);
        k_cg_direction<<<g0, kCellThreads, 0, c->stream>>>(n0, s, z, p, 1);
        c->launches += 3;
        while (it < maxIter) {
            ++it;
            k_mg_matvec_dot<<<g0, kCellThreads, 0, c->stream>>>(L0, dim, p, q, part);
            k_mg_sum<<<1, 1024, 0, c->stream>>>(part, (int)g0, s, 1);
            k_cg_update<<<g0, kCellThreads, 0, c->stream>>>(n0, s, x, r, p, q, wInv, part);
            k_mg_sum<<<1, 1024, 0, c->stream>>>(part, (int)g0, s, 2);
            c->launches += 4;
            LAUNCH_CHECK(c);
            CUDA_TRY(c, cudaMemcpyAsync(&hs[2], s + 2, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
            CUDA_TRY(c, cudaStreamSynchronize(c->stream));
            rr = hs[2];
            if (rr <= eps * bb || !(rr == rr)) break;
            mg_vcycle(c, 0, r, z);
            k_mg_dot<<<g0, kCellThreads, 0, c->stream>>>(n0, r, z, part);
            k_mg_sum<<<1, 1024, 0, c->stream>>>(part, (int)g0, s, 3);
            k_cg_direction<<<g0, kCellThreads, 0, c->stream>>>(n0, s, z, p, 0);
            k_cg_shift<<<1, 1, 0, c->stream>>>(s);
            c->launches += 4;
        }
    }
    k_mg_scatter<<<g0, kCellThreads, 0, c->stream>>>(c->P, Lf, c->F.pA);
    c->launches++;
    LAUNCH_CHECK(c);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    // relative residual of the last iteration where the semi-implicit step looks for it
    const double rel = (bb > 0.0) ? std::sqrt(rr / bb) : 0.0;
    iters = it;
    if (it > 0) std::memcpy(&c->ctlHost->res[it - 1], &rel, sizeof(double));
    result = c->F.pA;
    mark(c, "pcg_mg");
    return SIFV_OK;
}

// JacobiPressureSolver::solve with FP32 inner sweeps and FP64 refinement
// (SIFV_PREC_MIXED semi-implicit step): batches of FP32 sweeps between FP64
// Jacobi changes; result in place in F.pA.
int jacobi_mixed_run(sifv_ctx* c, const double* rho, const double* rhoc2, const double* rhs, double tol, int maxIter,
                     int& iters, const double*& result) {
    int st = ensure_res(c, maxIter);
    if (st != SIFV_OK) return st;
    const Params& P = c->P;
    const long long n = (long long)c->nint;
    if (!c->mxCoef) {
        int sa = SIFV_OK;
        c->mxCoef = dalloc(c, c->ncells * (size_t)(2 * P.dim + 2), sa);
        if (sa != SIFV_OK) return sa;
        void* p = nullptr;
        const size_t fl = sizeof(float) * (size_t)n;
        CUDA_TRY(c, cudaMalloc(&p, fl * (size_t)(2 * P.dim + 3)));
        c->allocs.push_back(p);
        c->mxW = static_cast<float*>(p);
        c->mxD = c->mxW + (size_t)(2 * P.dim) * n;
        c->mxE[0] = c->mxD + n;
        c->mxE[1] = c->mxE[0] + n;
    }
    CUDA_TRY(c, cudaMemsetAsync(&c->ctl->jacobiDone, 0, sizeof(int), c->stream));
    CUDA_TRY(c, cudaMemsetAsync(c->ctl->res, 0, sizeof(unsigned long long) * (size_t)maxIter, c->stream));
    const unsigned g = blocks(n, kCellThreads);
    k_jacobi_coef<<<g, kCellThreads, 0, c->stream>>>(P, rho, rhoc2, c->F, c->ctl, c->mxCoef, c->ncells);
    k_mx_weights<<<g, kCellThreads, 0, c->stream>>>(P, c->mxCoef, c->ncells, c->mxW, n);
    c->launches += 2;
    if (!c->mxGrid) {
        int sm = 0, nb = 0;
        CUDA_TRY(c, cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, c->device));
        CUDA_TRY(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_mx_sweep, kCellThreads, 0));
        c->mxGrid = (unsigned)std::max(1, sm * std::max(1, nb));
    }
    const unsigned gs = std::min(g, c->mxGrid);   // grid-stride FP32 sweeps
    const dim3 g3((unsigned)((P.nx + 31) / 32), (unsigned)((P.ny + 7) / 8), (unsigned)((P.nz + kJacZ - 1) / kJacZ));
    constexpr int kInner = 8;   // FP32 sweeps per FP64 refinement
    int it = 0, done = 0;
    while (it < maxIter && !done) {
        // iteration `it` in FP64: the change at p, also e_1
        k_mx_delta<<<g, kCellThreads, 0, c->stream>>>(P, c->mxCoef, c->ncells, rhs, c->F.pA, c->mxD, c->mxE[0],
                                                       c->ctl, it);
        int cur = 0;
        const int first = it;
        ++it;
        for (int q = 1; q < kInner && it < maxIter; ++q, ++it) {
            if (P.dim == 3)
                k_mx_sweep3<<<g3, 256, 0, c->stream>>>(P, c->mxW, c->mxD, c->mxE[cur], c->mxE[cur ^ 1], c->ctl, it,
                                                       tol);
            else
                k_mx_sweep<<<gs, kCellThreads, 0, c->stream>>>(P, c->mxW, c->mxD, c->mxE[cur], c->mxE[cur ^ 1], c->ctl,
                                                              it, tol);
            cur ^= 1;
        }
        c->launches += it - first;
        LAUNCH_CHECK(c);
        CUDA_TRY(c, cudaMemcpyAsync(c->ctlHost, c->ctl, sizeof(Ctl) + sizeof(unsigned long long) * (size_t)it,
                                    cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        int last = it;   // iterations whose update is in e
        if (c->ctlHost->jacobiDone) {
            done = last = c->ctlHost->jacobiDone;
        } else {
            double lr;
            unsigned long long b = c->ctlHost->res[it - 1];
            std::memcpy(&lr, &b, sizeof(double));
            if (lr < tol) done = it;
        }
        // the buffer written by the last sweep that ran: sweep q (1-based in the batch) writes mxE[q & 1]
        const int ran = last - first;   // 1 .. kInner
        k_mx_apply<<<g, kCellThreads, 0, c->stream>>>(P, c->mxE[(ran - 1) & 1], c->F.pA);
        c->launches++;
    }
    iters = done ? done : maxIter;
    result = c->F.pA;
    c->lastInPlace = 1;
    mark(c, "jacobi_mixed");
    return SIFV_OK;
}

int pressure_run(sifv_ctx* c, const double* rho, const double* rhoc2, const double* rhs, double tol, int maxIter,
                 int& iters, const double*& result) {
    if (c->exchangeFaces && (c->pressureKind == 2 || (c->pressureKind == 0 && c->cfg.precision == SIFV_PREC_MIXED)))
        return fail(c, SIFV_ERR_UNSUPPORTED,
                    "decomposed mesh: the pressure solve supports Jacobi (FP64) and Gauss-Seidel");
    c->lastInPlace = (c->pressureKind != 0) ? 1 : 0;
    if (c->pressureKind == 0 && c->cfg.precision == SIFV_PREC_MIXED)
        return jacobi_mixed_run(c, rho, rhoc2, rhs, tol, maxIter, iters, result);
    if (c->pressureKind == 2) return mg_run(c, rho, rhoc2, rhs, tol, maxIter, iters, result);
    if (c->pressureKind == 1) return gs_run(c, rho, rhoc2, rhs, tol, maxIter, iters, result);
    return jacobi_run(c, rho, rhoc2, rhs, tol, maxIter, iters, result);
}

void rk_coef(int order, int s, StageCoef& K) {
    // src/ExplicitSolver.cpp:92-103
    static const double t1[1][4] = {{1.0, 0.0, 1.0, 1.0}};
    static const double t2[2][4] = {{1.0, 0.0, 1.0, 1.0}, {1.0, 1.0, 1.0, 2.0}};
    static const double t3[3][4] = {{1.0, 0.0, 1.0, 1.0}, {1.0, 3.0, 1.0, 4.0}, {2.0, 1.0, 2.0, 3.0}};
    const double* r = (order == 1) ? t1[s] : (order == 2) ? t2[s] : t3[s];
    K.c1 = r[0]; K.c2 = r[1]; K.c3 = r[2]; K.c4 = r[3];
    K.s = s;
}

bool has_body_force(const sifv_config_t& c) {
    for (int d = 0; d < 3; ++d)
        if (c.bfA[d] != 0.0 || c.bfB[d] != 0.0) return true;
    return false;
}

void body_force(const sifv_config_t& c, double time, StageCoef& K) {
    K.hasBodyForce = has_body_force(c) ? 1 : 0;
    for (int d = 0; d < 3; ++d) K.accel[d] = c.bfA[d] + c.bfB[d] * std::cos(c.bfC[d] * time + c.bfD[d]);
}

// dt reduction + finalisation on the device.
// Halo exchange of a decomposed run (sifv_set_comm): the ghost layers of the
// SIFV_BC_EXCHANGE faces of `fields` from the neighbouring ranks.
int exchange_fields(sifv_ctx* c, double* const* fields, int n) {
    if (!c->exchangeFaces) return SIFV_OK;
    if (!c->comm.exchange)
        return fail(c, SIFV_ERR_BAD_ARG, "the mesh has SIFV_BC_EXCHANGE faces: set the halo exchange (sifv_set_comm)");
    if (c->comm.exchange(c->comm.user, fields, n, c->stream) != 0)
        return fail(c, SIFV_ERR_CUDA, "halo exchange failed");
    return SIFV_OK;
}

// ... of the conservative state the next stage converts (src/HaloExchange.cpp:
// the reference exchanges the primitives after converting; converting the
// exchanged conservative cells gives the same bits, as the conversion is
// per cell).
int exchange_cons(sifv_ctx* c) {
    if (!c->exchangeFaces) return SIFV_OK;
    double* f[6 + 2 * SIFV_MAX_PHASES];
    int n = 0;
    f[n++] = c->F.rho;
    f[n++] = c->F.rhoU;
    if (c->P.dim >= 2) f[n++] = c->F.rhoV;
    if (c->P.dim >= 3) f[n++] = c->F.rhoW;
    f[n++] = c->F.rhoE;
    for (int ph = 0; ph < c->P.nPh; ++ph) f[n++] = c->F.alphaRho[ph];
    for (int ph = 0; ph < c->P.nPh; ++ph) f[n++] = c->F.alpha[ph];
    // sigma travels with the reference's PRIM set; it matters with IGR and in
    // the semi-implicit correction
    if (c->cfg.useIGR || c->cfg.semiImplicit) f[n++] = c->F.sigma;
    return exchange_fields(c, f, n);
}

// The reference's PRIM exchange (HaloExchange::packState, VarSet::PRIM,
// src/HaloExchange.cpp:204-212) where the primitives are not functions of
// the conservative cells: after the semi-implicit star update and after the
// correction.
int exchange_prim(sifv_ctx* c) {
    if (!c->exchangeFaces) return SIFV_OK;
    double* f[6 + 2 * SIFV_MAX_PHASES];
    int n = 0;
    f[n++] = c->F.rho;
    f[n++] = c->F.velU;
    if (c->P.dim >= 2) f[n++] = c->F.velV;
    if (c->P.dim >= 3) f[n++] = c->F.velW;
    f[n++] = c->F.pres;
    f[n++] = c->F.sigma;
    for (int ph = 0; ph < c->P.nPh; ++ph) f[n++] = c->F.alphaRho[ph];
    for (int ph = 0; ph < c->P.nPh; ++ph) f[n++] = c->F.alpha[ph];
    return exchange_fields(c, f, n);
}

// One scalar field (fillScalarGhosts with a HaloExchange, src/RectilinearMesh.cpp:526-624).
int exchange_scalar(sifv_ctx* c, const double* f) {
    double* p = const_cast<double*>(f);
    return exchange_fields(c, &p, 1);
}

// Maximum over the ranks of a pressure-solver residual slot (the bits of a
// non-negative double): the MPI_Allreduce of src/JacobiPressureSolver.cpp:99-100.
int reduce_residual(sifv_ctx* c, unsigned long long* slot) {
    if (!c->exchangeFaces) return SIFV_OK;
    if (!c->comm.allreduce_max)
        return fail(c, SIFV_ERR_BAD_ARG, "the pressure solve of a decomposed mesh needs allreduce_max (sifv_set_comm)");
    if (c->comm.allreduce_max(c->comm.user, reinterpret_cast<double*>(slot), c->stream) != 0)
        return fail(c, SIFV_ERR_CUDA, "residual reduction over the ranks failed");
    return SIFV_OK;
}

int enqueue_dt(sifv_ctx* c, double targetDt, int useEnd) {
    const sifv_config_t& cfg = c->cfg;
    unsigned g = blocks((long long)c->nint, kCellThreads);
    if (cfg.semiImplicit) {
        k_dt_init<<<1, 1, 0, c->stream>>>(c->ctl, cfg.siMaxDt);
        k_dt_advective<<<g, kCellThreads, 0, c->stream>>>(c->P, c->F, c->ctl, cfg.siCfl);
        if (c->P.visc) {
            k_dt_viscous<<<g, kCellThreads, 0, c->stream>>>(c->P, c->F, c->ctl, cfg.siCfl);
            c->launches++;
        }
        if (c->P.cap) {
            k_dt_capillary<<<g, kCellThreads, 0, c->stream>>>(c->P, c->F, c->ctl, cfg.siCfl);
            c->launches++;
        }
        // decomposed run: the minimum over the ranks (src/RKTimeStepping.cpp:125-133)
        if (c->comm.allreduce_min &&
            c->comm.allreduce_min(c->comm.user, reinterpret_cast<double*>(&c->ctl->dtBits), c->stream) != 0)
            return fail(c, SIFV_ERR_CUDA, "dt reduction over the ranks failed");
        k_dt_finalize<<<1, 1, 0, c->stream>>>(c->ctl, -1.0, targetDt, 1, cfg.siMinDt, cfg.siMaxDt, useEnd);
        c->launches += 3;
    } else if (c->forcedDt > 0) {
        k_dt_finalize<<<1, 1, 0, c->stream>>>(c->ctl, c->forcedDt, -1.0, 0, 0.0, 0.0, 0);
        c->launches += 1;
    } else {
        if (cfg.constDt <= 0 && c->dtReady) {
            // the previous step's last stage left min(maxDt, acoustic dt) of this state in ctl->dtBits
        } else if (cfg.constDt <= 0) {
            k_dt_init<<<1, 1, 0, c->stream>>>(c->ctl, cfg.maxDt);
            NPH_DISPATCH(c, (k_dt_acoustic<NPHV><<<g, kCellThreads, 0, c->stream>>>(c->P, c->F, c->ctl, cfg.cfl)));
            if (c->P.visc) {
                k_dt_viscous<<<g, kCellThreads, 0, c->stream>>>(c->P, c->F, c->ctl, cfg.cfl);
                c->launches++;
            }
            if (c->P.cap) {
                k_dt_capillary<<<g, kCellThreads, 0, c->stream>>>(c->P, c->F, c->ctl, cfg.cfl);
                c->launches++;
            }
            c->launches += 2;
        }
        // decomposed run: the minimum over the ranks (src/RKTimeStepping.cpp:148-159)
        if (cfg.constDt <= 0 && c->comm.allreduce_min &&
            c->comm.allreduce_min(c->comm.user, reinterpret_cast<double*>(&c->ctl->dtBits), c->stream) != 0)
            return fail(c, SIFV_ERR_CUDA, "dt reduction over the ranks failed");
        c->dtReady = false;
        k_dt_finalize<<<1, 1, 0, c->stream>>>(c->ctl, cfg.constDt, targetDt, 0, 0.0, 0.0, useEnd);
        c->launches += 1;
    }
    mark(c, "dt");
    return SIFV_OK;
}

// One step, everything enqueued on the stream; semi-implicit steps
// synchronise once per Jacobi batch.
int enqueue_step(sifv_ctx* c, int step, double time, double targetDt, int useEnd, int& status) {
    const sifv_config_t& cfg = c->cfg;
    const Params& P = c->P;
    status = SIFV_OK;
    {
        int st = enqueue_dt(c, targetDt, useEnd);
        if (st != SIFV_OK) return st;
    }
    unsigned gc = blocks((long long)c->nint, kCellThreads);
    if (c->sweep && P.dim == 2) {
        // one fused tile kernel per stage; stage outputs ping-pong through two
        // scratch states, the last stage writes over the step-start state
        if (!c->tileB[0]) {
            int sa = SIFV_OK;
            for (int q = 0; q < 4; ++q) {
                c->tileB[q] = dalloc(c, c->ncells, sa);
                c->tileC[q] = dalloc(c, c->ncells, sa);
            }
            if (sa != SIFV_OK) return sa;
        }
        double* U[4] = {c->F.rho, c->F.rhoU, c->F.rhoV, c->F.rhoE};
        const int RK = cfg.RKOrder;
        for (int s = 0; s < RK; ++s) {
            StageCoef K{};
            rk_coef(RK, s, K);
            TileArgs T{};
            T.P = c->P;
            T.C.gamma = c->P.gamma;
            T.C.pInf = c->P.pInf;
            T.C.invGm1 = 1.0 / (c->P.gamma - 1.0);
            T.C.gPinf = c->P.gamma * c->P.pInf;
            T.eps = cfg.wenoEps;
            T.ctl = c->ctl;
            T.a1 = K.c1 / K.c4;
            T.a2 = K.c2 / K.c4;
            T.a3 = K.c3 / K.c4;
            T.inv[0] = c->invW[0];
            T.inv[1] = c->invW[1];
            T.last = (s == RK - 1) ? 1 : 0;
            T.dtNext = (T.last && cfg.constDt <= 0 && c->forcedDt <= 0) ? 1 : 0;
            T.cfl = cfg.cfl;
            T.dx = c->F.dx;
            T.dy = c->F.dy;
            if (T.dtNext) {   // accumulator of the next step's dt
                k_dt_init<<<1, 1, 0, c->stream>>>(c->ctl, cfg.maxDt);
                c->launches++;
            }
            T.velU = c->F.velU;
            T.velV = c->F.velV;
            T.pres = c->F.pres;
            T.unitScale = c->marchScale;
            double* const* in = (s == 0) ? U : (s == 1) ? c->tileB : c->tileC;
            double* const* out = (RK > 1 && s == RK - 1) ? U : (s == 0) ? c->tileB : c->tileC;
            for (int q = 0; q < 4; ++q) {
                T.in[q] = in[q];
                T.out[q] = out[q];
                T.u0[q] = (s > 0 && K.c2 != 0.0) ? U[q] : nullptr;
            }
            {
                int st = exchange_fields(c, const_cast<double* const*>(in), 4);
                if (st != SIFV_OK) return st;
            }
            if (tile2d_stage(T, c->stream, cfg.precision == SIFV_PREC_MIXED, c->launches,
                             c->profiling ? mark_cb : nullptr, c) != 0) {
                LAUNCH_CHECK(c);
                return fail(c, SIFV_ERR_CUDA, "tile launch failed");
            }
        }
        if (RK == 1 && tile2d_copy(c->ctl, c->tileB, U, c->ncells, c->stream, c->launches) != 0)
            return fail(c, SIFV_ERR_CUDA, "copy launch failed");
        launch_bc_prim(c);
        LAUNCH_CHECK(c);
        c->dtReady = cfg.constDt <= 0 && c->forcedDt <= 0;
        return SIFV_OK;
    }
    if (c->sweep) {
        SweepArgs A{};
        A.P = c->P;
        A.F = c->F;
        A.ctl = c->ctl;
        A.C.gamma = c->P.gamma;
        A.C.pInf = c->P.pInf;
        A.C.invGm1 = 1.0 / (c->P.gamma - 1.0);
        A.C.gPinf = c->P.gamma * c->P.pInf;
        A.eps = cfg.wenoEps;
        for (int q = 0; q < 5; ++q) A.rhs[q] = c->rhsBuf[q];
        A.rhoP = c->rhoP;
        for (int a = 0; a < 3; ++a) A.inv[a] = c->invW[a];
        for (int s = 0; s < cfg.RKOrder; ++s) {
            StageCoef K{};
            rk_coef(cfg.RKOrder, s, K);
            A.K.a1 = K.c1 / K.c4;
            A.K.a2 = K.c2 / K.c4;
            A.K.a3 = K.c3 / K.c4;
            A.K.save = (s == 0 && cfg.RKOrder > 1) ? 1 : 0;
            A.K.useU0 = (K.c2 != 0.0) ? 1 : 0;
            if (sweep_stage(A, c->stream, cfg.precision == SIFV_PREC_MIXED, c->launches,
                            c->profiling ? mark_cb : nullptr, c) != 0) {
                LAUNCH_CHECK(c);
                return fail(c, SIFV_ERR_CUDA, "sweep launch failed");
            }
        }
        if (sweep_finish_prim(c->P, c->F, c->ctl, c->stream, c->launches) != 0)
            return fail(c, SIFV_ERR_CUDA, "sweep launch failed");
        mark(c, "finish_prim");
        launch_bc_prim(c);
        LAUNCH_CHECK(c);
        return SIFV_OK;
    }
    for (int s = 0; s < cfg.RKOrder; ++s) {
        StageCoef K{};
        rk_coef(cfg.RKOrder, s, K);
        body_force(cfg, time, K);
        if (c->stageHook && c->stageHook(s, 0) != 0) return SIFV_ERR_CUDA;
        {
            int st = exchange_cons(c);
            if (st != SIFV_OK) return st;
        }
        launch_prim_bc(c);
        launch_ib_ghost(c);   // src/ExplicitSolver.cpp:116
        if (cfg.useIGR) {
            int st = igr_solve(c, step);
            if (st != SIFV_OK) return st;
        }
        for (int d = 0; d < P.dim; ++d) launch_face(c, d);
        if (P.visc) {
            for (int d = 0; d < P.dim; ++d) {
                long long nf = (long long)(P.nx + (d == 0)) * (P.ny + (d == 1)) * (P.nz + (d == 2));
                unsigned gf = blocks(nf, kCellThreads);
                if (d == 0) k_visc_face<0><<<gf, kCellThreads, 0, c->stream>>>(c->P, c->F, c->ctl);
                else if (d == 1) k_visc_face<1><<<gf, kCellThreads, 0, c->stream>>>(c->P, c->F, c->ctl);
                else k_visc_face<2><<<gf, kCellThreads, 0, c->stream>>>(c->P, c->F, c->ctl);
                c->launches++;
            }
            mark(c, "viscous");
        }
        if (P.cap) {
            for (int d = 0; d < P.dim; ++d) {
                long long nf = (long long)(P.nx + (d == 0)) * (P.ny + (d == 1)) * (P.nz + (d == 2));
                unsigned gf = blocks(nf, kCellThreads);
                if (d == 0) k_cap_face<0><<<gf, kCellThreads, 0, c->stream>>>(c->P, c->F, c->ctl);
                else if (d == 1) k_cap_face<1><<<gf, kCellThreads, 0, c->stream>>>(c->P, c->F, c->ctl);
                else k_cap_face<2><<<gf, kCellThreads, 0, c->stream>>>(c->P, c->F, c->ctl);
                c->launches++;
            }
            mark(c, "capillary");
        }
        if (!cfg.semiImplicit) {
            if (c->stageHook && c->stageHook(s, 1) != 0) return SIFV_ERR_CUDA;
            NPH_DISPATCH(c, (k_assemble<NPHV, 0><<<gc, kCellThreads, 0, c->stream>>>(c->P, c->F, c->ctl, K)));
            c->launches++;
            mark(c, "assemble");
            LAUNCH_CHECK(c);
            if (c->stageHook && c->stageHook(s, 2) != 0) return SIFV_ERR_CUDA;
        } else {
            NPH_DISPATCH(c, (k_assemble<NPHV, 1><<<gc, kCellThreads, 0, c->stream>>>(c->P, c->F, c->ctl, K)));
            c->launches++;
            mark(c, "assemble");
            {   // density + star velocity, src/SemiImplicitSolver.cpp:228-229
                int st = exchange_prim(c);
                if (st != SIFV_OK) return st;
            }
            launch_bc_prim(c);
            NPH_DISPATCH(c, (k_pressure_setup<NPHV><<<gc, kCellThreads, 0, c->stream>>>(c->P, c->F, c->ctl)));
            c->launches++;
            mark(c, "pressure_setup");
            LAUNCH_CHECK(c);
            int iters = 0;
            const double* pres = nullptr;
            int st = pressure_run(c, c->F.rho, c->F.rhoc2, c->F.pRhs, cfg.pressureTol, cfg.maxPressureIters, iters,
                                  pres);
            if (st != SIFV_OK) return st;
            c->lastIters = iters;
            if (iters >= cfg.maxPressureIters) {
                double last;
                unsigned long long b = c->ctlHost->res[iters - 1];
                std::memcpy(&last, &b, sizeof(double));
                if (!(last < cfg.pressureTol)) status = SIFV_NOT_CONVERGED;
            }
            if (c->exchangeFaces) {   // fillScalarGhosts(pressure_ / sigma, halo), src/SemiImplicitSolver.cpp:581-582
                int st = exchange_scalar(c, pres);
                if (st == SIFV_OK) st = exchange_scalar(c, c->F.sigma);
                if (st != SIFV_OK) return st;
            }
            NPH_DISPATCH(c, (k_correction<NPHV><<<gc, kCellThreads, 0, c->stream>>>(c->P, c->F, pres, c->ctl)));
            c->launches++;
            mark(c, "correction");
            {   // src/SemiImplicitSolver.cpp:642
                int st = exchange_prim(c);
                if (st != SIFV_OK) return st;
            }
            launch_bc_prim(c);
            LAUNCH_CHECK(c);
        }
    }
    if (!cfg.semiImplicit) {   // finalize: src/ExplicitSolver.cpp:192-200
        int st = exchange_cons(c);
        if (st != SIFV_OK) return st;
        launch_prim_bc(c);
        launch_ib_ghost(c);
    }
    LAUNCH_CHECK(c);
    return SIFV_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

void sifv_config_defaults(sifv_config_t* c) {
    std::memset(c, 0, sizeof(*c));
    c->dim = 3; c->nGhost = 2; c->RKOrder = 1; c->useIGR = 0; c->semiImplicit = 0;
    c->reconOrder = SIFV_WENO1; c->wenoEps = 1e-6;
    c->riemannSolver = SIFV_HLLC; c->eosKind = SIFV_EOS_IDEAL; c->gamma = 1.4; c->pInf = 0.0;
    c->cfl = 0.8; c->constDt = -1.0; c->maxDt = 1e-2; c->minDt = 1e-12;
    c->siCfl = 0.8; c->siMaxDt = 1e-2; c->siMinDt = 1e-12; c->maxPressureIters = 100; c->pressureTol = 1e-8;
    c->alphaCoeff = 1.0; c->IGRIters = 5; c->IGRWarmStartIters = 50;
    c->nPhases = 0; c->alphaMin = 1e-8;
    c->precision = SIFV_PREC_FP64;
    c->stSigma = 0.0; c->stEpsGradAlpha = 1e-8;
}

int sifv_config_validate(const sifv_config_t* cfg) {
    std::string m;
    int st = validate(cfg, m);
    if (st != SIFV_OK) g_err = m;
    return st;
}

const char* sifv_last_error(const sifv_ctx_t* ctx) { return ctx ? ctx->err.c_str() : g_err.c_str(); }

int sifv_create(const sifv_config_t* cfg, const sifv_mesh_t* mesh, int device, sifv_ctx_t** out) {
    if (!out || !cfg || !mesh) return fail(nullptr, SIFV_ERR_BAD_ARG, "null argument");
    *out = nullptr;
    std::string m;
    int st = validate(cfg, m);
    if (st != SIFV_OK) return fail(nullptr, st, m);
    const bool semiMixed = cfg->semiImplicit && cfg->precision == SIFV_PREC_MIXED;
    if (cfg->precision != SIFV_PREC_FP64 && !semiMixed) {
        bool bf = false;
        for (int d = 0; d < 3; ++d) bf = bf || cfg->bfA[d] != 0.0 || cfg->bfB[d] != 0.0;
        const bool visc = cfg->mu > 0.0 || cfg->nPhaseMu > 0 || cfg->stSigma > 0.0;
        if (cfg->semiImplicit || cfg->nPhases > 0 || cfg->useIGR || cfg->reconOrder != SIFV_WENO5 || bf || visc)
            return fail(nullptr, SIFV_ERR_UNSUPPORTED,
                        "SIFV_PREC_MIXED / SIFV_PREC_FP64_FAST run the explicit single-phase WENO5 step without "
                        "IGR, body force, viscosity or surface tension (the semi-implicit step takes SIFV_PREC_MIXED: "
                        "FP32 inner Jacobi sweeps); use SIFV_PREC_FP64 for this configuration");
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(nullptr, SIFV_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(nullptr, SIFV_ERR_BAD_ARG, "device index out of range");

    const int dim = cfg->dim;
    int nx = mesh->nx, ny = (dim >= 2) ? mesh->ny : 1, nz = (dim >= 3) ? mesh->nz : 1;
    int ng = cfg->nGhost;
    if (nx < 1 || ny < 1 || nz < 1) return fail(nullptr, SIFV_ERR_BAD_ARG, "mesh must have at least one cell per axis");
    if (nx < ng || (dim >= 2 && ny < ng) || (dim >= 3 && nz < ng))
        return fail(nullptr, SIFV_ERR_UNSUPPORTED, "every active axis needs at least nGhost cells");
    if (!mesh->xNodes || (dim >= 2 && !mesh->yNodes) || (dim >= 3 && !mesh->zNodes))
        return fail(nullptr, SIFV_ERR_BAD_ARG, "node arrays of the active axes are required");
    bool exchangeFaces = false;
    for (int f = 0; f < 6; ++f) {
        if (mesh->bc[f] == SIFV_BC_EXCHANGE && f < 2 * dim) {
            exchangeFaces = true;
            continue;
        }
        if (mesh->bc[f] < SIFV_BC_SYMMETRY || mesh->bc[f] > SIFV_BC_NOSLIPWALL)
            return fail(nullptr, SIFV_ERR_BAD_ARG, "unknown boundary condition");
    }
    if (exchangeFaces) {
        const bool visc = cfg->mu > 0.0 || cfg->nPhaseMu > 0 || cfg->stSigma > 0.0;
        if (visc)
            return fail(nullptr, SIFV_ERR_UNSUPPORTED,
                        "SIFV_BC_EXCHANGE faces (domain decomposition) are not supported with viscosity or surface "
                        "tension");
        if (cfg->semiImplicit && cfg->precision == SIFV_PREC_MIXED)
            return fail(nullptr, SIFV_ERR_UNSUPPORTED,
                        "SIFV_BC_EXCHANGE faces: the mixed-precision semi-implicit step is not supported (use "
                        "SIFV_PREC_FP64)");
        if (!cfg->semiImplicit && cfg->precision != SIFV_PREC_FP64 && (dim != 2 || cfg->useIGR))
            return fail(nullptr, SIFV_ERR_UNSUPPORTED,
                        "SIFV_BC_EXCHANGE faces on the fast / mixed path are supported in 2D without IGR (use "
                        "SIFV_PREC_FP64)");
    }

    sifv_ctx* c = new sifv_ctx();
    c->cfg = *cfg;
    c->device = device;
    c->exchangeFaces = exchangeFaces;
    {
        const char* e = std::getenv("SIFV_GS_MARCH");
        c->marchMode = (e && e[0] == '0') ? 0 : (e && e[0] == '1') ? 1 : -1;
        const char* es = std::getenv("SIFV_GS_MARCH_SEGMENTS");
        c->marchSegs = es ? std::atoi(es) : 0;
    }
    if (cudaSetDevice(device) != cudaSuccess) { delete c; return fail(nullptr, SIFV_ERR_CUDA, "cudaSetDevice failed"); }
    if (cudaStreamCreateWithFlags(&c->ownStream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return fail(nullptr, SIFV_ERR_CUDA, "cudaStreamCreate failed");
    }
    c->stream = c->ownStream;
    cudaEventCreate(&c->ev0);
    cudaEventCreate(&c->ev1);

    Params& P = c->P;
    P.dim = dim;
    P.nx = nx; P.ny = ny; P.nz = nz;
    P.ngx = ng; P.ngy = (dim >= 2) ? ng : 0; P.ngz = (dim >= 3) ? ng : 0;
    P.nxT = nx + 2 * P.ngx; P.nyT = ny + 2 * P.ngy; P.nzT = nz + 2 * P.ngz;
    for (int f = 0; f < 6; ++f) P.bc[f] = mesh->bc[f];
    P.nPh = cfg->nPhases;
    P.reconOrder = cfg->reconOrder;
    P.riemann = cfg->riemannSolver;
    P.includePressure = cfg->semiImplicit ? 0 : 1;
    P.useIGR = cfg->useIGR;
    P.reconSigma = (cfg->useIGR && cfg->riemannSolver == SIFV_LF) ? 1 : 0;
    P.eosStiffened = (cfg->eosKind == SIFV_EOS_STIFFENED) ? 1 : 0;
    P.RKOrder = cfg->RKOrder;
    P.wenoEps = cfg->wenoEps;
    P.gamma = cfg->gamma;
    P.pInf = (cfg->eosKind == SIFV_EOS_STIFFENED) ? cfg->pInf : 0.0;
    for (int p = 0; p < SIFV_MAX_PHASES; ++p) {
        P.phaseGamma[p] = cfg->phaseGamma[p];
        P.phasePInf[p] = cfg->phasePInf[p];
    }
    P.alphaMin = cfg->alphaMin;
    P.visc = (cfg->mu > 0.0 || cfg->nPhaseMu > 0) ? 1 : 0;
    P.perPhaseMu = cfg->nPhaseMu > 0 ? 1 : 0;
    P.mu = cfg->mu;
    for (int p = 0; p < SIFV_MAX_PHASES; ++p) P.phaseMu[p] = (p < cfg->nPhaseMu) ? cfg->phaseMu[p] : 0.0;
    P.cap = cfg->stSigma > 0.0 ? 1 : 0;
    P.stSigma = cfg->stSigma;
    P.stEps = cfg->stEpsGradAlpha;
    c->nphT = (cfg->nPhases == 0) ? 0 : (cfg->nPhases <= 2) ? 2 : 8;
    c->W = (cfg->reconOrder == SIFV_WENO1 || cfg->reconOrder == SIFV_UPWIND1) ? 1
         : (cfg->reconOrder == SIFV_WENO3 || cfg->reconOrder == SIFV_UPWIND3) ? 3 : 5;
    c->ncells = (size_t)P.nxT * P.nyT * P.nzT;
    c->nint = (size_t)nx * ny * nz;

    st = SIFV_OK;
    const size_t n = c->ncells;
    Fields& F = c->F;
    F.rho = dalloc(c, n, st); F.rhoU = dalloc(c, n, st); F.rhoE = dalloc(c, n, st);
    F.velU = dalloc(c, n, st); F.pres = dalloc(c, n, st); F.sigma = dalloc(c, n, st);
    if (dim >= 2) { F.rhoV = dalloc(c, n, st); F.velV = dalloc(c, n, st); }
    if (dim >= 3) { F.rhoW = dalloc(c, n, st); F.velW = dalloc(c, n, st); }
    for (int p = 0; p < cfg->nPhases; ++p) { F.alphaRho[p] = dalloc(c, n, st); F.alpha[p] = dalloc(c, n, st); }
    if (cfg->RKOrder > 1) {
        F.rho0 = dalloc(c, n, st); F.rhoU0 = dalloc(c, n, st); F.rhoE0 = dalloc(c, n, st); F.pres0 = dalloc(c, n, st);
        if (dim >= 2) F.rhoV0 = dalloc(c, n, st);
        if (dim >= 3) F.rhoW0 = dalloc(c, n, st);
        for (int p = 0; p < cfg->nPhases; ++p) { F.alphaRho0[p] = dalloc(c, n, st); F.alpha0[p] = dalloc(c, n, st); }
    }
    if (cfg->semiImplicit) {
        F.rhoUStar = dalloc(c, n, st); F.rhoEstar = dalloc(c, n, st); F.pAdvected = dalloc(c, n, st);
        F.rhoc2 = dalloc(c, n, st);
        if (dim >= 2) F.rhoVStar = dalloc(c, n, st);
        if (dim >= 3) F.rhoWStar = dalloc(c, n, st);
        F.pRhs = dalloc(c, n, st); F.divUstar = dalloc(c, n, st);
    }
    F.pA = dalloc(c, n, st); F.pB = dalloc(c, n, st);
    if (cfg->useIGR) { F.igrRhs = dalloc(c, n, st); F.igrDiag = dalloc(c, n, st); }
    for (int d = 0; d < dim; ++d) {
        size_t nf = (size_t)(nx + (d == 0)) * (ny + (d == 1)) * (nz + (d == 2));
        F.flux[d][FS_MASS] = dalloc(c, nf, st);
        F.flux[d][FS_MOMX] = dalloc(c, nf, st);
        if (dim >= 2) F.flux[d][FS_MOMY] = dalloc(c, nf, st);
        if (dim >= 3) F.flux[d][FS_MOMZ] = dalloc(c, nf, st);
        F.flux[d][FS_ENERGY] = dalloc(c, nf, st);
        if (cfg->semiImplicit) F.flux[d][FS_PFLUX] = dalloc(c, nf, st);
        if (cfg->semiImplicit || cfg->nPhases > 0) F.flux[d][FS_FVEL] = dalloc(c, nf, st);
        for (int p = 0; p < cfg->nPhases; ++p) {
            F.flux[d][FS_ALPHA + p] = dalloc(c, nf, st);
            F.flux[d][FS_AR + p] = dalloc(c, nf, st);
        }
        if (P.visc)
            for (int q = 0; q < 4; ++q) F.flux[d][FS_VISC + q] = (q == 0 || q == 3 || q < dim) ? dalloc(c, nf, st) : nullptr;
        if (P.cap)
            for (int q = 0; q < 4; ++q) F.flux[d][FS_CAP + q] = (q == 0 || q == 3 || q < dim) ? dalloc(c, nf, st) : nullptr;
    }
    // geometry: per-cell widths incl. ghosts, and IGR alpha/d^2
    static const double unit[2] = {0.0, 1.0};
    std::vector<double> xe = build_ext(mesh->xNodes, nx, P.ngx);
    std::vector<double> ye = build_ext((dim >= 2) ? mesh->yNodes : unit, ny, P.ngy);
    std::vector<double> ze = build_ext((dim >= 3) ? mesh->zNodes : unit, nz, P.ngz);
    auto centroids = [](const std::vector<double>& e, int ng, int n) {   // RectilinearMesh::cellCentroidX
        std::vector<double> cen(n);
        for (int i = 0; i < n; ++i) cen[i] = 0.5 * (e[i + ng] + e[i + ng + 1]);
        return cen;
    };
    c->cenX = centroids(xe, P.ngx, nx);
    c->cenY = centroids(ye, P.ngy, ny);
    c->cenZ = centroids(ze, P.ngz, nz);
    auto widths = [](const std::vector<double>& e) {
        std::vector<double> w(e.size() - 1);
        for (size_t i = 0; i + 1 < e.size(); ++i) w[i] = e[i + 1] - e[i];
        return w;
    };
    std::vector<double> dxv = widths(xe), dyv = widths(ye), dzv = widths(ze);
    auto uniform = [](const std::vector<double>& w, int ng, int n) {
        for (int i = 1; i < n; ++i)
            if (!(w[ng + i] == w[ng])) return false;
        return true;
    };
    c->uniformAxes = uniform(dxv, P.ngx, nx) && (dim < 2 || uniform(dyv, P.ngy, ny)) &&
                     (dim < 3 || uniform(dzv, P.ngz, nz));
    double dx0 = dxv[P.ngx];
    c->alphaIGR = cfg->alphaCoeff * dx0 * dx0;   // src/IGR.cpp:108
    auto a2 = [&](const std::vector<double>& w) {
        std::vector<double> r(w.size());
        for (size_t i = 0; i < w.size(); ++i) r[i] = c->alphaIGR * (1.0 / (w[i] * w[i]));
        return r;
    };
    std::vector<double> adx = a2(dxv), ady = a2(dyv), adz = a2(dzv);
    double* g[6];
    const std::vector<double>* src[6] = {&dxv, &dyv, &dzv, &adx, &ady, &adz};
    for (int q = 0; q < 6; ++q) {
        g[q] = dalloc(c, src[q]->size(), st);
        if (st == SIFV_OK)
            cudaMemcpyAsync(g[q], src[q]->data(), src[q]->size() * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    }
    F.dx = g[0]; F.dy = g[1]; F.dz = g[2]; F.adx2 = g[3]; F.ady2 = g[4]; F.adz2 = g[5];
    if (cfg->precision != SIFV_PREC_FP64 && !cfg->semiImplicit) {
        c->sweep = true;
        c->rhoP = dalloc(c, n, st);
        c->rhsBuf[0] = dalloc(c, n, st);
        c->rhsBuf[1] = dalloc(c, n, st);
        if (dim >= 2) c->rhsBuf[2] = dalloc(c, n, st);
        if (dim >= 3) c->rhsBuf[3] = dalloc(c, n, st);
        c->rhsBuf[4] = dalloc(c, n, st);
        const std::vector<double>* w[3] = {&dxv, &dyv, &dzv};
        for (int a = 0; a < 3; ++a) {
            std::vector<double> inv(w[a]->size());
            for (size_t q = 0; q < inv.size(); ++q) inv[q] = 1.0 / (*w[a])[q];
            c->invW[a] = dalloc(c, inv.size(), st);
            if (st == SIFV_OK)
                cudaMemcpyAsync(c->invW[a], inv.data(), inv.size() * sizeof(double), cudaMemcpyHostToDevice,
                                c->stream);
        }
        if (st == SIFV_OK) cudaStreamSynchronize(c->stream);   // host vectors above go out of scope
    }
    if (st == SIFV_OK) st = ensure_res(c, std::max(cfg->maxPressureIters, 1));
    if (st == SIFV_OK) {
        cudaError_t e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) st = fail(c, SIFV_ERR_CUDA, cudaGetErrorString(e));
    }
    if (st != SIFV_OK) {
        g_err = c->err;
        sifv_destroy(c);
        return st;
    }
    *out = c;
    return SIFV_OK;
}

int sifv_destroy(sifv_ctx_t* c) {
    if (!c) return SIFV_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (void* p : c->allocs) cudaFree(p);
    if (c->ctl) cudaFree(c->ctl);
    if (c->ctlHost) cudaFreeHost(c->ctlHost);
    if (c->sRho) { cudaFree(c->sRho); cudaFree(c->sRhoc2); cudaFree(c->sRhs); cudaFree(c->sP); }
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->ownStream) cudaStreamDestroy(c->ownStream);
    for (double* p : c->adjCkpt) cudaFree(p);
    if (c->adjStage) cudaFree(c->adjStage);
    if (c->loopLog) cudaFree(c->loopLog);
    for (void* p : c->ibAllocs) cudaFree(p);
    delete c;
    return SIFV_OK;
}

int sifv_extents(const sifv_ctx_t* c, int* nx, int* ny, int* nz) {
    if (!c) return fail(nullptr, SIFV_ERR_BAD_ARG, "null context");
    *nx = c->P.nxT; *ny = c->P.nyT; *nz = c->P.nzT;
    return SIFV_OK;
}

size_t sifv_total_cells(const sifv_ctx_t* c) { return c ? c->ncells : 0; }

int sifv_set_stream(sifv_ctx_t* c, void* stream) {
    c->stream = stream ? static_cast<cudaStream_t>(stream) : c->ownStream;
    return SIFV_OK;
}

int sifv_autotune(sifv_ctx_t* c, int reps, int* choice) {
    if (!c || reps <= 0 || !choice) return fail(c, SIFV_ERR_BAD_ARG, "bad argument");
    *choice = 0;
    if (!(c->sweep && c->P.dim == 2)) return SIFV_OK;   // only the 2D fused stage has a shape to tune
    cudaSetDevice(c->device);
    if (!c->tileB[0]) {
        int sa = SIFV_OK;
        for (int q = 0; q < 4; ++q) {
            c->tileB[q] = dalloc(c, c->ncells, sa);
            c->tileC[q] = dalloc(c, c->ncells, sa);
        }
        if (sa != SIFV_OK) return sa;
    }
    // probe: the first stage of a step from the current state into the scratch
    // state (the state itself is not written), no primitives, no dt
    const sifv_config_t& cfg = c->cfg;
    StageCoef K{};
    rk_coef(cfg.RKOrder, 0, K);
    TileArgs T{};
    T.P = c->P;
    T.C.gamma = c->P.gamma;
    T.C.pInf = c->P.pInf;
    T.C.invGm1 = 1.0 / (c->P.gamma - 1.0);
    T.C.gPinf = c->P.gamma * c->P.pInf;
    T.eps = cfg.wenoEps;
    T.ctl = c->ctl;
    T.a1 = K.c1 / K.c4;
    T.a2 = K.c2 / K.c4;
    T.a3 = K.c3 / K.c4;
    T.inv[0] = c->invW[0];
    T.inv[1] = c->invW[1];
    double* U[4] = {c->F.rho, c->F.rhoU, c->F.rhoV, c->F.rhoE};
    for (int q = 0; q < 4; ++q) {
        T.in[q] = U[q];
        T.out[q] = c->tileB[q];
        T.u0[q] = nullptr;
    }
    CUDA_TRY(c, cudaMemsetAsync(&c->ctl->skip, 0, sizeof(int), c->stream));
    const bool mixed = cfg.precision == SIFV_PREC_MIXED;
    int launches = 0, best = 1;
    float bestMs = 1e30f;
    for (int scale = 1; scale <= 4; ++scale) {
        T.unitScale = scale;
        if (tile2d_stage(T, c->stream, mixed, launches) != 0) return fail(c, SIFV_ERR_CUDA, "autotune launch failed");
        CUDA_TRY(c, cudaEventRecord(c->ev0, c->stream));
        for (int r = 0; r < reps; ++r)
            if (tile2d_stage(T, c->stream, mixed, launches) != 0)
                return fail(c, SIFV_ERR_CUDA, "autotune launch failed");
        CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
        CUDA_TRY(c, cudaEventSynchronize(c->ev1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        if (ms < bestMs) {
            bestMs = ms;
            best = scale;
        }
    }
    c->marchScale = best;
    *choice = best;
    return SIFV_OK;
}

int sifv_set_work_units(sifv_ctx_t* c, int unitsPerWarp) {
    if (!c || unitsPerWarp < 1 || unitsPerWarp > 4) return fail(c, SIFV_ERR_BAD_ARG, "units per warp must be 1-4");
    c->marchScale = unitsPerWarp;
    return SIFV_OK;
}

int sifv_set_comm(sifv_ctx_t* c, const sifv_comm_t* comm) {
    if (!c) return fail(nullptr, SIFV_ERR_BAD_ARG, "null context");
    c->comm = comm ? *comm : sifv_comm_t{};
    return SIFV_OK;
}

int sifv_synchronize(sifv_ctx_t* c) {
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SIFV_OK;
}

int sifv_field_device_ptr(sifv_ctx_t* c, int field, double** dptr) {
    double* p = field_ptr(c, field);
    if (!p) return fail(c, SIFV_ERR_BAD_ARG, "field not allocated for this configuration");
    *dptr = p;
    return SIFV_OK;
}

int sifv_set_field(sifv_ctx_t* c, int field, const double* src, int onDevice) {
    double* p = field_ptr(c, field);
    if (!p) return fail(c, SIFV_ERR_BAD_ARG, "field not allocated for this configuration");
    cudaSetDevice(c->device);
    CUDA_TRY(c, cudaMemcpyAsync(p, src, c->ncells * sizeof(double),
                                onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SIFV_OK;
}

int sifv_get_field(sifv_ctx_t* c, int field, double* dst, int onDevice) {
    double* p = field_ptr(c, field);
    if (!p) return fail(c, SIFV_ERR_BAD_ARG, "field not allocated for this configuration");
    cudaSetDevice(c->device);
    CUDA_TRY(c, cudaMemcpyAsync(dst, p, c->ncells * sizeof(double),
                                onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SIFV_OK;
}

int sifv_step(sifv_ctx_t* c, int step, double time, double targetDt, double* dtOut) {
    if (!c) return fail(nullptr, SIFV_ERR_BAD_ARG, "null context");
    cudaSetDevice(c->device);
    c->dtReady = false;   // the state may have changed since the last call
    c->launches = 0;
    CUDA_TRY(c, cudaMemsetAsync(&c->ctl->skip, 0, sizeof(int), c->stream));
    CUDA_TRY(c, cudaEventRecord(c->ev0, c->stream));
    int status = SIFV_OK;
    int st = enqueue_step(c, step, time, targetDt, false, status);
    if (st != SIFV_OK) return st;
    CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(c->ctlHost, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    cudaEventElapsedTime(&c->lastMs, c->ev0, c->ev1);
    c->lastLaunches = c->launches;
    if (dtOut) *dtOut = c->ctlHost->dt;
    return status;
}

int sifv_advance(sifv_ctx_t* c, int step0, double time0, double tEnd, int nSteps, double* timeOut, int* stepsTaken) {
    if (!c) return fail(nullptr, SIFV_ERR_BAD_ARG, "null context");
    if (c->cfg.semiImplicit) return fail(c, SIFV_ERR_UNSUPPORTED, "sifv_advance runs the explicit step only");
    if (c->cfg.useIGR) return fail(c, SIFV_ERR_UNSUPPORTED, "sifv_advance does not run IGR; use sifv_step");
    if (has_body_force(c->cfg)) return fail(c, SIFV_ERR_UNSUPPORTED, "sifv_advance does not run body forces");
    cudaSetDevice(c->device);
    c->dtReady = false;   // the state may have changed since the last call
    c->launches = 0;
    Ctl h{};
    h.time = time0;
    h.tEnd = (tEnd > 0) ? tEnd : INFINITY;
    CUDA_TRY(c, cudaMemcpyAsync(c->ctl, &h, sizeof(Ctl), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaEventRecord(c->ev0, c->stream));
    int status = SIFV_OK;
    for (int q = 0; q < nSteps; ++q) {
        int st = enqueue_step(c, step0 + q, time0, -1.0, true, status);
        if (st != SIFV_OK) return st;
        k_time_advance<<<1, 1, 0, c->stream>>>(c->ctl);
        c->launches++;
    }
    CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(c->ctlHost, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    cudaEventElapsedTime(&c->lastMs, c->ev0, c->ev1);
    c->lastLaunches = c->launches;
    if (timeOut) *timeOut = c->ctlHost->time;
    if (stepsTaken) *stepsTaken = c->ctlHost->stepsTaken;
    return SIFV_OK;
}

int sifv_profile_step(sifv_ctx_t* c, int step, double time, double targetDt, char* names, int namesCap,
                      double* ms, int* counts, int maxFamilies, int* nFamilies) {
    if (!c || !names || !ms || !counts || !nFamilies) return fail(c, SIFV_ERR_BAD_ARG, "null argument");
    cudaSetDevice(c->device);
    c->dtReady = false;   // the state may have changed since the last call
    c->launches = 0;
    c->marks.clear();
    c->profiling = true;
    cudaEvent_t start;
    cudaEventCreate(&start);
    CUDA_TRY(c, cudaMemsetAsync(&c->ctl->skip, 0, sizeof(int), c->stream));
    cudaEventRecord(start, c->stream);
    int status = SIFV_OK;
    int st = enqueue_step(c, step, time, targetDt, false, status);
    c->profiling = false;
    cudaError_t e = cudaStreamSynchronize(c->stream);
    std::vector<std::string> fam;
    std::vector<double> tot;
    std::vector<int> cnt;
    cudaEvent_t prev = start;
    for (auto& m : c->marks) {
        float t = 0.f;
        cudaEventElapsedTime(&t, prev, m.second);
        size_t k = 0;
        while (k < fam.size() && fam[k] != m.first) ++k;
        if (k == fam.size()) { fam.push_back(m.first); tot.push_back(0.0); cnt.push_back(0); }
        tot[k] += t;
        cnt[k] += 1;
        prev = m.second;
    }
    for (auto& m : c->marks) cudaEventDestroy(m.second);
    c->marks.clear();
    cudaEventDestroy(start);
    if (st != SIFV_OK) return st;
    if (e != cudaSuccess) return fail(c, SIFV_ERR_CUDA, cudaGetErrorString(e));
    std::string joined;
    int n = std::min<int>((int)fam.size(), maxFamilies);
    for (int k = 0; k < n; ++k) {
        ms[k] = tot[k];
        counts[k] = cnt[k];
        joined += fam[k];
        if (k + 1 < n) joined += "\n";
    }
    std::snprintf(names, (size_t)namesCap, "%s", joined.c_str());
    *nFamilies = n;
    return status;
}

int sifv_last_pressure_iterations(const sifv_ctx_t* c, int* iters) {
    *iters = c->lastIters;
    return SIFV_OK;
}

int sifv_last_step_stats(const sifv_ctx_t* c, double* ms, int* launches) {
    *ms = c->lastMs;
    *launches = c->lastLaunches;
    return SIFV_OK;
}

int sifv_pressure_solve(sifv_ctx_t* c, const double* rho, const double* rhoc2, const double* rhs, double* pressure,
                        double dt, double tol, int maxIter, int onDevice, int* iters) {
    if (!c || !rho || !rhoc2 || !rhs || !pressure || !iters) return fail(c, SIFV_ERR_BAD_ARG, "null argument");
    if (maxIter <= 0) return fail(c, SIFV_ERR_BAD_ARG, "maxIter must be > 0");
    cudaSetDevice(c->device);
    const size_t bytes = c->ncells * sizeof(double);
    const double *dRho = rho, *dRhoc2 = rhoc2, *dRhs = rhs;
    double* dP = pressure;
    if (!onDevice) {
        if (!c->sRho) {
            CUDA_TRY(c, cudaMalloc(&c->sRho, bytes));
            CUDA_TRY(c, cudaMalloc(&c->sRhoc2, bytes));
            CUDA_TRY(c, cudaMalloc(&c->sRhs, bytes));
            CUDA_TRY(c, cudaMalloc(&c->sP, bytes));
        }
        CUDA_TRY(c, cudaMemcpyAsync(c->sRho, rho, bytes, cudaMemcpyHostToDevice, c->stream));
        CUDA_TRY(c, cudaMemcpyAsync(c->sRhoc2, rhoc2, bytes, cudaMemcpyHostToDevice, c->stream));
        CUDA_TRY(c, cudaMemcpyAsync(c->sRhs, rhs, bytes, cudaMemcpyHostToDevice, c->stream));
        CUDA_TRY(c, cudaMemcpyAsync(c->sP, pressure, bytes, cudaMemcpyHostToDevice, c->stream));
        dRho = c->sRho; dRhoc2 = c->sRhoc2; dRhs = c->sRhs; dP = c->sP;
    }
    CUDA_TRY(c, cudaMemcpyAsync(c->F.pA, dP, bytes, cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(&c->ctl->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    int n = 0;
    const double* res = nullptr;
    int st = pressure_run(c, dRho, dRhoc2, dRhs, tol, maxIter, n, res);
    if (st != SIFV_OK) return st;
    if (c->lastInPlace)   // the whole array (ghosts as the reference's array leaves them)
        CUDA_TRY(c, cudaMemcpyAsync(dP, res, bytes, cudaMemcpyDeviceToDevice, c->stream));
    else
        k_jacobi_finish<<<blocks((long long)c->nint, kCellThreads), kCellThreads, 0, c->stream>>>(
            c->P, c->F.pA, c->F.pB, dP, c->ctl, maxIter);
    LAUNCH_CHECK(c);
    if (!onDevice) CUDA_TRY(c, cudaMemcpyAsync(pressure, dP, bytes, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    *iters = n;
    if (n >= maxIter) {
        double last;
        unsigned long long b = c->ctlHost->res[n - 1];
        std::memcpy(&last, &b, sizeof(double));
        if (!(last < tol)) return SIFV_NOT_CONVERGED;
    }
    return SIFV_OK;
}

int sifv_igr_solve(sifv_ctx_t* c, int step) {
    if (!c->cfg.useIGR) return fail(c, SIFV_ERR_BAD_ARG, "useIGR is off in this configuration");
    cudaSetDevice(c->device);
    int st = igr_solve(c, step);
    if (st != SIFV_OK) return st;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SIFV_OK;
}

int sifv_acoustic_dt(sifv_ctx_t* c, double cfl, double maxDt, double* dt) {
    cudaSetDevice(c->device);
    CUDA_TRY(c, cudaMemsetAsync(&c->ctl->skip, 0, sizeof(int), c->stream));
    k_dt_init<<<1, 1, 0, c->stream>>>(c->ctl, maxDt);
    Fields Fa = c->F;
    Fa.solid = nullptr;   // the standalone reduction takes every interior cell
    NPH_DISPATCH(c, (k_dt_acoustic<NPHV><<<blocks((long long)c->nint, kCellThreads), kCellThreads, 0, c->stream>>>(
                         c->P, Fa, c->ctl, cfl)));
    LAUNCH_CHECK(c);
    CUDA_TRY(c, cudaMemcpyAsync(c->ctlHost, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    unsigned long long b = c->ctlHost->dtBits;
    std::memcpy(dt, &b, sizeof(double));
    return SIFV_OK;
}

int sifv_advective_dt(sifv_ctx_t* c, double cfl, double maxDt, double* dt) {
    cudaSetDevice(c->device);
    CUDA_TRY(c, cudaMemsetAsync(&c->ctl->skip, 0, sizeof(int), c->stream));
    k_dt_init<<<1, 1, 0, c->stream>>>(c->ctl, maxDt);
    k_dt_advective<<<blocks((long long)c->nint, kCellThreads), kCellThreads, 0, c->stream>>>(c->P, c->F, c->ctl, cfl);
    LAUNCH_CHECK(c);
    CUDA_TRY(c, cudaMemcpyAsync(c->ctlHost, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    unsigned long long b = c->ctlHost->dtBits;
    std::memcpy(dt, &b, sizeof(double));
    return SIFV_OK;
}

int sifv_set_pressure_solver(sifv_ctx_t* c, int kind) {
    if (!c) return fail(nullptr, SIFV_ERR_BAD_ARG, "null context");
    if (kind != SIFV_PRESSURE_JACOBI && kind != SIFV_PRESSURE_GAUSS_SEIDEL && kind != SIFV_PRESSURE_PCG_MG)
        return fail(c, SIFV_ERR_BAD_ARG, "unknown pressure solver");
    c->pressureKind = kind;
    return SIFV_OK;
}

int sifv_convert_cons_to_prim(sifv_ctx_t* c) {
    // interior cells only, ghosts untouched (as the reference)
    cudaSetDevice(c->device);
    CUDA_TRY(c, cudaMemsetAsync(&c->ctl->skip, 0, sizeof(int), c->stream));
    launch_prim_bc(c, true);
    LAUNCH_CHECK(c);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SIFV_OK;
}

int sifv_apply_bc(sifv_ctx_t* c) {
    cudaSetDevice(c->device);
    launch_bc_prim(c);
    LAUNCH_CHECK(c);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SIFV_OK;
}

}  // extern "C"

// ===========================================================================
// Discrete adjoint and tangent of the explicit step
// ===========================================================================
namespace {

int nv_of(const sifv_ctx* c) { return c->cfg.dim + 2; }

// slot q of the conservative state: 0 rho, 1..dim momenta, dim + 1 energy
double* cons_field(sifv_ctx* c, int q) {
    const int dim = c->cfg.dim;
    if (q == 0) return c->F.rho;
    if (q == dim + 1) return c->F.rhoE;
    return (q == 1) ? c->F.rhoU : (q == 2) ? c->F.rhoV : c->F.rhoW;
}

int cons_slot(const sifv_ctx* c, int field) {
    const int dim = c->cfg.dim;
    switch (field) {
        case SIFV_F_RHO: return 0;
        case SIFV_F_RHOU: return 1;
        case SIFV_F_RHOV: return dim >= 2 ? 2 : -1;
        case SIFV_F_RHOW: return dim >= 3 ? 3 : -1;
        case SIFV_F_RHOE: return dim + 1;
        default: return -1;
    }
}

int adjoint_supported(sifv_ctx* c) {
    const sifv_config_t& g = c->cfg;
    if (g.semiImplicit || g.useIGR || g.nPhases > 0 || has_body_force(g) || g.precision != SIFV_PREC_FP64 ||
        (g.reconOrder != SIFV_WENO5 && g.reconOrder != SIFV_UPWIND5) || g.nGhost > 7 || c->P.visc || c->P.cap ||
        c->ib.count > 0)
        return fail(c, SIFV_ERR_UNSUPPORTED,
                    "the adjoint / tangent covers the explicit single-phase WENO5 / UPWIND5 step in SIFV_PREC_FP64 "
                    "without IGR, body force, viscosity, surface tension or immersed bodies (nGhost <= 7)");
    return SIFV_OK;
}

size_t face_count(const Params& P, int d) {
    return (size_t)(P.nx + (d == 0)) * (P.ny + (d == 1)) * (P.nz + (d == 2));
}

int ensure_adj_arrays(sifv_ctx* c, bool tangent) {
    int st = SIFV_OK;
    const int nv = nv_of(c), dim = c->cfg.dim;
    if (!tangent && !c->lam[0]) {
        for (int q = 0; q < nv; ++q) {
            c->lam[q] = dalloc(c, c->ncells, st);
            c->acc0[q] = dalloc(c, c->ncells, st);
        }
        for (int d = 0; d < dim; ++d) c->share[d] = dalloc(c, face_count(c->P, d) * 10 * nv, st);
    }
    if (tangent && !c->tan[0]) {
        for (int q = 0; q < nv; ++q) {
            c->tan[q] = dalloc(c, c->ncells, st);
            c->tan0[q] = dalloc(c, c->ncells, st);
            c->tanW[q] = dalloc(c, c->ncells, st);
        }
        for (int d = 0; d < dim; ++d)
            for (int q = 0; q < nv; ++q) c->tanF[d][q] = dalloc(c, face_count(c->P, d), st);
    }
    return st;
}

AdjArgs adj_args(sifv_ctx* c) {
    AdjArgs A{};
    A.P = c->P;
    A.F = c->F;
    for (int q = 0; q < 5; ++q) {
        A.lam[q] = c->lam[q];
        A.acc0[q] = c->acc0[q];
        A.tan[q] = c->tan[q];
        A.tan0[q] = c->tan0[q];
        A.tanW[q] = c->tanW[q];
    }
    for (int d = 0; d < 3; ++d) {
        A.share[d] = c->share[d];
        for (int q = 0; q < 5; ++q) A.tanF[d][q] = c->tanF[d][q];
    }
    A.fp32 = c->adjFp32;
    return A;
}

void set_stage_coef(AdjArgs& A, int order, int s) {
    StageCoef K{};
    rk_coef(order, s, K);
    A.a1 = K.c1 / K.c4;
    A.a2 = K.c2 / K.c4;
    A.a3 = K.c3 / K.c4;
}

void free_checkpoints(sifv_ctx* c) {
    for (double* p : c->adjCkpt) cudaFree(p);
    c->adjCkpt.clear();
    c->adjDts.clear();
    c->adjReady = false;
}

// copy of the conservative state appended to the checkpoint list
int push_checkpoint(sifv_ctx* c) {
    for (int q = 0; q < nv_of(c); ++q) {
        void* p = nullptr;
        if (cudaMalloc(&p, c->ncells * sizeof(double)) != cudaSuccess)
            return fail(c, SIFV_ERR_CUDA, "cudaMalloc for an adjoint checkpoint failed");
        c->adjCkpt.push_back(static_cast<double*>(p));
        CUDA_TRY(c, cudaMemcpyAsync(p, cons_field(c, q), c->ncells * sizeof(double), cudaMemcpyDeviceToDevice,
                                    c->stream));
    }
    return SIFV_OK;
}

int load_checkpoint(sifv_ctx* c, size_t idx) {
    const int nv = nv_of(c);
    for (int q = 0; q < nv; ++q)
        CUDA_TRY(c, cudaMemcpyAsync(cons_field(c, q), c->adjCkpt[idx * nv + q], c->ncells * sizeof(double),
                                    cudaMemcpyDeviceToDevice, c->stream));
    return SIFV_OK;
}

struct HookGuard {
    sifv_ctx* c;
    ~HookGuard() {
        c->stageHook = nullptr;
        c->forcedDt = -1.0;
    }
};

// Forward steps from the current state, either with a given time-step
// sequence or with the CFL dt and targetDt = tEnd - t; optionally records
// the sequence and a checkpoint every `every` steps.
int run_forward(sifv_ctx* c, int step0, double time0, double tEnd, int maxSteps, const double* sched, int nSched,
                int every, bool record, double& timeOut, int& stepsOut) {
    double t = time0;
    int q = 0;
    for (;;) {
        if (sched) {
            if (q >= nSched) break;
        } else if (!(t < tEnd) || (maxSteps > 0 && q >= maxSteps)) {
            break;
        }
        if (record && q % every == 0) {
            int st = push_checkpoint(c);
            if (st != SIFV_OK) return st;
        }
        c->forcedDt = sched ? sched[q] : -1.0;
        CUDA_TRY(c, cudaMemsetAsync(&c->ctl->skip, 0, sizeof(int), c->stream));
        int status = SIFV_OK;
        int st = enqueue_step(c, step0 + q, t, sched ? -1.0 : tEnd - t, false, status);
        c->forcedDt = -1.0;
        if (st != SIFV_OK) return st;
        CUDA_TRY(c, cudaMemcpyAsync(c->ctlHost, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        const double dt = c->ctlHost->dt;
        if (!(dt > 0.0)) return fail(c, SIFV_ERR_NAN, "time step not positive (state blew up)");
        if (record) c->adjDts.push_back(dt);
        t += dt;
        ++q;
    }
    timeOut = t;
    stepsOut = q;
    return SIFV_OK;
}

int check_ctx(sifv_ctx* c) {
    if (!c) return fail(nullptr, SIFV_ERR_BAD_ARG, "null context");
    cudaSetDevice(c->device);
    return adjoint_supported(c);
}

int copy_slot(sifv_ctx* c, double* const* arr, int field, const double* src, double* dst, int onDevice) {
    const int q = cons_slot(c, field);
    if (q < 0) return fail(c, SIFV_ERR_BAD_ARG, "field is not a conservative variable of this configuration");
    const size_t bytes = c->ncells * sizeof(double);
    if (src)
        CUDA_TRY(c, cudaMemcpyAsync(arr[q], src, bytes, onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                    c->stream));
    else
        CUDA_TRY(c, cudaMemcpyAsync(dst, arr[q], bytes, onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                    c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SIFV_OK;
}

}  // namespace

extern "C" {

int sifv_adjoint_forward(sifv_ctx_t* c, int step0, double time0, double tEnd, int maxSteps, int checkpointEvery,
                         const double* dtSchedule, int nSchedule, double* timeOut, int* stepsOut) {
    int st = check_ctx(c);
    if (st != SIFV_OK) return st;
    if (checkpointEvery <= 0) return fail(c, SIFV_ERR_BAD_ARG, "checkpointEvery must be > 0");
    if (!dtSchedule && !(tEnd < 1e300) && maxSteps <= 0)
        return fail(c, SIFV_ERR_BAD_ARG, "tEnd must be finite when there is no step limit");
    free_checkpoints(c);
    c->adjEvery = checkpointEvery;
    HookGuard guard{c};
    double t = 0.0;
    int n = 0;
    st = run_forward(c, step0, time0, tEnd, maxSteps, dtSchedule, nSchedule, checkpointEvery, true, t, n);
    if (st != SIFV_OK) {
        free_checkpoints(c);
        return st;
    }
    st = push_checkpoint(c);   // final state, restored after the reverse sweep
    if (st != SIFV_OK) {
        free_checkpoints(c);
        return st;
    }
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->adjReady = true;
    if (timeOut) *timeOut = t;
    if (stepsOut) *stepsOut = n;
    return SIFV_OK;
}

int sifv_adjoint_schedule(const sifv_ctx_t* c, double* dts, int cap, int* n) {
    if (!c || !n) return SIFV_ERR_BAD_ARG;
    *n = (int)c->adjDts.size();
    if (dts) std::memcpy(dts, c->adjDts.data(), sizeof(double) * std::min<size_t>(cap > 0 ? cap : 0, c->adjDts.size()));
    return SIFV_OK;
}

int sifv_adjoint_set_precision(sifv_ctx_t* c, int precision) {
    if (!c) return fail(nullptr, SIFV_ERR_BAD_ARG, "null context");
    if (precision != SIFV_PREC_FP64 && precision != SIFV_PREC_MIXED)
        return fail(c, SIFV_ERR_BAD_ARG, "the reverse sweep runs in SIFV_PREC_FP64 or SIFV_PREC_MIXED");
    c->adjFp32 = (precision == SIFV_PREC_MIXED) ? 1 : 0;
    return SIFV_OK;
}

int sifv_adjoint_set_seed(sifv_ctx_t* c, int field, const double* src, int onDevice) {
    int st = check_ctx(c);
    if (st != SIFV_OK) return st;
    if (!src) return fail(c, SIFV_ERR_BAD_ARG, "null seed");
    st = ensure_adj_arrays(c, false);
    if (st != SIFV_OK) return st;
    return copy_slot(c, c->lam, field, src, nullptr, onDevice);
}

int sifv_adjoint_get_gradient(sifv_ctx_t* c, int field, double* dst, int onDevice) {
    int st = check_ctx(c);
    if (st != SIFV_OK) return st;
    if (!dst) return fail(c, SIFV_ERR_BAD_ARG, "null output");
    st = ensure_adj_arrays(c, false);
    if (st != SIFV_OK) return st;
    return copy_slot(c, c->lam, field, nullptr, dst, onDevice);
}

int sifv_adjoint_backward(sifv_ctx_t* c, double* deviceMs) {
    int st = check_ctx(c);
    if (st != SIFV_OK) return st;
    if (!c->adjReady) return fail(c, SIFV_ERR_BAD_ARG, "no recorded forward run: call sifv_adjoint_forward first");
    st = ensure_adj_arrays(c, false);
    if (st != SIFV_OK) return st;
    const int nv = nv_of(c), RK = c->cfg.RKOrder, K = c->adjEvery, dim = c->cfg.dim;
    const int nSteps = (int)c->adjDts.size();
    const size_t nc = c->ncells;
    const size_t need = (size_t)K * RK * nv * nc;
    if (c->adjStageCap < need) {
        if (c->adjStage) cudaFree(c->adjStage);
        c->adjStage = nullptr;
        c->adjStageCap = 0;
        void* p = nullptr;
        if (cudaMalloc(&p, need * sizeof(double)) != cudaSuccess)
            return fail(c, SIFV_ERR_CUDA, "cudaMalloc for the adjoint stage states failed (lower checkpointEvery)");
        c->adjStage = static_cast<double*>(p);
        c->adjStageCap = need;
    }
    for (int q = 0; q < nv; ++q) CUDA_TRY(c, cudaMemsetAsync(c->acc0[q], 0, nc * sizeof(double), c->stream));
    CUDA_TRY(c, cudaEventRecord(c->ev0, c->stream));
    HookGuard guard{c};
    const int nSeg = (nSteps + K - 1) / K;
    for (int seg = nSeg - 1; seg >= 0; --seg) {
        const int q0 = seg * K, q1 = std::min(q0 + K, nSteps);
        st = load_checkpoint(c, (size_t)seg);
        if (st != SIFV_OK) return st;
        // recompute the segment, keeping every stage input
        int qLocal = 0;
        c->stageHook = [&](int s, int phase) -> int {
            if (phase != 0) return 0;
            double* dst = c->adjStage + (size_t)(qLocal * RK + s) * nv * nc;
            for (int v = 0; v < nv; ++v)
                if (cudaMemcpyAsync(dst + v * nc, cons_field(c, v), nc * sizeof(double), cudaMemcpyDeviceToDevice,
                                    c->stream) != cudaSuccess)
                    return -1;
            return 0;
        };
        for (int q = q0; q < q1; ++q) {
            qLocal = q - q0;
            c->forcedDt = c->adjDts[q];
            CUDA_TRY(c, cudaMemsetAsync(&c->ctl->skip, 0, sizeof(int), c->stream));
            int status = SIFV_OK;
            st = enqueue_step(c, q, 0.0, -1.0, false, status);
            if (st != SIFV_OK) return st;
        }
        c->stageHook = nullptr;
        c->forcedDt = -1.0;
        // reverse through the segment
        for (int q = q1 - 1; q >= q0; --q) {
            for (int s = RK - 1; s >= 0; --s) {
                Fields Fs = c->F;
                double* src = c->adjStage + (size_t)((q - q0) * RK + s) * nv * nc;
                Fs.rho = src;
                Fs.rhoU = src + nc;
                if (dim >= 2) Fs.rhoV = src + 2 * nc;
                if (dim >= 3) Fs.rhoW = src + 3 * nc;
                Fs.rhoE = src + (size_t)(dim + 1) * nc;
                k_prim_bc<0><<<blocks((long long)nc, kCellThreads), kCellThreads, 0, c->stream>>>(c->P, Fs, nullptr, 0);
                AdjArgs A = adj_args(c);
                A.F = Fs;
                set_stage_coef(A, RK, s);
                A.dt = c->adjDts[q];
                A.dtDev = nullptr;
                A.stage0 = (s == 0) ? 1 : 0;
                if (adjoint_stage(A, c->stream) != 0) {
                    LAUNCH_CHECK(c);
                    return fail(c, SIFV_ERR_CUDA, "adjoint launch failed");
                }
            }
        }
        LAUNCH_CHECK(c);
    }
    CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
    // the context's state is the end of the forward run again
    st = load_checkpoint(c, (size_t)nSeg);
    if (st != SIFV_OK) return st;
    launch_prim_bc(c);
    for (int q = 0; q < nv; ++q)
        if (zero_ghosts(c->P, c->lam[q], c->stream) != 0) return fail(c, SIFV_ERR_CUDA, "launch failed");
    LAUNCH_CHECK(c);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (deviceMs) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        *deviceMs = ms;
    }
    return SIFV_OK;
}

int sifv_tangent_set_direction(sifv_ctx_t* c, int field, const double* src, int onDevice) {
    int st = check_ctx(c);
    if (st != SIFV_OK) return st;
    if (!src) return fail(c, SIFV_ERR_BAD_ARG, "null direction");
    st = ensure_adj_arrays(c, true);
    if (st != SIFV_OK) return st;
    return copy_slot(c, c->tan, field, src, nullptr, onDevice);
}

int sifv_tangent_get(sifv_ctx_t* c, int field, double* dst, int onDevice) {
    int st = check_ctx(c);
    if (st != SIFV_OK) return st;
    if (!dst) return fail(c, SIFV_ERR_BAD_ARG, "null output");
    st = ensure_adj_arrays(c, true);
    if (st != SIFV_OK) return st;
    return copy_slot(c, c->tan, field, nullptr, dst, onDevice);
}

int sifv_tangent_forward(sifv_ctx_t* c, int step0, double time0, double tEnd, int maxSteps, const double* dtSchedule,
                         int nSchedule, double* timeOut, int* stepsOut) {
    int st = check_ctx(c);
    if (st != SIFV_OK) return st;
    if (!dtSchedule && !(tEnd < 1e300) && maxSteps <= 0)
        return fail(c, SIFV_ERR_BAD_ARG, "tEnd must be finite when there is no step limit");
    st = ensure_adj_arrays(c, true);
    if (st != SIFV_OK) return st;
    const int RK = c->cfg.RKOrder;
    HookGuard guard{c};
    c->stageHook = [&](int s, int phase) -> int {
        if (phase == 0) return 0;
        AdjArgs A = adj_args(c);
        set_stage_coef(A, RK, s);
        A.dtDev = &c->ctl->dt;
        if (phase == 1) return tangent_faces(A, c->stream);
        return tangent_update(A, (s == 0 && RK > 1) ? 1 : 0, c->stream);
    };
    double t = 0.0;
    int n = 0;
    st = run_forward(c, step0, time0, tEnd, maxSteps, dtSchedule, nSchedule, 1, false, t, n);
    if (st != SIFV_OK) return st;
    for (int q = 0; q < nv_of(c); ++q)
        if (zero_ghosts(c->P, c->tan[q], c->stream) != 0) return fail(c, SIFV_ERR_CUDA, "launch failed");
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (timeOut) *timeOut = t;
    if (stepsOut) *stepsOut = n;
    return SIFV_OK;
}

}  // extern "C"


// ===========================================================================
// Output path: NaN check, VTK snapshots from the device, runTimeLoop
// ===========================================================================
namespace {

// Device staging of one VTK session: two slots, each a device copy of the
// written fields (taken on the context's stream) and its pinned host copy
// (brought over on the session's copy stream).
struct VtkStage {
    int device = -1;
    size_t n = 0;
    int nf = 0;
    double* dev[2] = {nullptr, nullptr};
    double* host[2] = {nullptr, nullptr};
    cudaStream_t copy = nullptr;
    cudaEvent_t staged[2] = {nullptr, nullptr}, copied[2] = {nullptr, nullptr};
    bool busy[2] = {false, false};
    std::mutex mu;
};

void release_stage(void* p) {
    auto* s = static_cast<VtkStage*>(p);
    if (!s) return;
    cudaSetDevice(s->device);
    if (s->copy) cudaStreamSynchronize(s->copy);
    for (int q = 0; q < 2; ++q) {
        if (s->dev[q]) cudaFree(s->dev[q]);
        if (s->host[q]) cudaFreeHost(s->host[q]);
        if (s->staged[q]) cudaEventDestroy(s->staged[q]);
        if (s->copied[q]) cudaEventDestroy(s->copied[q]);
    }
    if (s->copy) cudaStreamDestroy(s->copy);
    delete s;
}

// The context's fields a snapshot writes, in a fixed order (pointers into
// `fields` are filled from the same order by vtk_fields_at).
std::vector<int> vtk_field_ids(const sifv::VtkLayout& L) {
    std::vector<int> ids = {SIFV_F_PRES};
    if (L.useIGR) ids.push_back(SIFV_F_SIGMA);
    ids.push_back(SIFV_F_RHOE);
    const int vel[3] = {SIFV_F_VELU, SIFV_F_VELV, SIFV_F_VELW}, mom[3] = {SIFV_F_RHOU, SIFV_F_RHOV, SIFV_F_RHOW};
    for (int d = 0; d < L.dim; ++d) ids.push_back(vel[d]);
    for (int d = 0; d < L.dim; ++d) ids.push_back(mom[d]);
    if (L.nPhases <= 0) ids.push_back(SIFV_F_RHO);
    for (int p = 0; p < L.nPhases; ++p) ids.push_back(SIFV_F_ALPHARHO(p));
    for (int p = 0; p < L.nPhases; ++p) ids.push_back(SIFV_F_ALPHA(p));
    return ids;
}

sifv_vtk_fields_t vtk_fields_at(const std::vector<int>& ids, const double* base, size_t n) {
    sifv_vtk_fields_t f{};
    for (size_t q = 0; q < ids.size(); ++q) {
        const double* a = base + q * n;
        const int id = ids[q];
        if (id == SIFV_F_PRES) f.pres = a;
        else if (id == SIFV_F_SIGMA) f.sigma = a;
        else if (id == SIFV_F_RHOE) f.rhoE = a;
        else if (id >= SIFV_F_VELU && id <= SIFV_F_VELW) f.vel[id - SIFV_F_VELU] = a;
        else if (id >= SIFV_F_RHOU && id <= SIFV_F_RHOW) f.mom[id - SIFV_F_RHOU] = a;
        else if (id == SIFV_F_RHO) f.rho = a;
        else if (id >= 16 && id < 32) f.alphaRho[id - 16] = a;
        else if (id >= 32) f.alpha[id - 32] = a;
    }
    return f;
}

int nan_scan(sifv_ctx* c, int& field, long long& cell) {
    field = -1;
    cell = -1;
    CUDA_TRY(c, cudaMemsetAsync(&c->ctl->nanCode, 0xff, sizeof(unsigned long long), c->stream));
    k_nan_scan<<<blocks((long long)c->nint, kCellThreads), kCellThreads, 0, c->stream>>>(c->P, c->F, c->ctl);
    LAUNCH_CHECK(c);
    unsigned long long code = 0;
    CUDA_TRY(c, cudaMemcpyAsync(&c->ctlHost->nanCode, &c->ctl->nanCode, sizeof(code), cudaMemcpyDeviceToHost,
                                c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    code = c->ctlHost->nanCode;
    if (code == ~0ull) return SIFV_OK;
    static const int order[6] = {SIFV_F_RHO, SIFV_F_RHOU, SIFV_F_RHOE, SIFV_F_PRES, SIFV_F_RHOV, SIFV_F_RHOW};
    field = order[code & 7ull];
    cell = (long long)(code >> 3);
    return SIFV_OK;
}

}  // namespace

extern "C" {

int sifv_check_nan(sifv_ctx_t* c, int* field, long long* cell) {
    if (!c || !field || !cell) return fail(c, SIFV_ERR_BAD_ARG, "null argument");
    cudaSetDevice(c->device);
    return nan_scan(c, *field, *cell);
}

int sifv_vtk_write(sifv_vtk_t* v, sifv_ctx_t* c, double time) {
    if (!v || !c) return fail(c, SIFV_ERR_BAD_ARG, "null argument");
    const sifv::VtkLayout& L = sifv::vtk_layout(v);
    const int ny = c->P.dim >= 2 ? c->P.ny : 1, nz = c->P.dim >= 3 ? c->P.nz : 1;
    if (L.dim != c->P.dim || L.nx != c->P.nx || L.ny != ny || L.nz != nz || L.ngx != c->P.ngx ||
        L.ngy != c->P.ngy || L.ngz != c->P.ngz || L.nPhases != c->cfg.nPhases || L.useIGR != (c->cfg.useIGR ? 1 : 0))
        return fail(c, SIFV_ERR_BAD_ARG, "the VTK session was opened for another mesh or configuration");
    cudaSetDevice(c->device);
    auto* S = static_cast<VtkStage*>(sifv::vtk_stage(v));
    const std::vector<int> ids = vtk_field_ids(L);
    if (!S) {
        S = new VtkStage();
        S->device = c->device;
        S->n = c->ncells;
        S->nf = (int)ids.size();
        if (cudaStreamCreateWithFlags(&S->copy, cudaStreamNonBlocking) != cudaSuccess) {
            delete S;
            return fail(c, SIFV_ERR_CUDA, "cannot create the VTK copy stream");
        }
        sifv::vtk_set_stage(v, S, release_stage);
    }
    if (S->device != c->device || S->n != c->ncells)
        return fail(c, SIFV_ERR_BAD_ARG, "the VTK session stages another context's device");
    int slot = -1;
    for (int attempt = 0; attempt < 2 && slot < 0; ++attempt) {
        {
            std::lock_guard<std::mutex> lk(S->mu);
            for (int q = 0; q < 2 && slot < 0; ++q)
                if (!S->busy[q]) slot = q;
            if (slot >= 0) S->busy[slot] = true;
        }
        if (slot < 0) sifv_vtk_flush(v);   // both slots in flight: wait for the writer
    }
    if (slot < 0) return fail(c, SIFV_ERR_CUDA, "no VTK staging slot");
    const size_t bytes = S->n * sizeof(double);
    if (!S->dev[slot]) {
        if (cudaMalloc(&S->dev[slot], bytes * S->nf) != cudaSuccess ||
            cudaHostAlloc(&S->host[slot], bytes * S->nf, cudaHostAllocDefault) != cudaSuccess ||
            cudaEventCreateWithFlags(&S->staged[slot], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&S->copied[slot], cudaEventDisableTiming) != cudaSuccess) {
            std::lock_guard<std::mutex> lk(S->mu);
            S->busy[slot] = false;
            return fail(c, SIFV_ERR_CUDA, "cannot allocate the VTK staging slot");
        }
    }
    for (int q = 0; q < S->nf; ++q)
        CUDA_TRY(c, cudaMemcpyAsync(S->dev[slot] + q * S->n, field_ptr(c, ids[q]), bytes, cudaMemcpyDeviceToDevice,
                                    c->stream));
    CUDA_TRY(c, cudaEventRecord(S->staged[slot], c->stream));
    CUDA_TRY(c, cudaStreamWaitEvent(S->copy, S->staged[slot], 0));
    CUDA_TRY(c, cudaMemcpyAsync(S->host[slot], S->dev[slot], bytes * S->nf, cudaMemcpyDeviceToHost, S->copy));
    CUDA_TRY(c, cudaEventRecord(S->copied[slot], S->copy));
    const int n = sifv::vtk_next_file(v);
    const size_t cells = S->n;
    sifv::vtk_enqueue(v, [v, S, slot, n, time, ids, cells](std::string& e) -> int {
        cudaSetDevice(S->device);
        int st = SIFV_OK;
        if (cudaEventSynchronize(S->copied[slot]) != cudaSuccess) {
            e = "VTK snapshot copy failed";
            st = SIFV_ERR_CUDA;
        } else {
            sifv_vtk_fields_t f = vtk_fields_at(ids, S->host[slot], cells);
            st = sifv::vtk_write_snapshot(v, n, time, &f, e);
        }
        std::lock_guard<std::mutex> lk(S->mu);
        S->busy[slot] = false;
        return st;
    });
    return SIFV_OK;
}

int sifv_run_time_loop(sifv_ctx_t* c, const sifv_time_loop_t* prm, sifv_vtk_t* vtk, sifv_progress_fn progress,
                       void* user, sifv_loop_result_t* res) {
    if (!c || !prm) return fail(c, SIFV_ERR_BAD_ARG, "null argument");
    if (!(prm->outputInterval > 0.0)) return fail(c, SIFV_ERR_BAD_ARG, "outputInterval must be > 0");
    if (!(prm->endTime < INFINITY)) return fail(c, SIFV_ERR_BAD_ARG, "endTime must be finite");
    sifv_loop_result_t r{};
    r.nanField = -1;
    r.nanCell = -1;
    const double endTime = prm->endTime, every = prm->outputInterval;
    const int printEvery = prm->printInterval > 0 ? prm->printInterval : 1;
    cudaSetDevice(c->device);
    c->dtReady = false;   // the state may have changed since the last call
    c->launches = 0;
    int st = SIFV_OK;
    double time = 0.0;
    int step = prm->step0;
    double nextOutput = every;
    // one output: the snapshot, then the NaN check (src/RKTimeStepping.cpp:275-311)
    auto output = [&](double t) -> int {
        r.outputs++;
        if (vtk) {
            int s = sifv_vtk_write(vtk, c, t);
            if (s != SIFV_OK) return s;
        }
        if (prm->checkNaN) {
            int f;
            long long cell;
            int s = nan_scan(c, f, cell);
            if (s != SIFV_OK) return s;
            if (f >= 0) {
                r.nanField = f;
                r.nanCell = cell;
                r.nanTime = t;
                r.nanStep = step;
                return fail(c, SIFV_ERR_NAN, "NaN detected at an output step");
            }
        }
        return SIFV_OK;
    };
    auto finish = [&](int s) -> int {
        r.time = time;
        r.steps = step;
        if (res) *res = r;
        if (vtk) {
            int f = sifv_vtk_flush(vtk);
            if (s == SIFV_OK && f != SIFV_OK) s = fail(c, f, sifv_vtk_last_error(vtk));
        }
        return s;
    };
    if (vtk) {
        st = sifv_vtk_write(vtk, c, 0.0);
        if (st != SIFV_OK) return finish(st);
    }
    r.outputs = 1;
    const bool resident = !c->cfg.semiImplicit && !c->cfg.useIGR && !has_body_force(c->cfg);
    if (!resident) {
        while (time < endTime) {
            double targetDt = endTime - time;
            if (nextOutput < endTime) targetDt = std::min(targetDt, nextOutput - time);
            double dt = 0.0;
            st = sifv_step(c, step, time, targetDt, &dt);
            if (st < 0) return finish(st);
            time += dt;
            step++;
            if (time >= nextOutput - 1e-12 * every) {
                nextOutput += every;
                st = output(time);
                if (st != SIFV_OK) return finish(st);
            }
            if (progress && (step % printEvery == 0 || step == 1)) progress(user, step, time, dt);
        }
        return finish(SIFV_OK);
    }
    const int batchMax = prm->batch > 0 ? prm->batch : 64;
    if (c->loopLogCap < batchMax) {
        if (c->loopLog) cudaFree(c->loopLog);
        c->loopLog = nullptr;
        c->loopLogCap = 0;
        CUDA_TRY(c, cudaMalloc(&c->loopLog, sizeof(double) * batchMax));
        c->loopLogCap = batchMax;
    }
    std::vector<double> log(batchMax);
    Ctl h{};
    h.time = 0.0;
    h.tEnd = endTime;
    h.nextOutput = nextOutput;
    h.outInterval = every;
    CUDA_TRY(c, cudaMemcpyAsync(c->ctl, &h, offsetof(Ctl, res), cudaMemcpyHostToDevice, c->stream));
    int perOutput = 0, sinceOutput = 0;   // steps of the last full output interval / of the current one
    while (time < endTime) {
        int B = batchMax;
        if (perOutput > 0) B = std::max(1, std::min(batchMax, perOutput - sinceOutput + 1));
        int status = SIFV_OK;
        for (int q = 0; q < B; ++q) {
            st = enqueue_step(c, step + q, 0.0, -1.0, 2, status);
            if (st != SIFV_OK) return finish(st);
            k_time_advance<<<1, 1, 0, c->stream>>>(c->ctl, c->loopLog, q);
            c->launches++;
        }
        LAUNCH_CHECK(c);
        CUDA_TRY(c, cudaMemcpyAsync(c->ctlHost, c->ctl, offsetof(Ctl, res), cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(c, cudaMemcpyAsync(log.data(), c->loopLog, sizeof(double) * B, cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        const bool due = c->ctlHost->outputDue != 0;
        int ran = 0;
        while (ran < B && log[ran] >= 0.0) ++ran;
        for (int q = 0; q < ran; ++q) {   // the host's copy of the device's time arithmetic
            time += log[q];
            step++;
            sinceOutput++;
            if (due && q == ran - 1) {
                nextOutput += every;
                perOutput = sinceOutput;
                sinceOutput = 0;
                st = output(time);
                if (st != SIFV_OK) return finish(st);
            }
            if (progress && (step % printEvery == 0 || step == 1)) progress(user, step, time, log[q]);
        }
        if (time != c->ctlHost->time) return finish(fail(c, SIFV_ERR_CUDA, "device and host time disagree"));
        if (due) {
            k_loop_resume<<<1, 1, 0, c->stream>>>(c->ctl);
            c->launches++;
        }
        if (ran == 0 && !due) break;   // nothing left to run (t >= endTime on the device)
    }
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return finish(SIFV_OK);
}

}  // extern "C"

// ===========================================================================
// Immersed boundaries
// ===========================================================================
namespace {

int set_ib(sifv_ctx* c, int nBodies, const int* wall, const sifv_ib_shapes_t* shapes) {
    if (nBodies > 0 && c->exchangeFaces)
        return fail(c, SIFV_ERR_UNSUPPORTED, "immersed boundaries are not supported with SIFV_BC_EXCHANGE faces");
    cudaSetDevice(c->device);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    for (void* p : c->ibAllocs) cudaFree(p);
    c->ibAllocs.clear();
    c->ib = IbDev{};
    c->F.solid = nullptr;
    c->ibTypes.clear();
    if (nBodies == 0) return SIFV_OK;
    if (c->cfg.semiImplicit) return fail(c, SIFV_ERR_UNSUPPORTED, "the semi-implicit step has no immersed boundary");
    if (c->sweep)
        return fail(c, SIFV_ERR_UNSUPPORTED, "immersed boundaries run in the SIFV_PREC_FP64 explicit step");
    for (int b = 0; b < nBodies; ++b)
        if (wall[b] != SIFV_IB_NOSLIP && wall[b] != SIFV_IB_SLIP) return fail(c, SIFV_ERR_BAD_ARG, "unknown wall type");
    sifv::IbGeometry g;
    g.dim = c->P.dim;
    g.nx = c->P.nx;
    g.ny = c->P.ny;
    g.nz = c->P.nz;
    g.ngx = c->P.ngx;
    g.ngy = c->P.ngy;
    g.ngz = c->P.ngz;
    g.nxT = c->P.nxT;
    g.nyT = c->P.nyT;
    g.ncells = c->ncells;
    g.cx = c->cenX;
    g.cy = c->cenY;
    g.cz = c->cenZ;
    sifv::IbTable t;
    sifv::ib_classify(g, nBodies, wall, *shapes, t);
    c->ibTypes = t.type;
    auto up = [&](const void* src, size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(bytes, 1)) != cudaSuccess) return nullptr;
        c->ibAllocs.push_back(p);
        if (bytes && cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
        return p;
    };
    const size_t m = t.cell.size();
    auto* solid = static_cast<const unsigned char*>(up(t.type.data(), t.type.size()));
    IbDev d{};
    d.count = (int)m;
    d.sequential = t.sequential;
    d.cell = static_cast<const long long*>(up(t.cell.data(), m * sizeof(long long)));
    d.wall = static_cast<const int*>(up(t.wall.data(), m * sizeof(int)));
    d.normal = static_cast<const double*>(up(t.normal.data(), m * 3 * sizeof(double)));
    d.n = static_cast<const int*>(up(t.n.data(), m * sizeof(int)));
    d.interp = static_cast<const long long*>(up(t.interp.data(), m * 8 * sizeof(long long)));
    d.w = static_cast<const double*>(up(t.w.data(), m * 8 * sizeof(double)));
    if (!solid || !d.cell || !d.wall || !d.normal || !d.n || !d.interp || !d.w) {
        for (void* p : c->ibAllocs) cudaFree(p);
        c->ibAllocs.clear();
        c->ibTypes.clear();
        return fail(c, SIFV_ERR_CUDA, "cannot upload the immersed-boundary tables");
    }
    c->ib = d;
    c->F.solid = solid;
    return SIFV_OK;
}

}  // namespace

extern "C" {

int sifv_set_immersed_bodies(sifv_ctx_t* c, const sifv_ib_body_t* bodies, int nBodies) {
    if (!c || nBodies < 0 || (nBodies > 0 && !bodies)) return fail(c, SIFV_ERR_BAD_ARG, "bad immersed-body list");
    std::vector<int> wall(nBodies);
    for (int b = 0; b < nBodies; ++b) {
        const sifv_ib_body_t& q = bodies[b];
        if (q.shape < SIFV_IB_CIRCLE || q.shape > SIFV_IB_PRISM) return fail(c, SIFV_ERR_BAD_ARG, "unknown body shape");
        if (q.shape == SIFV_IB_CYLINDER && (q.axis < 0 || q.axis > 2))
            return fail(c, SIFV_ERR_BAD_ARG, "cylinder axis must be 0, 1 or 2");
        wall[b] = q.wall;
    }
    sifv_ib_shapes_t s{};
    sifv::ib_builtin_shapes(bodies, s);
    return set_ib(c, nBodies, wall.data(), &s);
}

int sifv_set_immersed_shapes(sifv_ctx_t* c, int nBodies, const int* wall, const sifv_ib_shapes_t* shapes) {
    if (!c || nBodies < 0 || (nBodies > 0 && (!wall || !shapes || !shapes->signedDistance || !shapes->closestPoint ||
                                              !shapes->outwardNormal)))
        return fail(c, SIFV_ERR_BAD_ARG, "bad immersed-shape queries");
    return set_ib(c, nBodies, wall, shapes);
}

int sifv_ib_cell_types(sifv_ctx_t* c, unsigned char* types) {
    if (!c || !types) return fail(c, SIFV_ERR_BAD_ARG, "null argument");
    if (c->ibTypes.empty()) std::memset(types, SIFV_CELL_FLUID, c->ncells);
    else std::memcpy(types, c->ibTypes.data(), c->ncells);
    return SIFV_OK;
}

int sifv_apply_ib_ghost_cells(sifv_ctx_t* c) {
    if (!c) return fail(nullptr, SIFV_ERR_BAD_ARG, "null context");
    cudaSetDevice(c->device);
    CUDA_TRY(c, cudaMemsetAsync(&c->ctl->skip, 0, sizeof(int), c->stream));
    launch_ib_ghost(c);
    LAUNCH_CHECK(c);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SIFV_OK;
}

}  // extern "C"
