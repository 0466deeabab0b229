// sifv_ensemble.cu -- C ABI of batched ensembles (include/sifv.h,
// sifv_ensemble_*): many independent 1D problems of different sizes
// advanced to a common end time by one kernel launch (one CTA per
// instance, sifv_ensemble.cuh).  The FP64 instantiation here is compiled
// without FMA contraction and is bit-identical, instance by instance, to
// the single-problem reference-ordered path.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "sifv.h"
#include "sifv_ensemble.cuh"
#include "sifv_ensemble_api.h"

using namespace sifv;

struct sifv_ensemble {
    sifv_config_t cfg{};
    EnsArgs A{};
    int device = 0;
    int nInst = 0;
    int nphT = 0;
    cudaStream_t stream = nullptr;
    std::vector<void*> allocs;
    std::vector<long long> off;
    long long ncells = 0;
    int blockSize = 256;
    std::string err;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

thread_local std::string g_ens_err;

int efail(sifv_ensemble* e, int code, const std::string& m) {
    if (e) e->err = m; else g_ens_err = m;
    return code;
}

template <typename X>
X* ealloc(sifv_ensemble* e, size_t n, int& st) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(X)) != cudaSuccess) {
        st = efail(e, SIFV_ERR_CUDA, "cudaMalloc failed");
        return nullptr;
    }
    cudaMemsetAsync(p, 0, std::max<size_t>(n, 1) * sizeof(X), e->stream);
    e->allocs.push_back(p);
    return static_cast<X*>(p);
}

double* efield(sifv_ensemble* e, int f) {
    EnsArgs& A = e->A;
    switch (f) {
        case SIFV_F_RHO: return A.S[0].rho;
        case SIFV_F_RHOU: return A.S[0].rhoU;
        case SIFV_F_RHOE: return A.S[0].rhoE;
        case SIFV_F_VELU: return A.velU;
        case SIFV_F_PRES: return A.pres;
        default: break;
    }
    if (f >= 16 && f < 16 + e->cfg.nPhases) return A.S[0].alphaRho[f - 16];
    if (f >= 32 && f < 32 + e->cfg.nPhases) return A.S[0].alpha[f - 32];
    return nullptr;
}

template <typename T, int NPH>
int launch_t(const EnsArgs& A, int blockSize, cudaStream_t s) {
    const size_t bytes = ens_smem_bytes<T, NPH>(blockSize);
    if (cudaFuncSetAttribute(k_ensemble<T, NPH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) !=
        cudaSuccess)
        return -1;
    k_ensemble<T, NPH><<<A.nInst, blockSize, bytes, s>>>(A);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int launch(sifv_ensemble* e, int blockSize) {
    if (e->cfg.precision == SIFV_PREC_MIXED)
        return ensemble_launch_mixed(e->A, e->nphT, blockSize, e->stream);
    if (e->nphT == 0) return launch_t<double, 0>(e->A, blockSize, e->stream);
    if (e->nphT == 2) return launch_t<double, 2>(e->A, blockSize, e->stream);
    return launch_t<double, 8>(e->A, blockSize, e->stream);
}

// dynamic shared memory of one block, and the largest usable block size
size_t smem_bytes(const sifv_ensemble* e, int blockSize) {
    const bool f = e->cfg.precision == SIFV_PREC_MIXED;
    switch (e->nphT) {
        case 0: return f ? ens_smem_bytes<float, 0>(blockSize) : ens_smem_bytes<double, 0>(blockSize);
        case 2: return f ? ens_smem_bytes<float, 2>(blockSize) : ens_smem_bytes<double, 2>(blockSize);
        default: return f ? ens_smem_bytes<float, 8>(blockSize) : ens_smem_bytes<double, 8>(blockSize);
    }
}

int max_block(const sifv_ensemble* e) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    int m = (e->cfg.precision == SIFV_PREC_MIXED) ? 1024 : 512;
    while (m > 32 && smem_bytes(e, m) + 512 > (size_t)optin) m -= 32;
    return m;
}

// all packed state arrays (for the autotuner's save / restore)
std::vector<double*> state_arrays(sifv_ensemble* e) {
    EnsArgs& A = e->A;
    std::vector<double*> v = {A.S[0].rho, A.S[0].rhoU, A.S[0].rhoE, A.velU, A.pres};
    for (int p = 0; p < e->cfg.nPhases; ++p) { v.push_back(A.S[0].alphaRho[p]); v.push_back(A.S[0].alpha[p]); }
    return v;
}

}  // namespace

extern "C" {

const char* sifv_ensemble_last_error(const sifv_ensemble_t* e) { return e ? e->err.c_str() : g_ens_err.c_str(); }

int sifv_ensemble_create(const sifv_config_t* cfg, int nInst, const int* nCells, const double* xLo,
                         const double* xHi, const int bc[2], int device, sifv_ensemble_t** out) {
    if (!cfg || !nCells || !xLo || !xHi || !bc || !out || nInst <= 0)
        return efail(nullptr, SIFV_ERR_BAD_ARG, "null argument or empty ensemble");
    *out = nullptr;
    if (sifv_config_validate(cfg) != SIFV_OK) return efail(nullptr, SIFV_ERR_BAD_CONFIG, sifv_last_error(nullptr));
    bool bf = false;
    for (int d = 0; d < 3; ++d) bf = bf || cfg->bfA[d] != 0.0 || cfg->bfB[d] != 0.0;
    if (cfg->dim != 1 || cfg->semiImplicit || cfg->useIGR || bf || cfg->mu > 0.0 || cfg->nPhaseMu > 0 || cfg->stSigma > 0.0 ||
        (cfg->reconOrder != SIFV_WENO5 && cfg->reconOrder != SIFV_UPWIND5) ||
        (cfg->precision != SIFV_PREC_FP64 && cfg->precision != SIFV_PREC_MIXED))
        return efail(nullptr, SIFV_ERR_UNSUPPORTED,
                     "ensembles run the explicit 1D WENO5/UPWIND5 step (no IGR, body force, viscosity or surface tension) in "
                     "SIFV_PREC_FP64 or SIFV_PREC_MIXED");
    for (int k = 0; k < nInst; ++k)
        if (nCells[k] < cfg->nGhost || !(xHi[k] > xLo[k]))
            return efail(nullptr, SIFV_ERR_BAD_ARG, "each instance needs >= nGhost cells and xHi > xLo");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return efail(nullptr, SIFV_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= ndev) return efail(nullptr, SIFV_ERR_BAD_ARG, "device index out of range");
    cudaSetDevice(device);

    sifv_ensemble* e = new sifv_ensemble();
    e->cfg = *cfg;
    e->device = device;
    e->nInst = nInst;
    e->nphT = (cfg->nPhases == 0) ? 0 : (cfg->nPhases <= 2) ? 2 : 8;
    cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    cudaEventCreate(&e->ev0);
    cudaEventCreate(&e->ev1);
    const int ng = cfg->nGhost;
    e->off.resize(nInst + 1);
    e->off[0] = 0;
    for (int k = 0; k < nInst; ++k) {
        e->off[k + 1] = e->off[k] + nCells[k] + 2 * ng;
    }
    e->ncells = e->off[nInst];
    // cell widths: Runtime::createUniformMesh nodes a + (b - a) i / n
    // (src/Runtime.cpp:12-17) extended by RectilinearMesh::buildExtendedNodes
    // (src/RectilinearMesh.cpp:91-114)
    std::vector<double> dx(e->ncells);
    for (int k = 0; k < nInst; ++k) {
        int n = nCells[k];
        std::vector<double> ext(n + 2 * ng + 1), phys(n + 1);
        for (int i = 0; i <= n; ++i) phys[i] = xLo[k] + (xHi[k] - xLo[k]) * i / n;
        for (int i = 0; i <= n; ++i) ext[ng + i] = phys[i];
        for (int g = 1; g <= ng; ++g) {
            int mirror = std::min(g - 1, n - 1);
            ext[ng - g] = ext[ng - g + 1] - (phys[mirror + 1] - phys[mirror]);
        }
        for (int g = 1; g <= ng; ++g) {
            int mirror = std::max(n - g, 0);
            ext[ng + n + g] = ext[ng + n + g - 1] + (phys[mirror + 1] - phys[mirror]);
        }
        for (int q = 0; q < n + 2 * ng; ++q) dx[e->off[k] + q] = ext[q + 1] - ext[q];
    }
    // cost order: steps ~ n and work per step ~ n
    std::vector<int> order(nInst);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return nCells[a] > nCells[b]; });

    int st = SIFV_OK;
    EnsArgs& A = e->A;
    A.nInst = nInst;
    const size_t M = (size_t)e->ncells;
    const int nStates = (cfg->RKOrder >= 3) ? 3 : 2;   // the state and the stage outputs
    for (int k = 0; k < nStates; ++k) {
        EnsState& S = A.S[k];
        S.rho = ealloc<double>(e, M, st); S.rhoU = ealloc<double>(e, M, st); S.rhoE = ealloc<double>(e, M, st);
        for (int p = 0; p < cfg->nPhases; ++p) { S.alphaRho[p] = ealloc<double>(e, M, st); S.alpha[p] = ealloc<double>(e, M, st); }
    }
    A.velU = ealloc<double>(e, M, st); A.pres = ealloc<double>(e, M, st);
    double* dxd = ealloc<double>(e, M, st);
    A.dx = dxd;
    int* ord = ealloc<int>(e, nInst, st);
    int* nn = ealloc<int>(e, nInst, st);
    long long* offd = ealloc<long long>(e, nInst + 1, st);
    A.time = ealloc<double>(e, nInst, st);
    A.steps = ealloc<int>(e, nInst, st);
    A.lastDt = ealloc<double>(e, nInst, st);
    A.status = ealloc<int>(e, nInst, st);
    if (st == SIFV_OK) {
        cudaMemcpyAsync(dxd, dx.data(), M * sizeof(double), cudaMemcpyHostToDevice, e->stream);
        cudaMemcpyAsync(ord, order.data(), nInst * sizeof(int), cudaMemcpyHostToDevice, e->stream);
        cudaMemcpyAsync(nn, nCells, nInst * sizeof(int), cudaMemcpyHostToDevice, e->stream);
        cudaMemcpyAsync(offd, e->off.data(), (nInst + 1) * sizeof(long long), cudaMemcpyHostToDevice, e->stream);
        if (cudaStreamSynchronize(e->stream) != cudaSuccess) st = efail(e, SIFV_ERR_CUDA, "upload failed");
    }
    A.order = ord; A.n = nn; A.off = offd;
    Params& P = A.P;
    P.dim = 1; P.ny = P.nz = 1; P.ngx = ng; P.ngy = P.ngz = 0; P.nyT = P.nzT = 1;
    P.bc[0] = bc[0]; P.bc[1] = bc[1];
    for (int f = 2; f < 6; ++f) P.bc[f] = SIFV_BC_OUTFLOW;
    P.nPh = cfg->nPhases;
    P.reconOrder = cfg->reconOrder;
    P.riemann = cfg->riemannSolver;
    P.includePressure = 1;
    P.useIGR = 0; P.reconSigma = 0;
    P.eosStiffened = (cfg->eosKind == SIFV_EOS_STIFFENED) ? 1 : 0;
    P.RKOrder = cfg->RKOrder;
    P.wenoEps = cfg->wenoEps;
    P.gamma = cfg->gamma;
    P.pInf = P.eosStiffened ? cfg->pInf : 0.0;
    for (int p = 0; p < SIFV_MAX_PHASES; ++p) { P.phaseGamma[p] = cfg->phaseGamma[p]; P.phasePInf[p] = cfg->phasePInf[p]; }
    P.alphaMin = cfg->alphaMin;
    A.cfl = cfg->cfl; A.maxDt = cfg->maxDt; A.constDt = cfg->constDt;
    if (st != SIFV_OK) {
        g_ens_err = e->err;
        sifv_ensemble_destroy(e);
        return st;
    }
    *out = e;
    return SIFV_OK;
}

int sifv_ensemble_destroy(sifv_ensemble_t* e) {
    if (!e) return SIFV_OK;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    for (void* p : e->allocs) cudaFree(p);
    if (e->ev0) cudaEventDestroy(e->ev0);
    if (e->ev1) cudaEventDestroy(e->ev1);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return SIFV_OK;
}

int sifv_ensemble_layout(const sifv_ensemble_t* e, long long* offsets) {
    if (!e || !offsets) return SIFV_ERR_BAD_ARG;
    std::memcpy(offsets, e->off.data(), (e->nInst + 1) * sizeof(long long));
    return SIFV_OK;
}

int sifv_ensemble_set_field(sifv_ensemble_t* e, int field, const double* packed, int onDevice) {
    double* p = efield(e, field);
    if (!p) return efail(e, SIFV_ERR_BAD_ARG, "field not part of this ensemble");
    cudaSetDevice(e->device);
    if (cudaMemcpyAsync(p, packed, e->ncells * sizeof(double), onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                        e->stream) != cudaSuccess || cudaStreamSynchronize(e->stream) != cudaSuccess)
        return efail(e, SIFV_ERR_CUDA, "copy failed");
    return SIFV_OK;
}

int sifv_ensemble_get_field(sifv_ensemble_t* e, int field, double* packed, int onDevice) {
    double* p = efield(e, field);
    if (!p) return efail(e, SIFV_ERR_BAD_ARG, "field not part of this ensemble");
    cudaSetDevice(e->device);
    if (cudaMemcpyAsync(packed, p, e->ncells * sizeof(double), onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                        e->stream) != cudaSuccess || cudaStreamSynchronize(e->stream) != cudaSuccess)
        return efail(e, SIFV_ERR_CUDA, "copy failed");
    return SIFV_OK;
}

int sifv_ensemble_run(sifv_ensemble_t* e, double tEnd, int maxSteps, int blockSize, double* timesOut,
                      int* stepsOut, double* deviceMs) {
    if (!e) return efail(nullptr, SIFV_ERR_BAD_ARG, "null ensemble");
    int bs = blockSize > 0 ? blockSize : e->blockSize;
    const int maxBs = max_block(e);
    if (bs % 32 != 0 || bs < 32 || bs > maxBs)
        return efail(e, SIFV_ERR_BAD_ARG, "blockSize must be a multiple of 32 in [32, " + std::to_string(maxBs) + "]");
    if (!(tEnd < 1e300) && maxSteps <= 0) return efail(e, SIFV_ERR_BAD_ARG, "tEnd must be finite when there is no step limit");
    cudaSetDevice(e->device);
    e->A.tEnd = tEnd;
    e->A.maxSteps = maxSteps > 0 ? maxSteps : 0x7fffffff;
    cudaEventRecord(e->ev0, e->stream);
    if (launch(e, bs) != 0) return efail(e, SIFV_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(cudaGetLastError()));
    cudaEventRecord(e->ev1, e->stream);
    if (timesOut) cudaMemcpyAsync(timesOut, e->A.time, e->nInst * sizeof(double), cudaMemcpyDeviceToHost, e->stream);
    if (stepsOut) cudaMemcpyAsync(stepsOut, e->A.steps, e->nInst * sizeof(int), cudaMemcpyDeviceToHost, e->stream);
    std::vector<int> status(e->nInst);
    cudaMemcpyAsync(status.data(), e->A.status, e->nInst * sizeof(int), cudaMemcpyDeviceToHost, e->stream);
    cudaError_t err = cudaStreamSynchronize(e->stream);
    if (err != cudaSuccess) return efail(e, SIFV_ERR_CUDA, cudaGetErrorString(err));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    if (deviceMs) *deviceMs = ms;
    for (int k = 0; k < e->nInst; ++k)
        if (status[k] != 0)
            return efail(e, SIFV_ERR_NAN, "instance " + std::to_string(k) + ": time step not positive (state blew up)");
    return SIFV_OK;
}

// Pick the block size (128 / 256 / 512 threads per instance, and 1024 with
// FP32 bulk, as shared memory allows) with the shortest time for a probe in
// which every instance takes steps in proportion to its cell count (as in a
// run to a common end time at a fixed CFL), the largest probeSteps steps;
// the state is restored afterwards.
int sifv_ensemble_autotune(sifv_ensemble_t* e, int probeSteps, int* blockSizeOut) {
    if (!e) return efail(nullptr, SIFV_ERR_BAD_ARG, "null ensemble");
    cudaSetDevice(e->device);
    std::vector<double*> arrs = state_arrays(e);
    const size_t bytes = e->ncells * sizeof(double);
    std::vector<void*> saved;
    for (size_t q = 0; q < arrs.size(); ++q) {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            for (void* s : saved) cudaFree(s);
            return efail(e, SIFV_ERR_CUDA, "cudaMalloc failed");
        }
        saved.push_back(p);
        cudaMemcpyAsync(p, arrs[q], bytes, cudaMemcpyDeviceToDevice, e->stream);
    }
    std::vector<double> t0(e->nInst);
    std::vector<int> s0(e->nInst);
    cudaMemcpyAsync(t0.data(), e->A.time, e->nInst * sizeof(double), cudaMemcpyDeviceToHost, e->stream);
    cudaMemcpyAsync(s0.data(), e->A.steps, e->nInst * sizeof(int), cudaMemcpyDeviceToHost, e->stream);
    cudaStreamSynchronize(e->stream);
    int best = 256;
    float bestMs = 1e30f;
    const int cands[4] = {128, 256, 512, 1024};
    const int maxBs = max_block(e);
    std::vector<int> nc(e->nInst), lim(e->nInst);
    cudaMemcpy(nc.data(), e->A.n, e->nInst * sizeof(int), cudaMemcpyDeviceToHost);
    const int nMax = *std::max_element(nc.begin(), nc.end());
    for (int k = 0; k < e->nInst; ++k)
        lim[k] = s0[k] + std::max(1, (int)((long long)std::max(probeSteps, 1) * nc[k] / std::max(nMax, 1)));
    int* limD = nullptr;
    if (cudaMalloc(&limD, e->nInst * sizeof(int)) != cudaSuccess) {
        for (void* p : saved) cudaFree(p);
        return efail(e, SIFV_ERR_CUDA, "cudaMalloc failed");
    }
    cudaMemcpy(limD, lim.data(), e->nInst * sizeof(int), cudaMemcpyHostToDevice);
    e->A.stepLimit = limD;
    for (int bs : cands) {
        if (bs > maxBs) continue;
        e->A.tEnd = 1e300;
        e->A.maxSteps = 0x7fffffff;
        cudaEventRecord(e->ev0, e->stream);
        if (launch(e, bs) != 0) continue;
        cudaEventRecord(e->ev1, e->stream);
        cudaStreamSynchronize(e->stream);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e->ev0, e->ev1);
        if (ms < bestMs) { bestMs = ms; best = bs; }
        for (size_t q = 0; q < arrs.size(); ++q)
            cudaMemcpyAsync(arrs[q], saved[q], bytes, cudaMemcpyDeviceToDevice, e->stream);
        cudaMemcpyAsync(e->A.time, t0.data(), e->nInst * sizeof(double), cudaMemcpyHostToDevice, e->stream);
        cudaMemcpyAsync(e->A.steps, s0.data(), e->nInst * sizeof(int), cudaMemcpyHostToDevice, e->stream);
        cudaStreamSynchronize(e->stream);
    }
    e->A.stepLimit = nullptr;
    cudaFree(limD);
    for (void* s : saved) cudaFree(s);
    e->blockSize = best;
    if (blockSizeOut) *blockSizeOut = best;
    return cudaGetLastError() == cudaSuccess ? SIFV_OK : efail(e, SIFV_ERR_CUDA, "autotune failed");
}

}  // extern "C"
