// sifv_noalloc.cu -- a Jacobi pressure solve that allocates nothing.
//
// sifv_pressure_solve needs a context, and creating a context allocates
// device memory.  Some callers cannot do that: hosts whose whole GPU
// memory is handed out by their own pool allocator, and code that must not
// call cudaMalloc/cudaFree in the middle of stream work because those calls
// can synchronise the device.  sifv_pressure_solve_noalloc serves them: the
// caller passes the input and output arrays (device memory), and the
// solver's scratch -- the two Jacobi iterates, the per-iteration residual
// slots, the convergence flag and the cell widths -- lives in one
// file-scope static device array of fixed size, reserved on every GPU that
// loads this library until the process exits.
//
// The kernel is the same k_jacobi the context path runs (the kernel header
// is included with internal linkage so this file gets its own copy).
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "sifv.h"

namespace {
#include "sifv_kernels.cuh"
}  // namespace

namespace {

using sifv_nal_ctl = sifv::Ctl;
using CUresult_t = int;   // the driver API's CUresult (0 = success)

// Sizes of the static scratch (SIFV_NOALLOC_* in include/sifv.h).
constexpr size_t kMaxCells = SIFV_NOALLOC_MAX_CELLS;
constexpr int kMaxIters = SIFV_NOALLOC_MAX_ITERS;
constexpr int kMaxAxis = SIFV_NOALLOC_MAX_AXIS;

// Layout of the static array, in doubles:
//   [0, kCtl)                     control block (Ctl + kMaxIters residual slots)
//   [kCtl, + kMaxCells)           iterate A
//   [.., + kMaxCells)             iterate B
//   [.., + 3 * kMaxAxis)          dx, dy, dz (ghosts included)
constexpr size_t kCtl = (sizeof(sifv_nal_ctl) + sizeof(unsigned long long) * (kMaxIters + 1) + 255) / 256 * 32;
constexpr size_t kTotal = kCtl + 2 * kMaxCells + 3 * (size_t)kMaxAxis;

static __device__ __align__(256) double g_noalloc_scratch[kTotal];

constexpr int kMaxDevices = 64;
// Per device: the id of the CUDA context the address was looked up in, and
// the address.  A device reset, or another context made current on the same
// device, loads the module again, possibly at another address, so the
// address is looked up again whenever the current context's id changes.
struct ScratchSlot {
    unsigned long long ctxId;
    double* addr;
};
ScratchSlot g_scratch[kMaxDevices] = {};
std::mutex g_setup_mutex;
thread_local std::string g_noalloc_err;
thread_local double g_width_buf[kMaxAxis];   // host staging of one axis' widths

int nal_fail(int code, const char* msg) {
    g_noalloc_err = msg;
    return code;
}

// Driver entry points cuCtxGetCurrent / cuCtxGetId, reached through the
// runtime's entry-point table so that the library needs no link against
// the driver library.
using CtxGetCurrent = CUresult_t (*)(void**);
using CtxGetId = CUresult_t (*)(void*, unsigned long long*);

int driver_entry_points(CtxGetCurrent* getCurrent, CtxGetId* getId) {
    static CtxGetCurrent gc = nullptr;
    static CtxGetId gi = nullptr;
    if (!gc || !gi) {
        void* a = nullptr;
        void* b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
            qa != cudaDriverEntryPointSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
            qb != cudaDriverEntryPointSuccess)
            return nal_fail(SIFV_ERR_CUDA, "driver entry points cuCtxGetCurrent / cuCtxGetId not found");
        gc = reinterpret_cast<CtxGetCurrent>(a);
        gi = reinterpret_cast<CtxGetId>(b);
    }
    *getCurrent = gc;
    *getId = gi;
    return SIFV_OK;
}

// Device address of the static array on the current device.  The host-side
// name g_noalloc_scratch is only a stand-in, so the address is looked up
// (cudaGetSymbolAddress) with the device current, once per device and
// context, and kept for later calls.  When no context is current yet, the
// look-up itself initialises the device's primary context.
int scratch_for_current_device(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nal_fail(SIFV_ERR_CUDA, "cudaGetDevice failed");
    if (dev < 0 || dev >= kMaxDevices) return nal_fail(SIFV_ERR_UNSUPPORTED, "device index above 63");
    CtxGetCurrent getCurrent = nullptr;
    CtxGetId getId = nullptr;
    int st = driver_entry_points(&getCurrent, &getId);
    if (st != SIFV_OK) return st;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (getCurrent(&ctx) != 0) return nal_fail(SIFV_ERR_CUDA, "cuCtxGetCurrent failed");
    if (ctx && getId(ctx, &id) != 0) return nal_fail(SIFV_ERR_CUDA, "cuCtxGetId failed");
    if (!ctx || !g_scratch[dev].addr || g_scratch[dev].ctxId != id) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            g_noalloc_err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
            return SIFV_ERR_CUDA;
        }
        if (!ctx) {   // the look-up made the primary context current
            if (getCurrent(&ctx) != 0 || !ctx || getId(ctx, &id) != 0)
                return nal_fail(SIFV_ERR_CUDA, "no current CUDA context after initialisation");
        }
        g_scratch[dev].addr = static_cast<double*>(p);
        g_scratch[dev].ctxId = id;
    }
    *out = g_scratch[dev].addr;
    return SIFV_OK;
}

// Cell widths of one axis, ghosts included, into dst (length n + 2 ng):
// RectilinearMesh::buildExtendedNodes (src/RectilinearMesh.cpp:91-114)
// followed by dx(i) = ext[i+1] - ext[i], without a heap array.
void axis_widths(const double* phys, int nCells, int ng, double* dst) {
    // ext[q] for q in [0, nCells + 2 ng]; widths need consecutive pairs.
    auto ext = [&](int q) -> double {
        if (q >= ng && q <= ng + nCells) return phys[q - ng];
        if (q < ng) {
            double v = phys[0];
            for (int g = 1; g <= ng - q; ++g) {
                int mirror = (g - 1 < nCells - 1) ? g - 1 : nCells - 1;
                v = v - (phys[mirror + 1] - phys[mirror]);
            }
            return v;
        }
        double v = phys[nCells];
        for (int g = 1; g <= q - ng - nCells; ++g) {
            int mirror = (nCells - g > 0) ? nCells - g : 0;
            v = v + (phys[mirror + 1] - phys[mirror]);
        }
        return v;
    };
    for (int q = 0; q < nCells + 2 * ng; ++q) dst[q] = ext(q + 1) - ext(q);
}

}  // namespace

extern "C" {

const char* sifv_noalloc_last_error(void) { return g_noalloc_err.c_str(); }

int sifv_pressure_solve_noalloc(const sifv_mesh_t* mesh, int dim, int nGhost, const double* rho, const double* rhoc2,
                                const double* rhs, double* pressure, double dt, double tol, int maxIter,
                                void* stream, int* iters) {
    using namespace sifv;
    if (!mesh || !rho || !rhoc2 || !rhs || !pressure || !iters) return nal_fail(SIFV_ERR_BAD_ARG, "null argument");
    if (dim < 1 || dim > 3) return nal_fail(SIFV_ERR_BAD_ARG, "dim must be 1, 2 or 3");
    if (nGhost < 1) return nal_fail(SIFV_ERR_BAD_ARG, "nGhost must be >= 1");
    if (maxIter <= 0) return nal_fail(SIFV_ERR_BAD_ARG, "maxIter must be > 0");
    if (maxIter > kMaxIters) return nal_fail(SIFV_ERR_BAD_ARG, "maxIter exceeds SIFV_NOALLOC_MAX_ITERS");
    Params P{};
    P.dim = dim;
    P.nx = mesh->nx;
    P.ny = (dim >= 2) ? mesh->ny : 1;
    P.nz = (dim >= 3) ? mesh->nz : 1;
    P.ngx = nGhost;
    P.ngy = (dim >= 2) ? nGhost : 0;
    P.ngz = (dim >= 3) ? nGhost : 0;
    if (P.nx < nGhost || P.ny < (dim >= 2 ? nGhost : 1) || P.nz < (dim >= 3 ? nGhost : 1))
        return nal_fail(SIFV_ERR_UNSUPPORTED, "every active axis needs at least nGhost cells");
    if (!mesh->xNodes || (dim >= 2 && !mesh->yNodes) || (dim >= 3 && !mesh->zNodes))
        return nal_fail(SIFV_ERR_BAD_ARG, "node arrays of the active axes are required");
    P.nxT = P.nx + 2 * P.ngx;
    P.nyT = P.ny + 2 * P.ngy;
    P.nzT = P.nz + 2 * P.ngz;
    if (P.nxT > kMaxAxis || P.nyT > kMaxAxis || P.nzT > kMaxAxis)
        return nal_fail(SIFV_ERR_BAD_ARG, "an axis (ghosts included) exceeds SIFV_NOALLOC_MAX_AXIS cells");
    const size_t ncells = (size_t)P.nxT * P.nyT * P.nzT;
    if (ncells > kMaxCells)
        return nal_fail(SIFV_ERR_BAD_ARG, "mesh (ghosts included) exceeds SIFV_NOALLOC_MAX_CELLS cells");
    for (int f = 0; f < 6; ++f) P.bc[f] = mesh->bc[f];

    double* base = nullptr;
    int st = scratch_for_current_device(&base);
    if (st != SIFV_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Ctl* ctl = reinterpret_cast<Ctl*>(base);
    double* pA = base + kCtl;
    double* pB = pA + kMaxCells;
    double* dxs = pB + kMaxCells;
    Fields F{};
    F.pA = pA;
    F.pB = pB;
    F.dx = dxs;
    F.dy = dxs + kMaxAxis;
    F.dz = dxs + 2 * kMaxAxis;

    // cell widths: computed on the host into a fixed per-thread buffer, one
    // axis at a time, and copied into the static array
    static const double unit[2] = {0.0, 1.0};
    const double* nodes[3] = {mesh->xNodes, (dim >= 2) ? mesh->yNodes : unit, (dim >= 3) ? mesh->zNodes : unit};
    const int ncell[3] = {P.nx, P.ny, P.nz};
    const int ng[3] = {P.ngx, P.ngy, P.ngz};
    for (int a = 0; a < 3; ++a) {
        double* w = g_width_buf;
        axis_widths(nodes[a], ncell[a], ng[a], w);
        int len = ncell[a] + 2 * ng[a];
        if (cudaMemcpyAsync(const_cast<double*>(a == 0 ? F.dx : a == 1 ? F.dy : F.dz), w, len * sizeof(double),
                            cudaMemcpyHostToDevice, s) != cudaSuccess)
            return nal_fail(SIFV_ERR_CUDA, "copy of cell widths failed");
        if (cudaStreamSynchronize(s) != cudaSuccess) return nal_fail(SIFV_ERR_CUDA, "stream synchronize failed");
    }
    // the static array keeps the previous call's contents: reset the
    // convergence flag and residual slots, load dt and the initial iterate
    if (cudaMemsetAsync(ctl, 0, sizeof(Ctl) + sizeof(unsigned long long) * (size_t)maxIter, s) != cudaSuccess ||
        cudaMemcpyAsync(&ctl->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(pA, pressure, ncells * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return nal_fail(SIFV_ERR_CUDA, "scratch initialisation failed");

    const long long nint = (long long)P.nx * P.ny * P.nz;
    const unsigned g = (unsigned)((nint + 255) / 256);
    int it = 0, batch = 4, done = 0;
    double lastRes = 0.0;
    while (it < maxIter) {
        int nb = (batch < maxIter - it) ? batch : maxIter - it;
        for (int q = 0; q < nb; ++q, ++it) {
            const double* pin = (it & 1) ? pB : pA;
            double* pout = (it & 1) ? pA : pB;
            k_jacobi<<<g, 256, 0, s>>>(P, rho, rhoc2, rhs, pin, pout, F, ctl, it, tol);
        }
        if (cudaGetLastError() != cudaSuccess) return nal_fail(SIFV_ERR_CUDA, "Jacobi launch failed");
        int flag = 0;
        unsigned long long bits = 0;
        if (cudaMemcpyAsync(&flag, &ctl->jacobiDone, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaMemcpyAsync(&bits, &ctl->res[it - 1], sizeof(bits), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return nal_fail(SIFV_ERR_CUDA, "reading the convergence flag failed");
        std::memcpy(&lastRes, &bits, sizeof(double));
        if (flag) { done = flag; break; }
        if (lastRes < tol) { done = it; break; }
        batch = (batch * 2 < 32) ? batch * 2 : 32;
    }
    int n = done ? done : maxIter;
    const double* result = (n & 1) ? pB : pA;
    // interior cells of the result into the caller's array (ghosts untouched)
    k_jacobi_finish<<<g, 256, 0, s>>>(P, result, result, pressure, ctl, maxIter);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
        return nal_fail(SIFV_ERR_CUDA, "copy-out failed");
    *iters = n;
    // without convergence lastRes is the residual of iteration maxIter
    if (n >= maxIter && !(lastRes < tol)) return SIFV_NOT_CONVERGED;
    return SIFV_OK;
}

}  // extern "C"
