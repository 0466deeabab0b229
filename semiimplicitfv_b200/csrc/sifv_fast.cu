// sifv_fast.cu -- launchers of the fused sweep kernels (fast-FP64 and
// mixed-precision explicit step).  Compiled with FMA contraction enabled:
// these paths trade the reference's exact operation order for speed and
// are held to the relative tolerance of the parity tests instead of bit
// equality.
#include <cuda_runtime.h>

#include <cstring>

#include "sifv_sweep.cuh"
#include "sifv_sweep_api.h"
#include "sifv_march2d.cuh"

namespace sifv {

namespace {

constexpr int kSegment = 32;    // cells per thread along y / z
constexpr int kSegmentX = 510;  // cells per warp along x: 16 steps of 32 positions

template <int DIM, typename T>
int stage_dim(const SweepArgs& A, cudaStream_t s, int& launches, LaunchMark mark, void* user) {
    const Params& P = A.P;
    {
        long long warps = (long long)P.ny * P.nz * ((P.nx + A.segx - 1) / A.segx);
        unsigned g = (unsigned)((warps + 3) / 4);
        k_sweep_x<DIM, T><<<g, 128, 0, s>>>(A);
        ++launches;
        if (mark) mark(user, "sweep_x");
    }
    if (DIM == 1) {
        long long n = (long long)P.nx;
        k_rk_update<DIM><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(A);
        ++launches;
        if (mark) mark(user, "rk_update");
    } else {
        dim3 g1((P.nx + 127) / 128, (P.ny + A.seg - 1) / A.seg, P.nz);
        k_sweep_line<1, DIM, T, DIM == 2><<<g1, 128, 0, s>>>(A);
        ++launches;
        if (mark) mark(user, "sweep_y");
        if (DIM == 3) {
            dim3 g2((P.nx + 127) / 128, (P.nz + A.seg - 1) / A.seg, P.ny);
            k_sweep_line<2, DIM, T, true><<<g2, 128, 0, s>>>(A);
            ++launches;
            if (mark) mark(user, "sweep_z");
        }
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace

int sweep_stage(SweepArgs A, cudaStream_t s, bool mixed, int& launches, LaunchMark mark, void* user) {
    A.seg = kSegment;
    A.segx = kSegmentX;
    switch (A.P.dim) {
        case 1:
            return mixed ? stage_dim<1, float>(A, s, launches, mark, user)
                         : stage_dim<1, double>(A, s, launches, mark, user);
        case 2:
            return mixed ? stage_dim<2, float>(A, s, launches, mark, user)
                         : stage_dim<2, double>(A, s, launches, mark, user);
        default:
            return mixed ? stage_dim<3, float>(A, s, launches, mark, user)
                         : stage_dim<3, double>(A, s, launches, mark, user);
    }
}

namespace {

// Work units of the marching stage kernel: strips of 30 columns, each cut
// into segments so that every resident warp gets about unitScale units (1
// by default; sifv_autotune picks it by timing), segments at least 32 rows
// long (a segment first converts 6 rows and reconstructs 2 before its first
// update).
template <typename Kernel>
int march_launch(Kernel kernel, size_t bytes, int* residentWarps, TileArgs A, cudaStream_t s) {
    constexpr int kWarps = 4, kCols = 30;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return -1;
    if (residentWarps[dev] == 0) {
        if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
            return -1;
        int sms = 0, perSm = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, kWarps * 32, bytes) != cudaSuccess)
            return -1;
        residentWarps[dev] = (perSm > 0 ? perSm : 1) * sms * kWarps;
    }
    const int W = residentWarps[dev];
    A.strips = (A.P.nx + kCols - 1) / kCols;
    int segs = (W * (A.unitScale > 1 ? A.unitScale : 1)) / A.strips;
    const int maxSegs = (A.P.ny + 31) / 32;
    if (segs > maxSegs) segs = maxSegs;
    if (segs < 1) segs = 1;
    A.segRows = (A.P.ny + segs - 1) / segs;
    A.segs = (A.P.ny + A.segRows - 1) / A.segRows;
    const long long units = (long long)A.strips * A.segs;
    const long long blocksNeeded = (units + kWarps - 1) / kWarps;
    const long long maxBlocks = (W + kWarps - 1) / kWarps;
    const unsigned grid = (unsigned)(blocksNeeded < maxBlocks ? blocksNeeded : maxBlocks);
    kernel<<<grid, kWarps * 32, bytes, s>>>(A);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

template <int RS>
int march_fp64(const TileArgs& A, cudaStream_t s) {
    static int resident[64] = {0};
    return march_launch(k_march2d<double, RS>, sizeof(MarchWarpSmem<double>) * MarchShape<double>::warps, resident,
                        A, s);
}

template <int RS>
int march_mixed(const TileArgs& A, cudaStream_t s) {
    static int resident[64] = {0};
    return march_launch(k_march2d_mixed<RS>, march_mixed_smem(), resident, A, s);
}

int march_dispatch(const TileArgs& A, cudaStream_t s, bool mixed) {
    switch (A.P.riemann) {
        case SIFV_HLLC: return mixed ? march_mixed<SIFV_HLLC>(A, s) : march_fp64<SIFV_HLLC>(A, s);
        case SIFV_RUSANOV: return mixed ? march_mixed<SIFV_RUSANOV>(A, s) : march_fp64<SIFV_RUSANOV>(A, s);
        default: return mixed ? march_mixed<SIFV_LF>(A, s) : march_fp64<SIFV_LF>(A, s);
    }
}

}  // namespace

int tile2d_stage(const TileArgs& A, cudaStream_t s, bool mixed, int& launches, LaunchMark mark, void* user) {
    int st = march_dispatch(A, s, mixed);
    ++launches;
    if (mark) mark(user, "march2d");
    return st;
}

int tile2d_copy(const Ctl* ctl, const double* const in[4], double* const out[4], size_t n, cudaStream_t s,
                int& launches) {
    Copy4 C;
    for (int q = 0; q < 4; ++q) {
        C.src[q] = in[q];
        C.dst[q] = out[q];
    }
    k_copy4<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(ctl, C, n);
    ++launches;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

namespace {

// relative errors of frcp / fsqrt_pos against IEEE 1/x and sqrt(x) over
// x = m 2^e, m uniform in [1, 2) (a fixed 64-bit hash of the index), e in
// [-60, 60); maxima folded with atomicMax on the bit patterns
__global__ void k_fastmath_check(long long n, unsigned long long* out) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double eR = 0.0, eS = 0.0, eQ = 0.0;
    if (t < n) {
        unsigned long long h = (unsigned long long)t * 0x9E3779B97F4A7C15ull;
        h ^= h >> 29;
        h *= 0xBF58476D1CE4E5B9ull;
        h ^= h >> 32;
        const double m = 1.0 + (double)(h >> 11) * (1.0 / 9007199254740992.0);
        const int e = (int)(t % 120) - 60;
        const double x = ldexp(m, e);
        const double r0 = 1.0 / x, r1 = frcp(x);
        const double s0 = sqrt(x), s1 = fsqrt_pos(x);
        const double q0 = 1.0 / sqrt(x), q1 = frsqrt_pos(x);   // q0 carries two roundings
        eR = fabs(r1 - r0) / r0;
        eS = fabs(s1 - s0) / s0;
        eQ = fabs(q1 - q0) / q0;
        atomicAdd(&out[2], 1ull);
    }
    atomicMax(&out[0], (unsigned long long)__double_as_longlong(eR));
    atomicMax(&out[1], (unsigned long long)__double_as_longlong(eS));
    atomicMax(&out[3], (unsigned long long)__double_as_longlong(eQ));
}

}  // namespace

int sweep_finish_prim(const Params& P, const Fields& F, const Ctl* ctl, cudaStream_t s, int& launches) {
    long long n = (long long)P.nx * P.ny * P.nz;
    k_cons_to_prim_interior<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(P, F, ctl);
    ++launches;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace sifv

namespace sifv {
namespace {

// FP64 fused multiply-add throughput: every thread runs 8 independent
// chains of `iters` dependent FMAs (x <- x * a + b with |a| < 1, so the
// values stay finite) and stores their sum (so nothing is optimised away).
__global__ void __launch_bounds__(256) k_fp64_fma_probe(int iters, double a, double b, double* out) {
    double x[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) x[q] = (double)(threadIdx.x + q);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int q = 0; q < 8; ++q) x[q] = fma(x[q], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) s += x[q];
    if (s == 12345.678) out[blockIdx.x] = s;   // practically never: keeps the chains live
}

}  // namespace
}  // namespace sifv

// Measured FP64 FMA throughput of the current device (the FP64 co-bound of
// the fused stage kernels): a resident grid of the probe kernel, best of
// `reps` launches timed with CUDA events; *tflops = 2 flops per FMA.
extern "C" int sifv_fp64_peak_probe(int reps, double* tflops) {
    if (reps <= 0 || !tflops) return -2;
    int dev = 0, sms = 0, perSm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, sifv::k_fp64_fma_probe, 256, 0))
        return -3;
    const int blocks = sms * (perSm > 0 ? perSm : 1), iters = 4096;
    double* d = nullptr;
    if (cudaMalloc(&d, sizeof(double) * blocks) != cudaSuccess) return -3;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    cudaError_t err = cudaSuccess;
    for (int r = 0; r <= reps && err == cudaSuccess; ++r) {   // the first launch warms up
        cudaEventRecord(e0);
        sifv::k_fp64_fma_probe<<<blocks, 256>>>(iters, 0.999999, 1e-7, d);
        cudaEventRecord(e1);
        err = cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (r > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    if (err != cudaSuccess) return -3;
    const double flops = 2.0 * 8.0 * iters * 256.0 * blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    return 0;
}

extern "C" int sifv_fastmath_selftest(long long n, double* maxRelRcp, double* maxRelSqrt, double* maxRelRsqrt) {
    if (n <= 0 || !maxRelRcp || !maxRelSqrt) return -2;
    unsigned long long* d = nullptr;
    if (cudaMalloc(&d, 4 * sizeof(unsigned long long)) != cudaSuccess) return -3;
    cudaMemset(d, 0, 4 * sizeof(unsigned long long));
    sifv::k_fastmath_check<<<(unsigned)((n + 255) / 256), 256>>>(n, d);
    cudaError_t e = cudaGetLastError();
    unsigned long long h[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess || h[2] != (unsigned long long)n) return -3;   // every argument checked
    std::memcpy(maxRelRcp, &h[0], sizeof(double));
    std::memcpy(maxRelSqrt, &h[1], sizeof(double));
    if (maxRelRsqrt) std::memcpy(maxRelRsqrt, &h[3], sizeof(double));
    return 0;
}
