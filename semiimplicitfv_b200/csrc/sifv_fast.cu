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
// into segments so that every resident warp gets at most one unit (a
// segment first converts 6 rows and reconstructs 2 before its first update,
// so segments stay at least 32 rows long).
template <typename T, int RS>
int march_launch(TileArgs A, cudaStream_t s) {
    using S = MarchShape<T>;
    static int residentWarps[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t bytes = sizeof(MarchWarpSmem<T>) * S::warps;
    if (dev < 0 || dev >= 64) return -1;
    if (residentWarps[dev] == 0) {
        if (cudaFuncSetAttribute(k_march2d<T, RS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) !=
            cudaSuccess)
            return -1;
        int sms = 0, perSm = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_march2d<T, RS>, S::warps * 32, bytes) !=
                cudaSuccess)
            return -1;
        residentWarps[dev] = (perSm > 0 ? perSm : 1) * sms * S::warps;
    }
    const int W = residentWarps[dev];
    A.strips = (A.P.nx + S::cols - 1) / S::cols;
    int segs = W / A.strips;
    const int maxSegs = (A.P.ny + 31) / 32;
    if (segs > maxSegs) segs = maxSegs;
    if (segs < 1) segs = 1;
    A.segRows = (A.P.ny + segs - 1) / segs;
    A.segs = (A.P.ny + A.segRows - 1) / A.segRows;
    const long long units = (long long)A.strips * A.segs;
    const long long blocksNeeded = (units + S::warps - 1) / S::warps;
    const long long maxBlocks = (W + S::warps - 1) / S::warps;
    const unsigned grid = (unsigned)(blocksNeeded < maxBlocks ? blocksNeeded : maxBlocks);
    k_march2d<T, RS><<<grid, S::warps * 32, bytes, s>>>(A);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

template <typename T>
int march_dispatch(const TileArgs& A, cudaStream_t s) {
    switch (A.P.riemann) {
        case SIFV_HLLC: return march_launch<T, SIFV_HLLC>(A, s);
        case SIFV_RUSANOV: return march_launch<T, SIFV_RUSANOV>(A, s);
        default: return march_launch<T, SIFV_LF>(A, s);
    }
}

}  // namespace

int tile2d_stage(const TileArgs& A, cudaStream_t s, bool mixed, int& launches, LaunchMark mark, void* user) {
    int st = mixed ? march_dispatch<float>(A, s) : march_dispatch<double>(A, s);
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
    double eR = 0.0, eS = 0.0;
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
        eR = fabs(r1 - r0) / r0;
        eS = fabs(s1 - s0) / s0;
        atomicAdd(&out[2], 1ull);
    }
    atomicMax(&out[0], (unsigned long long)__double_as_longlong(eR));
    atomicMax(&out[1], (unsigned long long)__double_as_longlong(eS));
}

}  // namespace

int sweep_finish_prim(const Params& P, const Fields& F, const Ctl* ctl, cudaStream_t s, int& launches) {
    long long n = (long long)P.nx * P.ny * P.nz;
    k_cons_to_prim_interior<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(P, F, ctl);
    ++launches;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace sifv

extern "C" int sifv_fastmath_selftest(long long n, double* maxRelRcp, double* maxRelSqrt) {
    if (n <= 0 || !maxRelRcp || !maxRelSqrt) return -2;
    unsigned long long* d = nullptr;
    if (cudaMalloc(&d, 3 * sizeof(unsigned long long)) != cudaSuccess) return -3;
    cudaMemset(d, 0, 3 * sizeof(unsigned long long));
    sifv::k_fastmath_check<<<(unsigned)((n + 255) / 256), 256>>>(n, d);
    cudaError_t e = cudaGetLastError();
    unsigned long long h[3] = {0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess || h[2] != (unsigned long long)n) return -3;   // every argument checked
    std::memcpy(maxRelRcp, &h[0], sizeof(double));
    std::memcpy(maxRelSqrt, &h[1], sizeof(double));
    return 0;
}
