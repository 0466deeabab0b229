// sifv_fast.cu -- launchers of the fused sweep kernels (fast-FP64 and
// mixed-precision explicit step).  Compiled with FMA contraction enabled:
// these paths trade the reference's exact operation order for speed and
// are held to the relative tolerance of the parity tests instead of bit
// equality.
#include <cuda_runtime.h>

#include "sifv_sweep.cuh"
#include "sifv_sweep_api.h"

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

int sweep_finish_prim(const Params& P, const Fields& F, const Ctl* ctl, cudaStream_t s, int& launches) {
    long long n = (long long)P.nx * P.ny * P.nz;
    k_cons_to_prim_interior<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(P, F, ctl);
    ++launches;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace sifv
