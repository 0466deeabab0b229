// sifv_sweep_api.h -- host entry points and argument block of the fused
// sweep path, shared by the C ABI translation unit and the sweep
// translation unit.
#pragma once

#include <cuda_runtime.h>

#include "sifv_device.cuh"

namespace sifv {

// EOS constants of the single-phase face flux.
struct FluxConsts {
    double gamma, pInf, invGm1, gPinf;
};

// Stage update of one interior cell from its complete flux divergence
// (src/ExplicitSolver.cpp:127-188) as U = a1 U + a2 U0 + a3 dt R with
// (a1, a2, a3) = (c1, c2, c3) / c4; dt is read from device memory.
struct RKUpdate {
    double a1, a2, a3;
    int save;     // stage 0 of a multi-stage scheme: back up U into U0
    int useU0;
};

struct SweepArgs {
    Params P;
    Fields F;
    const Ctl* ctl;
    FluxConsts C;
    RKUpdate K;
    double eps;
    int seg;       // cells per thread segment (line sweeps)
    int segx;      // cells per warp segment of a row (x sweep), 32 m - 2
    double* rhs[5];  // FP64 rhs buffer (rho, rhoU, rhoV, rhoW, rhoE)
    double* rhoP;    // stage primitive density: the conservative rho is updated in place by the
                     // last sweep while neighbouring stencils still need the stage-start value
    const double* inv[3];   // 1 / d per cell (ghosts included)
};

// One RK stage of the 2D explicit step as one fused kernel
// (sifv_march2d.cuh): U' = a1 in + a2 u0 + a3 dt R(in), written to `out`
// (which may be u0, never `in`); `last` also writes the primitives of U'.
struct TileArgs {
    Params P;
    FluxConsts C;
    double eps;
    Ctl* ctl;
    const double* in[4];    // stage input: rho, rhoU, rhoV, rhoE
    const double* u0[4];    // step-start state (own cells), null when a2 == 0
    double* out[4];         // stage output
    double a1, a2, a3;
    const double* inv[2];   // 1 / dx, 1 / dy per cell (ghosts included)
    int last;               // write the primitives of the new state
    double *velU, *velV, *pres;
    int strips, segs, segRows;   // work units: strips of 30 columns x segments of segRows rows (set by the launcher)
    int unitScale;               // work units per resident warp (autotuned; 0 or 1: one)
    // last stage: fold the acoustic dt of the new state (k_dt_acoustic's
    // expressions) into ctl->dtBits for the next step
    int dtNext;
    double cfl;
    const double *dx, *dy;      // cell widths (ghosts included)
};

// Called after each kernel launch with the kernel family's name (per-kernel
// timing); may be null.
typedef void (*LaunchMark)(void* user, const char* family);

// One RK stage of the explicit step on the fused sweep kernels
// (mixed: FP32 reconstruction / Riemann bulk).  Returns 0 on success.
int sweep_stage(SweepArgs A, cudaStream_t s, bool mixed, int& launches, LaunchMark mark = nullptr,
                void* user = nullptr);

int tile2d_stage(const TileArgs& A, cudaStream_t s, bool mixed, int& launches, LaunchMark mark = nullptr,
                 void* user = nullptr);
// out[q] = in[q] over n values, skipped when the step is (device-side loops).
int tile2d_copy(const Ctl* ctl, const double* const in[4], double* const out[4], size_t n, cudaStream_t s,
                int& launches);

// End-of-step conservative -> primitive on interior cells.
int sweep_finish_prim(const Params& P, const Fields& F, const Ctl* ctl, cudaStream_t s, int& launches);

}  // namespace sifv
