// sifv_adjoint_api.h -- arguments and launchers of the discrete adjoint /
// tangent kernels (sifv_adjoint.cuh), used by the C ABI translation unit.
#pragma once

#include <cuda_runtime.h>

#include "sifv_device.cuh"

namespace sifv {

struct AdjArgs {
    Params P;
    Fields F;            // stage input: cons (and prims incl. ghosts once filled)
    double* lam[5];      // dJ/dU' in, dJ/dU out (rho, momenta, rhoE; interior cells)
    double* acc0[5];     // dJ/dU0 accumulated through the RK combination
    double* share[3];    // per direction: 10 * (dim + 2) doubles per face
    double dt, a1, a2, a3;   // dt and c1/c4, c2/c4, c3/c4 of the stage
    const double* dtDev;     // non-null: dt is read from device memory (the step's CFL dt)
    int stage0;          // stage 0 of a step: lam += acc0, acc0 = 0
    int fp32;            // local Jacobians of the reverse sweep in FP32
    double* tan[5];      // tangent dU (interior cells)
    double* tan0[5];     // tangent of the step-start state
    double* tanW[5];     // tangent of the primitives (all cells)
    double* tanF[3][5];  // tangent face fluxes per direction
};

// Reverse of one RK stage (prims of the stage input must be filled).
int adjoint_stage(const AdjArgs& A, cudaStream_t s);
// Tangent of one stage before the forward update (prim + face tangents) and
// after it (the RK combination; save = stage 0 of a multi-stage step).
int tangent_faces(const AdjArgs& A, cudaStream_t s);
int tangent_update(const AdjArgs& A, int save, cudaStream_t s);
// Zero the ghost entries of a cell array.
int zero_ghosts(const Params& P, double* f, cudaStream_t s);

}  // namespace sifv
