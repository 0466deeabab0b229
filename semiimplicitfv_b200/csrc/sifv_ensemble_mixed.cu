// sifv_ensemble_mixed.cu -- the FP32-bulk instantiation of the ensemble
// kernel, compiled with FMA contraction (mixed precision is held to an L1
// error bound, not to bit equality).
#include "sifv_ensemble.cuh"
#include "sifv_ensemble_api.h"

namespace sifv {

// The mixture pressure recovery from total energy (where pInf ~ 6e8
// cancels), the carried state and the update stay FP64 inside the kernel.
int ensemble_launch_mixed(const EnsArgs& A, int nph, int blockSize, cudaStream_t s) {
    if (nph == 0) k_ensemble<float, 0><<<A.nInst, blockSize, 0, s>>>(A);
    else if (nph == 2) k_ensemble<float, 2><<<A.nInst, blockSize, 0, s>>>(A);
    else k_ensemble<float, 8><<<A.nInst, blockSize, 0, s>>>(A);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace sifv
