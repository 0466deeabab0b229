// sifv_ensemble_mixed.cu -- the FP32-bulk instantiation of the ensemble
// kernel, compiled with FMA contraction and the approximate single-precision
// division / square root of --use_fast_math (FP64 arithmetic is unaffected;
// mixed precision is held to an L1 error bound, not to bit equality).
#include "sifv_ensemble.cuh"
#include "sifv_ensemble_api.h"

namespace sifv {

// The mixture pressure recovery from total energy (where pInf ~ 6e8
// cancels), the carried state and the update stay FP64 inside the kernel.
namespace {
template <int NPH>
int launch_f(const EnsArgs& A, int blockSize, cudaStream_t s) {
    const size_t bytes = ens_smem_bytes<float, NPH>(blockSize);
    if (cudaFuncSetAttribute(k_ensemble<float, NPH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) !=
        cudaSuccess)
        return -1;
    k_ensemble<float, NPH><<<A.nInst, blockSize, bytes, s>>>(A);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
}  // namespace

int ensemble_launch_mixed(const EnsArgs& A, int nph, int blockSize, cudaStream_t s) {
    if (nph == 0) return launch_f<0>(A, blockSize, s);
    if (nph == 2) return launch_f<2>(A, blockSize, s);
    return launch_f<8>(A, blockSize, s);
}

}  // namespace sifv
