// sifv_ensemble_api.h -- launchers of the ensemble kernel, shared by the
// reference-ordered and the mixed-precision translation units.
#pragma once

#include <cuda_runtime.h>

namespace sifv {

struct EnsArgs;

// FP32-bulk instantiation (sifv_ensemble_mixed.cu).  Returns 0 on success.
int ensemble_launch_mixed(const EnsArgs& A, int nph, int blockSize, cudaStream_t s);

}  // namespace sifv
