// fkd_mlp.h -- the learned split predictor shared by the MLP kernels and the
// build (see fkd_mlp.cu, fkd_features.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/fkdtree_b200.h"

namespace fkd {
const float* mlp_params(fkd_mlp m);
cudaError_t mlp_infer(const float* params, const float* x, uint64_t n, float* y, cudaStream_t stream);
}  // namespace fkd
