// mlp.hpp -- launchers of the learned decision network used by the
// correction pipeline (the kernels live in mlp.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace careb200 {

constexpr int kMlpFeatures = 24;
constexpr int kMlpFloats = 5873;

// Logits of rows x[n][24] (n read from *n_dev when it is non-null, capped at
// n). err gets bit 1 when a tensor-core completion wait ran out.
cudaError_t mlp_infer(const float* params, const float* x, uint64_t n, const unsigned long long* n_dev,
                      float* logits, int* err, cudaStream_t stream);

}  // namespace careb200
