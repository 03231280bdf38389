// Internal launcher declarations (not part of the C ABI).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace evoc {

// prep.cu
cudaError_t launch_prepare_float(float* X, int64_t n, int ld, int d, float* norms, int* not_unit, int sms,
                                 cudaStream_t stream);

// exact_f32.cu: plain FP32 exact search with fused top-k.
size_t knn_f32_simt_smem();
cudaError_t launch_knn_f32_simt(const float* X, int64_t n, int ld, int k, int cap, uint64_t* scratch, int grid,
                                int32_t* out_idx, float* out_raw, float* out_dist, int64_t q_begin, int64_t q_end,
                                cudaStream_t stream);

// Candidate-buffer capacity used by every fused top-k epilogue for k kept keys.
inline int topk_capacity(int k) {
  int cap = 2 * k;
  if (cap < k + 64) cap = k + 64;
  return (cap + 7) & ~7;
}

}  // namespace evoc
