// The reference's integer brute-force branch, reproduced bit for bit.
//
// knn_graph_impl (src/knn.rs:418-421) sends i8 and u8 data with
// n <= brute_force_max_n to brute_force_knn (src/knn.rs:189-281): for each row
// i it walks j = 0 .. n-1 (skipping i) in order, computes the dissimilarity
// (-(i8 dot as f32); -(popcount(a & b) / popcount(a | b)) in f32, 0.0 for an
// empty union) and, when it is strictly below the root of a k-slot max-heap
// (initially +inf / -1), replaces the root and sifts it down; the heap array
// itself is the output row (not sorted).  The order of the replacements
// decides the heap's final arrangement, so this kernel keeps it: one warp per
// row computes the dissimilarities of 32 consecutive j at a time (each lane
// its own j, 16-byte loads, dp4a or popc), a ballot marks those below the
// root, and lane 0 applies them in j order with the reference's exact
// sift-down (strict < compares, left child before right).  A candidate that
// fails against the root from before the ballot fails against every later
// root (the root never grows), so nothing is skipped that the serial loop
// would take.  Work is O(n^2 d) on the SIMT units: the branch is meant, as in
// the reference, for small n.
#include <algorithm>
#include <cstdint>

#include "common.cuh"
#include "kernels.h"

namespace evoc {

namespace {

// Shared memory of one warp: the query row, the heap's k distances and k
// indices, rounded up so the next warp's query row stays 16-byte aligned.
__host__ __device__ __forceinline__ size_t warp_bytes(int64_t row_bytes, int k) {
  return (size_t(row_bytes) + size_t(k) * 8 + 15) / 16 * 16;
}

template <int DT>  // 1: i8, 2: u8
__device__ __forceinline__ float brute_dissimilarity(const uint4* __restrict__ a, const uint4* __restrict__ b,
                                                     int words16) {
  if (DT == 1) {
    int32_t acc = 0;
    for (int w = 0; w < words16; w++) {
      const uint4 x = a[w], y = __ldg(b + w);
      acc = __dp4a(int32_t(x.x), int32_t(y.x), acc);
      acc = __dp4a(int32_t(x.y), int32_t(y.y), acc);
      acc = __dp4a(int32_t(x.z), int32_t(y.z), acc);
      acc = __dp4a(int32_t(x.w), int32_t(y.w), acc);
    }
    return -__int2float_rn(acc);
  }
  uint32_t inter = 0, uni = 0;
  for (int w = 0; w < words16; w++) {
    const uint4 x = a[w], y = __ldg(b + w);
    inter += __popc(x.x & y.x) + __popc(x.y & y.y) + __popc(x.z & y.z) + __popc(x.w & y.w);
    uni += __popc(x.x | y.x) + __popc(x.y | y.y) + __popc(x.z | y.z) + __popc(x.w | y.w);
  }
  return uni > 0 ? -__fdiv_rn(__uint2float_rn(inter), __uint2float_rn(uni)) : 0.0f;
}

}  // namespace

// Rows q_begin .. q_end-1 (output rows 0 ..); X: n rows of row_bytes (a
// multiple of 16, zero padded).  Shared memory per warp: the query row, then
// the heap (k f32 distances, k int32 indices).
template <int DT>
__global__ void brute_force_heap_kernel(const uint8_t* __restrict__ X, int64_t n, int64_t row_bytes, int k,
                                        int64_t q_begin, int64_t q_end, int32_t* __restrict__ out_idx,
                                        float* __restrict__ out_raw, float* __restrict__ out_dist) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  uint8_t* base = smem + size_t(warp) * warp_bytes(row_bytes, k);
  uint4* qrow = reinterpret_cast<uint4*>(base);
  float* hd = reinterpret_cast<float*>(base + row_bytes);
  int32_t* hi = reinterpret_cast<int32_t*>(base + row_bytes + size_t(k) * 4);
  const int words16 = int(row_bytes / 16);
  for (int64_t i = q_begin + int64_t(blockIdx.x) * wpb + warp; i < q_end; i += int64_t(gridDim.x) * wpb) {
    const uint4* src = reinterpret_cast<const uint4*>(X + i * row_bytes);
    for (int w = lane; w < words16; w += 32) qrow[w] = src[w];
    for (int t = lane; t < k; t += 32) {
      hd[t] = __int_as_float(0x7f800000);  // f32::INFINITY
      hi[t] = -1;
    }
    __syncwarp();
    for (int64_t j0 = 0; j0 < n; j0 += 32) {
      const int64_t j = j0 + lane;
      float dj = 0.0f;
      const bool live = j < n && j != i;
      if (live) dj = brute_dissimilarity<DT>(qrow, reinterpret_cast<const uint4*>(X + j * row_bytes), words16);
      const float root = hd[0];
      uint32_t mask = __ballot_sync(0xffffffffu, live && dj < root);
      while (mask) {
        const int src_lane = __ffs(mask) - 1;
        mask &= mask - 1;
        const float d = __shfl_sync(0xffffffffu, dj, src_lane);
        if (lane == 0 && d < hd[0]) {
          // replace the root, then the reference's sift-down
          hd[0] = d;
          hi[0] = int32_t(j0 + src_lane);
          int pos = 0;
          for (;;) {
            const int left = 2 * pos + 1;
            if (left >= k) break;
            const int right = left + 1;
            int swap = pos;
            if (hd[swap] < hd[left]) swap = left;
            if (right < k && hd[swap] < hd[right]) swap = right;
            if (swap == pos) break;
            const float td = hd[pos];
            hd[pos] = hd[swap];
            hd[swap] = td;
            const int32_t ti = hi[pos];
            hi[pos] = hi[swap];
            hi[swap] = ti;
            pos = swap;
          }
        }
        __syncwarp();
      }
    }
    const int64_t orow = (i - q_begin) * k;
    for (int t = lane; t < k; t += 32) {
      const float raw = hd[t];
      out_idx[orow + t] = hi[t];
      if (out_raw) out_raw[orow + t] = raw;
      if (out_dist) out_dist[orow + t] = transform_raw(DT, raw);
    }
    __syncwarp();
  }
}

size_t brute_force_smem_per_warp(int64_t row_bytes, int k) { return warp_bytes(row_bytes, k); }

cudaError_t launch_brute_force_heap(int dtype, const void* X, int64_t n, int64_t row_bytes, int k, int64_t q_begin,
                                    int64_t q_end, int32_t* out_idx, float* out_raw, float* out_dist, int sms,
                                    cudaStream_t stream) {
  if ((dtype != 1 && dtype != 2) || row_bytes % 16 != 0 || k < 1 || q_begin < 0 || q_end > n || q_begin >= q_end)
    return cudaErrorInvalidValue;
  const size_t per_warp = brute_force_smem_per_warp(row_bytes, k);
  if (per_warp > 200 * 1024) return cudaErrorInvalidValue;
  int wpb = int(std::min<size_t>(8, std::max<size_t>(1, (96 * 1024) / per_warp)));
  const size_t smem = per_warp * size_t(wpb);
  const int64_t rows = q_end - q_begin;
  int64_t blocks = (rows + wpb - 1) / wpb;
  if (blocks > int64_t(sms) * 32) blocks = int64_t(sms) * 32;
  auto kern = dtype == 1 ? brute_force_heap_kernel<1> : brute_force_heap_kernel<2>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  kern<<<unsigned(blocks), wpb * 32, smem, stream>>>(static_cast<const uint8_t*>(X), n, row_bytes, k, q_begin, q_end,
                                                      out_idx, out_raw, out_dist);
  return cudaGetLastError();
}

}  // namespace evoc
