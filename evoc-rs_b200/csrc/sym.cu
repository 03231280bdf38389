// Symmetric 16-bit scan: the pieces around the scan kernel's symmetric mode
// (tc_scan.cu).
//
// The n x n score matrix of a self-join is symmetric, so the scan multiplies
// only the key tiles from each query block's own rows on: about half the
// tensor-core work.  A score of query row r against key row c > r's block
// then has to reach row c's kept keys too.  Row c cannot hold a heap that
// other CTAs update, so those "mirror" scores go to a per-row mailbox, and
// only the ones that can still matter: a score must reach a threshold that is
// provably no better than row c's final C-th kept key.
//
// Threshold.  A pre-scan keeps, for every row, the C+1 best of a strided
// sample of m rows (the same tensor-core scan, no self rule; its (C+1)-th
// raw value is T_c).  At least C of those are not row c itself, and every
// score the main scan computes for the same pair differs from the pre-scan's
// by at most twice the tensor-core accumulation bound A_c = (L/4 + 2) 2^-21
// |x~_c| max|y~| (both sum the same exact products of the same 16-bit
// operands; the rerank's certificate uses the same model).  So row c's C-th
// best score over all keys has a raw value of at most T_c + 2 A_c, and a
// mirror score whose raw value lies beyond that cannot be among the C kept:
// it is dropped.  The scan compares scores (raw = -score for positive
// scores), so the threshold is stored as a score, rounded towards -inf.
//
// Merge.  Each row's own-side kept keys (the scan's sorted candidates) and
// its mailbox are folded into one heap of C keys; the result is what the
// non-symmetric scan keeps, and the C-th kept raw value is the certificate's
// bound.  A row whose mailbox overflowed gets the bound -f32::MAX, so the
// certificate fails it and the row is scanned again by the non-symmetric
// rescan: nothing depends on the mailbox being large enough.
#include <algorithm>
#include <cfloat>

#include "common.cuh"
#include "kernels.h"

namespace evoc {
namespace {

// Row j of dst = row j * stride of src (j < m); rows m .. m_pad - 1 zero.
// One block per row, 16-byte words.
__global__ void gather_strided_rows_kernel(const uint4* __restrict__ src, int64_t words, int64_t stride, int64_t m,
                                           int64_t m_pad, uint4* __restrict__ dst) {
  for (int64_t j = blockIdx.x; j < m_pad; j += gridDim.x) {
    const uint4* s = src + j * stride * words;
    uint4* d = dst + j * words;
    for (int64_t w = threadIdx.x; w < words; w += blockDim.x) d[w] = j < m ? s[w] : make_uint4(0u, 0u, 0u, 0u);
  }
}

// thr[c] (score threshold of scanned row c's mailbox, +inf past n), umin[c /
// 32] (the smallest of 32 thresholds), count[c] = 0 (count is indexed by
// data-set row; all n are cleared).  One warp per 32 rows.
__global__ void sym_thresholds_kernel(int64_t n, int64_t n_pad, const float* __restrict__ T,
                                      const float* __restrict__ hnorm, const int32_t* __restrict__ perm,
                                      const unsigned int* __restrict__ maxes,
                                      int half_len, float* __restrict__ thr, float* __restrict__ umin,
                                      int32_t* __restrict__ count) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
  const double hm = double(__uint_as_float(maxes[1]));
  for (int64_t w = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); w * 32 < n_pad; w += warps) {
    const int64_t c = w * 32 + lane;
    float u = __int_as_float(0x7f800000);  // +inf: never reached
    if (c < n) {
      const double a = (double(half_len) / 4.0 + 2.0) * 0x1p-21 * double(hnorm[perm[c]]) * hm;
      const double t = double(T[c]) + 2.0 * a;  // raw value no better than row c's C-th kept
      // raw = -score for positive scores; a threshold at or above zero admits every score
      u = t < 0.0 ? __double2float_rd(-t) : __int_as_float(0xff800000);
      count[c] = 0;
    }
    thr[c] = u;
    float mn = u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    if (lane == 0) umin[w] = mn;
  }
}

// One warp per row: the own-side keys (sorted ascending, C of them, idx -1
// past the valid ones) seed a max-heap held by lane 0 in shared memory (a
// descending array is one); the mailbox is read 32 keys at a time and the
// keys below the heap's root are offered.  Writes the row's C candidates and
// its bound (C-th kept raw value; -f32::MAX after an overflow).  stats[0]
// counts overflowed rows, stats[1] the most keys a row was offered.
constexpr int kMergeWarps = 8;

__global__ void __launch_bounds__(kMergeWarps * 32)
sym_merge_kernel(int64_t n, int C, int32_t* __restrict__ cand, const float* __restrict__ own_raw,
                 const int32_t* __restrict__ count, const uint64_t* __restrict__ mail, int cap,
                 float* __restrict__ bound, int32_t* __restrict__ stats) {
  extern __shared__ uint64_t merge_heaps[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  uint64_t* h = merge_heaps + int64_t(wib) * C;
  const int64_t warps = int64_t(gridDim.x) * kMergeWarps;
  for (int64_t r = int64_t(blockIdx.x) * kMergeWarps + wib; r < n; r += warps) {
    int32_t* ci = cand + r * C;
    const float* cr = own_raw + r * C;
    for (int j = lane; j < C; j += 32) {
      const int32_t id = ci[j];
      h[C - 1 - j] = id >= 0 ? make_key(cr[j], id) : kKeyInf;
    }
    __syncwarp();
    KeyHeap heap;
    heap.h = h;
    heap.size = C;
    heap.cap = C;
    const int32_t got = count[r];
    const int64_t cnt = got < cap ? got : cap;
    const uint64_t* mb = mail + r * int64_t(cap);
    for (int64_t b = 0; b < cnt; b += 32) {
      const uint64_t key = b + lane < cnt ? mb[b + lane] : kKeyInf;
      uint32_t pass = __ballot_sync(0xffffffffu, key < h[0]);
      while (pass) {
        const int src = __ffs(pass) - 1;
        pass &= pass - 1;
        const uint64_t k = __shfl_sync(0xffffffffu, key, src);
        if (lane == 0) heap.offer(k);  // re-checks against the moved root
        __syncwarp();
      }
    }
    if (lane == 0) heap.finish();
    __syncwarp();
    for (int j = lane; j < C; j += 32) ci[j] = h[j] == kKeyInf ? -1 : key_index(h[j]);
    if (lane == 0) {
      const bool over = got > cap;
      bound[r] = over ? -FLT_MAX : (h[C - 1] == kKeyInf ? kHeapInf : from_orderable(uint32_t(h[C - 1] >> 32)));
      if (over) atomicAdd(stats, 1);
      if (got > 0) atomicMax(stats + 1, got);
    }
    __syncwarp();
  }
}

}  // namespace

cudaError_t launch_gather_strided_rows(const void* src, int64_t row_bytes, int64_t stride, int64_t m, int64_t m_pad,
                                       void* dst, int sms, cudaStream_t stream) {
  if (row_bytes % 16 || stride < 1 || m < 0 || m_pad < m) return cudaErrorInvalidValue;
  if (m_pad == 0) return cudaSuccess;
  const int64_t grid = std::min<int64_t>(m_pad, int64_t(sms) * 16);
  gather_strided_rows_kernel<<<unsigned(grid), 128, 0, stream>>>(static_cast<const uint4*>(src), row_bytes / 16,
                                                                 stride, m, m_pad, static_cast<uint4*>(dst));
  return cudaGetLastError();
}

cudaError_t launch_sym_thresholds(int64_t n, int64_t n_pad, const float* T, const float* hnorm,
                                  const int32_t* perm, const unsigned int* maxes, int half_len, float* thr,
                                  float* umin, int32_t* count, int sms, cudaStream_t stream) {
  if (n <= 0 || n_pad < n || n_pad % 32) return cudaErrorInvalidValue;
  const int64_t warps = n_pad / 32;
  const int64_t grid = std::min<int64_t>((warps + 7) / 8, int64_t(sms) * 8);
  sym_thresholds_kernel<<<unsigned(grid), 256, 0, stream>>>(n, n_pad, T, hnorm, perm, maxes, half_len, thr, umin,
                                                            count);
  return cudaGetLastError();
}

cudaError_t launch_sym_merge(int64_t n, int C, int32_t* cand, const float* own_raw, const int32_t* count,
                             const uint64_t* mail, int cap, float* bound, int32_t* stats, int sms,
                             cudaStream_t stream) {
  if (n <= 0 || C < 1 || C > 1024 || cap < 1) return cudaErrorInvalidValue;
  const size_t smem = size_t(kMergeWarps) * size_t(C) * 8;
  const int64_t grid = std::min<int64_t>((n + kMergeWarps - 1) / kMergeWarps, int64_t(sms) * 8);
  sym_merge_kernel<<<unsigned(grid), kMergeWarps * 32, smem, stream>>>(n, C, cand, own_raw, count, mail, cap, bound,
                                                                       stats);
  return cudaGetLastError();
}

}  // namespace evoc
