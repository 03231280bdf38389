// Second stage of the 16-bit form: FP32 rerank of the oversampled candidates,
// and the certificate that the candidates hold the row's true k nearest.
//
// The FP16 (or BF16) tensor-core scan (tc_scan.cu) keeps C = oversample*k
// candidates per row.  Here each warp takes one query row, recomputes the C
// dot products in FP32 from the original (renormalised) f32 rows, ranks them
// by the reference's dissimilarity (src/fast_cosine.rs:33-45; self = -1.0)
// with ties by index, and only for candidates whose FP32 value lies within
// 1e-6 of the k-th value recomputes the dot product in FP64 to settle the
// order at the boundary.  Output is the final sorted row with transformed
// distances (src/knn.rs:156-171).
//
// Certificate.  Every key the scan did not keep scored no better than its
// C-th kept key (raw value b_C).  With x~, y~ the 16-bit operands and
// r = x - x~ their residuals (exact in f32), the scan's score of (x, y)
// differs from the exact dot x.y by at most
//   E = |r_x| |y~| + |x~| |r_y| + |r_x| |r_y|          (Cauchy-Schwarz on
//       x.y - x~.y~ = x~.r_y + r_x.y~ + r_x.r_y)
//     + (L/4 + 2) 2^-21 |x~| |y~|                      (tensor-core f32
//       accumulation of L products, exact products, at most two units of
//       2^-22 of the running magnitude lost per four-term step),
// taking the maxima of |r_y| and |y~| over all keys.  So every key not kept
// has an exact dissimilarity of at least min(b_C, 0) - E.  The k-th value
// found here is within e32 = (ceil(d/32) + 8) 2^-24 of exact (this kernel's
// FP32 summation: ceil(d/32) FMAs per lane and five shuffle additions, on
// rows of norm at most 1 + 1e-5).  A row is certified when
//   min(b_C, 0) - E >= min(r_k + e32, 0) - 1e-6,
// i.e. a key the scan dropped can at most tie the k-th within the 1e-6 the
// exact FP32 form also allows.  Rows that fail are listed for a second scan
// with a larger candidate set and, failing that, an exact FP32 scan
// (evoc_gpu.cu).  FP16 operands (11-bit significands) make E about 8x smaller
// than BF16 (8-bit) on unit rows, which is what lets nearly every row pass.
//
// The candidate rows are gathered from HBM, so the order in which query rows
// are reranked decides how often those rows are found in L2.  Rows are
// processed grouped by their nearest pivot (a deterministic sample of the
// data found with the same tensor-core scan), so the warps in flight at any
// moment work on nearby points whose candidates overlap.
#include <cuda_bf16.h>

#include "batch.h"
#include "common.cuh"
#include "kernels.h"

namespace evoc {

namespace {
constexpr int RW = 8;          // warps per block
constexpr int MAXC = 256;      // candidates per row handled in shared memory
constexpr int GROUP = 4;       // candidates per pass over the query row

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void warp_bitonic(uint64_t* keys, int P, int lane) {
  for (int size = 2; size <= P; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = lane; i < (P >> 1); i += 32) {
        const int lo = 2 * stride * (i / stride) + (i % stride);
        const int hi = lo + stride;
        const bool up = (lo & size) == 0;
        const uint64_t a = keys[lo], b = keys[hi];
        if ((a > b) == up) {
          keys[lo] = b;
          keys[hi] = a;
        }
      }
      __syncwarp();
    }
  }
}

__device__ __forceinline__ float key_raw(uint64_t key) { return from_orderable(uint32_t(key >> 32)); }

// The certificate above for one reranked row (kw holds its C sorted keys).
// Warp-uniform result.
__device__ __forceinline__ bool certify_row(const CertArgs& ct, const uint64_t* kw, int C, int k, int d,
                                            int64_t n_keys, int64_t qg, float b_c, int lane) {
  if (C >= n_keys) return true;  // every key was a candidate
  bool self_in = false;
  float worst = -3.0e38f;  // largest FP32 raw value among the k reported
  bool full = true;
  for (int j = lane; j < C; j += 32) {
    const uint64_t key = kw[j];
    if (key != kKeyInf && key_index(key) == qg) self_in = true;
    if (j < k) {
      if (key == kKeyInf) full = false;
      else worst = fmaxf(worst, key_raw(key));
    }
  }
  self_in = __any_sync(0xffffffffu, self_in);
  full = __all_sync(0xffffffffu, full);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) worst = fmaxf(worst, __shfl_xor_sync(0xffffffffu, worst, o));
  if (!self_in || !full || k > C) return false;
  const double e32 = (double((d + 31) / 32) + 8.0) * 0x1p-24 * 1.0001;
  const double U = fmin(double(worst) + e32, 0.0);
  const double rq = ct.rnorm[qg], hq = ct.hnorm[qg];
  const double rm = double(__uint_as_float(ct.maxes[0])), hm = double(__uint_as_float(ct.maxes[1]));
  const double E = rq * hm + hq * rm + rq * rm + (double(ct.half_len) / 4.0 + 2.0) * 0x1p-21 * hq * hm;
  const double LB = fmin(double(b_c), 0.0) - E;
  return LB >= U - 1e-6 + 1e-12;
}
}  // namespace

// One query row: FP32 dot products with its C candidates, a warp bitonic
// sort of (raw, index) keys, FP64 at the k-th boundary, the sorted row
// written to output row q.  kw: this warp's P key slots; dw: its 32 doubles.
// With ct (and b_c, the scan's C-th kept raw value), returns whether the row
// is certified (always true without).
__device__ __forceinline__ bool rerank_row(const float* __restrict__ X, int ld, int d, int64_t n_keys, int64_t q,
                                           int64_t qg, const int32_t* __restrict__ cq, int C, int P, int k,
                                           int32_t* __restrict__ out_idx, float* __restrict__ out_raw,
                                           float* __restrict__ out_dist, int* status, uint64_t* kw, double* dw,
                                           int lane, const CertArgs* ct = nullptr, float b_c = 0.0f) {
  const float* xq = X + qg * ld;
  for (int j0 = 0; j0 < C; j0 += GROUP) {
    int32_t id[GROUP];
    float acc[GROUP];
#pragma unroll
    for (int u = 0; u < GROUP; u++) {
      id[u] = (j0 + u < C) ? cq[j0 + u] : -1;
      if (id[u] >= n_keys) {  // never written by a finished scan: record it, skip the candidate
        if (status) atomicCAS(status, 0, kStatusBadCandidate);
        id[u] = -1;
      }
      acc[u] = 0.0f;
    }
    for (int t = lane; t < d; t += 32) {
      const float xv = xq[t];
#pragma unroll
      for (int u = 0; u < GROUP; u++)
        if (id[u] >= 0) acc[u] = fmaf(xv, X[int64_t(id[u]) * ld + t], acc[u]);
    }
#pragma unroll
    for (int u = 0; u < GROUP; u++) {
      const float dot = warp_sum(acc[u]);
      if (lane == u && j0 + u < C) {
        uint64_t key = kKeyInf;
        if (id[u] >= 0) key = make_key(id[u] == qg ? -1.0f : raw_cosine(dot), id[u]);
        kw[j0 + u] = key;
      }
    }
  }
  for (int j = C + lane; j < P; j += 32) kw[j] = kKeyInf;
  __syncwarp();
  warp_bitonic(kw, P, lane);

  // FP64 only where FP32 cannot separate candidates at the k-th boundary.
  const int kk = k < C ? k : C;
  if (kk < C && kw[kk - 1] != kKeyInf && kw[kk] != kKeyInf) {
    const float rk = key_raw(kw[kk - 1]);
    int lo = kk - 1, hi = kk;
    while (lo > 0 && kw[lo - 1] != kKeyInf && key_raw(kw[lo - 1]) >= rk - 1e-6f) lo--;
    while (hi < C && kw[hi] != kKeyInf && key_raw(kw[hi]) <= rk + 1e-6f) hi++;
    const int g = hi - lo;
    if (g > 1 && g <= 32) {
      for (int j = 0; j < g; j++) {
        const int32_t c = key_index(kw[lo + j]);
        double acc = 0.0;
        for (int t = lane; t < d; t += 32) acc = fma(double(xq[t]), double(X[int64_t(c) * ld + t]), acc);
        acc = warp_sum_d(acc);
        // FP64 dissimilarity under the reference's rule: self -1, -dot, or the
        // MIN_POSITIVE sentinel for dots <= 0 (a true tie, broken by index).
        if (lane == 0) dw[j] = (c == qg) ? -1.0 : (acc > 0.0 ? -acc : double(kMinPositive));
      }
      __syncwarp();
      if (lane == 0) {
        // insertion sort of the boundary group by (FP64 dissimilarity, index)
        for (int i = 1; i < g; i++) {
          const double dv = dw[i];
          const uint64_t kv = kw[lo + i];
          int j = i - 1;
          while (j >= 0 && (dw[j] > dv || (dw[j] == dv && key_index(kw[lo + j]) > key_index(kv)))) {
            dw[j + 1] = dw[j];
            kw[lo + j + 1] = kw[lo + j];
            j--;
          }
          dw[j + 1] = dv;
          kw[lo + j + 1] = kv;
        }
      }
      __syncwarp();
    }
  }
  const bool certified = ct ? certify_row(*ct, kw, C, k, d, n_keys, qg, b_c, lane) : true;
  // Write the row (lane j writes entries j, j+32, ...).
  for (int j = lane; j < k; j += 32) {
    const uint64_t key = j < C ? kw[j] : kKeyInf;
    const bool ok = key != kKeyInf;
    const float raw = ok ? key_raw(key) : kHeapInf;
    out_idx[q * k + j] = ok ? key_index(key) : -1;
    if (out_raw) out_raw[q * k + j] = raw;
    if (out_dist) out_dist[q * k + j] = transform_raw(0, raw);
  }
  __syncwarp();
  return certified;
}

__global__ void __launch_bounds__(RW * 32)
rerank_f32_kernel(const float* __restrict__ X, int ld, int d, int64_t n, int64_t n_keys, int64_t q_row0,
                  const int32_t* __restrict__ cand, int C, int k, const int32_t* __restrict__ order,
                  int32_t* __restrict__ out_idx, float* __restrict__ out_raw, float* __restrict__ out_dist,
                  int* status, const CertArgs cert, bool use_cert, bool by_item, int64_t n_out) {
  __shared__ uint64_t keys[RW][MAXC];
  __shared__ double d64[RW][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // The candidates are only complete when the scan that wrote them finished.
  if (status && *reinterpret_cast<volatile int*>(status) != 0) return;
  int P = 1;
  while (P < C) P <<= 1;
  for (int64_t w = int64_t(blockIdx.x) * RW + warp; w < n; w += int64_t(gridDim.x) * RW) {
    int64_t q = order ? order[w] : w;  // output row
    if (q < 0 || q >= n_out) {           // a malformed order: record it, skip the row
      if (lane == 0 && status) atomicCAS(status, 0, kStatusBadOrder);
      continue;
    }
    const int64_t ci = by_item ? w : q;  // candidate row
    const bool ok = rerank_row(X, ld, d, n_keys, q, q_row0 + q, cand + ci * C, C, P, k, out_idx, out_raw, out_dist,
                               status, keys[warp], d64[warp], lane, use_cert ? &cert : nullptr,
                               use_cert ? cert.bound[ci] : 0.0f);
    if (!ok && lane == 0) {
      const int slot = atomicAdd(cert.fail_count, 1);
      if (slot < cert.fail_cap) cert.fail_list[slot] = int32_t(q);
    }
  }
}

// The same per row over the requests of a batch: warp per global row, the
// request found by binary search over the rows' prefix offsets.
__global__ void __launch_bounds__(RW * 32)
batch_rerank_kernel(BatchHeader* hdr, const BatchRowJob* __restrict__ jobs) {
  __shared__ uint64_t keys[RW][MAXC];
  __shared__ double d64[RW][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* status = &hdr->status;
  if (*reinterpret_cast<volatile int*>(status) != 0) return;
  const int nj = hdr->n_jobs;
  const int64_t total = hdr->total_rows;
  for (int64_t w = int64_t(blockIdx.x) * RW + warp; w < total; w += int64_t(gridDim.x) * RW) {
    int lo = 0, hi = nj - 1;
    while (lo < hi) {  // last job with row_base <= w
      const int mid = (lo + hi + 1) >> 1;
      if (jobs[mid].row_base <= w) lo = mid;
      else hi = mid - 1;
    }
    const BatchRowJob& J = jobs[lo];
    const int64_t q = w - J.row_base;
    if (q < 0 || q >= J.n) {
      if (lane == 0) atomicCAS(status, 0, kStatusBadOrder);
      continue;
    }
    int P = 1;
    while (P < J.C) P <<= 1;
    CertArgs ct{J.bound, J.rnorm, J.hnorm, J.maxes, int(J.ldb / 2), nullptr, nullptr, 0};
    const bool ok = rerank_row(J.x, int(J.ld), int(J.dim), J.n, q, q, J.cand + q * J.C, J.C, P, J.keff, J.out_idx,
                               J.out_raw, J.out_dist, status, keys[warp], d64[warp], lane,
                               J.certify ? &ct : nullptr, J.certify ? J.bound[q] : 0.0f);
    if (!ok && lane == 0) {
      const int slot = atomicAdd(&hdr->fail_count, 1);
      if (slot < hdr->fail_cap) {
        hdr->fail_list[2 * slot] = lo;
        hdr->fail_list[2 * slot + 1] = int32_t(q);
      }
    }
  }
}

cudaError_t launch_rerank_f32(const float* X, int ld, int d, int64_t n, int64_t n_keys, int64_t q_row0,
                              const int32_t* cand, int C, int k, const int32_t* order, int32_t* out_idx, float* out_raw,
                              float* out_dist, int* status, int sms, cudaStream_t stream, const CertArgs* cert,
                              bool by_item, int64_t n_out) {
  if (C > MAXC || C < 1) return cudaErrorInvalidValue;
  if (by_item && !order) return cudaErrorInvalidValue;
  if (cert && (!cert->bound || !cert->rnorm || !cert->hnorm || !cert->maxes || !cert->fail_list || !cert->fail_count))
    return cudaErrorInvalidValue;
  int64_t blocks = (n + RW - 1) / RW;
  if (blocks > int64_t(sms) * 16) blocks = int64_t(sms) * 16;
  CertArgs ct{};
  if (cert) ct = *cert;
  rerank_f32_kernel<<<unsigned(blocks), RW * 32, 0, stream>>>(X, ld, d, n, n_keys, q_row0, cand, C, k, order,
                                                               out_idx, out_raw, out_dist, status, ct, cert != nullptr,
                                                               by_item, n_out < 0 ? n : n_out);
  return cudaGetLastError();
}

cudaError_t launch_batch_rerank(BatchHeader* hdr, const BatchRowJob* jobs, int grid, cudaStream_t stream) {
  batch_rerank_kernel<<<unsigned(grid), RW * 32, 0, stream>>>(hdr, jobs);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Locality order: pivot rows, nearest-pivot labels, counting sort.
// ---------------------------------------------------------------------------
__global__ void gather_rows_kernel(const uint8_t* __restrict__ src, int64_t row_bytes, int64_t n, int64_t n_piv,
                                   uint8_t* __restrict__ dst) {
  // pivot p is row floor(p * n / n_piv)
  const int64_t total = n_piv * row_bytes;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t p = e / row_bytes, b = e % row_bytes;
    const int64_t r = p * n / n_piv;
    dst[e] = src[r * row_bytes + b];
  }
}

__global__ void label_hist_kernel(const int32_t* __restrict__ label, int64_t n, int nb, int32_t* __restrict__ hist) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    int b = label[i];
    b = (b < 0 || b >= nb) ? 0 : b;
    atomicAdd(&hist[b], 1);
  }
}

// Single block: exclusive prefix sum of hist[0..nb) into cursor.
__global__ void exclusive_scan_kernel(const int32_t* __restrict__ hist, int nb, int32_t* __restrict__ cursor) {
  __shared__ int32_t part[1024];
  const int t = threadIdx.x;
  const int per = (nb + blockDim.x - 1) / blockDim.x;
  int32_t s = 0;
  for (int i = 0; i < per; i++) {
    const int b = t * per + i;
    if (b < nb) s += hist[b];
  }
  part[t] = s;
  __syncthreads();
  for (int off = 1; off < blockDim.x; off <<= 1) {
    const int32_t v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int32_t run = part[t] - s;
  for (int i = 0; i < per; i++) {
    const int b = t * per + i;
    if (b < nb) {
      cursor[b] = run;
      run += hist[b];
    }
  }
}

__global__ void label_scatter_kernel(const int32_t* __restrict__ label, int64_t n, int nb, int32_t* __restrict__ cursor,
                                     int32_t* __restrict__ order) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    int b = label[i];
    b = (b < 0 || b >= nb) ? 0 : b;
    const int32_t pos = atomicAdd(&cursor[b], 1);
    if (pos >= 0 && pos < n) order[pos] = int32_t(i);
  }
}

// Rows inside each cell sorted by index, so the order does not depend on the
// order the scatter's atomics ran in (Shell sort, one thread per cell).
__global__ void sort_cells_kernel(const int32_t* __restrict__ cell_end, const int32_t* __restrict__ cell_cnt, int nb,
                                  int32_t* __restrict__ order) {
  const int gaps[] = {701, 301, 132, 57, 23, 10, 4, 1};
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    const int64_t m = cell_cnt[b];
    int32_t* r = order + (cell_end[b] - m);
    for (int gi = 0; gi < 8; gi++) {
      const int64_t g = gaps[gi];
      if (g >= m) continue;
      for (int64_t a = g; a < m; a++) {
        const int32_t v = r[a];
        int64_t j = a;
        while (j >= g && r[j - g] > v) {
          r[j] = r[j - g];
          j -= g;
        }
        r[j] = v;
      }
    }
  }
}

cudaError_t launch_gather_pivots(const void* src, int64_t row_bytes, int64_t n, int64_t n_piv, void* dst, int sms,
                                 cudaStream_t stream) {
  gather_rows_kernel<<<sms * 4, 256, 0, stream>>>(static_cast<const uint8_t*>(src), row_bytes, n, n_piv,
                                                  static_cast<uint8_t*>(dst));
  return cudaGetLastError();
}

cudaError_t launch_order_by_label(const int32_t* label, int64_t n, int nb, int32_t* hist, int32_t* cursor,
                                  int32_t* order, bool sorted_cells, int sms, cudaStream_t stream) {
  if (nb > 1024 * 64) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(hist, 0, size_t(nb) * sizeof(int32_t), stream);
  if (e != cudaSuccess) return e;
  label_hist_kernel<<<sms * 4, 256, 0, stream>>>(label, n, nb, hist);
  exclusive_scan_kernel<<<1, 1024, 0, stream>>>(hist, nb, cursor);
  label_scatter_kernel<<<sms * 4, 256, 0, stream>>>(label, n, nb, cursor, order);
  if (sorted_cells) sort_cells_kernel<<<(nb + 127) / 128, 128, 0, stream>>>(cursor, hist, nb, order);
  return cudaGetLastError();
}

}  // namespace evoc
