// Fuzzy simplicial set from the kNN graph, on the device.
//
// Restates src/graph_construction.rs:16-248 and the SciPy-compatible sparse
// binops of src/csr_matmul.rs:62-150:
//   smooth_knn_dist       per row: rho = first distance > 0; sigma by 64 steps
//                         of bisection in f64 on sum_{j>=1} exp(-(d_j-rho)/sigma)
//                         = log2(k), tolerance 1e-5; floored at 1e-3 * mean(row)
//                         (rho > 0) or 1e-3 * mean(all distances) (rho == 0)
//   membership strengths  w = 0 for self, 1 when d - rho <= 0 or sigma == 0,
//                         else f32 exp(-(d - rho) / sigma)
//   fuzzy union           A + A^T - A o A^T, each element rounded in f32 in the
//                         order SciPy's row-wise merge rounds it, zeros dropped,
//                         rows sorted by column (canonical CSR)
//
// One thread owns one row for sigma/rho/membership (any k: the row's
// membership entries are insertion-sorted in place in its output slots); the
// transpose is a column-count / scan / scatter / per-bucket sort; the union
// is a per-row two-pointer merge done twice (count, then write).
#include "common.cuh"
#include "kernels.h"

namespace evoc {

// Sets *need_mean when some row has no positive distance (its sigma floor uses
// the mean of all distances).
__global__ void rho_zero_flag_kernel(const float* __restrict__ dist, int64_t n, int k, int* __restrict__ need_mean) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    bool pos = false;
    for (int j = 0; j < k; j++) pos |= double(dist[i * k + j]) > 0.0;
    if (!pos) atomicOr(need_mean, 1);
  }
}

// ndarray's contiguous f32 sum (eight partial sums, then a short tail) divided
// by the element count in f32: the order that mean() rounds in.  Sequential by
// nature, so one thread runs it, and only when a row needs it.
__global__ void ndarray_mean_kernel(const float* __restrict__ x, int64_t len, const int* __restrict__ need_mean,
                                    float* __restrict__ mean_out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (*need_mean == 0) {
    *mean_out = 0.0f;
    return;
  }
  float p[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  int64_t i = 0;
  for (; i + 8 <= len; i += 8)
#pragma unroll
    for (int j = 0; j < 8; j++) p[j] = __fadd_rn(p[j], x[i + j]);
  float acc = 0.0f;
  acc = __fadd_rn(acc, __fadd_rn(p[0], p[4]));
  acc = __fadd_rn(acc, __fadd_rn(p[1], p[5]));
  acc = __fadd_rn(acc, __fadd_rn(p[2], p[6]));
  acc = __fadd_rn(acc, __fadd_rn(p[3], p[7]));
  for (int64_t j = 0; i < len && j < 7; i++, j++) acc = __fadd_rn(acc, x[i]);
  *mean_out = len > 0 ? __fdiv_rn(acc, float(len)) : 0.0f;
}

// sigma/rho and the membership row of A (nonzero weights, sorted by column).
__global__ void fuzzy_rows_kernel(const int32_t* __restrict__ idx, const float* __restrict__ dist, int64_t n, int k,
                                  float n_neighbors, const float* __restrict__ mean_all, float* __restrict__ sigma_out,
                                  float* __restrict__ rho_out, int32_t* __restrict__ a_cols, float* __restrict__ a_vals,
                                  int32_t* __restrict__ a_cnt, int32_t* __restrict__ indeg) {
  const double target = log2(double(n_neighbors));
  const double tol = double(1e-5f);
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const float* row = dist + i * k;
    double r = 0.0;
    for (int j = 0; j < k; j++) {
      const double d = double(row[j]);
      if (d > 0.0) {
        r = d;
        break;
      }
    }
    double lo = 0.0, hi = __longlong_as_double(0x7ff0000000000000ll), mid = 1.0;
    for (int it = 0; it < 64; it++) {
      double ps = 0.0;
      for (int j = 1; j < k; j++) {
        const double d = double(row[j]) - r;
        ps += d > 0.0 ? exp(-(d / mid)) : 1.0;
      }
      if (fabs(ps - target) < tol) break;
      if (ps > target) {
        hi = mid;
        mid = (lo + hi) / 2.0;
      } else {
        lo = mid;
        if (isinf(hi)) mid *= 2.0;
        else mid = (lo + hi) / 2.0;
      }
    }
    double s = mid;
    if (r > 0.0) {
      double m = 0.0;
      for (int j = 0; j < k; j++) m += double(row[j]);
      m /= double(k);
      const double fl = double(1e-3f) * m;
      if (s < fl) s = fl;
    } else {
      const double fl = double(1e-3f) * double(*mean_all);
      if (s < fl) s = fl;
    }
    const float sig = float(s), rh = float(r);
    sigma_out[i] = sig;
    rho_out[i] = rh;

    int32_t* cols = a_cols + i * k;  // the row's k output slots, filled in column order
    float* vals = a_vals + i * k;
    int cnt = 0;
    for (int j = 0; j < k; j++) {
      const int32_t c = idx[i * k + j];
      if (c == -1) continue;
      float w;
      if (c == int32_t(i)) w = 0.0f;
      else {
        const float dr = __fsub_rn(row[j], rh);
        w = (dr <= 0.0f || sig == 0.0f) ? 1.0f : expf(-__fdiv_rn(dr, sig));
      }
      if (w == 0.0f) continue;
      int p = cnt++;
      while (p > 0 && cols[p - 1] > c) {  // insertion by column
        cols[p] = cols[p - 1];
        vals[p] = vals[p - 1];
        p--;
      }
      cols[p] = c;
      vals[p] = w;
    }
    for (int t = 0; t < cnt; t++) atomicAdd(&indeg[cols[t]], 1);
    a_cnt[i] = cnt;
  }
}

// out[0] = 0, out[i+1] = cnt[0] + ... + cnt[i] (single block).
__global__ void scan_counts_kernel(const int32_t* __restrict__ cnt, int64_t n, int64_t* __restrict__ out) {
  __shared__ int64_t part[1024];
  const int t = threadIdx.x;
  const int64_t per = (n + blockDim.x - 1) / blockDim.x;
  int64_t s = 0;
  for (int64_t q = 0; q < per; q++) {
    const int64_t b = t * per + q;
    if (b < n) s += cnt[b];
  }
  part[t] = s;
  __syncthreads();
  for (int off = 1; off < int(blockDim.x); off <<= 1) {
    const int64_t v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int64_t run = part[t] - s;
  if (t == 0) out[0] = 0;
  for (int64_t q = 0; q < per; q++) {
    const int64_t b = t * per + q;
    if (b < n) {
      run += cnt[b];
      out[b + 1] = run;
    }
  }
}

__global__ void scatter_transpose_kernel(const int32_t* __restrict__ a_cols, const float* __restrict__ a_vals,
                                         const int32_t* __restrict__ a_cnt, int64_t n, int k,
                                         const int64_t* __restrict__ colptr, int32_t* __restrict__ fill,
                                         int32_t* __restrict__ at_rows, float* __restrict__ at_vals) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    for (int t = 0; t < a_cnt[i]; t++) {
      const int32_t c = a_cols[i * k + t];
      const int64_t pos = colptr[c] + atomicAdd(&fill[c], 1);
      at_rows[pos] = int32_t(i);
      at_vals[pos] = a_vals[i * k + t];
    }
  }
}

// Each column bucket of A^T sorted by row.  A row appears at most once in a
// column, so sorting the packed (row << 32 | value bits) keys sorts by row.
// Buckets hold k entries on average but hubs can hold thousands: a warp sorts
// each bucket of up to kWarpSort entries (bitonic, in registers up to 32, in
// the warp's shared-memory slice above); larger buckets are listed and sorted
// by a whole block each (kBlockSort entries in shared memory), and any larger
// still by one thread (Shell sort).
constexpr int kWarpSort = 1024;
constexpr int kBlockSort = 8192;
constexpr int kSortWarps = 4;

__device__ __forceinline__ uint64_t bucket_key(int32_t r, float v) {
  return (uint64_t(uint32_t(r)) << 32) | __float_as_uint(v);
}

template <int P_MAX>
__device__ __forceinline__ void bitonic_shared(uint64_t* keys, int P, int tid, int nthreads, bool block) {
  for (int size = 2; size <= P; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = tid; i < (P >> 1); i += nthreads) {
        const int lo = 2 * stride * (i / stride) + (i % stride);
        const int hi = lo + stride;
        const bool up = (lo & size) == 0;
        const uint64_t a = keys[lo], b = keys[hi];
        if ((a > b) == up) {
          keys[lo] = b;
          keys[hi] = a;
        }
      }
      if (block) __syncthreads();
      else __syncwarp();
    }
  }
}

__device__ void shell_sort_bucket(int32_t* r, float* v, int64_t m) {
  const int gaps[] = {701, 301, 132, 57, 23, 10, 4, 1};
  for (int gi = 0; gi < 8; gi++) {
    const int64_t g = gaps[gi];
    if (g >= m) continue;
    for (int64_t a = g; a < m; a++) {
      const int32_t kr = r[a];
      const float kv = v[a];
      int64_t b = a;
      while (b >= g && r[b - g] > kr) {
        r[b] = r[b - g];
        v[b] = v[b - g];
        b -= g;
      }
      r[b] = kr;
      v[b] = kv;
    }
  }
}

__global__ void __launch_bounds__(kSortWarps * 32)
sort_buckets_warp_kernel(const int64_t* __restrict__ colptr, int64_t n, int32_t* __restrict__ rows,
                         float* __restrict__ vals, int32_t* __restrict__ big, int32_t* __restrict__ n_big) {
  __shared__ uint64_t slice[kSortWarps][kWarpSort];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t* keys = slice[warp];
  const int64_t wstride = int64_t(gridDim.x) * kSortWarps;
  for (int64_t c = int64_t(blockIdx.x) * kSortWarps + warp; c < n; c += wstride) {
    const int64_t s = colptr[c], m = colptr[c + 1] - s;
    if (m <= 1) continue;
    if (m > kWarpSort) {
      if (lane == 0) big[atomicAdd(n_big, 1)] = int32_t(c);
      continue;
    }
    int32_t* r = rows + s;
    float* v = vals + s;
    int P = 32;
    while (P < m) P <<= 1;
    for (int i = lane; i < P; i += 32) keys[i] = i < m ? bucket_key(r[i], v[i]) : ~0ull;
    __syncwarp();
    bitonic_shared<kWarpSort>(keys, P, lane, 32, false);
    for (int i = lane; i < m; i += 32) {
      r[i] = int32_t(keys[i] >> 32);
      v[i] = __uint_as_float(uint32_t(keys[i]));
    }
    __syncwarp();
  }
}

__global__ void sort_buckets_big_kernel(const int64_t* __restrict__ colptr, int32_t* __restrict__ rows,
                                        float* __restrict__ vals, const int32_t* __restrict__ big,
                                        const int32_t* __restrict__ n_big) {
  extern __shared__ uint64_t keys[];
  for (int b = blockIdx.x; b < *n_big; b += gridDim.x) {
    const int64_t c = big[b];
    const int64_t s = colptr[c], m = colptr[c + 1] - s;
    int32_t* r = rows + s;
    float* v = vals + s;
    if (m > kBlockSort) {  // beyond a block's shared memory: one thread
      if (threadIdx.x == 0) shell_sort_bucket(r, v, m);
      __syncthreads();
      continue;
    }
    int P = 1;
    while (P < m) P <<= 1;
    for (int i = threadIdx.x; i < P; i += blockDim.x) keys[i] = i < m ? bucket_key(r[i], v[i]) : ~0ull;
    __syncthreads();
    bitonic_shared<kBlockSort>(keys, P, threadIdx.x, blockDim.x, true);
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
      r[i] = int32_t(keys[i] >> 32);
      v[i] = __uint_as_float(uint32_t(keys[i]));
    }
    __syncthreads();
  }
}

// Row i of (A + A^T) - (A o A^T) in SciPy's rounding: s = a + b (missing side
// is 0.0), p = a * b only where both exist (dropped when 0), result s - p,
// dropped when 0.  write == false: count only.
__device__ __forceinline__ int64_t merge_row(int64_t i, int k, const int32_t* __restrict__ a_cols,
                                             const float* __restrict__ a_vals, int ca,
                                             const int64_t* __restrict__ colptr, const int32_t* __restrict__ at_rows,
                                             const float* __restrict__ at_vals, int symmetrize, int32_t* out_cols,
                                             float* out_vals, bool write) {
  int64_t out = 0;
  int ja = 0;
  int64_t jb = symmetrize ? colptr[i] : 0, eb = symmetrize ? colptr[i + 1] : 0;
  while (ja < ca || jb < eb) {
    const int64_t col_a = ja < ca ? a_cols[i * k + ja] : INT64_MAX;
    const int64_t col_b = jb < eb ? at_rows[jb] : INT64_MAX;
    const int64_t col = col_a < col_b ? col_a : col_b;
    const bool ha = col_a == col, hb = col_b == col;
    const float va = ha ? a_vals[i * k + ja] : 0.0f;
    const float vb = hb ? at_vals[jb] : 0.0f;
    float v;
    if (!symmetrize) v = va;
    else {
      const float s = __fadd_rn(va, vb);
      float p = 0.0f;
      if (ha && hb) p = __fmul_rn(va, vb);
      v = __fsub_rn(s, p);
    }
    if (v != 0.0f) {
      if (write) {
        out_cols[out] = int32_t(col);
        out_vals[out] = v;
      }
      out++;
    }
    if (ha) ja++;
    if (hb) jb++;
  }
  return out;
}

__global__ void union_count_kernel(int64_t n, int k, const int32_t* __restrict__ a_cols,
                                   const float* __restrict__ a_vals, const int32_t* __restrict__ a_cnt,
                                   const int64_t* __restrict__ colptr, const int32_t* __restrict__ at_rows,
                                   const float* __restrict__ at_vals, int symmetrize, int32_t* __restrict__ row_cnt) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    row_cnt[i] = int32_t(merge_row(i, k, a_cols, a_vals, a_cnt[i], colptr, at_rows, at_vals, symmetrize, nullptr,
                                   nullptr, false));
}

__global__ void union_write_kernel(int64_t n, int k, const int32_t* __restrict__ a_cols,
                                   const float* __restrict__ a_vals, const int32_t* __restrict__ a_cnt,
                                   const int64_t* __restrict__ colptr, const int32_t* __restrict__ at_rows,
                                   const float* __restrict__ at_vals, int symmetrize, const int64_t* __restrict__ indptr,
                                   int32_t* __restrict__ indices, float* __restrict__ data) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    merge_row(i, k, a_cols, a_vals, a_cnt[i], colptr, at_rows, at_vals, symmetrize, indices + indptr[i],
              data + indptr[i], true);
}

cudaError_t launch_scan_counts(const int32_t* cnt, int64_t n, int64_t* out, cudaStream_t stream) {
  scan_counts_kernel<<<1, 1024, 0, stream>>>(cnt, n, out);
  return cudaGetLastError();
}

cudaError_t launch_smooth_and_membership(const int32_t* idx, const float* dist, int64_t n, int k, float n_neighbors,
                                         const FuzzyWork& w, float* sigma, float* rho, int sms, cudaStream_t stream) {
  if (k < 1) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(w.flags, 0, 2 * sizeof(int), stream);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(w.indeg, 0, size_t(n) * sizeof(int32_t), stream);
  if (e != cudaSuccess) return e;
  rho_zero_flag_kernel<<<sms * 4, 256, 0, stream>>>(dist, n, k, w.flags);
  ndarray_mean_kernel<<<1, 32, 0, stream>>>(dist, n * int64_t(k), w.flags, w.mean);
  fuzzy_rows_kernel<<<sms * 8, 128, 0, stream>>>(idx, dist, n, k, n_neighbors, w.mean, sigma, rho, w.a_cols,
                                                 w.a_vals, w.a_cnt, w.indeg);
  return cudaGetLastError();
}

cudaError_t launch_fuzzy_union_count(int64_t n, int k, int symmetrize, const FuzzyWork& w, int64_t* indptr, int sms,
                                     cudaStream_t stream) {
  cudaError_t e;
  if (symmetrize) {
    scan_counts_kernel<<<1, 1024, 0, stream>>>(w.indeg, n, w.colptr);
    e = cudaMemsetAsync(w.fill, 0, size_t(n) * sizeof(int32_t), stream);
    if (e != cudaSuccess) return e;
    scatter_transpose_kernel<<<sms * 8, 128, 0, stream>>>(w.a_cols, w.a_vals, w.a_cnt, n, k, w.colptr, w.fill,
                                                          w.at_rows, w.at_vals);
    cudaError_t e = cudaMemsetAsync(w.n_big, 0, sizeof(int32_t), stream);
    if (e != cudaSuccess) return e;
    sort_buckets_warp_kernel<<<sms * 16, kSortWarps * 32, 0, stream>>>(w.colptr, n, w.at_rows, w.at_vals, w.big,
                                                                       w.n_big);
    e = cudaFuncSetAttribute(sort_buckets_big_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(kBlockSort * sizeof(uint64_t)));
    if (e != cudaSuccess) return e;
    sort_buckets_big_kernel<<<sms, 1024, kBlockSort * sizeof(uint64_t), stream>>>(w.colptr, w.at_rows, w.at_vals,
                                                                                  w.big, w.n_big);
  }
  union_count_kernel<<<sms * 8, 128, 0, stream>>>(n, k, w.a_cols, w.a_vals, w.a_cnt, w.colptr, w.at_rows, w.at_vals,
                                                  symmetrize, w.row_cnt);
  scan_counts_kernel<<<1, 1024, 0, stream>>>(w.row_cnt, n, indptr);
  return cudaGetLastError();
}

cudaError_t launch_fuzzy_union_write(int64_t n, int k, int symmetrize, const FuzzyWork& w, const int64_t* indptr,
                                     int32_t* indices, float* data, int sms, cudaStream_t stream) {
  union_write_kernel<<<sms * 8, 128, 0, stream>>>(n, k, w.a_cols, w.a_vals, w.a_cnt, w.colptr, w.at_rows, w.at_vals,
                                                  symmetrize, indptr, indices, data);
  return cudaGetLastError();
}

}  // namespace evoc
