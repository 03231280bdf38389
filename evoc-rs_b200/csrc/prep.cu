// Input preparation on the device.
//
// prepare_float (src/knn.rs:78-113): if any row's L2 norm differs from 1 by
// more than 1e-5, every row is divided by its norm (a zero norm divides by 1).
// The norm is the serial f32 sum of squares followed by sqrt, exactly as the
// reference rounds it: each product and each partial sum is rounded on its
// own (no FMA contraction), sqrt and division are IEEE.  One thread owns one
// row; rows are staged through shared memory in 32-column slabs so the
// global reads stay coalesced.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "batch.h"
#include "common.cuh"
#include "kernels.h"

namespace evoc {

namespace {
constexpr int kRows = 128;
constexpr int kSlab = 32;
}

// Norms of rows r0 .. r0+127 (one thread per row, serial f32 sum of squares).
__device__ __forceinline__ void row_norms_block(const float* __restrict__ X, int64_t n, int ld, int d,
                                                float* __restrict__ norms, int* __restrict__ not_unit, int64_t r0,
                                                float (*slab)[kSlab + 1]) {
  const int tid = threadIdx.x;
  float acc = 0.0f;
  for (int c0 = 0; c0 < d; c0 += kSlab) {
    // cooperative coalesced load: 128 rows x 32 columns
    for (int e = tid; e < kRows * kSlab; e += kRows) {
      const int r = e / kSlab, c = e % kSlab;
      const int64_t g = r0 + r;
      slab[r][c] = (g < n && c0 + c < d) ? X[g * ld + c0 + c] : 0.0f;
    }
    __syncthreads();
    const int lim = min(kSlab, d - c0);
    for (int c = 0; c < lim; c++) {
      const float v = slab[tid][c];
      acc = __fadd_rn(acc, __fmul_rn(v, v));
    }
    __syncthreads();
  }
  const int64_t row = r0 + tid;
  if (row < n) {
    const float nrm = __fsqrt_rn(acc);
    norms[row] = nrm;
    if (fabsf(__fsub_rn(nrm, 1.0f)) > 1e-5f) atomicOr(not_unit, 1);
  }
}

__global__ void __launch_bounds__(kRows)
row_norms_kernel(const float* __restrict__ X, int64_t n, int ld, int d, float* __restrict__ norms,
                 int* __restrict__ not_unit) {
  __shared__ float slab[kRows][kSlab + 1];
  row_norms_block(X, n, ld, d, norms, not_unit, int64_t(blockIdx.x) * kRows, slab);
}

__global__ void normalize_rows_kernel(float* __restrict__ X, int64_t n, int ld, int d,
                                      const float* __restrict__ norms, const int* __restrict__ not_unit) {
  if (*not_unit == 0) return;
  const int64_t total = n * int64_t(d);
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / d, c = e % d;
    float nrm = norms[r];
    if (nrm == 0.0f) nrm = 1.0f;
    X[r * ld + c] = __fdiv_rn(X[r * ld + c], nrm);
  }
}

cudaError_t launch_prepare_float(float* X, int64_t n, int ld, int d, float* norms, int* not_unit, int sms,
                                 cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(not_unit, 0, sizeof(int), stream);
  if (e != cudaSuccess) return e;
  const int64_t blocks = (n + kRows - 1) / kRows;
  row_norms_kernel<<<unsigned(blocks), kRows, 0, stream>>>(X, n, ld, d, norms, not_unit);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  normalize_rows_kernel<<<sms * 8, 256, 0, stream>>>(X, n, ld, d, norms, not_unit);
  return cudaGetLastError();
}

}  // namespace evoc

namespace evoc {

// One f32 value as the 16-bit operand of the tensor-core scan.  FP16: round
// to nearest even, with values below the smallest normal (2^-14) flushed to
// zero, so no subnormal ever reaches the tensor cores and the residual
// x - half(x) below accounts for the whole difference whatever the hardware
// does with subnormal inputs.  BF16: round to nearest even.
__device__ __forceinline__ uint16_t half_bits(float v, int half_type) {
  if (half_type == kHalfBf16) return __bfloat16_as_ushort(__float2bfloat16_rn(v));
  if (fabsf(v) < 6.103515625e-05f) return 0;
  return __half_as_ushort(__float2half_rn(v));
}

__device__ __forceinline__ float half_value(uint16_t b, int half_type) {
  return half_type == kHalfBf16 ? __bfloat162float(__ushort_as_bfloat16(b)) : __half2float(__ushort_as_half(b));
}

// f32 rows (ld floats) -> 16-bit rows (ldb elements, zero padded).  Warp per
// row.  With `cert`, also the two norms the BF16/FP16 form certifies its rows
// with: |x - half(x)| (the residual, exact in f32) and |half(x)|, summed in
// f64 and rounded up to f32, and their maxima over all rows (non-negative
// floats compare as their bit patterns).
__global__ void to_half_kernel(const float* __restrict__ X, int64_t n_rows, int64_t n, int ld, int d,
                               uint16_t* __restrict__ Y, int ldb, int half_type, float* __restrict__ rnorm,
                               float* __restrict__ hnorm, unsigned int* __restrict__ maxes) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
  for (int64_t r = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); r < n_rows; r += warps) {
    double rr = 0.0, hh = 0.0;
    for (int c = lane; c < ldb; c += 32) {
      const float v = (c < d && r < n) ? X[r * ld + c] : 0.0f;
      const uint16_t b = half_bits(v, half_type);
      Y[r * ldb + c] = b;
      const float h = half_value(b, half_type);
      const double res = double(v) - double(h);
      rr += res * res;
      hh += double(h) * double(h);
    }
    if (rnorm && r < n) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        rr += __shfl_xor_sync(0xffffffffu, rr, o);
        hh += __shfl_xor_sync(0xffffffffu, hh, o);
      }
      if (lane == 0) {
        // f64 sums of at most 2^16 squares are within a relative 2^-36 of
        // exact: one part in 2^-30 more before rounding up covers them.
        const float a = __double2float_ru(__dsqrt_ru(rr * (1.0 + 0x1p-30)));
        const float b = __double2float_ru(__dsqrt_ru(hh * (1.0 + 0x1p-30)));
        rnorm[r] = a;
        hnorm[r] = b;
        atomicMax(&maxes[0], __float_as_uint(a));
        atomicMax(&maxes[1], __float_as_uint(b));
      }
    }
  }
}

cudaError_t launch_to_half(const float* X, int64_t n_rows, int64_t n, int ld, int d, void* Y, int ldb, int half_type,
                           float* rnorm, float* hnorm, unsigned int* maxes, int sms, cudaStream_t stream) {
  if (rnorm) {
    cudaError_t e = cudaMemsetAsync(maxes, 0, 2 * sizeof(unsigned int), stream);
    if (e != cudaSuccess) return e;
  }
  to_half_kernel<<<sms * 8, 256, 0, stream>>>(X, n_rows, n, ld, d, static_cast<uint16_t*>(Y), ldb, half_type, rnorm,
                                               hnorm, maxes);
  return cudaGetLastError();
}

// Rows list[i] (+ row0) of src -> row i of dst (row_bytes each, 16-byte
// multiples); dst rows count .. rows_out-1 are zeroed.
__global__ void gather_rows_list_kernel(const uint8_t* __restrict__ src, int64_t row_bytes, int64_t row0,
                                        const int32_t* __restrict__ list, int64_t count, int64_t rows_out,
                                        uint8_t* __restrict__ dst) {
  const int64_t wpr = row_bytes / 16, total = rows_out * wpr;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e / wpr, w = e % wpr;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (i < count) v = reinterpret_cast<const uint4*>(src + (row0 + list[i]) * row_bytes)[w];
    reinterpret_cast<uint4*>(dst + i * row_bytes)[w] = v;
  }
}

cudaError_t launch_gather_rows_list(const void* src, int64_t row_bytes, int64_t row0, const int32_t* list,
                                    int64_t count, int64_t rows_out, void* dst, int sms, cudaStream_t stream) {
  if (row_bytes % 16 != 0 || rows_out < count) return cudaErrorInvalidValue;
  gather_rows_list_kernel<<<sms * 4, 256, 0, stream>>>(static_cast<const uint8_t*>(src), row_bytes, row0, list, count,
                                                       rows_out, static_cast<uint8_t*>(dst));
  return cudaGetLastError();
}

}  // namespace evoc

namespace evoc {

// Row copy with padding.  Wide path: 16-byte words when both strides and
// both base addresses allow it; otherwise 4-byte words; otherwise bytes.
template <typename W>
__global__ void copy_rows_kernel(const uint8_t* __restrict__ src, int64_t n, int64_t row_bytes,
                                 uint8_t* __restrict__ dst, int64_t rows, int64_t ld_bytes) {
  const int64_t wpr = ld_bytes / int64_t(sizeof(W));      // words per destination row
  const int64_t src_w = row_bytes / int64_t(sizeof(W));   // words of data per row
  const int64_t total = rows * wpr;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / wpr, c = e % wpr;
    W v{};
    if (r < n && c < src_w) v = reinterpret_cast<const W*>(src + r * row_bytes)[c];
    reinterpret_cast<W*>(dst + r * ld_bytes)[c] = v;
  }
}

cudaError_t launch_copy_rows(const void* src, int64_t n, int64_t row_bytes, void* dst, int64_t rows, int64_t ld_bytes,
                             int sms, cudaStream_t stream) {
  if (ld_bytes < row_bytes || rows < n) return cudaErrorInvalidValue;
  const uintptr_t a = reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst);
  const auto* s8 = static_cast<const uint8_t*>(src);
  auto* d8 = static_cast<uint8_t*>(dst);
  const int grid = sms * 8;
  if (row_bytes % 16 == 0 && ld_bytes % 16 == 0 && (a & 15) == 0)
    copy_rows_kernel<uint4><<<grid, 256, 0, stream>>>(s8, n, row_bytes, d8, rows, ld_bytes);
  else if (row_bytes % 4 == 0 && ld_bytes % 4 == 0 && (a & 3) == 0)
    copy_rows_kernel<uint32_t><<<grid, 256, 0, stream>>>(s8, n, row_bytes, d8, rows, ld_bytes);
  else
    copy_rows_kernel<uint8_t><<<grid, 256, 0, stream>>>(s8, n, row_bytes, d8, rows, ld_bytes);
  return cudaGetLastError();
}

}  // namespace evoc

// ---------------------------------------------------------------------------
// Batches: the same per-request steps over the request table of a batch.
// ---------------------------------------------------------------------------
namespace evoc {

namespace {
__device__ __forceinline__ int find_block_job(const BatchRowJob* __restrict__ jobs, int nj, int64_t g) {
  int lo = 0, hi = nj - 1;
  while (lo < hi) {  // last request with blk_base <= g
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].blk_base <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
}  // namespace

// Packed input rows -> padded rows (f32: x, ld floats; i8: xb, ldb bytes),
// zero-filled past the data; also clears each request's prepare_float flag.
__global__ void batch_copy_kernel(const BatchHeader* __restrict__ hdr, const BatchRowJob* __restrict__ jobs,
                                  bool f32) {
  const int nj = hdr->n_jobs;
  for (int j = 0; j < nj; j++) {
    const BatchRowJob& J = jobs[j];
    if (blockIdx.x == 0 && threadIdx.x == 0 && J.flag) *J.flag = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0 && J.maxes) J.maxes[0] = J.maxes[1] = 0u;
    uint8_t* dst = f32 ? reinterpret_cast<uint8_t*>(J.x) : J.xb;
    const int64_t ld_bytes = f32 ? J.ld * 4 : J.ldb;
    if (J.row_bytes % 4 == 0) {
      const int64_t wpr = ld_bytes / 4, src_w = J.row_bytes / 4, total = J.rows * wpr;
      for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
           e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t r = e / wpr, c = e % wpr;
        uint32_t v = 0u;
        if (r < J.n && c < src_w) v = reinterpret_cast<const uint32_t*>(J.src + r * J.row_bytes)[c];
        reinterpret_cast<uint32_t*>(dst + r * ld_bytes)[c] = v;
      }
    } else {
      const int64_t total = J.rows * ld_bytes;
      for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
           e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t r = e / ld_bytes, c = e % ld_bytes;
        dst[e] = (r < J.n && c < J.row_bytes) ? J.src[r * J.row_bytes + c] : uint8_t(0);
      }
    }
  }
}

__global__ void __launch_bounds__(kRows)
batch_row_norms_kernel(const BatchHeader* __restrict__ hdr, const BatchRowJob* __restrict__ jobs) {
  __shared__ float slab[kRows][kSlab + 1];
  const int nj = hdr->n_jobs;
  const int64_t total = hdr->total_blocks;
  for (int64_t g = blockIdx.x; g < total; g += gridDim.x) {
    const BatchRowJob& J = jobs[find_block_job(jobs, nj, g)];
    row_norms_block(J.x, J.n, int(J.ld), int(J.dim), J.norms, J.flag, (g - J.blk_base) * kRows, slab);
  }
}

__global__ void batch_normalize_kernel(const BatchHeader* __restrict__ hdr, const BatchRowJob* __restrict__ jobs) {
  const int nj = hdr->n_jobs;
  for (int j = 0; j < nj; j++) {
    const BatchRowJob& J = jobs[j];
    if (*J.flag == 0) continue;
    const int64_t d = J.dim, total = J.n * d;
    for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
      const int64_t r = e / d, c = e % d;
      float nrm = J.norms[r];
      if (nrm == 0.0f) nrm = 1.0f;
      J.x[r * J.ld + c] = __fdiv_rn(J.x[r * J.ld + c], nrm);
    }
  }
}

__global__ void batch_to_half_kernel(const BatchHeader* __restrict__ hdr, const BatchRowJob* __restrict__ jobs) {
  const int nj = hdr->n_jobs;
  for (int j = 0; j < nj; j++) {
    const BatchRowJob& J = jobs[j];
    const int64_t lde = J.ldb / 2, total = J.rows * lde;
    uint16_t* Y = reinterpret_cast<uint16_t*>(J.xb);
    for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
      const int64_t r = e / lde, c = e % lde;
      Y[e] = half_bits((c < J.dim && r < J.n) ? J.x[r * J.ld + c] : 0.0f, J.half_type);
    }
  }
}

// The certificate's row norms of every f32 request (warp per row, as
// to_half_kernel computes them).
__global__ void batch_half_norms_kernel(const BatchHeader* __restrict__ hdr, const BatchRowJob* __restrict__ jobs) {
  const int nj = hdr->n_jobs;
  const int64_t total = hdr->total_rows;
  const int lane = threadIdx.x & 31;
  const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
  for (int64_t w = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); w < total; w += warps) {
    int lo = 0, hi = nj - 1;
    while (lo < hi) {  // last request with row_base <= w
      const int mid = (lo + hi + 1) >> 1;
      if (jobs[mid].row_base <= w) lo = mid;
      else hi = mid - 1;
    }
    const BatchRowJob& J = jobs[lo];
    if (!J.rnorm) continue;
    const int64_t r = w - J.row_base;
    double rr = 0.0, hh = 0.0;
    for (int c = lane; c < J.dim; c += 32) {
      const float v = J.x[r * J.ld + c];
      const float h = half_value(half_bits(v, J.half_type), J.half_type);
      const double res = double(v) - double(h);
      rr += res * res;
      hh += double(h) * double(h);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      rr += __shfl_xor_sync(0xffffffffu, rr, o);
      hh += __shfl_xor_sync(0xffffffffu, hh, o);
    }
    if (lane == 0) {
      const float a = __double2float_ru(__dsqrt_ru(rr * (1.0 + 0x1p-30)));
      const float b = __double2float_ru(__dsqrt_ru(hh * (1.0 + 0x1p-30)));
      J.rnorm[r] = a;
      J.hnorm[r] = b;
      atomicMax(&J.maxes[0], __float_as_uint(a));
      atomicMax(&J.maxes[1], __float_as_uint(b));
    }
  }
}

cudaError_t launch_batch_rows(bool f32, const BatchHeader* hdr, const BatchRowJob* jobs, int grid_rows,
                              int grid_norms, cudaStream_t stream) {
  batch_copy_kernel<<<grid_rows, 256, 0, stream>>>(hdr, jobs, f32);
  if (!f32) return cudaGetLastError();
  batch_row_norms_kernel<<<grid_norms, kRows, 0, stream>>>(hdr, jobs);
  batch_normalize_kernel<<<grid_rows, 256, 0, stream>>>(hdr, jobs);
  batch_to_half_kernel<<<grid_rows, 256, 0, stream>>>(hdr, jobs);
  batch_half_norms_kernel<<<grid_norms, kRows, 0, stream>>>(hdr, jobs);
  return cudaGetLastError();
}

}  // namespace evoc

namespace evoc {

namespace {
__device__ __forceinline__ uint64_t fill_hash(uint64_t z) {  // splitmix64 finaliser
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
}  // namespace

__global__ void fill_random_kernel(int mode, uint8_t* __restrict__ rows, int64_t n_rows_mem, int64_t row_bytes,
                                   int64_t n, int64_t bytes, uint64_t seed) {
  const int64_t total = n_rows_mem * row_bytes;
  const int64_t eb = mode == 0 ? 2 : 1;
  for (int64_t e = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) * eb; e < total;
       e += int64_t(gridDim.x) * blockDim.x * eb) {
    const int64_t r = e / row_bytes, c = e % row_bytes;
    const bool live = r < n && c < bytes;
    const uint64_t h = fill_hash(seed ^ uint64_t(e));
    if (mode == 0) {
      const float v = live ? float(int32_t(h & 0xffff) - 32768) / 32768.0f : 0.0f;
      *reinterpret_cast<__half*>(rows + e) = __float2half_rn(v);
    } else if (mode == 1) {
      rows[e] = live ? uint8_t(int8_t(int32_t(h % 255) - 127)) : uint8_t(0);
    } else {
      const uint64_t b = h & (h >> 8) & (h >> 16);  // each bit set with probability 1/8
      rows[e] = live ? uint8_t(b) : uint8_t(0);
    }
  }
}

cudaError_t launch_fill_random(int mode, void* rows, int64_t n_rows_mem, int64_t row_bytes, int64_t n,
                               int64_t bytes, uint64_t seed, int sms, cudaStream_t stream) {
  if (mode < 0 || mode > 2 || (mode == 0 && (row_bytes % 2 || bytes % 2))) return cudaErrorInvalidValue;
  fill_random_kernel<<<sms * 8, 256, 0, stream>>>(mode, static_cast<uint8_t*>(rows), n_rows_mem, row_bytes, n, bytes,
                                                  seed);
  return cudaGetLastError();
}

}  // namespace evoc
