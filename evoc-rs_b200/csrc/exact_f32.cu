// Plain FP32 exact kNN: tiled FP32 SIMT dot products with the top-k
// selection fused into the tile epilogue (the n x n matrix never reaches HBM).
//
// Replaces the distance evaluations of the reference's NN-descent local join
// (src/nndescent/float.rs:552-660, fast_cosine in src/fast_cosine.rs:33-45)
// with an exact search under the contract in common.cuh.
//
// Layout: X is the row-normalised embedding, n rows of `ld` floats (ld is a
// multiple of 16, zero padded).  A persistent grid walks 128-row query blocks;
// for each, every 128-row key tile is multiplied in 16-wide k-steps
// (register-prefetched double buffer), the 128x128 score tile is staged in
// shared memory, and 128 owner threads (one per query row) feed their row's
// scores to a thread-private candidate buffer in global scratch.
//
// Key splits: with n_splits > 1 a query block is n_splits work items, each
// over a contiguous range of key tiles, writing its rows' sorted top-k keys
// to `partial` (split-major); merge_key_splits_kernel then takes each row's k
// smallest keys of all splits.  A few query rows (the certificate's failed
// rows) then still spread over every SM.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace evoc {

namespace {
constexpr int BM = 128, BN = 128, BK = 16, NT = 256;
constexpr int SPAD = 129;  // score tile row stride (conflict-free row scans)
constexpr int APAD = 132;  // k-major operand stride

struct F32Smem {
  float a[2][BK][APAD];
  float b[2][BK][APAD];
  float s[BM][SPAD];
};

__device__ __forceinline__ void load_tile(const float* __restrict__ X, int64_t n, int ld, int64_t row0, int k0,
                                          int tid, float4 (&r)[2]) {
  const int row = tid >> 2, c4 = (tid & 3) * 4;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    int64_t g = row0 + row + h * 64;
    if (g < n) r[h] = *reinterpret_cast<const float4*>(X + g * ld + k0 + c4);
    else r[h] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

__device__ __forceinline__ void store_tile(float (*dst)[APAD], int tid, const float4 (&r)[2]) {
  const int row = tid >> 2, c4 = (tid & 3) * 4;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    dst[c4 + 0][row + h * 64] = r[h].x;
    dst[c4 + 1][row + h * 64] = r[h].y;
    dst[c4 + 2][row + h * 64] = r[h].z;
    dst[c4 + 3][row + h * 64] = r[h].w;
  }
}
}  // namespace

__global__ void __launch_bounds__(NT, 2)
knn_f32_simt_kernel(const float* __restrict__ X, int64_t n, int ld, int k, int cap,
                    uint64_t* __restrict__ scratch, int32_t* __restrict__ out_idx, float* __restrict__ out_raw,
                    float* __restrict__ out_dist, int64_t q_begin, int64_t q_end, const float* __restrict__ Q,
                    const int32_t* __restrict__ q_list, int64_t q_row0, int n_splits, uint64_t* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  F32Smem& sm = *reinterpret_cast<F32Smem*>(smem_raw);
  const int tid = threadIdx.x;
  const int ty = tid >> 4, tx = tid & 15;
  const int64_t n_qblocks = (q_end - q_begin + BM - 1) / BM;
  const int64_t n_tiles_all = (n + BN - 1) / BN;
  const int64_t tiles_per = (n_tiles_all + n_splits - 1) / n_splits;
  const int64_t n_items = n_qblocks * n_splits;
  uint64_t* my_buf = scratch + (int64_t(blockIdx.x) * BM + (tid & (BM - 1))) * cap;

  for (int64_t item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int64_t qb = item / n_splits;
    const int sp = int(item % n_splits);
    const int64_t kt_begin = sp * tiles_per;
    const int64_t n_ktiles = kt_begin + tiles_per < n_tiles_all ? kt_begin + tiles_per : n_tiles_all;
    const int64_t q0 = q_begin + qb * BM;
    RowTopK top;
    top.init(my_buf, k, cap);
    const int64_t my_q = q0 + tid;
    // this query's row of X (the self rule) and its output row
    const int64_t my_self = (q_list && tid < BM && my_q < q_end) ? q_row0 + q_list[my_q] : my_q;

    for (int64_t kt = kt_begin; kt < n_ktiles; kt++) {
      const int64_t c0 = kt * BN;
      float acc[8][8];
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = 0.f;

      float4 ra[2], rb[2];
      load_tile(Q, q_end, ld, q0, 0, tid, ra);
      load_tile(X, n, ld, c0, 0, tid, rb);
      store_tile(sm.a[0], tid, ra);
      store_tile(sm.b[0], tid, rb);
      __syncthreads();
      int buf = 0;
      for (int k0 = 0; k0 < ld; k0 += BK) {
        const bool more = k0 + BK < ld;
        if (more) {
          load_tile(Q, q_end, ld, q0, k0 + BK, tid, ra);
          load_tile(X, n, ld, c0, k0 + BK, tid, rb);
        }
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
          float av[8], bv[8];
          float4 t0 = *reinterpret_cast<const float4*>(&sm.a[buf][kk][ty * 4]);
          float4 t1 = *reinterpret_cast<const float4*>(&sm.a[buf][kk][64 + ty * 4]);
          float4 u0 = *reinterpret_cast<const float4*>(&sm.b[buf][kk][tx * 4]);
          float4 u1 = *reinterpret_cast<const float4*>(&sm.b[buf][kk][64 + tx * 4]);
          av[0] = t0.x; av[1] = t0.y; av[2] = t0.z; av[3] = t0.w;
          av[4] = t1.x; av[5] = t1.y; av[6] = t1.z; av[7] = t1.w;
          bv[0] = u0.x; bv[1] = u0.y; bv[2] = u0.z; bv[3] = u0.w;
          bv[4] = u1.x; bv[5] = u1.y; bv[6] = u1.z; bv[7] = u1.w;
#pragma unroll
          for (int i = 0; i < 8; i++)
#pragma unroll
            for (int j = 0; j < 8; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
        if (more) {
          store_tile(sm.a[buf ^ 1], tid, ra);
          store_tile(sm.b[buf ^ 1], tid, rb);
        }
        __syncthreads();
        buf ^= 1;
      }
      // Stage the score tile.
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const int r = (i < 4) ? ty * 4 + i : 64 + ty * 4 + (i - 4);
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const int c = (j < 4) ? tx * 4 + j : 64 + tx * 4 + (j - 4);
          sm.s[r][c] = acc[i][j];
        }
      }
      __syncthreads();
      if (tid < BM && my_q < q_end) {
        const int lim = (n - c0 < BN) ? int(n - c0) : BN;
        for (int c = 0; c < lim; c++) {
          const int64_t key = c0 + c;
          const float raw = (key == my_self) ? -1.0f : raw_cosine(sm.s[tid][c]);
          top.offer(raw, int32_t(key));
        }
      }
      __syncthreads();
    }
    if (tid < BM && my_q < q_end && partial) {
      // this split's sorted top-k keys of the row (kKeyInf past the end)
      const int got = top.finish();
      uint64_t* dst = partial + (int64_t(sp) * (q_end - q_begin) + (my_q - q_begin)) * k;
      for (int j = 0; j < k; j++) dst[j] = j < got ? top.buf[j] : kKeyInf;
    } else if (tid < BM && my_q < q_end) {
      const int got = top.finish();
      const int64_t orow = (q_list ? int64_t(q_list[my_q]) : my_q - q_begin) * k;
      for (int j = 0; j < k; j++) {
        float raw = kHeapInf;
        int32_t idx = -1;
        if (j < got) {
          raw = from_orderable(uint32_t(top.buf[j] >> 32));
          idx = key_index(top.buf[j]);
        }
        out_idx[orow + j] = idx;
        if (out_raw) out_raw[orow + j] = raw;
        if (out_dist) out_dist[orow + j] = transform_raw(0, raw);
      }
    }
  }
}

// Warp per row r of `rows`: the k smallest of the row's n_splits sorted
// partial lists (keys are unique but for kKeyInf), taken one at a time as the
// smallest key above the last one taken; written to output row q_list[r] (or
// r) as (index, raw, transformed distance).
__global__ void merge_key_splits_kernel(const uint64_t* __restrict__ partial, int64_t rows, int k, int n_splits,
                                        const int32_t* __restrict__ q_list, int32_t* __restrict__ out_idx,
                                        float* __restrict__ out_raw, float* __restrict__ out_dist) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
  for (int64_t r = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += warps) {
    const int64_t orow = (q_list ? int64_t(q_list[r]) : r) * k;
    const int total = n_splits * k;
    uint64_t last = 0;
    bool first = true;
    for (int j = 0; j < k; j++) {
      uint64_t best = kKeyInf;
      for (int e = lane; e < total; e += 32) {
        const int s = e / k, t = e - s * k;
        const uint64_t key = partial[(int64_t(s) * rows + r) * k + t];
        if ((first || key > last) && key < best) best = key;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const uint64_t other = __shfl_xor_sync(0xffffffffu, best, o);
        best = other < best ? other : best;
      }
      first = false;
      last = best;
      if (lane == 0) {
        const bool ok = best != kKeyInf;
        const float raw = ok ? from_orderable(uint32_t(best >> 32)) : kHeapInf;
        out_idx[orow + j] = ok ? key_index(best) : -1;
        if (out_raw) out_raw[orow + j] = raw;
        if (out_dist) out_dist[orow + j] = transform_raw(0, raw);
      }
    }
  }
}

size_t knn_f32_simt_smem() { return sizeof(F32Smem); }

cudaError_t launch_knn_f32_simt(const float* X, int64_t n, int ld, int k, int cap, uint64_t* scratch,
                                int grid, int32_t* out_idx, float* out_raw, float* out_dist, int64_t q_begin,
                                int64_t q_end, cudaStream_t stream, const float* Q, const int32_t* q_list,
                                int64_t q_row0, int n_splits, uint64_t* partial) {
  if ((Q == nullptr) != (q_list == nullptr)) return cudaErrorInvalidValue;
  if (n_splits < 1 || (n_splits > 1 && partial == nullptr)) return cudaErrorInvalidValue;
  const size_t smem = sizeof(F32Smem);
  cudaError_t e = cudaFuncSetAttribute(knn_f32_simt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  knn_f32_simt_kernel<<<grid, NT, smem, stream>>>(X, n, ld, k, cap, scratch, out_idx, out_raw, out_dist, q_begin,
                                                   q_end, Q ? Q : X, q_list, q_row0, n_splits,
                                                   n_splits > 1 ? partial : nullptr);
  return cudaGetLastError();
}

cudaError_t launch_merge_key_splits(const uint64_t* partial, int64_t rows, int k, int n_splits,
                                    const int32_t* q_list, int32_t* out_idx, float* out_raw, float* out_dist,
                                    int sms, cudaStream_t stream) {
  if (rows <= 0) return cudaSuccess;
  const int64_t blocks = std::min<int64_t>((rows + 7) / 8, int64_t(sms) * 8);
  merge_key_splits_kernel<<<int(blocks), 256, 0, stream>>>(partial, rows, k, n_splits, q_list, out_idx, out_raw,
                                                          out_dist);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// The k-major form of the same search.  XT holds the rows transposed: ld rows
// (one per coordinate) of `cols` floats, cols = round_up(n, 128) + 128, with
// zeros past row n-1.  An operand tile (16 coordinates x 128 rows) is then 16
// contiguous 512-byte runs, copied to shared memory by cp.async with no
// register staging or transposition; a two-stage pipeline keeps one k-step in
// flight and takes one barrier per k-step.  The score tile has its own shared
// memory, so the next tile's first copy overlaps the top-k epilogue.
//
// Epilogue: every thread filters its 8 x 8 scores against their rows'
// current admission thresholds (published in shared memory by the row
// owners) and marks the survivors in a per-row 128-bit mask; a row owner
// then offers only the marked columns, in column order.  The filter drops
// exactly the scores the owner's offer would reject on the raw value, so the
// kept sets are those of a full scan.
//
// Alignment: query block starts q_begin + 128 i must be multiples of 4 floats
// (the host takes this form only when q_begin % 4 == 0); key tiles start at
// multiples of 128.  Bounds: a query tile reads columns q0 .. q0+127 with
// q0 < n, so below round_up(n, 128) + 128 = cols.

namespace {
struct F32KtSmem {
  float a[2][BK][APAD];
  float b[2][BK][APAD];
  float s[BM][SPAD];      // surviving scores (raw), at their columns
  uint32_t mask[BM][4];   // survivor columns of each row
  float thr[BM];          // each row's admission threshold (raw); -inf: no row
};

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Queues the copies of k-step `ks` of the (q0, c0) tile pair into stage `st`:
// 2 x 16 runs of 128 floats, 512 16-byte chunks each, two per thread.
__device__ __forceinline__ void kt_issue(F32KtSmem& sm, int st, const float* __restrict__ XT, int64_t cols,
                                         int64_t q0, int64_t c0, int ks, int tid) {
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int id = tid + h * NT;
    const int r = id >> 5, c = (id & 31) * 4;
    const float* src = XT + int64_t(ks * BK + r) * cols;
    cp_async16(&sm.a[st][r][c], src + q0 + c);
    cp_async16(&sm.b[st][r][c], src + c0 + c);
  }
  cp_async_commit();
}
}  // namespace

__global__ void __launch_bounds__(NT, 2)
knn_f32_kt_kernel(const float* __restrict__ XT, int64_t cols, int64_t n, int ld, int k, int cap,
                  uint64_t* __restrict__ scratch, int32_t* __restrict__ out_idx, float* __restrict__ out_raw,
                  float* __restrict__ out_dist, int64_t q_begin, int64_t q_end) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  F32KtSmem& sm = *reinterpret_cast<F32KtSmem*>(smem_raw);
  const int tid = threadIdx.x;
  const int ty = tid >> 4, tx = tid & 15;
  const int nk = ld / BK;
  const int64_t n_qblocks = (q_end - q_begin + BM - 1) / BM;
  const int64_t n_ktiles = (n + BN - 1) / BN;
  uint64_t* my_buf = scratch + (int64_t(blockIdx.x) * BM + (tid & (BM - 1))) * cap;

  for (int64_t qb = blockIdx.x; qb < n_qblocks; qb += gridDim.x) {
    const int64_t q0 = q_begin + qb * BM;
    const int64_t my_q = q0 + tid;
    RowTopK top;
    top.init(my_buf, k, cap);
    if (tid < BM) {
      sm.thr[tid] = (my_q < q_end) ? top.thr_raw : __int_as_float(0xff800000);
#pragma unroll
      for (int w = 0; w < 4; w++) sm.mask[tid][w] = 0u;
    }
    float acc[8][8];
    int stage = 0;
    kt_issue(sm, 0, XT, cols, q0, 0, 0, tid);
    int64_t kt = 0;
    int ks = 0;
    while (kt < n_ktiles) {
      cp_async_wait_all();
      __syncthreads();  // stage `stage` landed for all threads; stage^1 is free (its k-step is done)
      {
        int64_t nkt = kt;
        int nks = ks + 1;
        if (nks == nk) {
          nks = 0;
          nkt++;
        }
        if (nkt < n_ktiles) kt_issue(sm, stage ^ 1, XT, cols, q0, nkt * BN, nks, tid);
      }
      if (ks == 0) {
#pragma unroll
        for (int i = 0; i < 8; i++)
#pragma unroll
          for (int j = 0; j < 8; j++) acc[i][j] = 0.f;
      }
#pragma unroll
      for (int kk = 0; kk < BK; kk++) {
        float av[8], bv[8];
        const float4 t0 = *reinterpret_cast<const float4*>(&sm.a[stage][kk][ty * 4]);
        const float4 t1 = *reinterpret_cast<const float4*>(&sm.a[stage][kk][64 + ty * 4]);
        const float4 u0 = *reinterpret_cast<const float4*>(&sm.b[stage][kk][tx * 4]);
        const float4 u1 = *reinterpret_cast<const float4*>(&sm.b[stage][kk][64 + tx * 4]);
        av[0] = t0.x; av[1] = t0.y; av[2] = t0.z; av[3] = t0.w;
        av[4] = t1.x; av[5] = t1.y; av[6] = t1.z; av[7] = t1.w;
        bv[0] = u0.x; bv[1] = u0.y; bv[2] = u0.z; bv[3] = u0.w;
        bv[4] = u1.x; bv[5] = u1.y; bv[6] = u1.z; bv[7] = u1.w;
#pragma unroll
        for (int i = 0; i < 8; i++)
#pragma unroll
          for (int j = 0; j < 8; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
      }
      stage ^= 1;
      if (++ks == nk) {
        // The tile is complete: filter it, then let the 128 row owners take
        // the survivors.  Scores, masks and thresholds are next written a full
        // tile later, after at least one more top-of-step barrier, so the
        // owners' reads and updates below are done by then.
        const int64_t c0 = kt * BN;
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const int r = (i < 4) ? ty * 4 + i : 64 + ty * 4 + (i - 4);
          const float t = sm.thr[r];
          const int64_t qrow = q0 + r;
          uint32_t lo = 0u, hi = 0u;
#pragma unroll
          for (int j = 0; j < 8; j++) {
            const int c = (j < 4) ? tx * 4 + j : 64 + tx * 4 + (j - 4);
            const int64_t key = c0 + c;
            const float raw = (key == qrow) ? -1.0f : raw_cosine(acc[i][j]);
            if (key < n && raw <= t) {
              sm.s[r][c] = raw;
              if (j < 4) lo |= 1u << ((tx & 7) * 4 + j);
              else hi |= 1u << ((tx & 7) * 4 + (j - 4));
            }
          }
          if (lo) atomicOr(&sm.mask[r][tx >> 3], lo);
          if (hi) atomicOr(&sm.mask[r][2 + (tx >> 3)], hi);
        }
        __syncthreads();
        if (tid < BM) {
          if (my_q < q_end) {
#pragma unroll
            for (int w = 0; w < 4; w++) {
              uint32_t m = sm.mask[tid][w];
              while (m) {
                const int c = w * 32 + __ffs(m) - 1;
                m &= m - 1u;
                top.offer(sm.s[tid][c], int32_t(c0 + c));
              }
            }
            sm.thr[tid] = top.thr_raw;
          }
#pragma unroll
          for (int w = 0; w < 4; w++) sm.mask[tid][w] = 0u;
        }
        ks = 0;
        kt++;
      }
    }
    if (tid < BM && my_q < q_end) {
      const int got = top.finish();
      const int64_t orow = (my_q - q_begin) * k;
      for (int j = 0; j < k; j++) {
        float raw = kHeapInf;
        int32_t idx = -1;
        if (j < got) {
          raw = from_orderable(uint32_t(top.buf[j] >> 32));
          idx = key_index(top.buf[j]);
        }
        out_idx[orow + j] = idx;
        if (out_raw) out_raw[orow + j] = raw;
        if (out_dist) out_dist[orow + j] = transform_raw(0, raw);
      }
    }
    __syncthreads();  // the score tile and both stages are free before the next query block
  }
}

// XT[c][j] = X[j][c] for rows j < n, zero for n <= j < cols.  One 64-row x
// 16-coordinate tile per step: reads of 64-byte row pieces, writes of
// 256-byte runs of XT.
__global__ void __launch_bounds__(256) transpose_rows_kernel(const float* __restrict__ X, int64_t n, int ld,
                                                             float* __restrict__ XT, int64_t cols) {
  __shared__ float t[16][65];
  const int tid = threadIdx.x;
  const int64_t ctiles = cols / 64;
  const int64_t tiles = ctiles * (ld / 16);
  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int64_t j0 = (tile % ctiles) * 64;
    const int k0 = int(tile / ctiles) * 16;
    {
      const int r = tid >> 2, c4 = (tid & 3) * 4;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (j0 + r < n) v = *reinterpret_cast<const float4*>(X + (j0 + r) * ld + k0 + c4);
      t[c4 + 0][r] = v.x;
      t[c4 + 1][r] = v.y;
      t[c4 + 2][r] = v.z;
      t[c4 + 3][r] = v.w;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int id = tid + i * 256;
      const int kk = id >> 6, jj = id & 63;
      XT[int64_t(k0 + kk) * cols + j0 + jj] = t[kk][jj];
    }
    __syncthreads();
  }
}

int64_t knn_f32_kt_cols(int64_t n) { return (n + 127) / 128 * 128 + 128; }

cudaError_t launch_knn_f32_kt(const float* X, int64_t n, int ld, float* XT, int k, int cap, uint64_t* scratch,
                              int grid, int32_t* out_idx, float* out_raw, float* out_dist, int64_t q_begin,
                              int64_t q_end, int sms, cudaStream_t stream) {
  if (ld % BK != 0 || q_begin % 4 != 0 || q_begin < 0 || q_end > n || q_begin > q_end) return cudaErrorInvalidValue;
  const int64_t cols = knn_f32_kt_cols(n);
  const int64_t tiles = cols / 64 * (ld / 16);
  const int tgrid = int(std::min<int64_t>(tiles, int64_t(sms) * 8));
  transpose_rows_kernel<<<tgrid, 256, 0, stream>>>(X, n, ld, XT, cols);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || q_begin == q_end) return e;
  const size_t smem = sizeof(F32KtSmem);
  e = cudaFuncSetAttribute(knn_f32_kt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  knn_f32_kt_kernel<<<grid, NT, smem, stream>>>(XT, cols, n, ld, k, cap, scratch, out_idx, out_raw, out_dist,
                                                q_begin, q_end);
  return cudaGetLastError();
}

}  // namespace evoc
