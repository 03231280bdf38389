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
                    const int32_t* __restrict__ q_list, int64_t q_row0) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  F32Smem& sm = *reinterpret_cast<F32Smem*>(smem_raw);
  const int tid = threadIdx.x;
  const int ty = tid >> 4, tx = tid & 15;
  const int64_t n_qblocks = (q_end - q_begin + BM - 1) / BM;
  const int64_t n_ktiles = (n + BN - 1) / BN;
  uint64_t* my_buf = scratch + (int64_t(blockIdx.x) * BM + (tid & (BM - 1))) * cap;

  for (int64_t qb = blockIdx.x; qb < n_qblocks; qb += gridDim.x) {
    const int64_t q0 = q_begin + qb * BM;
    RowTopK top;
    top.init(my_buf, k, cap);
    const int64_t my_q = q0 + tid;
    // this query's row of X (the self rule) and its output row
    const int64_t my_self = (q_list && tid < BM && my_q < q_end) ? q_row0 + q_list[my_q] : my_q;

    for (int64_t kt = 0; kt < n_ktiles; kt++) {
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
    if (tid < BM && my_q < q_end) {
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

size_t knn_f32_simt_smem() { return sizeof(F32Smem); }

cudaError_t launch_knn_f32_simt(const float* X, int64_t n, int ld, int k, int cap, uint64_t* scratch,
                                int grid, int32_t* out_idx, float* out_raw, float* out_dist, int64_t q_begin,
                                int64_t q_end, cudaStream_t stream, const float* Q, const int32_t* q_list,
                                int64_t q_row0) {
  if ((Q == nullptr) != (q_list == nullptr)) return cudaErrorInvalidValue;
  const size_t smem = sizeof(F32Smem);
  cudaError_t e = cudaFuncSetAttribute(knn_f32_simt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  knn_f32_simt_kernel<<<grid, NT, smem, stream>>>(X, n, ld, k, cap, scratch, out_idx, out_raw, out_dist, q_begin,
                                                   q_end, Q ? Q : X, q_list, q_row0);
  return cudaGetLastError();
}

}  // namespace evoc
