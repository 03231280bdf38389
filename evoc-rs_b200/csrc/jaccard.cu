// Exact bitwise-Jaccard kNN for packed binary rows (EmbeddingData::UInt8),
// with the top-k selection fused into the tile epilogue.
//
// Dissimilarity (src/nndescent/uint8.rs:21-35): -(inter / union) with f32
// division, 0.0 when union == 0.  inter = sum popc(a & b) over 32-bit words;
// union = |a| + |b| - inter, which equals popc(a | b) exactly, so only the
// AND+POPC pair runs per word and the row popcounts are computed once.
//
// Layout: rows of `ldw` 32-bit words (the byte rows zero-padded to a
// multiple of 64 bytes).  A persistent grid walks 128-row query blocks; each
// 128-row key tile is accumulated in 16-word steps with 128-bit loads into
// a double-buffered shared-memory stage and 8x8 per-thread register tiles of
// intersection counts; the counts are staged in shared memory and 128 owner
// threads (one per query row) offer the survivors to a bounded max-heap of
// (raw, index) keys in shared memory.
#include "common.cuh"
#include "kernels.h"

namespace evoc {

namespace {
constexpr int BM = 128, BN = 128, BKW = 16, NT = 256;
constexpr int SPAD = 129;
constexpr int APAD = 132;

struct JacSmem {
  uint32_t a[2][BKW][APAD];
  uint32_t b[2][BKW][APAD];
  int32_t s[BM][SPAD];
  int32_t pb[BN];
};

__device__ __forceinline__ void load_words(const uint32_t* __restrict__ X, int64_t n, int ldw, int64_t row0, int k0,
                                           int tid, uint4 (&r)[2]) {
  const int row = tid >> 2, c4 = (tid & 3) * 4;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int64_t g = row0 + row + h * 64;
    if (g < n) r[h] = *reinterpret_cast<const uint4*>(X + g * ldw + k0 + c4);
    else r[h] = make_uint4(0u, 0u, 0u, 0u);
  }
}

__device__ __forceinline__ void store_words(uint32_t (*dst)[APAD], int tid, const uint4 (&r)[2]) {
  const int row = tid >> 2, c4 = (tid & 3) * 4;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    dst[c4 + 0][row + h * 64] = r[h].x;
    dst[c4 + 1][row + h * 64] = r[h].y;
    dst[c4 + 2][row + h * 64] = r[h].z;
    dst[c4 + 3][row + h * 64] = r[h].w;
  }
}

// Jaccard dissimilarity from exact counts, as the reference computes it.
__device__ __forceinline__ float jaccard_raw(int32_t inter, int32_t uni) {
  return uni > 0 ? -__fdiv_rn(__int2float_rn(inter), __int2float_rn(uni)) : 0.0f;
}
}  // namespace

__global__ void popcount_rows_kernel(const uint32_t* __restrict__ X, int64_t n, int ldw, int32_t* __restrict__ pc) {
  for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += int64_t(gridDim.x) * blockDim.x) {
    int32_t c = 0;
    for (int w = 0; w < ldw; w++) c += __popc(X[r * ldw + w]);
    pc[r] = c;
  }
}

__global__ void __launch_bounds__(NT, 1)
knn_jaccard_kernel(const uint32_t* __restrict__ X, const int32_t* __restrict__ pc, int64_t n, int ldw, int k,
                   int heap_stride, int32_t* __restrict__ out_idx, float* __restrict__ out_raw,
                   float* __restrict__ out_dist, int64_t q_begin, int64_t q_end) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  JacSmem& sm = *reinterpret_cast<JacSmem*>(smem_raw);
  uint64_t* heaps = reinterpret_cast<uint64_t*>(smem_raw + sizeof(JacSmem));
  const int tid = threadIdx.x;
  const int ty = tid >> 4, tx = tid & 15;
  const int64_t n_qblocks = (q_end - q_begin + BM - 1) / BM;
  const int64_t n_ktiles = (n + BN - 1) / BN;

  for (int64_t qb = blockIdx.x; qb < n_qblocks; qb += gridDim.x) {
    const int64_t q0 = q_begin + qb * BM;
    const int64_t my_q = q0 + tid;
    const bool owner = tid < BM && my_q < q_end;
    KeyHeap heap;
    heap.init(heaps + (tid & (BM - 1)) * heap_stride, k);
    const int32_t pa = owner ? pc[my_q] : 0;
    if (owner) heap.offer(make_key(-1.0f, int32_t(my_q)));  // self, the NN-descent leaf-init rule
    float thr_j = -1.0f;  // Jaccard similarity a key must reach (negative: heap not full)

    for (int64_t kt = 0; kt < n_ktiles; kt++) {
      const int64_t c0 = kt * BN;
      int32_t acc[8][8];
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = 0;
      uint4 ra[2], rb[2];
      load_words(X, q_end, ldw, q0, 0, tid, ra);
      load_words(X, n, ldw, c0, 0, tid, rb);
      store_words(sm.a[0], tid, ra);
      store_words(sm.b[0], tid, rb);
      if (tid < BN) sm.pb[tid] = (c0 + tid < n) ? pc[c0 + tid] : 0;
      __syncthreads();
      int buf = 0;
      for (int k0 = 0; k0 < ldw; k0 += BKW) {
        const bool more = k0 + BKW < ldw;
        if (more) {
          load_words(X, q_end, ldw, q0, k0 + BKW, tid, ra);
          load_words(X, n, ldw, c0, k0 + BKW, tid, rb);
        }
#pragma unroll
        for (int kk = 0; kk < BKW; kk++) {
          const uint4 t0 = *reinterpret_cast<const uint4*>(&sm.a[buf][kk][ty * 4]);
          const uint4 t1 = *reinterpret_cast<const uint4*>(&sm.a[buf][kk][64 + ty * 4]);
          const uint4 u0 = *reinterpret_cast<const uint4*>(&sm.b[buf][kk][tx * 4]);
          const uint4 u1 = *reinterpret_cast<const uint4*>(&sm.b[buf][kk][64 + tx * 4]);
          const uint32_t av[8] = {t0.x, t0.y, t0.z, t0.w, t1.x, t1.y, t1.z, t1.w};
          const uint32_t bv[8] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w};
#pragma unroll
          for (int i = 0; i < 8; i++)
#pragma unroll
            for (int j = 0; j < 8; j++) acc[i][j] += __popc(av[i] & bv[j]);
        }
        if (more) {
          store_words(sm.a[buf ^ 1], tid, ra);
          store_words(sm.b[buf ^ 1], tid, rb);
        }
        __syncthreads();
        buf ^= 1;
      }
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
      if (owner) {
        const int lim = (n - c0 < BN) ? int(n - c0) : BN;
        for (int c = 0; c < lim; c++) {
          const int32_t inter = sm.s[tid][c];
          const int32_t uni = pa + sm.pb[c] - inter;
          // inter/uni >= thr_j  <=>  inter >= thr_j * uni (uni > 0); loosened so
          // rounding never rejects a key the exact compare would admit.
          if (thr_j >= 0.0f && float(inter) < thr_j * float(uni) * (1.0f - 1e-6f) - 0.5f) continue;
          const int64_t key = c0 + c;
          if (key == my_q) continue;
          heap.offer(make_key(jaccard_raw(inter, uni), int32_t(key)));
          const uint64_t t = heap.threshold();
          thr_j = (t == kKeyInf) ? -1.0f : -from_orderable(uint32_t(t >> 32));
        }
      }
      __syncthreads();
    }
    if (owner) {
      const int got = heap.finish();
      const int64_t orow = (my_q - q_begin) * k;
      for (int j = 0; j < k; j++) {
        float raw = kHeapInf;
        int32_t idx = -1;
        if (j < got) {
          raw = from_orderable(uint32_t(heap.h[j] >> 32));
          idx = key_index(heap.h[j]);
          // The key folds -0.0 onto +0.0; the reference gives -0.0 for an empty
          // intersection with a non-empty union and +0.0 when both rows are empty.
          if (raw == 0.0f) raw = (pa + pc[idx] == 0) ? 0.0f : -0.0f;
        }
        out_idx[orow + j] = idx;
        if (out_raw) out_raw[orow + j] = raw;
        if (out_dist) out_dist[orow + j] = transform_raw(2, raw);
      }
    }
    __syncthreads();
  }
}

// One thread per 16 output bytes (two input bytes): each input bit becomes a
// 0/1 byte, most significant bit first (the order np.packbits uses; any fixed
// order gives the same intersection counts).
__global__ void expand_bits_kernel(const uint8_t* __restrict__ X, int64_t n, int64_t ld_in, int64_t nbytes,
                                   uint8_t* __restrict__ Y, int64_t rows, int64_t ld_out) {
  const int64_t per_row = ld_out / 16;
  const int64_t total = rows * per_row;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / per_row, c = e % per_row;  // c-th 16-byte group = input bytes 2c, 2c+1
    uint32_t w[4] = {0u, 0u, 0u, 0u};
    if (r < n) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int64_t b = 2 * c + h;
        const uint32_t v = b < nbytes ? X[r * ld_in + b] : 0u;
        // bits 7..4 -> bytes 0..3 of word 2h, bits 3..0 -> bytes 0..3 of word 2h+1
        w[2 * h] = ((v >> 7) & 1u) | (((v >> 6) & 1u) << 8) | (((v >> 5) & 1u) << 16) | (((v >> 4) & 1u) << 24);
        w[2 * h + 1] = ((v >> 3) & 1u) | (((v >> 2) & 1u) << 8) | (((v >> 1) & 1u) << 16) | ((v & 1u) << 24);
      }
    }
    *reinterpret_cast<uint4*>(Y + r * ld_out + c * 16) = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

cudaError_t launch_expand_bits(const void* X, int64_t n, int64_t ld_in, int64_t nbytes, void* Y, int64_t rows,
                               int64_t ld_out, int sms, cudaStream_t stream) {
  if (ld_out % 16 != 0 || ld_out < 8 * nbytes || rows < n || (reinterpret_cast<uintptr_t>(Y) & 15))
    return cudaErrorInvalidValue;
  expand_bits_kernel<<<sms * 8, 256, 0, stream>>>(static_cast<const uint8_t*>(X), n, ld_in, nbytes,
                                                   static_cast<uint8_t*>(Y), rows, ld_out);
  return cudaGetLastError();
}

cudaError_t launch_popcount_rows(const void* X, int64_t n, int ldw, int32_t* pc, int sms, cudaStream_t stream) {
  popcount_rows_kernel<<<sms * 4, 256, 0, stream>>>(static_cast<const uint32_t*>(X), n, ldw, pc);
  return cudaGetLastError();
}

size_t knn_jaccard_smem(int k) { return sizeof(JacSmem) + size_t(BM) * size_t(k | 1) * 8; }

cudaError_t launch_knn_jaccard(const void* X, int64_t n, int ldw, int k, int32_t* pc, int grid, int32_t* out_idx,
                               float* out_raw, float* out_dist, int64_t q_begin, int64_t q_end, int sms,
                               cudaStream_t stream) {
  const size_t smem = knn_jaccard_smem(k);
  if (smem > 232448) return cudaErrorInvalidValue;
  popcount_rows_kernel<<<sms * 4, 256, 0, stream>>>(static_cast<const uint32_t*>(X), n, ldw, pc);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // The opt-in limit rather than `smem` (which varies with k), so concurrent
  // callers never lower each other's limit before their launch.
  e = cudaFuncSetAttribute(knn_jaccard_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 232448);
  if (e != cudaSuccess) return e;
  knn_jaccard_kernel<<<grid, NT, smem, stream>>>(static_cast<const uint32_t*>(X), pc, n, ldw, k, k | 1, out_idx,
                                                 out_raw, out_dist, q_begin, q_end);
  return cudaGetLastError();
}

}  // namespace evoc
