// GPU NN-descent (approximate kNN), the device counterpart of the reference's
// nn_descent_*_sorted drivers (src/nndescent/float.rs:775-879, int8.rs:575-678,
// uint8.rs:563-666).
//
// The reference alternates candidate sampling (src/heap.rs:203-343), a local
// join over each row's new/old candidates (float.rs:517-669) and bucketed
// heap updates (heap.rs:425-502), and stops when an iteration changes at most
// delta * k * n heap entries.  On the GPU the join is done pull-wise so that
// every row's list has exactly one writer:
//   * row u's candidates are its current neighbours, its (sampled) reverse
//     neighbours, and their neighbours -- only pairs that involve at least one
//     new edge, as in the reference's new x new / new x old join;
//   * a warp owns row u: the candidate ids are de-duplicated with a warp
//     bitonic sort in shared memory, each distance is one coalesced 16-byte
//     gather of the candidate row, and the row's top-k (k <= 32) lives in the
//     warp's registers, one key per lane, updated by warp-shuffle insertion;
//   * the graph is double buffered (reads from the current list of every row,
//     writes the next), so no row is read while it is being rewritten.
// Rows are visited in nearest-pivot order (the same cells that seed the
// initial graph), so concurrently processed rows share gathered rows in L2.
// f32 joins compute FP32 dot products from the f32 rows (BF16 rounding would
// blur the k-th boundary of tight clusters); the final k per row are
// recomputed by the FP32 rerank (rerank.cu).
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels.h"

namespace evoc {

namespace {
constexpr int NW = 4;          // warps per block
constexpr int CMAX = 4096;     // candidate ids per row per iteration
constexpr int KMAX = 32;

__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// Warp-cooperative raw dissimilarity between rows a and b (all lanes get it).
template <int DT>
__device__ __forceinline__ float warp_raw(const uint8_t* __restrict__ X, int64_t row_bytes, const int32_t* pc,
                                          int64_t a, int64_t b, int lane) {
  const uint4* ra = reinterpret_cast<const uint4*>(X + a * row_bytes);
  const uint4* rb = reinterpret_cast<const uint4*>(X + b * row_bytes);
  const int chunks = int(row_bytes / 16);
  if (DT == 0) {
    float acc = 0.0f;
    for (int c = lane; c < chunks; c += 32) {
      const float4 x = reinterpret_cast<const float4*>(ra)[c], y = reinterpret_cast<const float4*>(rb)[c];
      acc = fmaf(x.x, y.x, acc);
      acc = fmaf(x.y, y.y, acc);
      acc = fmaf(x.z, y.z, acc);
      acc = fmaf(x.w, y.w, acc);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return raw_cosine(acc);
  } else if (DT == 1) {
    int acc = 0;
    for (int c = lane; c < chunks; c += 32) {
      const uint4 x = ra[c], y = rb[c];
      acc = __dp4a(int(x.x), int(y.x), acc);
      acc = __dp4a(int(x.y), int(y.y), acc);
      acc = __dp4a(int(x.z), int(y.z), acc);
      acc = __dp4a(int(x.w), int(y.w), acc);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return raw_int8(acc);
  } else {
    int inter = 0;
    for (int c = lane; c < chunks; c += 32) {
      const uint4 x = ra[c], y = rb[c];
      inter += __popc(x.x & y.x) + __popc(x.y & y.y) + __popc(x.z & y.z) + __popc(x.w & y.w);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) inter += __shfl_xor_sync(0xffffffffu, inter, o);
    return raw_jaccard(uint32_t(inter), uint32_t(pc[a] + pc[b] - inter));
  }
}

// Sorted top-k held one key per lane (lanes >= k hold kKeyInf).  Inserts key
// unless its index is already present or it does not beat the k-th; returns
// whether it was inserted.
__device__ __forceinline__ bool warp_insert(uint64_t& mine, uint64_t key, int k, int lane) {
  const uint32_t same = __ballot_sync(0xffffffffu, lane < k && key_index(mine) == key_index(key) && mine != kKeyInf);
  if (same) return false;
  const uint64_t kth = __shfl_sync(0xffffffffu, mine, k - 1);
  if (key >= kth) return false;
  const uint32_t below = __ballot_sync(0xffffffffu, lane < k && mine < key);
  const int pos = __popc(below);
  const uint64_t up = __shfl_up_sync(0xffffffffu, mine, 1);
  if (lane < k) {
    if (lane == pos) mine = key;
    else if (lane > pos) mine = up;
  }
  return true;
}

__device__ __forceinline__ void warp_sort_u32(uint32_t* a, int P, int lane) {
  for (int size = 2; size <= P; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = lane; i < (P >> 1); i += 32) {
        const int lo = 2 * stride * (i / stride) + (i % stride), hi = lo + stride;
        const bool up = (lo & size) == 0;
        const uint32_t x = a[lo], y = a[hi];
        if ((x > y) == up) {
          a[lo] = y;
          a[hi] = x;
        }
      }
      __syncwarp();
    }
}
}  // namespace

// Initial graph: self (raw -1.0), the nearest of rows drawn from the row's
// pivot cell, and a third of the list kept for random rows from anywhere.
// The random entries keep the initial graph connected across cells: with
// cell-only lists, neighbours of neighbours never leave the cell and true
// neighbours just across a cell boundary are never reached.  Every entry is
// new.
template <int DT>
__global__ void __launch_bounds__(NW * 32)
nnd_init_kernel(const uint8_t* __restrict__ X, int64_t row_bytes, const int32_t* __restrict__ pc, int64_t n, int k,
                const int32_t* __restrict__ order, const int32_t* __restrict__ label,
                const int32_t* __restrict__ cell_end, const int32_t* __restrict__ cell_cnt, uint64_t seed,
                uint64_t* __restrict__ keys, uint8_t* __restrict__ isnew) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kr = label ? k / 3 : k;  // slots for random rows
  const int kc = k - kr;             // slots for cell rows (self included)
  for (int64_t w = int64_t(blockIdx.x) * NW + warp; w < n; w += int64_t(gridDim.x) * NW) {
    const int64_t u = order ? order[w] : w;
    uint64_t cellk = kKeyInf, randk = kKeyInf;
    if (kc > 0) warp_insert(cellk, make_key(-1.0f, int32_t(u)), kc, lane);
    else warp_insert(randk, make_key(-1.0f, int32_t(u)), kr, lane);
    if (label && kc > 0) {
      const int lb = label[u];
      const int64_t cn = cell_cnt[lb], c0 = cell_end[lb] - cn;
      for (int t = 0; t < 2 * kc + 8 && cn > 1; t++) {
        const uint64_t h = mix64(seed ^ (uint64_t(u) << 20) ^ uint64_t(t));
        const int64_t v = order[c0 + int64_t(h % uint64_t(cn))];
        if (v == u) continue;
        warp_insert(cellk, make_key(warp_raw<DT>(X, row_bytes, pc, u, v, lane), int32_t(v)), kc, lane);
      }
    }
    for (int t = 0; t < 2 * kr + 8 && kr > 0; t++) {
      const uint64_t h = mix64(seed ^ 0xabcdefull ^ (uint64_t(u) << 20) ^ uint64_t(t));
      const int64_t v = int64_t(h % uint64_t(n));
      if (v == u) continue;
      const uint64_t key = make_key(warp_raw<DT>(X, row_bytes, pc, u, v, lane), int32_t(v));
      // skip rows already taken from the cell
      if (__ballot_sync(0xffffffffu, lane < kc && cellk != kKeyInf && key_index(cellk) == int32_t(v))) continue;
      warp_insert(randk, key, kr, lane);
    }
    // merge: cell entries then random entries into one sorted list of k
    uint64_t mine = kKeyInf;
    for (int s = 0; s < kc; s++) {
      const uint64_t kv = __shfl_sync(0xffffffffu, cellk, s);
      if (kv != kKeyInf) warp_insert(mine, kv, k, lane);
    }
    for (int s = 0; s < kr; s++) {
      const uint64_t kv = __shfl_sync(0xffffffffu, randk, s);
      if (kv != kKeyInf) warp_insert(mine, kv, k, lane);
    }
    if (lane < k) {
      keys[u * k + lane] = mine;
      isnew[u * k + lane] = 1;
    }
  }
}

// Reverse edges: for every edge u -> v, count v (pass 0) or place u in v's
// bucket (pass 1), tagged with the edge's newness in bit 31.
__global__ void nnd_reverse_kernel(const uint64_t* __restrict__ keys, const uint8_t* __restrict__ isnew, int64_t n,
                                   int k, int pass, int32_t* __restrict__ cnt, const int64_t* __restrict__ ptr,
                                   int32_t* __restrict__ fill, int32_t* __restrict__ rows) {
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n * k; e += int64_t(gridDim.x) * blockDim.x) {
    if (keys[e] == kKeyInf) continue;
    const int32_t v = key_index(keys[e]);
    const int32_t u = int32_t(e / k);
    if (v == u) continue;
    if (pass == 0) atomicAdd(&cnt[v], 1);
    else rows[ptr[v] + atomicAdd(&fill[v], 1)] = int32_t(uint32_t(u) | (isnew[e] ? 0x80000000u : 0u));
  }
}

// Keeps, per row, rcap reverse neighbours: new edges first, then by hash
// priority (a deterministic sample; the reference samples by random priority).
// Entries keep the newness tag in bit 31.
__global__ void nnd_reverse_select_kernel(const int64_t* __restrict__ ptr, const int32_t* __restrict__ rows, int64_t n,
                                          int rcap, uint64_t seed, int32_t* __restrict__ sel, int32_t* __restrict__ nsel) {
  for (int64_t v = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += int64_t(gridDim.x) * blockDim.x) {
    const int64_t s = ptr[v], m = ptr[v + 1] - s;
    int got = 0;
    uint64_t best[KMAX];
    int32_t bid[KMAX];
    for (int64_t j = 0; j < m; j++) {
      const int32_t u = rows[s + j];  // tagged
      const uint32_t id = uint32_t(u) & 0x7fffffffu;
      const uint64_t old_bit = (uint32_t(u) & 0x80000000u) ? 0ull : (1ull << 63);
      const uint64_t pr = old_bit | ((mix64(seed ^ (uint64_t(id) << 32) ^ uint64_t(v)) >> 1) & 0x7fffffff00000000ull) | id;
      if (got < rcap) {
        int p = got++;
        while (p > 0 && best[p - 1] > pr) {
          best[p] = best[p - 1];
          bid[p] = bid[p - 1];
          p--;
        }
        best[p] = pr;
        bid[p] = u;
      } else if (pr < best[rcap - 1]) {
        int p = rcap - 1;
        while (p > 0 && best[p - 1] > pr) {
          best[p] = best[p - 1];
          bid[p] = bid[p - 1];
          p--;
        }
        best[p] = pr;
        bid[p] = u;
      }
    }
    for (int j = 0; j < got; j++) sel[v * rcap + j] = bid[j];
    nsel[v] = got;
  }
}

template <int DT>
__global__ void __launch_bounds__(NW * 32)
nnd_join_kernel(const uint8_t* __restrict__ X, int64_t row_bytes, const int32_t* __restrict__ pc, int64_t n, int k,
                const int32_t* __restrict__ order, const uint64_t* __restrict__ keys, const uint8_t* __restrict__ isnew,
                const int32_t* __restrict__ rsel, const int32_t* __restrict__ rn, int rcap,
                uint64_t* __restrict__ keys_out, uint8_t* __restrict__ new_out, unsigned long long* __restrict__ changes) {
  extern __shared__ uint32_t nnd_cand[];  // NW x CMAX candidate ids
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* cw = nnd_cand + warp * CMAX;
  for (int64_t w = int64_t(blockIdx.x) * NW + warp; w < n; w += int64_t(gridDim.x) * NW) {
    const int64_t u = order ? order[w] : w;
    uint64_t mine = lane < k ? keys[u * k + lane] : kKeyInf;
    const uint64_t orig = mine;
    const uint8_t mynew = lane < k ? isnew[u * k + lane] : 0;
    // Sources: the current neighbours (newness from the list) and the sampled
    // reverse neighbours (newness of the reverse edge).  Second hop: each
    // source's neighbours and reverse neighbours; a pair counts when the edge
    // to the source or the edge out of it is new (the reference joins new x
    // new and new x old candidates of every row, src/nndescent/float.rs:517-669).
    const int nr = rn[u];
    int nc = 0;
    for (int s = 0; s < k + nr; s++) {
      int32_t src;
      int src_new;
      if (s < k) {
        const uint64_t kv = __shfl_sync(0xffffffffu, mine, s);
        src_new = __shfl_sync(0xffffffffu, int(mynew), s);
        if (kv == kKeyInf) continue;
        src = key_index(kv);
      } else {
        const uint32_t t = uint32_t(rsel[u * rcap + (s - k)]);
        src = int32_t(t & 0x7fffffffu);
        src_new = (t & 0x80000000u) ? 1 : 0;
      }
      if (src < 0 || src == u) continue;
      if (lane == 0 && nc < CMAX) cw[nc] = uint32_t(src);
      nc = nc < CMAX ? nc + 1 : nc;
      // forward neighbours of src (lanes < k), then its reverse sample (lanes < rn[src])
      for (int part = 0; part < 2; part++) {
        int32_t w = -1;
        int wn = 0;
        if (part == 0) {
          const uint64_t nk = lane < k ? keys[int64_t(src) * k + lane] : kKeyInf;
          if (nk != kKeyInf) {
            w = key_index(nk);
            wn = isnew[int64_t(src) * k + lane];
          }
        } else {
          if (lane < rn[src]) {
            const uint32_t t = uint32_t(rsel[int64_t(src) * rcap + lane]);
            w = int32_t(t & 0x7fffffffu);
            wn = (t & 0x80000000u) ? 1 : 0;
          }
        }
        const bool take = w >= 0 && w != int32_t(u) && (src_new || wn);
        const uint32_t m = __ballot_sync(0xffffffffu, take);
        const int off = __popc(m & ((1u << lane) - 1u));
        if (take && nc + off < CMAX) cw[nc + off] = uint32_t(w);
        nc += __popc(m);
        if (nc > CMAX) nc = CMAX;
      }
      __syncwarp();
    }
    int P = 1;
    while (P < nc) P <<= 1;
    for (int j = nc + lane; j < P; j += 32) cw[j] = 0xffffffffu;
    __syncwarp();
    warp_sort_u32(cw, P, lane);
    // Walk the unique ids; each distance is one warp-wide gather.
    for (int j = 0; j < nc; j++) {
      const uint32_t c = cw[j];
      if (c == 0xffffffffu) break;
      if (j > 0 && cw[j - 1] == c) continue;
      const uint32_t inl = __ballot_sync(0xffffffffu, lane < k && orig != kKeyInf && key_index(orig) == int32_t(c));
      if (inl) continue;
      const float raw = warp_raw<DT>(X, row_bytes, pc, u, int64_t(c), lane);
      warp_insert(mine, make_key(raw, int32_t(c)), k, lane);
    }
    // New flag: the entry was not in the list at the start of the iteration.
    bool was = false;
    for (int s = 0; s < k; s++) {
      const uint64_t o = __shfl_sync(0xffffffffu, orig, s);
      was |= (o == mine);
    }
    if (lane < k) {
      keys_out[u * k + lane] = mine;
      new_out[u * k + lane] = (mine != kKeyInf && !was) ? 1 : 0;
    }
    const uint32_t ch = __ballot_sync(0xffffffffu, lane < k && mine != kKeyInf && !was);
    if (lane == 0 && ch) atomicAdd(changes, (unsigned long long)__popc(ch));
    __syncwarp();
  }
}

// Final rows: sorted keys -> (index, raw, transformed distance); optionally the
// index list only (for the FP32 rerank of f32 data).
__global__ void nnd_emit_kernel(const uint64_t* __restrict__ keys, int64_t n, int k, int dtype,
                                const int32_t* __restrict__ pc, int32_t* __restrict__ out_idx,
                                float* __restrict__ out_raw, float* __restrict__ out_dist) {
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n * k; e += int64_t(gridDim.x) * blockDim.x) {
    const uint64_t kv = keys[e];
    const bool ok = kv != kKeyInf;
    float raw = ok ? from_orderable(uint32_t(kv >> 32)) : kHeapInf;
    const int32_t id = ok ? key_index(kv) : -1;
    if (ok && raw == 0.0f) {
      if (dtype == 1) raw = -0.0f;
      else if (dtype == 2) raw = (pc[e / k] + pc[id] == 0) ? 0.0f : -0.0f;
    }
    out_idx[e] = id;
    if (out_raw) out_raw[e] = raw;
    if (out_dist) out_dist[e] = transform_raw(dtype, raw);
  }
}

namespace {
template <int DT>
cudaError_t nnd_run(const NndArgs& a, cudaStream_t stream) {
  const int blocks = a.sms * 8;
  nnd_init_kernel<DT><<<blocks, NW * 32, 0, stream>>>(a.X, a.row_bytes, a.pc, a.n, a.k, a.order, a.label, a.cell_end,
                                                      a.cell_cnt, a.seed, a.keys[0], a.isnew[0]);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_nnd_init(const NndArgs& a, cudaStream_t stream) {
  if (a.k < 1 || a.k > KMAX || a.row_bytes % 16 != 0) return cudaErrorInvalidValue;
  if (a.dtype == 0) return nnd_run<0>(a, stream);
  if (a.dtype == 1) return nnd_run<1>(a, stream);
  return nnd_run<2>(a, stream);
}

cudaError_t launch_nnd_iteration(const NndArgs& a, int cur, int iter, cudaStream_t stream) {
  const int blocks = a.sms * 8;
  cudaError_t e = cudaMemsetAsync(a.rcnt, 0, size_t(a.n) * 4, stream);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(a.rfill, 0, size_t(a.n) * 4, stream);
  if (e != cudaSuccess) return e;
  nnd_reverse_kernel<<<blocks, 256, 0, stream>>>(a.keys[cur], a.isnew[cur], a.n, a.k, 0, a.rcnt, nullptr, nullptr,
                                                 nullptr);
  e = launch_scan_counts(a.rcnt, a.n, a.rptr, stream);
  if (e != cudaSuccess) return e;
  nnd_reverse_kernel<<<blocks, 256, 0, stream>>>(a.keys[cur], a.isnew[cur], a.n, a.k, 1, a.rcnt, a.rptr, a.rfill,
                                                 a.rrows);
  nnd_reverse_select_kernel<<<blocks, 128, 0, stream>>>(a.rptr, a.rrows, a.n, a.rcap, a.seed + uint64_t(iter) * 7919u,
                                                        a.rsel, a.rn);
  const int nxt = cur ^ 1;
  const size_t smem = size_t(NW) * CMAX * sizeof(uint32_t);
  if (a.dtype == 0) {
    e = cudaFuncSetAttribute(nnd_join_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    nnd_join_kernel<0><<<blocks, NW * 32, smem, stream>>>(a.X, a.row_bytes, a.pc, a.n, a.k, a.order, a.keys[cur],
                                                          a.isnew[cur], a.rsel, a.rn, a.rcap, a.keys[nxt],
                                                          a.isnew[nxt], a.changes);
  } else if (a.dtype == 1) {
    e = cudaFuncSetAttribute(nnd_join_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    nnd_join_kernel<1><<<blocks, NW * 32, smem, stream>>>(a.X, a.row_bytes, a.pc, a.n, a.k, a.order, a.keys[cur],
                                                          a.isnew[cur], a.rsel, a.rn, a.rcap, a.keys[nxt],
                                                          a.isnew[nxt], a.changes);
  } else {
    e = cudaFuncSetAttribute(nnd_join_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    nnd_join_kernel<2><<<blocks, NW * 32, smem, stream>>>(a.X, a.row_bytes, a.pc, a.n, a.k, a.order, a.keys[cur],
                                                          a.isnew[cur], a.rsel, a.rn, a.rcap, a.keys[nxt],
                                                          a.isnew[nxt], a.changes);
  }
  return cudaGetLastError();
}

cudaError_t launch_nnd_emit(const NndArgs& a, int cur, int32_t* out_idx, float* out_raw, float* out_dist,
                            cudaStream_t stream) {
  nnd_emit_kernel<<<a.sms * 8, 256, 0, stream>>>(a.keys[cur], a.n, a.k, a.dtype, a.pc, out_idx, out_raw, out_dist);
  return cudaGetLastError();
}

}  // namespace evoc
