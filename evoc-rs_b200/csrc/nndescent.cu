// GPU NN-descent (approximate kNN), the device counterpart of the reference's
// nn_descent_*_sorted drivers (src/nndescent/float.rs:775-879, int8.rs:575-678,
// uint8.rs:563-666).
//
// Each iteration follows the reference's steps:
//   * candidates (build_candidates, src/heap.rs:203-343): for every row, up to
//     max_candidates new and max_candidates old candidates drawn from its
//     forward and reverse edges, the ones with the smallest priority kept
//     (priority: a hash of the edge and the iteration, the same for both
//     directions of an edge, as the reference draws one tau value per edge);
//   * local join (generate_sorted_graph_update_array, float.rs:517-669): the
//     reference pairs the candidates of every row v (new x new, new x old)
//     and pushes each pair into both rows' heaps.  Here the join is pulled so
//     that every row's list has one writer: row u takes, from every candidate
//     src of u, the candidates w of src, when the edge to src or the one out
//     of src is new;
//   * update (flagged_heap_push / apply_sorted_graph_updates, heap.rs:143-200,
//     425-502): a warp owns row u and keeps its sorted top-k (k <= 64) in
//     registers, two keys per lane, inserting by warp ballots and shuffles;
//     an index already in the list is not inserted twice;
//   * stop (float.rs:853-872): after an iteration that changed at most
//     delta * k * n entries, or whose sum of distances moved by less than
//     delta_improv relative to the previous iteration.
// The graph is double buffered (reads from the current lists of every row,
// writes the next), so no row is read while it is rewritten.  A row's
// second-hop ids go through a per-warp hash set in shared memory, so each
// distance is computed once per row and iteration, and four candidate rows
// are gathered at a time (16-byte loads from each, four independent streams
// in flight per lane).  Rows are visited in nearest-pivot order (the cells
// that seed the initial graph), so concurrently processed rows share gathered
// rows in L2.  f32 data is joined on its FP16 rows (half the bytes of f32; the
// candidates' final distances and order are recomputed by the FP32 rerank,
// rerank.cu, from the f32 rows).
#include <cuda_fp16.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace evoc {

namespace {
constexpr int NW = 4;           // warps per block
constexpr int HSLOTS = 2048;    // hash-set slots per warp (ids evaluated for the current row): 8 KB,
                                // so seven 4-warp blocks fit an SM's shared memory
constexpr int KMAX = 64;
constexpr int MCMAX = 64;       // max_candidates
constexpr uint32_t kEmpty = 0xffffffffu;

__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// Dot-product partial sums of one 16-byte chunk.
template <int DT>
__device__ __forceinline__ float chunk_dot(uint4 x, uint4 y) {
  if (DT == 0) {  // FP16 rows
    const __half2* a = reinterpret_cast<const __half2*>(&x);
    const __half2* b = reinterpret_cast<const __half2*>(&y);
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const float2 fa = __half22float2(a[i]), fb = __half22float2(b[i]);
      s = fmaf(fa.x, fb.x, s);
      s = fmaf(fa.y, fb.y, s);
    }
    return s;
  }
  return 0.0f;
}

template <int DT>
__device__ __forceinline__ int chunk_int(uint4 x, uint4 y) {
  if (DT == 1) {
    int s = 0;
    s = __dp4a(int(x.x), int(y.x), s);
    s = __dp4a(int(x.y), int(y.y), s);
    s = __dp4a(int(x.z), int(y.z), s);
    s = __dp4a(int(x.w), int(y.w), s);
    return s;
  }
  return __popc(x.x & y.x) + __popc(x.y & y.y) + __popc(x.z & y.z) + __popc(x.w & y.w);
}

// Raw dissimilarities of row a to rows b[0..G) (b < 0: skipped), computed by
// the whole warp with the G gathers interleaved.  Every lane gets all G.
template <int DT, int G>
__device__ __forceinline__ void warp_raw_g(const uint8_t* __restrict__ X, int64_t row_bytes,
                                           const int32_t* __restrict__ pc, int64_t a, const int32_t (&b)[G],
                                           float (&raw)[G], int lane) {
  const uint4* ra = reinterpret_cast<const uint4*>(X + a * row_bytes);
  const int chunks = int(row_bytes / 16);
  float fs[G];
  int is[G];
#pragma unroll
  for (int g = 0; g < G; g++) {
    fs[g] = 0.0f;
    is[g] = 0;
  }
  for (int c = lane; c < chunks; c += 32) {
    const uint4 x = ra[c];
    uint4 y[G];
#pragma unroll
    for (int g = 0; g < G; g++)
      y[g] = b[g] >= 0 ? reinterpret_cast<const uint4*>(X + int64_t(b[g]) * row_bytes)[c] : make_uint4(0, 0, 0, 0);
#pragma unroll
    for (int g = 0; g < G; g++) {
      if (DT == 0) fs[g] += chunk_dot<DT>(x, y[g]);
      else is[g] += chunk_int<DT>(x, y[g]);
    }
  }
#pragma unroll
  for (int g = 0; g < G; g++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      if (DT == 0) fs[g] += __shfl_xor_sync(0xffffffffu, fs[g], o);
      else is[g] += __shfl_xor_sync(0xffffffffu, is[g], o);
    }
    if (DT == 0) raw[g] = raw_cosine(fs[g]);
    else if (DT == 1) raw[g] = raw_int8(is[g]);
    else raw[g] = b[g] >= 0 ? raw_jaccard(uint32_t(is[g]), uint32_t(pc[a] + pc[b[g]] - is[g])) : 0.0f;
  }
}

// A row's sorted top-k (k <= 64): position p < 32 in lane p of `a`, position
// 32 + p in lane p of `b`; unused positions hold kKeyInf.
struct WarpList {
  uint64_t a, b;

  __device__ __forceinline__ uint64_t at(int p) const {
    return p < 32 ? __shfl_sync(0xffffffffu, a, p) : __shfl_sync(0xffffffffu, b, p - 32);
  }
  __device__ __forceinline__ bool contains(int32_t id, int k, int lane) const {
    const bool m = (lane < k && a != kKeyInf && key_index(a) == id) ||
                   (lane + 32 < k && b != kKeyInf && key_index(b) == id);
    return __any_sync(0xffffffffu, m);
  }
  // Inserts key unless its index is present or it does not beat the k-th.
  __device__ __forceinline__ bool insert(uint64_t key, int k, int lane) {
    if (contains(key_index(key), k, lane)) return false;
    if (key >= at(k - 1)) return false;
    const int pos = __popc(__ballot_sync(0xffffffffu, lane < k && a < key)) +
                    __popc(__ballot_sync(0xffffffffu, lane + 32 < k && b < key));
    uint64_t aup = __shfl_up_sync(0xffffffffu, a, 1);
    uint64_t bup = __shfl_up_sync(0xffffffffu, b, 1);
    const uint64_t a31 = __shfl_sync(0xffffffffu, a, 31);
    if (lane == 0) bup = a31;
    if (lane < k) {
      if (lane == pos) a = key;
      else if (lane > pos) a = aup;
    }
    if (lane + 32 < k) {
      if (lane + 32 == pos) b = key;
      else if (lane + 32 > pos) b = bup;
    }
    return true;
  }
};

// Per-warp hash set of the ids whose distance to the current row was taken.
// Returns true when id was absent (and is now recorded); when the probe
// sequence finds neither, the id is reported absent (computed once more --
// the list itself rejects a repeated index).
__device__ __forceinline__ bool hash_claim(uint32_t* hs, uint32_t id) {
  uint32_t h = uint32_t(mix64(id)) & (HSLOTS - 1);
  for (int t = 0; t < 16; t++) {
    const uint32_t prev = atomicCAS(&hs[h], kEmpty, id);
    if (prev == kEmpty) return true;
    if (prev == id) return false;
    h = (h + 1) & (HSLOTS - 1);
  }
  return true;
}

// Candidate buffer of a lane set: the ids in `take` lanes are evaluated four
// at a time and offered to the list.
template <int DT>
__device__ __forceinline__ void eval_taken(const uint8_t* __restrict__ X, int64_t row_bytes,
                                           const int32_t* __restrict__ pc, int64_t u, int32_t w, bool take,
                                           WarpList& L, int k, int lane, uint32_t& evals) {
  uint32_t m = __ballot_sync(0xffffffffu, take);
  evals += __popc(m);
  while (m) {
    int32_t b[4];
#pragma unroll
    for (int g = 0; g < 4; g++) {
      const int src = m ? __ffs(m) - 1 : 0;
      const int32_t v = __shfl_sync(0xffffffffu, w, src);
      b[g] = m ? v : -1;
      m &= m ? m - 1 : 0u;
    }
    float raw[4];
    warp_raw_g<DT, 4>(X, row_bytes, pc, u, b, raw, lane);
#pragma unroll
    for (int g = 0; g < 4; g++)
      if (b[g] >= 0) L.insert(make_key(raw[g], b[g]), k, lane);
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
    WarpList cell{kKeyInf, kKeyInf}, rnd{kKeyInf, kKeyInf};
    if (kc > 0) cell.insert(make_key(-1.0f, int32_t(u)), kc, lane);
    else rnd.insert(make_key(-1.0f, int32_t(u)), kr, lane);
    if (label && kc > 0) {
      const int lb = label[u];
      const int64_t cn = cell_cnt[lb], c0 = cell_end[lb] - cn;
      for (int t = 0; t < 2 * kc + 8 && cn > 1; t += 4) {
        int32_t b[4];
#pragma unroll
        for (int g = 0; g < 4; g++) {
          const uint64_t h = mix64(seed ^ (uint64_t(u) << 20) ^ uint64_t(t + g));
          const int64_t v = order[c0 + int64_t(h % uint64_t(cn))];
          b[g] = v == u ? -1 : int32_t(v);
        }
        float raw[4];
        warp_raw_g<DT, 4>(X, row_bytes, pc, u, b, raw, lane);
#pragma unroll
        for (int g = 0; g < 4; g++)
          if (b[g] >= 0) cell.insert(make_key(raw[g], b[g]), kc, lane);
      }
    }
    for (int t = 0; t < 2 * kr + 8 && kr > 0; t += 4) {
      int32_t b[4];
#pragma unroll
      for (int g = 0; g < 4; g++) {
        const uint64_t h = mix64(seed ^ 0xabcdefull ^ (uint64_t(u) << 20) ^ uint64_t(t + g));
        const int64_t v = int64_t(h % uint64_t(n));
        // skip the row itself and rows already taken from the cell
        b[g] = (v == u || cell.contains(int32_t(v), kc, lane)) ? -1 : int32_t(v);
      }
      float raw[4];
      warp_raw_g<DT, 4>(X, row_bytes, pc, u, b, raw, lane);
#pragma unroll
      for (int g = 0; g < 4; g++)
        if (b[g] >= 0) rnd.insert(make_key(raw[g], b[g]), kr, lane);
    }
    // merge: cell entries then random entries into one sorted list of k
    WarpList L{kKeyInf, kKeyInf};
    for (int s = 0; s < kc; s++) {
      const uint64_t kv = cell.at(s);
      if (kv != kKeyInf) L.insert(kv, k, lane);
    }
    for (int s = 0; s < kr; s++) {
      const uint64_t kv = rnd.at(s);
      if (kv != kKeyInf) L.insert(kv, k, lane);
    }
    if (lane < k) {
      keys[u * k + lane] = L.a;
      isnew[u * k + lane] = 1;
    }
    if (lane + 32 < k) {
      keys[u * k + 32 + lane] = L.b;
      isnew[u * k + 32 + lane] = 1;
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

namespace {
// Keeps, of a row's new or old candidates, the mc ids of smallest priority,
// an id offered more than once (u -> v and v -> u both listed) counting at
// its smallest priority.  The kept set is then independent of the order the
// reverse edges were filled in (atomics): it always equals the mc smallest
// of {id -> min priority} over the pushes so far.
__device__ __forceinline__ void cand_push(uint64_t* best, int32_t* bid, int& got, int mc, uint64_t pr, int32_t id) {
  for (int j = 0; j < got; j++)
    if ((bid[j] & 0x7fffffff) == (id & 0x7fffffff)) {
      if (pr >= best[j]) return;
      int p = j;  // smaller priority: move the entry up
      while (p > 0 && best[p - 1] > pr) {
        best[p] = best[p - 1];
        bid[p] = bid[p - 1];
        p--;
      }
      best[p] = pr;
      bid[p] = id;
      return;
    }
  if (got == mc && pr >= best[mc - 1]) return;
  int p = got < mc ? got++ : mc - 1;
  while (p > 0 && best[p - 1] > pr) {
    best[p] = best[p - 1];
    bid[p] = bid[p - 1];
    p--;
  }
  best[p] = pr;
  bid[p] = id;
}
}  // namespace

// build_candidates (src/heap.rs:203-343): per row, up to mc new and mc old
// candidates from its forward edges (its list) and reverse edges (the rows
// listing it), by smallest priority.  Output: 2*mc tagged ids per row (bit 31
// = new), -1 past the end.
__global__ void nnd_candidates_kernel(const uint64_t* __restrict__ keys, const uint8_t* __restrict__ isnew,
                                      const int64_t* __restrict__ rptr, const int32_t* __restrict__ rrows, int64_t n,
                                      int k, int mc, uint64_t seed, int32_t* __restrict__ cand) {
  for (int64_t u = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; u < n; u += int64_t(gridDim.x) * blockDim.x) {
    uint64_t bn[MCMAX], bo[MCMAX];
    int32_t in_[MCMAX], io[MCMAX];
    int gn = 0, go = 0;
    // forward edges u -> v
    for (int j = 0; j < k; j++) {
      const uint64_t kv = keys[u * k + j];
      if (kv == kKeyInf) continue;
      const int32_t v = key_index(kv);
      if (v == u) continue;
      const uint64_t pr = mix64(seed ^ (uint64_t(u) << 32) ^ uint64_t(uint32_t(v)));  // the edge's priority
      if (isnew[u * k + j]) cand_push(bn, in_, gn, mc, pr, v | int32_t(0x80000000u));
      else cand_push(bo, io, go, mc, pr, v);
    }
    // reverse edges w -> u (tagged with that edge's newness)
    for (int64_t j = rptr[u]; j < rptr[u + 1]; j++) {
      const uint32_t t = uint32_t(rrows[j]);
      const int32_t w = int32_t(t & 0x7fffffffu);
      const uint64_t pr = mix64(seed ^ (uint64_t(uint32_t(w)) << 32) ^ uint64_t(u));
      if (t & 0x80000000u) cand_push(bn, in_, gn, mc, pr, int32_t(t));
      else cand_push(bo, io, go, mc, pr, w);
    }
    int32_t* out = cand + u * 2 * mc;
    for (int j = 0; j < 2 * mc; j++) out[j] = j < gn ? in_[j] : (j - gn < go ? io[j - gn] : -1);
  }
}

// The pull-style local join: warp per row u (in pivot order).  Sources: u's
// candidates; second hop: each source's candidates, taken when the edge to
// the source or the one out of it is new.
template <int DT>
__global__ void __launch_bounds__(NW * 32)
nnd_join_kernel(const uint8_t* __restrict__ X, int64_t row_bytes, const int32_t* __restrict__ pc, int64_t n, int k,
                const int32_t* __restrict__ order, const uint64_t* __restrict__ keys, const int32_t* __restrict__ cand,
                int mc2, uint64_t* __restrict__ keys_out, uint8_t* __restrict__ new_out,
                unsigned long long* __restrict__ changes, unsigned long long* __restrict__ n_evals) {
  extern __shared__ uint32_t nnd_hash[];  // NW x HSLOTS
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* hs = nnd_hash + warp * HSLOTS;
  uint32_t evals = 0;  // distances this warp computed (uniform across the warp)
  for (int64_t w = int64_t(blockIdx.x) * NW + warp; w < n; w += int64_t(gridDim.x) * NW) {
    const int64_t u = order ? order[w] : w;
    WarpList L{lane < k ? keys[u * k + lane] : kKeyInf, lane + 32 < k ? keys[u * k + 32 + lane] : kKeyInf};
    const WarpList orig = L;
    for (int j = lane; j < HSLOTS; j += 32) hs[j] = kEmpty;
    __syncwarp();
    // the list's own ids are never recomputed
    if (lane < k && L.a != kKeyInf) hash_claim(hs, uint32_t(key_index(L.a)));
    if (lane + 32 < k && L.b != kKeyInf) hash_claim(hs, uint32_t(key_index(L.b)));
    __syncwarp();
    const int32_t* cu = cand + u * int64_t(mc2);
    for (int s = 0; s < mc2; s++) {
      const int32_t st = cu[s];  // same address for every lane; -1 ends the list (ids stay below 2^31 - 1)
      if (st == -1) break;
      const int32_t src = int32_t(uint32_t(st) & 0x7fffffffu);
      const bool src_new = (uint32_t(st) & 0x80000000u) != 0;
      if (src == u) continue;
      // the source itself
      bool take = false;
      if (lane == 0) take = hash_claim(hs, uint32_t(src));
      eval_taken<DT>(X, row_bytes, pc, u, src, take, L, k, lane, evals);
      // its candidates
      const int32_t* cs = cand + int64_t(src) * mc2;
      for (int c0 = 0; c0 < mc2; c0 += 32) {
        int32_t wv = -1;
        bool wn = false;
        if (c0 + lane < mc2) {
          const int32_t t = cs[c0 + lane];
          if (t != -1) {
            wv = int32_t(uint32_t(t) & 0x7fffffffu);
            wn = (uint32_t(t) & 0x80000000u) != 0;
          }
        }
        bool tk = wv >= 0 && wv != int32_t(u) && (src_new || wn);
        if (tk) tk = hash_claim(hs, uint32_t(wv));
        eval_taken<DT>(X, row_bytes, pc, u, wv, tk, L, k, lane, evals);
      }
    }
    // New flag: the entry was not in the list at the start of the iteration.
    bool wa = false, wb = false;
    for (int s = 0; s < k; s++) {
      const uint64_t o = orig.at(s);
      wa |= (o == L.a);
      wb |= (o == L.b);
    }
    if (lane < k) {
      keys_out[u * k + lane] = L.a;
      new_out[u * k + lane] = (L.a != kKeyInf && !wa) ? 1 : 0;
    }
    if (lane + 32 < k) {
      keys_out[u * k + 32 + lane] = L.b;
      new_out[u * k + 32 + lane] = (L.b != kKeyInf && !wb) ? 1 : 0;
    }
    const uint32_t ch = __ballot_sync(0xffffffffu, lane < k && L.a != kKeyInf && !wa) ;
    const uint32_t ch2 = __ballot_sync(0xffffffffu, lane + 32 < k && L.b != kKeyInf && !wb);
    if (lane == 0 && (ch | ch2)) atomicAdd(changes, (unsigned long long)(__popc(ch) + __popc(ch2)));
    __syncwarp();
  }
  if (lane == 0 && evals) atomicAdd(n_evals, (unsigned long long)evals);
}

// Sum over the graph of the finite raw dissimilarities, in f64 (the
// delta_improv test, src/nndescent/float.rs:857-870).
// Per-block partial sums into sum[1 + block]; nnd_sum_final_kernel adds them
// in block order into sum[0], so the total does not depend on scheduling.
__global__ void nnd_sum_kernel(const uint64_t* __restrict__ keys, int64_t total, double* __restrict__ sum) {
  __shared__ double part[8];
  double s = 0.0;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const uint64_t kv = keys[e];
    if (kv != kKeyInf) {
      const float r = from_orderable(uint32_t(kv >> 32));
      if (r < kHeapInf) s += double(r);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < int(blockDim.x >> 5); i++) t += part[i];
    sum[1 + blockIdx.x] = t;
  }
}

__global__ void nnd_sum_final_kernel(double* __restrict__ sum, int parts) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double t = 0.0;
  for (int i = 0; i < parts; i++) t += sum[1 + i];
  sum[0] = t;
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

template <int DT>
cudaError_t join(const NndArgs& a, int cur, int blocks, size_t smem, cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(nnd_join_kernel<DT>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  const int nxt = cur ^ 1;
  nnd_join_kernel<DT><<<blocks, NW * 32, smem, stream>>>(a.X, a.row_bytes, a.pc, a.n, a.k, a.order, a.keys[cur],
                                                         a.cand, 2 * a.mc, a.keys[nxt], a.isnew[nxt], a.changes,
                                                         a.evals);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_nnd_init(const NndArgs& a, cudaStream_t stream) {
  if (a.k < 1 || a.k > KMAX || a.mc < 1 || a.mc > MCMAX || a.row_bytes % 16 != 0) return cudaErrorInvalidValue;
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
  nnd_candidates_kernel<<<blocks, 128, 0, stream>>>(a.keys[cur], a.isnew[cur], a.rptr, a.rrows, a.n, a.k, a.mc,
                                                    a.seed + uint64_t(iter) * 7919u, a.cand);
  const size_t smem = size_t(NW) * HSLOTS * sizeof(uint32_t);
  if (a.dtype == 0) e = join<0>(a, cur, blocks, smem, stream);
  else if (a.dtype == 1) e = join<1>(a, cur, blocks, smem, stream);
  else e = join<2>(a, cur, blocks, smem, stream);
  if (e != cudaSuccess) return e;
  const int parts = std::min(a.sms * 4, kNndSumParts);
  nnd_sum_kernel<<<parts, 256, 0, stream>>>(a.keys[cur ^ 1], a.n * a.k, a.sum);
  nnd_sum_final_kernel<<<1, 32, 0, stream>>>(a.sum, parts);
  return cudaGetLastError();
}

cudaError_t launch_nnd_emit(const NndArgs& a, int cur, int32_t* out_idx, float* out_raw, float* out_dist,
                            cudaStream_t stream) {
  nnd_emit_kernel<<<a.sms * 8, 256, 0, stream>>>(a.keys[cur], a.n, a.k, a.dtype, a.pc, out_idx, out_raw, out_dist);
  return cudaGetLastError();
}

}  // namespace evoc
