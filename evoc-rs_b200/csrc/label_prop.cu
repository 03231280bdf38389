// Label-propagation initialisation and reproducible node-embedding kernels.
//
//   label_prop_iteration ........ src/label_prop.rs:39-91     lp_iteration_kernel
//   label_outliers .............. src/label_prop.rs:94-132    outlier_walk_kernel + pointer jumping
//   remap_labels ................ src/label_prop.rs:135-157   remap_* kernels
//   partition reduction maps .... src/label_prop.rs:188-230   part_* kernels
//   csr_matmul_dense ............ src/label_prop.rs:233-250   reduce_data_kernel, expand_kernel
//   scipy_csr_matmul (SMMP) ..... src/csr_matmul.rs:6-59      launch_reduce_graph, expand_kernel
//   hadamard_symmetric .......... src/label_prop.rs:450-461   launch_hadamard_sym
//   pca_init + small-graph norm . src/label_prop.rs:251-309   pca_kernel
//   final centring / scaling .... src/label_prop.rs:660-672   center_* kernels
//   make_epochs_per_sample ...... src/embed.rs:10-23          ne_schedule_kernel
//   node_embedding_epoch_repr ... src/embed.rs:138-248        ne_block_kernel, ne_heavy_kernel, ne_apply_kernel
//   node_embedding_epoch ........ src/embed.rs:57-135         ne_hogwild_kernel (lock-free, not bit-exact)
//
// Every result matches the reference's rounding: f32 expressions are written
// with __fmul_rn / __fadd_rn / __fsub_rn / __fdiv_rn / __fsqrt_rn so nvcc
// cannot contract them into FMAs, and every order-dependent sum runs in the
// reference's order.  Where the reference is serial (the outlier walk, the
// per-part and per-row sums) the GPU runs independent rows / parts / columns
// in parallel and each of them serially.
//
// The SciPy SMMP products keep SciPy's output order (each row's columns in
// reverse order of first appearance), which the recursion's vote order and
// the embedding's edge order depend on.  Instead of a per-row linked list the
// product is formed by stable radix sorts:
//   temp = N^T G:  edge e of row i (part p = part[i]) contributes x_p * g_e to
//     (p, j); sorting the edges by (p, j), stable in e, lists each group's
//     contributions in the reference's accumulation order (members ascending,
//     then row order), and the group's first e is its first appearance.
//   reduced = temp R:  temp entries sorted by (p, q = part[j], descending first
//     e) list each (p, q) group in temp's row order; a group's head (largest
//     first e) is where q first appears, so the row's output order is the
//     heads' first e ascending.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "lp.h"

namespace evoc {
namespace lp {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int32_t kNoKey = INT32_MIN;
constexpr int64_t kOutlierStack = 4096;  // per-warp stack entries of the parallel outlier walks

// tau RNG step, src/rng.rs:5-35 (int64 state words, 32-bit result).
__device__ int32_t tau_rand_int(int64_t st[3]) {
  auto shl = [](int64_t v, int sh) { return (int64_t)((uint64_t)v << sh); };
  st[0] = (shl(st[0] & 4294967294LL, 12) & 0xFFFFFFFFLL) ^ (((shl(st[0], 13) & 0xFFFFFFFFLL) ^ st[0]) >> 19);
  st[1] = (shl(st[1] & 4294967288LL, 4) & 0xFFFFFFFFLL) ^ (((shl(st[1], 2) & 0xFFFFFFFFLL) ^ st[1]) >> 25);
  st[2] = (shl(st[2] & 4294967280LL, 17) & 0xFFFFFFFFLL) ^ (((shl(st[2], 3) & 0xFFFFFFFFLL) ^ st[2]) >> 11);
  return (int32_t)(uint32_t)(uint64_t)(st[0] ^ st[1] ^ st[2]);
}

__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

// Adds one chunk of up to 32 consecutive entries (lane order = entry order)
// to an ordered table: keys in order of first appearance, each key's sum
// built by adding its values in entry order, the first value stored as is.
// Returns false, with the table as before the chunk, when the chunk's new
// keys do not fit in `cap` slots.
// With `dix` (overflow rows), the slot of key k is dix[k + dix_off] (-1 when
// absent) instead of a search of the table; the caller clears the entries it
// set once the row is done.
template <class Acc>
__device__ bool table_chunk(int32_t key, Acc val, bool valid, int32_t* tkey, Acc* tsum, int cap, int& cnt,
                            int32_t* dix = nullptr, int32_t dix_off = 0) {
  const int lane = threadIdx.x & 31;
  const int32_t k = valid ? key : kNoKey;
  const unsigned peers = __match_any_sync(kFull, k);
  const bool leader = valid && (__ffs(peers) - 1 == lane);
  int slot = -1;
  if (leader) {
    if (dix) {
      slot = dix[k + dix_off];
    } else {
      for (int t = 0; t < cnt; t++)
        if (tkey[t] == k) {
          slot = t;
          break;
        }
    }
  }
  const unsigned newm = __ballot_sync(kFull, leader && slot < 0);
  if (cnt + __popc(newm) > cap) return false;
  const bool fresh = leader && slot < 0;
  if (fresh) slot = cnt + __popc(newm & ((1u << lane) - 1u));
  const int gmax = __reduce_max_sync(kFull, leader ? __popc(peers) : 0);
  Acc acc = (leader && !fresh) ? tsum[slot] : Acc(0);
  unsigned rem = leader ? peers : 0u;
  for (int it = 0; it < gmax; it++) {
    const int src = rem ? __ffs(rem) - 1 : lane;
    const Acc v = __shfl_sync(kFull, val, src);
    if (rem) {
      acc = (fresh && it == 0) ? v : add_rn(acc, v);
      rem &= rem - 1u;
    }
  }
  if (leader) {
    if (fresh) {
      tkey[slot] = k;
      if (dix) dix[k + dix_off] = slot;
    }
    tsum[slot] = acc;
  }
  cnt += __popc(newm);
  __syncwarp();
  return true;
}

__device__ __forceinline__ void table_clear(const int32_t* tkey, int cnt, int32_t* dix, int32_t dix_off) {
  for (int t = threadIdx.x & 31; t < cnt; t += 32) dix[tkey[t] + dix_off] = -1;
  __syncwarp();
}

// ------------------------------------------------------------------ label propagation

// Votes of row r in first-appearance order; *res = the label of the last vote
// equal to max(1.0, largest vote), skipping label -1; cur when there is none
// (the reference's loop, src/label_prop.rs:71-88, with cur == -1 for every
// row that reaches it).
__device__ bool vote_row(const Csr& g, int64_t r, const int32_t* lab, int32_t* tkey, double* tsum, int cap,
                         int32_t cur, int32_t* res, int32_t* dix = nullptr) {
  const int lane = threadIdx.x & 31;
  const int64_t s = g.indptr[r], e = g.indptr[r + 1];
  int cnt = 0;
  for (int64_t b = s; b < e; b += 32) {
    const int64_t k = b + lane;
    const bool valid = k < e;
    int32_t l = 0;
    double w = 0.0;
    if (valid) {
      l = lab[g.indices[k]];
      w = (double)g.data[k];
    }
    if (!table_chunk<double>(l, w, valid, tkey, tsum, cap, cnt, dix, 1)) return false;
  }
  double m = 1.0;
  for (int t = lane; t < cnt; t += 32)
    if (tkey[t] != -1) m = fmax(m, tsum[t]);
  for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(kFull, m, o));
  int last = -1;
  for (int t = lane; t < cnt; t += 32)
    if (tkey[t] != -1 && tsum[t] == m) last = t;
  last = __reduce_max_sync(kFull, last);
  *res = last >= 0 ? tkey[last] : cur;
  if (dix) table_clear(tkey, cnt, dix, 1);
  return true;
}

__global__ void __launch_bounds__(kRowWarps * 32)
    lp_iteration_kernel(Csr g, const int32_t* lab_in, int32_t* lab_out, int32_t* overflow, int32_t* n_overflow) {
  __shared__ int32_t skey[kRowWarps][kVoteSlots];
  __shared__ double ssum[kRowWarps][kVoteSlots];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * kRowWarps;
  for (int64_t r = (int64_t)blockIdx.x * kRowWarps + warp; r < g.n; r += nw) {
    const int32_t cur = lab_in[r];
    int32_t res = cur;
    if (cur < 0 && !vote_row(g, r, lab_in, skey[warp], ssum[warp], kVoteSlots, cur, &res)) {
      if (lane == 0) overflow[atomicAdd(n_overflow, 1)] = (int32_t)r;
      continue;
    }
    if (lane == 0) lab_out[r] = res;
  }
}

__global__ void __launch_bounds__(kRowWarps * 32)
    lp_overflow_kernel(Csr g, const int32_t* lab_in, int32_t* lab_out, const int32_t* overflow,
                       const int32_t* n_overflow, int32_t* skey, double* ssum, int64_t cap, int32_t* dix,
                       int64_t key_bound) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t gw = (int64_t)blockIdx.x * kRowWarps + warp, nw = (int64_t)gridDim.x * kRowWarps;
  const int32_t cnt = *n_overflow;
  for (int64_t i = gw; i < cnt; i += nw) {
    const int64_t r = overflow[i];
    int32_t res = lab_in[r];
    vote_row(g, r, lab_in, skey + gw * cap, ssum + gw * cap, (int)cap, res, &res,
             dix ? dix + gw * key_bound : nullptr);
    if (lane == 0) lab_out[r] = res;
  }
}

__global__ void max_degree_kernel(const int64_t* indptr, int64_t n, int64_t* out) {
  int64_t m = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    m = max(m, indptr[i + 1] - indptr[i]);
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(kFull, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax((unsigned long long*)out, (unsigned long long)m);
}

// Caller graphs: indptr[0] == 0, non-decreasing, indptr[n] == nnz, columns in [0, n).
__global__ void validate_csr_kernel(Csr g, int32_t* bad) {
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, step = (int64_t)gridDim.x * blockDim.x;
  if (i0 == 0 && (g.indptr[0] != 0 || g.indptr[g.n] != g.nnz)) atomicExch(bad, 1);
  for (int64_t i = i0; i < g.n; i += step)
    if (g.indptr[i + 1] < g.indptr[i]) atomicExch(bad, 1);
  for (int64_t e = i0; e < g.nnz; e += step)
    if (g.indices[e] < 0 || g.indices[e] >= g.n) atomicExch(bad, 1);
}

__global__ void seed_labels_kernel(int32_t* labels, const int64_t* idx, int64_t count) {
  for (int64_t i = 0; i < count; i++) labels[idx[i]] = (int32_t)i;
}

// Unlabelled-row flags and the largest label, before the outlier walk.
__global__ void outlier_flags_kernel(const int32_t* labels, int64_t n, int32_t* flag, int32_t* max_label) {
  int32_t m = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t l = labels[i];
    flag[i] = l < 0;
    m = max(m, l);
  }
  m = __reduce_max_sync(kFull, m);
  if ((threadIdx.x & 31) == 0) atomicMax(max_label, m);
}

// label_outliers, all unlabelled rows at once.  In the reference's row-order
// pass, row j reads as labelled at row i's turn exactly when it was labelled
// before the pass or is an unlabelled row before i (those are all assigned by
// then), so every walk's path is fixed in advance: each row's walk runs on
// its own warp against the labels from before the pass.  A walk that stops at
// an earlier unlabelled row records that row (its label is copied once
// known); one that runs 64 pops or empties its stack takes the random label
// from its own tau stream.
struct WalkOut {
  int32_t fin;  // label, or -1 when copied from `ptr`
  int32_t ptr;  // earlier unlabelled row whose label is copied, or -1
};

// Returns false (nothing written) when the walk outgrows `cap` stack entries.
__device__ bool outlier_walk(const Csr& g, const int32_t* labels, int64_t i, int32_t ml, int64_t rs0, int64_t rs1,
                             int64_t rs2, int32_t* stack, int64_t cap, WalkOut* out) {
  const int lane = threadIdx.x & 31;
  if (lane == 0) stack[0] = (int32_t)i;
  __syncwarp();
  int64_t top = 1;
  bool unl = true;
  int it = 0;
  int32_t fin = -1, ptr = -1;
  while (unl && it < 64 && top > 0) {
    it++;
    top--;
    const int64_t node = stack[top];
    const int64_t s = g.indptr[node], e = g.indptr[node + 1];
    for (int64_t b = s; b < e; b += 32) {
      const int64_t k = b + lane;
      const bool valid = k < e;
      const int32_t j = valid ? g.indices[k] : 0;
      const int32_t lj = valid ? labels[j] : -1;
      const unsigned hit = __ballot_sync(kFull, valid && (lj >= 0 || (int64_t)j < i));
      const int npush = hit ? __ffs(hit) - 1 : __popc(__ballot_sync(kFull, valid));
      if (top + npush > cap) return false;
      if (lane < npush) stack[top + lane] = j;
      top += npush;
      if (hit) {
        const int f = __ffs(hit) - 1;
        const int32_t jj = __shfl_sync(kFull, j, f), ll = __shfl_sync(kFull, lj, f);
        if (ll >= 0) fin = ll;
        else ptr = jj;
        unl = false;
        break;
      }
    }
    __syncwarp();
  }
  if (it >= 64 || unl) {
    int64_t st[3] = {(int64_t)((uint64_t)rs0 + (uint64_t)i), (int64_t)((uint64_t)rs1 + (uint64_t)i),
                     (int64_t)((uint64_t)rs2 + (uint64_t)i)};
    const int64_t draw = tau_rand_int(st);
    const int64_t mod = (int64_t)ml + 1;
    const int64_t v = draw % mod;
    fin = (int32_t)(v < 0 ? v + mod : v);
    ptr = -1;
  }
  if (lane == 0) *out = WalkOut{fin, ptr};
  __syncwarp();
  return true;
}

__global__ void __launch_bounds__(kRowWarps * 32)
    outlier_walk_kernel(Csr g, const int32_t* labels, const int64_t* rs, const int32_t* rows, const int32_t* count,
                        const int32_t* max_label, int32_t* stacks, int64_t scap, WalkOut* out, int32_t* big,
                        int32_t* n_big) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t gw = (int64_t)blockIdx.x * kRowWarps + warp, nw = (int64_t)gridDim.x * kRowWarps;
  const int32_t cnt = *count, ml = *max_label;
  for (int64_t oi = gw; oi < cnt; oi += nw)
    if (!outlier_walk(g, labels, rows[oi], ml, rs[0], rs[1], rs[2], stacks + gw * scap, scap, out + oi) && lane == 0)
      big[atomicAdd(n_big, 1)] = (int32_t)oi;
}

// The walks that outgrew the per-warp stacks, one warp with the full stack.
__global__ void outlier_walk_big_kernel(Csr g, const int32_t* labels, const int64_t* rs, const int32_t* rows,
                                        const int32_t* max_label, const int32_t* big, const int32_t* n_big,
                                        int32_t* stack, int64_t cap, WalkOut* out, int32_t* status) {
  const int32_t nb = *n_big, ml = *max_label;
  for (int32_t b = 0; b < nb; b++) {
    const int32_t oi = big[b];
    if (!outlier_walk(g, labels, rows[oi], ml, rs[0], rs[1], rs[2], stack, cap, out + oi)) {
      if ((threadIdx.x & 31) == 0) atomicExch(status, 1);
      return;
    }
  }
}

// Copied labels by pointer jumping over the unlabelled rows (pointers go to
// earlier rows, so the chains end): nxt = -1 marks a row whose label is known.
// First, each unlabelled row's position in the list.
__global__ void outlier_index_kernel(const int32_t* count, const int32_t* rows, int32_t* oidx) {
  const int32_t cnt = *count;
  for (int64_t oi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; oi < cnt; oi += (int64_t)gridDim.x * blockDim.x)
    oidx[rows[oi]] = (int32_t)oi;
}

__global__ void outlier_resolve_start_kernel(const WalkOut* out, const int32_t* count, const int32_t* oidx,
                                             int32_t* lab, int32_t* nxt) {
  const int32_t cnt = *count;
  for (int64_t oi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; oi < cnt;
       oi += (int64_t)gridDim.x * blockDim.x) {
    const WalkOut w = out[oi];
    lab[oi] = w.fin;
    nxt[oi] = w.ptr < 0 ? -1 : oidx[w.ptr];
  }
}

__global__ void outlier_resolve_round_kernel(const int32_t* count, const int32_t* lab_a, const int32_t* nxt_a,
                                             int32_t* lab_b, int32_t* nxt_b, int32_t* pending) {
  const int32_t cnt = *count;
  for (int64_t oi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; oi < cnt;
       oi += (int64_t)gridDim.x * blockDim.x) {
    const int32_t t = nxt_a[oi];
    if (t < 0) {
      lab_b[oi] = lab_a[oi];
      nxt_b[oi] = -1;
    } else if (nxt_a[t] < 0) {
      lab_b[oi] = lab_a[t];
      nxt_b[oi] = -1;
    } else {
      lab_b[oi] = -1;
      nxt_b[oi] = nxt_a[t];
      *pending = 1;
    }
  }
}

__global__ void outlier_scatter_kernel(const int32_t* count, const int32_t* rows, const int32_t* lab, int32_t* labels) {
  const int32_t cnt = *count;
  for (int64_t oi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; oi < cnt; oi += (int64_t)gridDim.x * blockDim.x)
    labels[rows[oi]] = lab[oi];
}

__global__ void remap_flags_kernel(const int32_t* labels, int64_t n, int32_t bound, int32_t* flags,
                                   int32_t* status) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t l = labels[i];
    if (l < 0 || l >= bound) atomicExch(status, 2);
    else flags[l] = 1;
  }
}

__global__ void remap_apply_kernel(int32_t* labels, int64_t n, int32_t bound, const int32_t* flags,
                                   const int32_t* map, int32_t* n_parts) {
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i0 == 0) *n_parts = map[bound - 1] + flags[bound - 1];
  for (int64_t i = i0; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t l = labels[i];
    if (l >= 0 && l < bound) labels[i] = map[l];
  }
}

// ------------------------------------------------------------------ partition maps

__global__ void part_count_kernel(const int32_t* part, int64_t n, int32_t* count, int32_t* iota) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    atomicAdd(&count[part[i]], 1);
    iota[i] = (int32_t)i;
  }
}

__global__ void part_start_kernel(const int32_t* sorted_part, int64_t n, int64_t* start) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (i == 0 || sorted_part[i] != sorted_part[i - 1]) start[sorted_part[i]] = i;
}

// normalize_cols_l2 of the 0/1 reduction map (column sums of 1.0*1.0 = the
// part size) and normalize_rows_l1 of its transpose (|x_p| added c_p times).
__global__ void part_norm_kernel(const int32_t* count, int32_t n_parts, float* xnorm, float* wred) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n_parts; p += gridDim.x * blockDim.x) {
    const int32_t c = count[p];
    float sq = 0.0f;
    for (int32_t t = 0; t < c; t++) sq = __fadd_rn(sq, 1.0f);
    const float norm = fmaxf(__fsqrt_rn(sq), 1e-12f);
    const float x = __fdiv_rn(1.0f, norm);
    float s = 0.0f;
    for (int32_t t = 0; t < c; t++) s = __fadd_rn(s, fabsf(x));
    s = fmaxf(s, 1e-12f);
    xnorm[p] = x;
    wred[p] = __fdiv_rn(x, s);
  }
}

// One warp per (part, 32 columns): each lane sums its column over the part's
// members in order; the members' rows are loaded 32 at a time ahead of the adds.
__global__ void __launch_bounds__(256)
    reduce_data_kernel(const float* x, int64_t d, const int32_t* members, const int64_t* start, const int32_t* count,
                       const float* wred, int32_t n_parts, float* out) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t chunks = (d + 31) / 32;
  const int64_t tasks = (int64_t)n_parts * chunks;
  for (int64_t task = gw; task < tasks; task += nw) {
    const int64_t p = task / chunks, col = (task % chunks) * 32 + lane;
    const bool in = col < d;
    const double w = (double)wred[p];
    const int32_t* mem = members + start[p];
    const int32_t c = count[p];
    float acc = 0.0f;
    for (int32_t t0 = 0; t0 < c; t0 += 32) {
      const int nb = min(32, c - t0);
      const int32_t mine = lane < nb ? mem[t0 + lane] : 0;
      float v[32];
#pragma unroll
      for (int u = 0; u < 32; u++) {
        const int32_t m = __shfl_sync(kFull, mine, u);
        v[u] = (in && u < nb) ? x[(int64_t)m * d + col] : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < 32; u++)
        if (u < nb) acc = __fadd_rn(acc, __double2float_rn(__dmul_rn(w, (double)v[u])));
    }
    if (in) out[p * d + col] = acc;
  }
}

// ------------------------------------------------------------------ SMMP reduction

__device__ __forceinline__ int64_t row_of(const int64_t* indptr, int64_t n, int64_t e) {
  int64_t lo = 0, hi = n;  // largest r with indptr[r] <= e
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (indptr[mid] <= e) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Step 1: key (part of the edge's row, column), value = edge index.
__global__ void edge_keys_kernel(Csr g, const int32_t* part, uint64_t* key, uint32_t* val) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < g.nnz; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = row_of(g.indptr, g.n, e);
    key[e] = ((uint64_t)(uint32_t)part[r] << 32) | (uint32_t)g.indices[e];
    val[e] = (uint32_t)e;
  }
}

// Head flags of runs of equal (key >> shift).
__global__ void head_flags_kernel(const uint64_t* key, int64_t m, int shift, int32_t* flag) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    flag[i] = (i == 0 || (key[i] >> shift) != (key[i - 1] >> shift)) ? 1 : 0;
}

// Step 2: temp entries.  One thread per (p, j) group: the f32 sum of x_p * g_e
// in edge order; nonzero sums become (p, q = part[j], ~first e) keys whose
// value is the sum's bits.
__global__ void temp_groups_kernel(const uint64_t* key, const uint32_t* val, int64_t m, const int32_t* pos,
                                   const int32_t* n_groups, const float* gdata, const float* xnorm,
                                   const int32_t* part, int qshift, uint64_t* okey, uint32_t* oval,
                                   int32_t* counter) {
  const int32_t ng = *n_groups;
  for (int64_t gi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gi < ng; gi += (int64_t)gridDim.x * blockDim.x) {
    const int64_t st = pos[gi], en = gi + 1 < ng ? pos[gi + 1] : m;
    const uint32_t p = (uint32_t)(key[st] >> 32);
    const uint32_t j = (uint32_t)key[st];
    const float x = xnorm[p];
    float acc = 0.0f;
    for (int64_t t = st; t < en; t++) acc = __fadd_rn(acc, __fmul_rn(x, gdata[val[t]]));
    if (acc != 0.0f) {
      const int32_t o = atomicAdd(counter, 1);
      const uint32_t q = (uint32_t)part[j];
      okey[o] = ((uint64_t)p << (32 + qshift)) | ((uint64_t)q << 32) | (uint64_t)(0xffffffffu - val[st]);
      oval[o] = __float_as_uint(acc);
    }
  }
}

// Step 3: reduced entries.  One thread per (p, q) group of sorted temp
// entries: the f32 sum of temp * 1.0 in temp's row order; nonzero sums become
// (p, first e of the group's head) keys with (q, sum) kept aside by index.
__global__ void reduced_groups_kernel(const uint64_t* key, const uint32_t* val, int64_t m, const int32_t* pos,
                                      const int32_t* n_groups, int qshift, uint64_t* okey, uint32_t* oidx,
                                      uint32_t* oq, uint32_t* osum, int32_t* counter) {
  const int32_t ng = *n_groups;
  const uint64_t qmask = (1ull << qshift) - 1ull;
  for (int64_t gi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gi < ng; gi += (int64_t)gridDim.x * blockDim.x) {
    const int64_t st = pos[gi], en = gi + 1 < ng ? pos[gi + 1] : m;
    float acc = 0.0f;
    for (int64_t t = st; t < en; t++) acc = __fadd_rn(acc, __fmul_rn(__uint_as_float(val[t]), 1.0f));
    if (acc != 0.0f) {
      const int32_t o = atomicAdd(counter, 1);
      const uint64_t k = key[st];
      const uint32_t p = (uint32_t)(k >> (32 + qshift));
      const uint32_t q = (uint32_t)((k >> 32) & qmask);
      const uint32_t head_e = 0xffffffffu - (uint32_t)k;
      okey[o] = ((uint64_t)p << 32) | head_e;
      oidx[o] = (uint32_t)o;
      oq[o] = q;
      osum[o] = __float_as_uint(acc);
    }
  }
}

__global__ void row_count_kernel(const uint64_t* key, int64_t m, int shift, int64_t* count) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    atomicAdd((unsigned long long*)&count[key[i] >> shift], 1ull);
}

// Step 4: the reduced CSR, clamped to [0, 1].
__global__ void reduced_write_kernel(const uint32_t* idx, int64_t m, const uint32_t* oq, const uint32_t* osum,
                                     int32_t* r_indices, float* r_data) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t i = idx[t];
    r_indices[t] = (int32_t)oq[i];
    r_data[t] = fminf(fmaxf(__uint_as_float(osum[i]), 0.0f), 1.0f);
  }
}

// Exclusive scan of `count` (m entries) into indptr (m + 1), one block.
__global__ void __launch_bounds__(1024) scan_i64_kernel(const int64_t* count, int64_t m, int64_t* indptr) {
  __shared__ int64_t part[1024];
  const int t = threadIdx.x;
  const int64_t per = (m + 1023) / 1024;
  const int64_t b = t * per, e = min(m, b + per);
  int64_t s = 0;
  for (int64_t i = b; i < e; i++) s += count[i];
  part[t] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const int64_t v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int64_t run = part[t] - s;
  for (int64_t i = b; i < e; i++) {
    indptr[i] = run;
    run += count[i];
  }
  if (t == 1023) indptr[m] = part[1023];
}

// ------------------------------------------------------------------ hadamard_symmetric

__global__ void sorted_flag_kernel(Csr g, int32_t* unsorted) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < g.nnz; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = row_of(g.indptr, g.n, e);
    if (e > g.indptr[r] && g.indices[e] <= g.indices[e - 1]) atomicExch(unsorted, 1);
  }
}

__global__ void row_col_keys_kernel(Csr g, uint64_t* key, uint32_t* val) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < g.nnz; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = row_of(g.indptr, g.n, e);
    key[e] = ((uint64_t)r << 32) | (uint32_t)g.indices[e];
    val[e] = __float_as_uint(g.data[e]);
  }
}

// Entry (r, c, v) of the row-sorted graph keeps v * G[c, r] when G[c, r] != 0.
__global__ void sym_keep_kernel(const int64_t* indptr, int64_t n, int64_t nnz, const uint64_t* key,
                                const uint32_t* val, int32_t* keep, uint32_t* prod, int64_t* rcount) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t r = (uint32_t)(key[e] >> 32), c = (uint32_t)key[e];
    int64_t lo = indptr[c], hi = indptr[c + 1];
    const uint64_t want = ((uint64_t)c << 32) | r;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (key[mid] < want) lo = mid + 1;
      else hi = mid;
    }
    const float other = (lo < indptr[c + 1] && key[lo] == want) ? __uint_as_float(val[lo]) : 0.0f;
    const int k = other != 0.0f;
    keep[e] = k;
    prod[e] = __float_as_uint(__fmul_rn(__uint_as_float(val[e]), other));
    if (k) atomicAdd((unsigned long long*)&rcount[r], 1ull);
  }
}

__global__ void sym_write_kernel(const uint64_t* key, const uint32_t* prod, const int32_t* keep,
                                 const int32_t* dst, int64_t nnz, int32_t* s_indices, float* s_data) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x)
    if (keep[e]) {
      s_indices[dst[e]] = (int32_t)(uint32_t)key[e];
      s_data[dst[e]] = __uint_as_float(prod[e]);
    }
}

// ------------------------------------------------------------------ expander

// Row r of data_expander = SMMP(sym, N): part sums in first-appearance order,
// stored (and summed for the L1 norm, and multiplied into the layout) in
// reverse order; then the average with the row's own part layout.
__device__ bool expand_row(const Csr& sym, int64_t r, const int32_t* part, const float* xnorm, const float* layout,
                           int ncomp, int32_t* tkey, float* tsum, int cap, float* result, int32_t* dix = nullptr) {
  const int lane = threadIdx.x & 31;
  const int64_t s = sym.indptr[r], e = sym.indptr[r + 1];
  int cnt = 0;
  for (int64_t b = s; b < e; b += 32) {
    const int64_t k = b + lane;
    const bool valid = k < e;
    int32_t q = 0;
    float v = 0.0f;
    if (valid) {
      q = part[sym.indices[k]];
      v = __fmul_rn(sym.data[k], xnorm[q]);
    }
    if (!table_chunk<float>(q, v, valid, tkey, tsum, cap, cnt, dix, 0)) return false;
  }
  float rs = 0.0f;
  for (int t = cnt - 1; t >= 0; t--) {
    const float v = tsum[t];
    if (v != 0.0f) rs = __fadd_rn(rs, fabsf(v));
  }
  rs = fmaxf(rs, 1e-12f);
  if (lane < ncomp) {
    float a = 0.0f;
    for (int t = cnt - 1; t >= 0; t--) {
      const float v = tsum[t];
      if (v == 0.0f) continue;
      const double vn = (double)__fdiv_rn(v, rs);
      a = __fadd_rn(a, __double2float_rn(__dmul_rn(vn, (double)layout[(int64_t)tkey[t] * ncomp + lane])));
    }
    const float bb = __fadd_rn(0.0f, layout[(int64_t)part[r] * ncomp + lane]);
    result[r * ncomp + lane] = __double2float_rn(__dmul_rn(__dadd_rn((double)a, (double)bb), 0.5));
  }
  __syncwarp();
  if (dix) table_clear(tkey, cnt, dix, 0);
  return true;
}

__global__ void __launch_bounds__(kRowWarps * 32)
    expand_kernel(Csr sym, const int32_t* part, const float* xnorm, const float* layout, int ncomp, float* result,
                  int32_t* overflow, int32_t* n_overflow) {
  __shared__ int32_t skey[kRowWarps][kVoteSlots];
  __shared__ float ssum[kRowWarps][kVoteSlots];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * kRowWarps;
  for (int64_t r = (int64_t)blockIdx.x * kRowWarps + warp; r < sym.n; r += nw)
    if (!expand_row(sym, r, part, xnorm, layout, ncomp, skey[warp], ssum[warp], kVoteSlots, result) && lane == 0)
      overflow[atomicAdd(n_overflow, 1)] = (int32_t)r;
}

__global__ void __launch_bounds__(kRowWarps * 32)
    expand_overflow_kernel(Csr sym, const int32_t* part, const float* xnorm, const float* layout, int ncomp,
                           float* result, const int32_t* overflow, const int32_t* n_overflow, int32_t* skey,
                           float* ssum, int64_t cap, int32_t* dix, int64_t key_bound) {
  const int warp = threadIdx.x >> 5;
  const int64_t gw = (int64_t)blockIdx.x * kRowWarps + warp, nw = (int64_t)gridDim.x * kRowWarps;
  const int32_t cnt = *n_overflow;
  for (int64_t i = gw; i < cnt; i += nw)
    expand_row(sym, overflow[i], part, xnorm, layout, ncomp, skey + gw * cap, ssum + gw * cap, (int)cap, result,
               dix ? dix + gw * key_bound : nullptr);
}

// Column means summed in row order (f64).  The block streams tiles of rows
// into shared memory (double-buffered) while lane c of warp 0 adds column c
// of the previous tile in row order.
constexpr int kCenterTile = 6144;  // floats per tile buffer

__global__ void __launch_bounds__(1024) center_mean_kernel(const float* result, int64_t n, int ncomp, double* mean) {
  __shared__ float tile[2][kCenterTile];
  const int rows_per = kCenterTile / ncomp;
  const int64_t tiles = (n + rows_per - 1) / rows_per;
  auto load = [&](int64_t t) {
    const int64_t r0 = t * rows_per;
    const int64_t cnt = min((int64_t)rows_per, n - r0) * ncomp;
    for (int64_t i = threadIdx.x; i < cnt; i += blockDim.x) tile[t & 1][i] = result[r0 * ncomp + i];
  };
  double acc = 0.0;
  if (tiles > 0) load(0);
  __syncthreads();
  for (int64_t t = 0; t < tiles; t++) {
    if (threadIdx.x < 32) {
      if (threadIdx.x < ncomp) {
        const int rows = (int)min((int64_t)rows_per, n - t * rows_per);
        const float* src = tile[t & 1] + threadIdx.x;
        int r = 0;
        for (; r + 8 <= rows; r += 8) {
          float v[8];
#pragma unroll
          for (int u = 0; u < 8; u++) v[u] = src[(r + u) * ncomp];
#pragma unroll
          for (int u = 0; u < 8; u++) acc = __dadd_rn(acc, (double)v[u]);
        }
        for (; r < rows; r++) acc = __dadd_rn(acc, (double)src[r * ncomp]);
      }
    } else if (t + 1 < tiles) {
      const int64_t r0 = (t + 1) * rows_per;
      const int64_t cnt = min((int64_t)rows_per, n - r0) * ncomp;
      for (int64_t i = threadIdx.x - 32; i < cnt; i += blockDim.x - 32) tile[(t + 1) & 1][i] = result[r0 * ncomp + i];
    }
    __syncthreads();
  }
  if (threadIdx.x < ncomp) mean[threadIdx.x] = __ddiv_rn(acc, (double)n);
}

__global__ void center_apply_kernel(const float* result, int64_t n, int ncomp, float scaling, const double* mean,
                                    float* out) {
  const int64_t total = n * ncomp;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = __double2float_rn(__dmul_rn((double)scaling, __dsub_rn((double)result[i], mean[i % ncomp])));
}

// ------------------------------------------------------------------ PCA base init

constexpr int kPcaMax = 64;

// Cyclic Jacobi rotations by one warp on the symmetric nn x nn matrix A (row
// stride kPcaMax, f64, in shared memory), accumulating the eigenvectors into
// V (columns; V starts as the identity).  Stops when the off-diagonal mass is
// below 1e-30 of the total, or after 60 sweeps.
__device__ void jacobi_warp(double* A, double* V, int nn, int lane) {
  for (int sweep = 0; sweep < 60; sweep++) {
    double off = 0.0, tot = 0.0;
    for (int i = lane; i < nn * nn; i += 32) {
      const int a = i / nn, b = i % nn;
      const double v = A[a * kPcaMax + b] * A[a * kPcaMax + b];
      tot += v;
      if (a != b) off += v;
    }
    for (int o = 16; o; o >>= 1) {
      off += __shfl_xor_sync(kFull, off, o);
      tot += __shfl_xor_sync(kFull, tot, o);
    }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int p = 0; p < nn - 1; p++)
      for (int q = p + 1; q < nn; q++) {
        const double apq = A[p * kPcaMax + q];
        if (apq == 0.0) continue;
        const double tau = (A[q * kPcaMax + q] - A[p * kPcaMax + p]) / (2.0 * apq);
        const double tt = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        const double c = 1.0 / sqrt(1.0 + tt * tt), s = tt * c;
        for (int k = lane; k < nn; k += 32) {
          const double akp = A[k * kPcaMax + p], akq = A[k * kPcaMax + q];
          A[k * kPcaMax + p] = c * akp - s * akq;
          A[k * kPcaMax + q] = s * akp + c * akq;
          const double vkp = V[k * kPcaMax + p], vkq = V[k * kPcaMax + q];
          V[k * kPcaMax + p] = c * vkp - s * vkq;
          V[k * kPcaMax + q] = s * vkp + c * vkq;
        }
        __syncwarp();
        for (int k = lane; k < nn; k += 32) {
          const double apk = A[p * kPcaMax + k], aqk = A[q * kPcaMax + k];
          A[p * kPcaMax + k] = c * apk - s * aqk;
          A[q * kPcaMax + k] = s * apk + c * aqk;
        }
        __syncwarp();
      }
  }
}

// normalize_small_graph_init_like_python (src/label_prop.rs:251-262), by one
// thread: subtract the f64 mean of all entries (element order), then divide
// by (max - min) / 2 in f32 when positive.
__device__ void small_init_normalise(float* out, int count) {
  double m = 0.0;
  for (int i = 0; i < count; i++) m = __dadd_rn(m, (double)out[i]);
  m = __ddiv_rn(m, (double)count);
  float lo = INFINITY, hi = -INFINITY;
  for (int i = 0; i < count; i++) {
    const float v = __double2float_rn(__dsub_rn((double)out[i], m));
    out[i] = v;
    lo = fminf(lo, v);
    hi = fmaxf(hi, v);
  }
  const float scale = __fdiv_rn(__fsub_rn(hi, lo), 2.0f);
  if (scale > 0.0f)
    for (int i = 0; i < count; i++) out[i] = __fdiv_rn(out[i], scale);
}

// One block.  Centred rows X (f64, f32 column means), Gram G = X X^T, cyclic
// Jacobi (one warp) for G's eigenpairs; component j = sign_j * sqrt(l_j) *
// u_j with the sign that makes the largest-|.| entry of X^T u_j (the last on
// ties) non-negative; then the small-graph normalisation.
__global__ void __launch_bounds__(256) pca_kernel(const float* x, int64_t n, int64_t d, int ncomp, float* out,
                                                  float* mean_ws, double* vws, int32_t* status) {
  extern __shared__ double sh[];
  double* A = sh;                    // n x n
  double* V = sh + kPcaMax * kPcaMax;  // n x n
  __shared__ double s_eval[kPcaMax];
  __shared__ int s_order[kPcaMax];
  __shared__ double s_sign[kPcaMax];
  const int t = threadIdx.x;
  const int nn = (int)n;
  for (int64_t c = t; c < d; c += blockDim.x) {
    float m = 0.0f;
    for (int i = 0; i < nn; i++) m = __fadd_rn(m, x[(int64_t)i * d + c]);
    mean_ws[c] = __fdiv_rn(m, (float)nn);
  }
  __syncthreads();
  for (int pq = t; pq < nn * nn; pq += blockDim.x) {
    const int a = pq / nn, b = pq % nn;
    if (b < a) continue;
    double s = 0.0;
    for (int64_t c = 0; c < d; c++) {
      const double mc = (double)mean_ws[c];
      s += ((double)x[(int64_t)a * d + c] - mc) * ((double)x[(int64_t)b * d + c] - mc);
    }
    A[a * kPcaMax + b] = s;
    A[b * kPcaMax + a] = s;
  }
  for (int i = t; i < kPcaMax * kPcaMax; i += blockDim.x) V[i] = (i / kPcaMax == i % kPcaMax) ? 1.0 : 0.0;
  __syncthreads();
  if (t < 32) {
    const int lane = t;
    jacobi_warp(A, V, nn, lane);
    if (lane == 0) {
      for (int i = 0; i < nn; i++) {
        s_eval[i] = A[i * kPcaMax + i];
        s_order[i] = i;
      }
      for (int i = 0; i < nn; i++)  // descending eigenvalues (stable selection)
        for (int j = i + 1; j < nn; j++)
          if (s_eval[s_order[j]] > s_eval[s_order[i]]) {
            const int tmp = s_order[i];
            s_order[i] = s_order[j];
            s_order[j] = tmp;
          }
    }
  }
  __syncthreads();
  const int kc = min(ncomp, min(nn, d < kPcaMax ? (int)d : kPcaMax));
  // signs from X^T u_j: per component, the block finds the last largest |entry|
  for (int j = 0; j < kc; j++) {
    const int col = s_order[j];
    for (int64_t c = t; c < d; c += blockDim.x) {
      const double mc = (double)mean_ws[c];
      double v = 0.0;
      for (int i = 0; i < nn; i++) v += ((double)x[(int64_t)i * d + c] - mc) * V[i * kPcaMax + col];
      vws[c] = v;
    }
    __syncthreads();
    if (t == 0) {
      double best = -1.0, bv = 0.0;
      for (int64_t c = 0; c < d; c++)
        if (fabs(vws[c]) >= best) {
          best = fabs(vws[c]);
          bv = vws[c];
        }
      s_sign[j] = bv >= 0.0 ? 1.0 : -1.0;
    }
    __syncthreads();
  }
  for (int i = t; i < nn * ncomp; i += blockDim.x) {
    const int r = i / ncomp, j = i % ncomp;
    float v = 0.0f;
    if (j < kc) {
      const int col = s_order[j];
      const double sv = sqrt(fmax(s_eval[col], 0.0));
      v = (float)(s_sign[j] * V[r * kPcaMax + col] * sv);
    }
    out[i] = v;
  }
  __syncthreads();
  if (t == 0) small_init_normalise(out, nn * ncomp);
}

// ------------------------------------------------------------------ spectral / MDS / random base inits

// pairwise_sq_distances (src/label_prop.rs:322-337): f32, coordinates summed
// in order with separate multiply and add; D is nn x nn (row stride kPcaMax).
__device__ void pairwise_sq(const float* x, int nn, int64_t d, float* D) {
  for (int pq = threadIdx.x; pq < nn * nn; pq += blockDim.x) {
    const int a = pq / nn, b = pq % nn;
    if (b < a) continue;
    float sq = 0.0f;
    for (int64_t c = 0; c < d; c++) {
      const float diff = __fsub_rn(x[(int64_t)a * d + c], x[(int64_t)b * d + c]);
      sq = __fadd_rn(sq, __fmul_rn(diff, diff));
    }
    D[a * kPcaMax + b] = sq;
    D[b * kPcaMax + a] = sq;
  }
}

// One block: spectral_init (mode 0, src/label_prop.rs:364-423) or mds_init
// (mode 1, 339-362) of nn <= 64 rows, then the small-graph normalisation.
// The symmetric eigen-decomposition is cyclic Jacobi in f64 on the f32
// matrix (the reference: faer's f32 solver), eigenvalues ascending (stable
// in index order), each eigenvector's largest-|.| entry (the first on ties)
// made non-negative.
__global__ void __launch_bounds__(256) spectral_mds_kernel(const float* x, int64_t n, int64_t d, int ncomp, int mode,
                                                           float* out) {
  extern __shared__ double sh[];
  double* A = sh;                         // nn x nn
  double* V = sh + kPcaMax * kPcaMax;     // nn x nn
  double* T = sh + 2 * kPcaMax * kPcaMax; // nn x nn (MDS: H D)
  float* D = reinterpret_cast<float*>(sh + 3 * kPcaMax * kPcaMax);  // nn x nn
  __shared__ float s_deg[kPcaMax];
  __shared__ double s_eval[kPcaMax];
  __shared__ int s_order[kPcaMax];
  __shared__ float s_sigma;
  const int t = threadIdx.x;
  const int nn = (int)n;
  pairwise_sq(x, nn, d, D);
  for (int i = t; i < kPcaMax * kPcaMax; i += blockDim.x) V[i] = (i / kPcaMax == i % kPcaMax) ? 1.0 : 0.0;
  __syncthreads();
  if (mode == 0) {
    // sigma: sqrt of the element at index len/2 of the sorted positive
    // distances (both triangles), floored at 1e-8; 1 when none is positive.
    int npos = 0;
    for (int i = 0; i < nn * nn; i++) npos += D[(i / nn) * kPcaMax + i % nn] > 0.0f;
    if (t == 0) s_sigma = 1.0f;
    __syncthreads();
    const int r = npos / 2;
    for (int i = t; i < nn * nn; i += blockDim.x) {
      const float v = D[(i / nn) * kPcaMax + i % nn];
      if (!(v > 0.0f)) continue;
      int less = 0, le = 0;
      for (int j = 0; j < nn * nn; j++) {
        const float w = D[(j / nn) * kPcaMax + j % nn];
        if (w > 0.0f) {
          less += w < v;
          le += w <= v;
        }
      }
      if (less <= r && r < le) s_sigma = fmaxf(sqrtf(v), 1e-8f);  // every writer writes the same value
    }
    __syncthreads();
    const float sg = s_sigma;
    const float den = __fmul_rn(__fmul_rn(2.0f, sg), sg);
    // affinities W (i != j, kept above 1e-12) into T as f32 values, degrees by rows in column order
    for (int i = t; i < nn * nn; i += blockDim.x) {
      const int a = i / nn, b = i % nn;
      float w = 0.0f;
      if (a != b) {
        w = expf(__fdiv_rn(-D[a * kPcaMax + b], den));
        if (!(w > 1e-12f)) w = 0.0f;
      }
      T[a * kPcaMax + b] = (double)w;
    }
    __syncthreads();
    for (int a = t; a < nn; a += blockDim.x) {
      float s = 0.0f;
      for (int b = 0; b < nn; b++)
        if (T[a * kPcaMax + b] != 0.0) s = __fadd_rn(s, (float)T[a * kPcaMax + b]);
      s_deg[a] = s;
    }
    __syncthreads();
    for (int i = t; i < nn * nn; i += blockDim.x) {
      const int a = i / nn, b = i % nn;
      float l = (a == b) ? 1.0f : 0.0f;
      const float w = (float)T[a * kPcaMax + b];
      if (w != 0.0f) {
        const float dn = fmaxf(sqrtf(__fmul_rn(s_deg[a], s_deg[b])), 1e-12f);
        l = __fsub_rn(l, __fdiv_rn(w, dn));
      }
      A[a * kPcaMax + b] = (double)l;
    }
  } else {
    // B = -0.5 * (H D) H with H = I - 1/n, in f64, then rounded to f32
    const double inv = 1.0 / (double)nn;
    for (int i = t; i < nn * nn; i += blockDim.x) {
      const int a = i / nn, b = i % nn;
      double s = 0.0;
      for (int c = 0; c < nn; c++) s += ((a == c ? 1.0 : 0.0) - inv) * (double)D[c * kPcaMax + b];
      T[a * kPcaMax + b] = s;
    }
    __syncthreads();
    for (int i = t; i < nn * nn; i += blockDim.x) {
      const int a = i / nn, b = i % nn;
      double s = 0.0;
      for (int c = 0; c < nn; c++) s += T[a * kPcaMax + c] * ((c == b ? 1.0 : 0.0) - inv);
      A[a * kPcaMax + b] = (double)(float)(-0.5 * s);
    }
  }
  __syncthreads();
  if (t < 32) {
    jacobi_warp(A, V, nn, t);
    if (t == 0) {
      for (int i = 0; i < nn; i++) {  // ascending eigenvalues, equal ones in index order (insertion sort)
        s_eval[i] = A[i * kPcaMax + i];
        int p = i;
        while (p > 0 && s_eval[s_order[p - 1]] > s_eval[i]) {
          s_order[p] = s_order[p - 1];
          p--;
        }
        s_order[p] = i;
      }
    }
  }
  __syncthreads();
  // spectral: eigenvectors 1 .. ncomp of the ascending order; MDS: 0 .. ncomp-1 scaled by sqrt(max(l, 0))
  const int first = mode == 0 ? 1 : 0;
  const int kc = max(0, min(ncomp, nn - first));
  for (int i = t; i < nn * ncomp; i += blockDim.x) {
    const int r = i / ncomp, j = i % ncomp;
    float v = 0.0f;
    if (j < kc) {
      const int col = s_order[j + first];
      int best = 0;
      for (int q = 1; q < nn; q++)
        if (fabs(V[q * kPcaMax + col]) > fabs(V[best * kPcaMax + col])) best = q;
      const float sign = V[best * kPcaMax + col] < 0.0 ? -1.0f : 1.0f;
      const float u = __fmul_rn(sign, (float)V[r * kPcaMax + col]);
      v = mode == 0 ? u : __fmul_rn(u, sqrtf(fmaxf((float)s_eval[col], 0.0f)));
    }
    out[i] = v;
  }
  __syncthreads();
  if (t == 0) small_init_normalise(out, nn * ncomp);
}

// random_unit_init's rows (src/label_prop.rs:311-320): each row of the drawn
// normals divided by sqrt of its f32 dot with itself (ndarray's unrolled dot:
// eight partial sums over whole blocks of eight, paired 0+4, 1+5, 2+6, 3+7,
// then the tail in order), when positive.
__global__ void unit_rows_kernel(float* r, int64_t n, int ncomp) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float* row = r + i * ncomp;
    float p[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int c = 0;
    for (; c + 8 <= ncomp; c += 8)
      for (int j = 0; j < 8; j++) p[j] = __fadd_rn(p[j], __fmul_rn(row[c + j], row[c + j]));
    float s = 0.0f;
    s = __fadd_rn(s, __fadd_rn(p[0], p[4]));
    s = __fadd_rn(s, __fadd_rn(p[1], p[5]));
    s = __fadd_rn(s, __fadd_rn(p[2], p[6]));
    s = __fadd_rn(s, __fadd_rn(p[3], p[7]));
    for (; c < ncomp; c++) s = __fadd_rn(s, __fmul_rn(row[c], row[c]));
    const float norm = sqrtf(s);
    if (norm > 0.0f)
      for (int j = 0; j < ncomp; j++) row[j] = __fdiv_rn(row[j], norm);
  }
}

// The jitter and node-embedding upscalers (src/label_prop.rs:606-656):
// j = f32(layout[part[r], c] (0 for part < 0) + noise[r, c]); the jitter
// expander writes f32((f64(result) + f64(j)) * 0.5), the node-embedding
// upscaler writes j.
__global__ void upscale_kernel(float* result, const int32_t* part, const float* layout, const float* noise,
                               int64_t n, int ncomp, int jitter) {
  const int64_t total = n * ncomp;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / ncomp;
    const int c = (int)(i % ncomp);
    const int32_t p = part[r];
    const float base = p >= 0 ? layout[(int64_t)p * ncomp + c] : 0.0f;
    const float j = __fadd_rn(base, noise[i]);
    result[i] = jitter ? __double2float_rn(__dmul_rn(__dadd_rn((double)result[i], (double)j), 0.5)) : j;
  }
}

// ------------------------------------------------------------------ node embedding

// Largest positive weight (as int bits: positive floats order like their bits).
__global__ void ne_maxw_kernel(const float* w, int64_t m, float* max_w) {
  int best = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    if (w[i] > 0.0f) best = max(best, __float_as_int(w[i]));
  best = __reduce_max_sync(kFull, best);
  if ((threadIdx.x & 31) == 0 && best > 0) atomicMax((int*)max_w, best);
}

__global__ void ne_schedule_kernel(const float* w, int64_t m, float nf, float nsr, float neg_scale,
                                   const float* max_w, float* eps, float* epns, float* eonn, float* eons) {
  const float mx = *max_w;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    float e;
    if (mx == 0.0f) {
      e = nf;
    } else {
      float ns = __fmul_rn(nf, __fdiv_rn(w[i], mx));
      if (!(ns >= 1.0f)) ns = 1.0f;
      e = __fdiv_rn(nf, ns);
    }
    float en = __fdiv_rn(e, nsr);
    en = __fmul_rn(en, neg_scale);
    eps[i] = e;
    eons[i] = e;
    epns[i] = en;
    eonn[i] = en;
  }
}

__device__ __forceinline__ uint64_t neg_count(float nf, float eon, float rate) {
  const float v = __fdiv_rn(__fsub_rn(nf, eon), rate);
  if (v <= 0.0f) return 0;
  if (v != v) return 0;
  if (v >= 2147483648.0f) return 2147483647ull;
  return (uint64_t)(int32_t)v;
}

__device__ __forceinline__ float clip4(float v) { return v > 4.0f ? 4.0f : (v < -4.0f ? -4.0f : v); }

// Rows of more than min_deg edges, deferred by ne_block_kernel to ne_heavy_kernel.
struct HeavyRows {
  int64_t min_deg;
  uint32_t* rows;
  int32_t* count;
};

// The positive move of one edge (scaled by alpha); false when the squared
// distance is 0 (the reference adds nothing then).
template <int MAXD>
__device__ __forceinline__ bool ne_pos(const float* cur, const float* yt, int ncomp, float noise, float alpha,
                                       float* out) {
  float ds = 0.0f;
#pragma unroll
  for (int d = 0; d < MAXD; d++)
    if (d < ncomp) {
      const float df = __fsub_rn(cur[d], yt[d]);
      ds = __fadd_rn(ds, __fmul_rn(df, df));
    }
  if (!(ds > 0.0f)) return false;
  const float dist = __fsqrt_rn(ds);
  const float num = __fsub_rn(__fmul_rn(__fmul_rn(-2.0f, noise), dist), 2.0f);
  const float den = __fadd_rn(__fsub_rn(__fmul_rn(2.0f, ds), __fmul_rn(0.5f, dist)), 1.0f);
  const float gc = __fdiv_rn(num, den);
#pragma unroll
  for (int d = 0; d < MAXD; d++)
    if (d < ncomp) out[d] = __fmul_rn(__fmul_rn(gc, __fsub_rn(cur[d], yt[d])), alpha);
  return true;
}

// Negative sample p of edge `raw` (scaled and clipped); false when it adds nothing.
template <int MAXD>
__device__ __forceinline__ bool ne_neg(const float* cur, const float* emb, const uint32_t* order, uint64_t nv,
                                       uint64_t raw, uint64_t p, uint32_t epoch, uint32_t rng_state, int ncomp,
                                       float gamma, float alpha, float* out) {
  const uint64_t idx = (raw * ((uint64_t)epoch + p + 1ull) * (uint64_t)rng_state) % nv;
  const uint64_t tn = order[idx];
  if (tn >= nv) return false;
  const float* yn = emb + tn * ncomp;
  float dn = 0.0f;
#pragma unroll
  for (int d = 0; d < MAXD; d++)
    if (d < ncomp) {
      const float df = __fsub_rn(cur[d], yn[d]);
      dn = __fadd_rn(dn, __fmul_rn(df, df));
    }
  if (!(dn > 1e-2f)) return false;
  const float gc = __fdiv_rn(__fmul_rn(gamma, 4.0f), __fmul_rn(__fadd_rn(1.0f, __fmul_rn(0.25f, dn)), dn));
  if (!(gc > 0.0f)) return false;
#pragma unroll
  for (int d = 0; d < MAXD; d++)
    if (d < ncomp) out[d] = __fmul_rn(clip4(__fmul_rn(gc, __fsub_rn(cur[d], yn[d]))), alpha);
  return true;
}

constexpr int kHeavyWarps = 16;
constexpr int kHeavySlots = 4;  // positive move + 3 negative samples staged per edge
constexpr uint32_t kHeavyOverflow = 0x80000000u;

__host__ __device__ inline int heavy_tile_edges(int ncomp) { return ncomp <= 8 ? 512 : (ncomp <= 16 ? 256 : 128); }
__host__ __device__ inline size_t heavy_smem_bytes(int ncomp) {
  return size_t(2) * heavy_tile_edges(ncomp) * (size_t(kHeavySlots) * ncomp + 2) * sizeof(float) +
         size_t(heavy_tile_edges(ncomp)) * kHeavySlots * sizeof(uint32_t);
}

// One CTA per deferred row.  Warps 1..15 compute the contributions of a tile
// of the row's edges into shared memory while warp 0 adds the previous
// tile's, in edge order, lane d keeping component d of the update row (the
// reference's order of f32 additions for that component).  An edge wanting
// more negative samples than the staging holds is flagged and its samples
// are computed by warp 0 in order.
template <int MAXD, int MINB>
__global__ void __launch_bounds__(kHeavyWarps * 32, MINB)
    ne_heavy_kernel(Csr g, float* emb, float* upd, const uint32_t* order, const float* eps, const float* epns,
                    float* eonn, float* eons, uint32_t rng_state, int ncomp, float alpha, uint32_t epoch,
                    float noise, float gamma, float decay, int apply_decay, HeavyRows heavy) {
  extern __shared__ float hv_sh[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int te = heavy_tile_edges(ncomp);
  const int stride = kHeavySlots * ncomp + 2;  // floats per staged edge: slots, mask, count
  const uint64_t nv = (uint64_t)g.n;
  const float nf = (float)epoch;
  const int32_t cnt = *heavy.count;
  for (int32_t h = blockIdx.x; h < cnt; h += gridDim.x) {
    const uint64_t from = heavy.rows[h];
    float cur[MAXD];
#pragma unroll
    for (int d = 0; d < MAXD; d++)
      if (d < ncomp) cur[d] = emb[from * ncomp + d];
    const uint64_t e0 = (uint64_t)g.indptr[from], e1 = (uint64_t)g.indptr[from + 1];
    const int64_t tiles = (int64_t)((e1 - e0 + te - 1) / te);
    float ud = 0.0f;
    if (warp == 0 && lane < ncomp)
      ud = apply_decay ? __fmul_rn(upd[from * ncomp + lane], decay) : upd[from * ncomp + lane];
    auto stage = [&](int64_t tile, int first_thread, int threads) {
      float* buf = hv_sh + (size_t)(tile & 1) * te * stride;
      for (int i = (int)threadIdx.x - first_thread; i < te; i += threads) {
        const uint64_t raw = e0 + (uint64_t)tile * te + i;
        float* ent = buf + (size_t)i * stride;
        uint32_t m = 0, nn = 0;
        if (raw < e1 && !(eons[raw] > nf)) {
          const uint64_t to = (uint64_t)(uint32_t)g.indices[raw];
          if (to < nv) {
            if (ne_pos<MAXD>(cur, emb + to * ncomp, ncomp, noise, alpha, ent)) m |= 1u;
            eons[raw] = __fadd_rn(eons[raw], eps[raw]);
            const float rate = epns[raw];
            const uint64_t nneg = neg_count(nf, eonn[raw], rate);
            nn = (uint32_t)nneg;
            if (nneg < (uint64_t)kHeavySlots) {
              for (uint64_t p = 0; p < nneg; p++)
                if (ne_neg<MAXD>(cur, emb, order, nv, raw, p, epoch, rng_state, ncomp, gamma, alpha,
                                 ent + (1 + p) * ncomp))
                  m |= 2u << p;
            } else {
              m |= kHeavyOverflow;
            }
            eonn[raw] = __fadd_rn(eonn[raw], __fmul_rn(__ull2float_rn(nneg), rate));
          }
        }
        reinterpret_cast<uint32_t*>(ent)[kHeavySlots * ncomp] = m;
        reinterpret_cast<uint32_t*>(ent)[kHeavySlots * ncomp + 1] = nn;
      }
    };
    stage(0, 0, blockDim.x);
    __syncthreads();
    uint32_t* offs = reinterpret_cast<uint32_t*>(hv_sh + (size_t)2 * te * stride);  // te * kHeavySlots
    for (int64_t t = 0; t < tiles; t++) {
      if (warp == 0) {
        const float* buf = hv_sh + (size_t)(t & 1) * te * stride;
        const int64_t left = (int64_t)(e1 - e0) - t * te;
        const int n_in = (int)(left < te ? left : te);
        // offsets (in floats) of the applied contributions, in edge order and slot order; an edge
        // whose negative samples were not staged is listed as 0x80000000 | edge
        const int per = (n_in + 31) / 32;
        const int i0 = lane * per, i1 = min(n_in, i0 + per);
        int mine = 0;
        for (int i = i0; i < i1; i++) {
          const uint32_t m = reinterpret_cast<const uint32_t*>(buf + (size_t)i * stride)[kHeavySlots * ncomp];
          mine += (m & kHeavyOverflow) ? (int)(m & 1u) + 1 : __popc(m);
        }
        int at = mine;
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(kFull, at, o);
          if (lane >= o) at += v;
        }
        const int total = __shfl_sync(kFull, at, 31);
        at -= mine;
        for (int i = i0; i < i1; i++) {
          const uint32_t m = reinterpret_cast<const uint32_t*>(buf + (size_t)i * stride)[kHeavySlots * ncomp];
          for (uint32_t bits = m & ~kHeavyOverflow; bits; bits &= bits - 1u)
            offs[at++] = (uint32_t)(i * stride + (__ffs(bits) - 1) * ncomp);
          if (m & kHeavyOverflow) offs[at++] = kHeavyOverflow | (uint32_t)i;
        }
        __syncwarp();
        int q = 0;
        for (; q + 4 <= total; q += 4) {
          uint32_t o4[4];
          float v4[4];
#pragma unroll
          for (int j = 0; j < 4; j++) o4[j] = offs[q + j];
          if ((o4[0] | o4[1] | o4[2] | o4[3]) & kHeavyOverflow) break;
#pragma unroll
          for (int j = 0; j < 4; j++) v4[j] = lane < ncomp ? buf[o4[j] + lane] : 0.0f;
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (lane < ncomp) ud = __fadd_rn(ud, v4[j]);
        }
        for (; q < total; q++) {
          const uint32_t o = offs[q];
          if (o & kHeavyOverflow) {
            const int i = (int)(o & ~kHeavyOverflow);
            const uint32_t nn = reinterpret_cast<const uint32_t*>(buf + (size_t)i * stride)[kHeavySlots * ncomp + 1];
            const uint64_t raw = e0 + (uint64_t)t * te + i;
            float c[MAXD];
            for (uint64_t p = 0; p < nn; p++)
              if (ne_neg<MAXD>(cur, emb, order, nv, raw, p, epoch, rng_state, ncomp, gamma, alpha, c)) {
#pragma unroll
                for (int d = 0; d < MAXD; d++)
                  if (d == lane && d < ncomp) ud = __fadd_rn(ud, c[d]);
              }
          } else if (lane < ncomp) {
            ud = __fadd_rn(ud, buf[o + lane]);
          }
        }
      } else if (t + 1 < tiles) {
        stage(t + 1, 32, blockDim.x - 32);
      }
      __syncthreads();
    }
    if (warp == 0 && lane < ncomp) upd[from * ncomp + lane] = ud;
    __syncthreads();
  }
}

constexpr int kNeWarps = 4;    // warps (nodes in flight) per CTA
constexpr int kNegSlots = 3;   // negative samples per edge staged at once

// Per-warp staging: [32 lanes][1 + kNegSlots][ncomp] contributions, then 32
// flags (and 32 spare words).
__host__ __device__ inline int ne_stage_floats(int ncomp) { return 32 * (1 + kNegSlots) * ncomp + 64; }

// One warp per node of the block.  The lanes take 32 consecutive edges and
// compute their contributions (positive move, then each negative sample)
// from the embedding as it stood at the block's start; then every lane adds
// them, in edge order and within an edge in sample order, to its own copy of
// the node's update row -- the reference's serial order of f32 additions.
// Edges wanting more than kNegSlots negative samples in a chunk are handed
// through the staging one contribution at a time instead.
template <int MAXD, int MINB>
__global__ void __launch_bounds__(kNeWarps * 32, MINB)
    ne_block_kernel(Csr g, float* emb, float* upd, const uint32_t* order, int64_t bs, int64_t be, const float* eps,
                    const float* epns, float* eonn, float* eons, uint32_t rng_state, int ncomp, float alpha,
                    uint32_t epoch, float noise, float gamma, float decay, int apply_decay, HeavyRows heavy) {
  extern __shared__ float ne_sh[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int kSlots = 1 + kNegSlots;
  float* vec = ne_sh + (size_t)warp * ne_stage_floats(ncomp);
  uint32_t* fmask = reinterpret_cast<uint32_t*>(vec + 32 * kSlots * ncomp);
  const uint64_t nv = (uint64_t)g.n;
  const float nf = (float)epoch;
  const int64_t step = (int64_t)gridDim.x * kNeWarps;
  int64_t ni = bs + (int64_t)blockIdx.x * kNeWarps + warp;
  // the next node's id and row bounds are loaded while the current one runs
  uint64_t nfrom = ni < be ? order[ni] : nv;
  uint64_t ne0 = 0, ne1 = 0;
  if (nfrom < nv) {
    ne0 = (uint64_t)g.indptr[nfrom];
    ne1 = (uint64_t)g.indptr[nfrom + 1];
  }
  for (; ni < be; ni += step) {
    const uint64_t from = nfrom, e0 = ne0, e1 = ne1;
    nfrom = ni + step < be ? order[ni + step] : nv;
    if (nfrom < nv) {
      ne0 = (uint64_t)g.indptr[nfrom];
      ne1 = (uint64_t)g.indptr[nfrom + 1];
    }
    if (from >= nv) continue;
    if ((int64_t)(e1 - e0) > heavy.min_deg) {  // deferred to ne_heavy_kernel
      if (lane == 0) heavy.rows[atomicAdd(heavy.count, 1)] = (uint32_t)from;
      continue;
    }
    float cur[MAXD], u[MAXD];
#pragma unroll
    for (int d = 0; d < MAXD; d++)
      if (d < ncomp) {
        cur[d] = emb[from * ncomp + d];
        u[d] = apply_decay ? __fmul_rn(upd[from * ncomp + d], decay) : upd[from * ncomp + d];
      }
    for (uint64_t base = e0; base < e1; base += 32) {
      const uint64_t raw = base + lane;
      bool act = false;
      uint64_t to = 0;
      if (raw < e1 && !(eons[raw] > nf)) {
        to = (uint64_t)(uint32_t)g.indices[raw];
        act = to < nv;
      }
      if (!__any_sync(kFull, act)) continue;
      uint32_t fl = 0;
      uint64_t nneg = 0;
      float rate = 0.0f;
      float cp[MAXD];
      if (act) {
        if (ne_pos<MAXD>(cur, emb + to * ncomp, ncomp, noise, alpha, cp)) fl = 1u;
        eons[raw] = __fadd_rn(eons[raw], eps[raw]);
        rate = epns[raw];
        nneg = neg_count(nf, eonn[raw], rate);
      }
      auto add_slot = [&](int L, int slot) {
        const float* src = vec + ((size_t)L * kSlots + slot) * ncomp;
#pragma unroll
        for (int d = 0; d < MAXD; d++)
          if (d < ncomp) u[d] = __fadd_rn(u[d], src[d]);
      };
      const int maxneg = (int)__reduce_max_sync(kFull, (unsigned)(nneg < (1ull << 30) ? nneg : (1ull << 30)));
      if (maxneg <= kNegSlots) {
        if (fl) {
          float* dst = vec + (size_t)lane * kSlots * ncomp;
#pragma unroll
          for (int d = 0; d < MAXD; d++)
            if (d < ncomp) dst[d] = cp[d];
        }
        for (int p = 0; p < maxneg; p++)
          if ((uint64_t)p < nneg &&
              ne_neg<MAXD>(cur, emb, order, nv, raw, (uint64_t)p, epoch, rng_state, ncomp, gamma, alpha,
                           vec + ((size_t)lane * kSlots + 1 + p) * ncomp))
            fl |= 2u << p;
        __syncwarp();
        // lanes with something to add, in lane (= edge) order; their slots in sample order
        for (unsigned live = __ballot_sync(kFull, fl != 0); live; live &= live - 1u) {
          const int L = __ffs(live) - 1;
          const uint32_t f = __shfl_sync(kFull, fl, L);
          for (uint32_t bits = f; bits; bits &= bits - 1u) add_slot(L, __ffs(bits) - 1);
        }
        __syncwarp();
      } else {
        for (int L = 0; L < 32; L++) {
          const uint64_t nL = __shfl_sync(kFull, nneg, L);
          const uint32_t fL = __shfl_sync(kFull, fl, L);
          if (fL) {
            if (lane == L) {
              float* dst = vec + (size_t)lane * kSlots * ncomp;
#pragma unroll
              for (int d = 0; d < MAXD; d++)
                if (d < ncomp) dst[d] = cp[d];
            }
            __syncwarp();
            add_slot(L, 0);
            __syncwarp();
          }
          for (uint64_t p = 0; p < nL; p++) {
            if (lane == L)
              fmask[L] = ne_neg<MAXD>(cur, emb, order, nv, raw, p, epoch, rng_state, ncomp, gamma, alpha,
                                      vec + (size_t)lane * kSlots * ncomp + ncomp)
                             ? 1u
                             : 0u;
            __syncwarp();
            if (fmask[L]) add_slot(L, 1);
            __syncwarp();
          }
        }
      }
      if (act) eonn[raw] = __fadd_rn(eonn[raw], __fmul_rn(__ull2float_rn(nneg), rate));
    }
    if (lane == 0) {
#pragma unroll
      for (int d = 0; d < MAXD; d++)
        if (d < ncomp) upd[from * ncomp + d] = u[d];
    }
  }
}

// node_embedding_epoch (the non-reproducible epoch, src/embed.rs:57-135): the
// reference walks the edges in order and updates both ends in place; here
// every edge of the epoch runs at once (lock-free, as Python's parallel
// version does), the updates landing with atomic adds.  The per-edge sample
// schedules advance exactly as in the serial loop; the embedding agrees with
// it in distribution, not bit for bit.
__global__ void edge_head_kernel(const int64_t* indptr, int64_t n, uint32_t* head) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
    for (int64_t e = indptr[r]; e < indptr[r + 1]; e++) head[e] = (uint32_t)r;
}

template <int MAXD>
__global__ void __launch_bounds__(256)
    ne_hogwild_kernel(Csr g, const uint32_t* head, float* emb, const float* eps, const float* epns, float* eonn,
                      float* eons, uint32_t rng_state, int ncomp, float alpha, uint32_t epoch, float noise) {
  const uint64_t nv = (uint64_t)g.n;
  const float nf = (float)epoch;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < g.nnz; i += (int64_t)gridDim.x * blockDim.x) {
    if (eons[i] > nf) continue;
    const uint64_t j = head[i], k = (uint64_t)(uint32_t)g.indices[i];
    if (j >= nv || k >= nv) continue;
    float ej[MAXD], ek[MAXD];
#pragma unroll
    for (int d = 0; d < MAXD; d++)
      if (d < ncomp) {
        ej[d] = emb[j * ncomp + d];
        ek[d] = emb[k * ncomp + d];
      }
    float ds = 0.0f;
#pragma unroll
    for (int d = 0; d < MAXD; d++)
      if (d < ncomp) {
        const float df = __fsub_rn(ej[d], ek[d]);
        ds = __fadd_rn(ds, __fmul_rn(df, df));
      }
    if (ds > 0.0f) {
      const float dist = __fsqrt_rn(ds);
      const float num = __fsub_rn(__fmul_rn(__fmul_rn(-2.0f, noise), dist), 2.0f);
      const float den = __fadd_rn(__fsub_rn(__fmul_rn(2.0f, ds), __fmul_rn(0.5f, dist)), 1.0f);
      const float gc = __fdiv_rn(num, den);
#pragma unroll
      for (int d = 0; d < MAXD; d++)
        if (d < ncomp) {
          const float step = __fmul_rn(__fmul_rn(gc, __fsub_rn(ej[d], ek[d])), alpha);
          atomicAdd(&emb[j * ncomp + d], step);
          atomicAdd(&emb[k * ncomp + d], -step);
          ej[d] = __fadd_rn(ej[d], step);
        }
    }
    eons[i] = __fadd_rn(eons[i], eps[i]);
    const float rate = epns[i];
    const uint64_t nneg = neg_count(nf, eonn[i], rate);
    for (uint64_t p = 0; p < nneg; p++) {
      const uint64_t nk = (((uint64_t)epoch + p) * (uint64_t)i * (uint64_t)rng_state) % nv;
      const float* en = emb + nk * ncomp;
      float dn = 0.0f;
#pragma unroll
      for (int d = 0; d < MAXD; d++)
        if (d < ncomp) {
          const float df = __fsub_rn(ej[d], en[d]);
          dn = __fadd_rn(dn, __fmul_rn(df, df));
        }
      if (dn > 1e-2f) {
        const float gc = __fdiv_rn(4.0f, __fmul_rn(__fadd_rn(1.0f, __fmul_rn(0.25f, dn)), dn));
#pragma unroll
        for (int d = 0; d < MAXD; d++)
          if (d < ncomp) {
            const float step = __fmul_rn(clip4(__fmul_rn(gc, __fsub_rn(ej[d], en[d]))), alpha);
            atomicAdd(&emb[j * ncomp + d], step);
            ej[d] = __fadd_rn(ej[d], step);
          }
      }
    }
    eonn[i] = __fadd_rn(eonn[i], __fmul_rn(__ull2float_rn(nneg), rate));
  }
}

__global__ void ne_apply_kernel(float* emb, const float* upd, const uint32_t* order, int64_t bs, int64_t be,
                                uint64_t nv, int ncomp) {
  const int64_t total = (be - bs) * ncomp;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t from = order[bs + i / ncomp];
    if (from >= nv) continue;
    const uint64_t o = from * ncomp + i % ncomp;
    emb[o] = __fadd_rn(emb[o], upd[o]);
  }
}

inline int grid_for(int64_t work, int threads, int cap) {
  const int64_t b = (work + threads - 1) / threads;
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

int bits_for(int64_t v) {  // bits to hold values 0..v-1
  int b = 1;
  while ((int64_t(1) << b) < v) b++;
  return b;
}

}  // namespace

// ------------------------------------------------------------------ launchers

cudaError_t launch_max_degree(const int64_t* indptr, int64_t n, int64_t* out, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(out, 0, 8, s);
  if (e != cudaSuccess) return e;
  max_degree_kernel<<<grid_for(n, 256, 1184), 256, 0, s>>>(indptr, n, out);
  return cudaGetLastError();
}

cudaError_t launch_validate_csr(const Csr& g, int32_t* bad, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(bad, 0, 4, s);
  if (e != cudaSuccess) return e;
  validate_csr_kernel<<<grid_for(std::max(g.n, g.nnz), 256, 4096), 256, 0, s>>>(g, bad);
  return cudaGetLastError();
}

cudaError_t launch_seed_labels(int32_t* labels, const int64_t* idx, int64_t count, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  seed_labels_kernel<<<1, 1, 0, s>>>(labels, idx, count);
  return cudaGetLastError();
}

cudaError_t launch_lp_iteration(const Csr& g, const int32_t* lab_in, int32_t* lab_out, int32_t* overflow,
                                int32_t* n_overflow, int32_t* scratch_key, double* scratch_sum, int64_t max_deg,
                                int32_t* dix, int64_t key_bound, int sms, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(n_overflow, 0, 4, s);
  if (e != cudaSuccess) return e;
  const int grid = grid_for(g.n, kRowWarps, sms * 8);
  lp_iteration_kernel<<<grid, kRowWarps * 32, 0, s>>>(g, lab_in, lab_out, overflow, n_overflow);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (max_deg > kVoteSlots) {
    lp_overflow_kernel<<<sms, kRowWarps * 32, 0, s>>>(g, lab_in, lab_out, overflow, n_overflow, scratch_key,
                                                      scratch_sum, max_deg, dix, key_bound);
    e = cudaGetLastError();
  }
  return e;
}

size_t lp_outliers_tmp_bytes(int64_t n) {
  size_t b = 0;
  cub::DeviceSelect::Flagged(nullptr, b, thrust::counting_iterator<int32_t>(0), (const int32_t*)nullptr,
                             (int32_t*)nullptr, (int32_t*)nullptr, (int)n);
  return b;
}

size_t outlier_stack_entries(int sms) { return size_t(sms) * 4 * kRowWarps * kOutlierStack; }

cudaError_t run_lp_outliers(const Csr& g, int32_t* labels, const int64_t* rs, const OutlierScratch& w, int64_t max_deg,
                            int sms, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(w.max_label, 0, 4, s);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(w.n_big, 0, 4, s)) != cudaSuccess) return e;
  outlier_flags_kernel<<<grid_for(g.n, 256, 2048), 256, 0, s>>>(labels, g.n, w.flag, w.max_label);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  size_t tb = w.tmp_bytes;
  e = cub::DeviceSelect::Flagged(w.tmp, tb, thrust::counting_iterator<int32_t>(0), w.flag, w.rows, w.count, (int)g.n,
                                 s);
  if (e != cudaSuccess) return e;
  int32_t cnt = 0;
  if ((e = cudaMemcpyAsync(&cnt, w.count, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
  if (cnt == 0) return cudaSuccess;
  WalkOut* out = reinterpret_cast<WalkOut*>(w.walk);
  outlier_walk_kernel<<<sms * 4, kRowWarps * 32, 0, s>>>(g, labels, rs, w.rows, w.count, w.max_label, w.stacks,
                                                         kOutlierStack, out, w.big, w.n_big);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  outlier_walk_big_kernel<<<1, 32, 0, s>>>(g, labels, rs, w.rows, w.max_label, w.big, w.n_big, w.big_stack,
                                           64 * max_deg + 1, out, w.status);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const int grid = grid_for(cnt, 256, 4096);
  outlier_index_kernel<<<grid, 256, 0, s>>>(w.count, w.rows, w.oidx);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  outlier_resolve_start_kernel<<<grid, 256, 0, s>>>(out, w.count, w.oidx, w.lab[0], w.nxt[0]);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  int cur = 0;
  for (int round = 0; round < 64; round++) {  // chains halve each round: 2^64 > any row count
    if ((e = cudaMemsetAsync(w.pending, 0, 4, s)) != cudaSuccess) return e;
    outlier_resolve_round_kernel<<<grid, 256, 0, s>>>(w.count, w.lab[cur], w.nxt[cur], w.lab[cur ^ 1],
                                                      w.nxt[cur ^ 1], w.pending);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    cur ^= 1;
    int32_t pend = 0;
    if ((e = cudaMemcpyAsync(&pend, w.pending, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    if (!pend) break;
  }
  outlier_scatter_kernel<<<grid, 256, 0, s>>>(w.count, w.rows, w.lab[cur], labels);
  return cudaGetLastError();
}

size_t lp_remap_tmp_bytes(int32_t bound) {
  size_t b = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, b, (int32_t*)nullptr, (int32_t*)nullptr, bound);
  return b;
}

cudaError_t launch_lp_remap(int32_t* labels, int64_t n, int32_t bound, int32_t* flags, int32_t* map,
                            int32_t* n_parts, int32_t* status, void* tmp, size_t tmp_bytes, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(flags, 0, size_t(bound) * 4, s);
  if (e != cudaSuccess) return e;
  remap_flags_kernel<<<grid_for(n, 256, 1184), 256, 0, s>>>(labels, n, bound, flags, status);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, flags, map, bound, s);
  if (e != cudaSuccess) return e;
  remap_apply_kernel<<<grid_for(n, 256, 1184), 256, 0, s>>>(labels, n, bound, flags, map, n_parts);
  return cudaGetLastError();
}

size_t part_members_tmp_bytes(int64_t n, int32_t n_parts) {
  size_t b = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, b, (const int32_t*)nullptr, (int32_t*)nullptr, (const int32_t*)nullptr,
                                  (int32_t*)nullptr, (int)n, 0, bits_for(n_parts));
  return b;
}

cudaError_t launch_part_members(const int32_t* part, int64_t n, int32_t n_parts, int32_t* count, int64_t* start,
                                int32_t* members, float* xnorm, float* wred, void* tmp, size_t tmp_bytes,
                                int32_t* keys_tmp, int32_t* vals_tmp, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(count, 0, size_t(n_parts) * 4, s);
  if (e != cudaSuccess) return e;
  part_count_kernel<<<grid_for(n, 256, 1184), 256, 0, s>>>(part, n, count, vals_tmp);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, part, keys_tmp, vals_tmp, members, (int)n, 0,
                                      bits_for(n_parts), s);
  if (e != cudaSuccess) return e;
  part_start_kernel<<<grid_for(n, 256, 1184), 256, 0, s>>>(keys_tmp, n, start);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  part_norm_kernel<<<grid_for(n_parts, 128, 1184), 128, 0, s>>>(count, n_parts, xnorm, wred);
  return cudaGetLastError();
}

cudaError_t launch_reduce_data(const float* x, int64_t d, const int32_t* members, const int64_t* start,
                               const int32_t* count, const float* wred, int32_t n_parts, float* out, int sms,
                               cudaStream_t s) {
  const int64_t tasks = int64_t(n_parts) * ((d + 31) / 32);
  reduce_data_kernel<<<grid_for(tasks * 32, 256, sms * 64), 256, 0, s>>>(x, d, members, start, count, wred, n_parts,
                                                                        out);
  return cudaGetLastError();
}

size_t reduce_sort_tmp_bytes(int64_t nnz) {
  size_t a = 0, b = 0, c = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, a, (const uint64_t*)nullptr, (uint64_t*)nullptr, (const uint32_t*)nullptr,
                                  (uint32_t*)nullptr, (int)nnz, 0, 64);
  cub::DeviceSelect::Flagged(nullptr, b, thrust::counting_iterator<int32_t>(0), (const int32_t*)nullptr,
                             (int32_t*)nullptr, (int32_t*)nullptr, (int)nnz);
  cub::DeviceScan::ExclusiveSum(nullptr, c, (const int64_t*)nullptr, (int64_t*)nullptr, (int)nnz + 1);
  return std::max(a, std::max(b, c));
}

namespace {

// Start positions of runs of equal (key >> shift): pos[0..*count).
cudaError_t group_starts(const uint64_t* key, int64_t m, int shift, const ReduceScratch& w, int32_t* pos,
                         int32_t* count, cudaStream_t s) {
  head_flags_kernel<<<grid_for(m, 256, 4096), 256, 0, s>>>(key, m, shift, w.head);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  size_t tb = w.tmp_bytes;
  return cub::DeviceSelect::Flagged(w.tmp, tb, thrust::counting_iterator<int32_t>(0), w.head, pos, count, (int)m,
                                    s);
}

}  // namespace

cudaError_t launch_reduce_graph(const Csr& g, const int32_t* part, const float* xnorm, int32_t n_parts,
                                const ReduceScratch& w, int64_t* r_indptr, int32_t* r_indices, float* r_data,
                                int64_t* r_nnz, cudaStream_t s) {
  const int pb = bits_for(n_parts);
  cudaError_t e;
  int32_t* ctr = w.counter;  // [0] temp groups, [1] temp entries, [2] reduced groups, [3] reduced entries
  if ((e = cudaMemsetAsync(ctr, 0, 16, s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(w.rcount, 0, size_t(n_parts + 1) * 8, s)) != cudaSuccess) return e;
  int32_t n_temp = 0, n_red = 0;
  if (g.nnz > 0) {
    // (part of row, column) keys, stable in edge order
    edge_keys_kernel<<<grid_for(g.nnz, 256, 8192), 256, 0, s>>>(g, part, w.k0, w.v0);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    size_t tb = w.tmp_bytes;
    e = cub::DeviceRadixSort::SortPairs(w.tmp, tb, w.k0, w.k1, w.v0, w.v1, (int)g.nnz, 0, 32 + pb, s);
    if (e != cudaSuccess) return e;
    if ((e = group_starts(w.k1, g.nnz, 0, w, w.pos, ctr + 0, s)) != cudaSuccess) return e;
    temp_groups_kernel<<<grid_for(g.nnz, 256, 8192), 256, 0, s>>>(w.k1, w.v1, g.nnz, w.pos, ctr + 0, g.data, xnorm,
                                                                  part, pb, w.k0, w.v0, ctr + 1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(&n_temp, ctr + 1, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
  }
  if (n_temp > 0) {
    // (p, q, descending first e): each (p, q) group in temp's row order
    size_t tb = w.tmp_bytes;
    e = cub::DeviceRadixSort::SortPairs(w.tmp, tb, w.k0, w.k1, w.v0, w.v1, n_temp, 0, 32 + 2 * pb, s);
    if (e != cudaSuccess) return e;
    if ((e = group_starts(w.k1, n_temp, 32, w, w.pos, ctr + 2, s)) != cudaSuccess) return e;
    reduced_groups_kernel<<<grid_for(n_temp, 256, 8192), 256, 0, s>>>(w.k1, w.v1, n_temp, w.pos, ctr + 2, pb, w.k0,
                                                                      w.v0, w.v2, w.v3, ctr + 3);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(&n_red, ctr + 3, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
  }
  if (n_red > 0) {
    // rows in order of p, each row's parts by the first e of their heads
    size_t tb = w.tmp_bytes;
    e = cub::DeviceRadixSort::SortPairs(w.tmp, tb, w.k0, w.k1, w.v0, w.v1, n_red, 0, 32 + pb, s);
    if (e != cudaSuccess) return e;
    row_count_kernel<<<grid_for(n_red, 256, 8192), 256, 0, s>>>(w.k1, n_red, 32, w.rcount);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    reduced_write_kernel<<<grid_for(n_red, 256, 8192), 256, 0, s>>>(w.v1, n_red, w.v2, w.v3, r_indices, r_data);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  scan_i64_kernel<<<1, 1024, 0, s>>>(w.rcount, n_parts, r_indptr);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const int64_t nr = n_red;
  return cudaMemcpyAsync(r_nnz, &nr, 8, cudaMemcpyHostToDevice, s);
}

cudaError_t launch_hadamard_sym(const Csr& g, const ReduceScratch& w, int64_t* s_indptr, int32_t* s_indices,
                                float* s_data, int64_t* s_nnz, cudaStream_t s) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(w.rcount, 0, size_t(g.n + 1) * 8, s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(w.counter, 0, 16, s)) != cudaSuccess) return e;
  if (g.nnz > 0) {
    sorted_flag_kernel<<<grid_for(g.nnz, 256, 8192), 256, 0, s>>>(g, w.counter);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    int32_t unsorted = 0;
    if ((e = cudaMemcpyAsync(&unsorted, w.counter, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    // (row, column) keys; rows already in column order skip the sort
    row_col_keys_kernel<<<grid_for(g.nnz, 256, 8192), 256, 0, s>>>(g, unsorted ? w.k0 : w.k1,
                                                                   unsorted ? w.v0 : w.v1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (unsorted) {
      size_t tb = w.tmp_bytes;
      e = cub::DeviceRadixSort::SortPairs(w.tmp, tb, w.k0, w.k1, w.v0, w.v1, (int)g.nnz, 0, 32 + bits_for(g.n), s);
      if (e != cudaSuccess) return e;
    }
    sym_keep_kernel<<<grid_for(g.nnz, 256, 8192), 256, 0, s>>>(g.indptr, g.n, g.nnz, w.k1, w.v1, w.head, w.v2,
                                                               w.rcount);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    size_t tb = w.tmp_bytes;
    e = cub::DeviceScan::ExclusiveSum(w.tmp, tb, w.head, w.pos, (int)g.nnz, s);
    if (e != cudaSuccess) return e;
  }
  scan_i64_kernel<<<1, 1024, 0, s>>>(w.rcount, g.n, s_indptr);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (g.nnz > 0) {
    sym_write_kernel<<<grid_for(g.nnz, 256, 8192), 256, 0, s>>>(w.k1, w.v2, w.head, w.pos, g.nnz, s_indices, s_data);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaMemcpyAsync(s_nnz, s_indptr + g.n, 8, cudaMemcpyDeviceToDevice, s);
}

cudaError_t launch_expand(const Csr& sym, const int32_t* part, const float* xnorm, const float* layout, int ncomp,
                          float* result, int32_t* overflow, int32_t* n_overflow, int32_t* scratch_key,
                          float* scratch_sum, int64_t max_deg, int32_t* dix, int64_t key_bound, int sms,
                          cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(n_overflow, 0, 4, s);
  if (e != cudaSuccess) return e;
  expand_kernel<<<grid_for(sym.n, kRowWarps, sms * 8), kRowWarps * 32, 0, s>>>(sym, part, xnorm, layout, ncomp,
                                                                               result, overflow, n_overflow);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (max_deg > kVoteSlots) {
    expand_overflow_kernel<<<sms, kRowWarps * 32, 0, s>>>(sym, part, xnorm, layout, ncomp, result, overflow,
                                                          n_overflow, scratch_key, scratch_sum, max_deg, dix,
                                                          key_bound);
    e = cudaGetLastError();
  }
  return e;
}

cudaError_t launch_center_scale(const float* result, int64_t n, int ncomp, float scaling, float* out,
                                double* mean, cudaStream_t s) {
  center_mean_kernel<<<1, 1024, 0, s>>>(result, n, ncomp, mean);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  center_apply_kernel<<<grid_for(n * ncomp, 256, 4096), 256, 0, s>>>(result, n, ncomp, scaling, mean, out);
  return cudaGetLastError();
}

cudaError_t launch_pca_init(const float* x, int64_t n, int64_t d, int ncomp, float* out, float* mean_ws,
                            double* vws, int32_t* status, cudaStream_t s) {
  if (n <= 0 || n > kPcaMax) return cudaErrorInvalidValue;
  const size_t smem = size_t(2) * kPcaMax * kPcaMax * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(pca_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  pca_kernel<<<1, 256, smem, s>>>(x, n, d, ncomp, out, mean_ws, vws, status);
  return cudaGetLastError();
}

cudaError_t launch_spectral_mds_init(const float* x, int64_t n, int64_t d, int ncomp, int mode, float* out,
                                    cudaStream_t s) {
  if (n <= 0 || n > kPcaMax || (mode != 0 && mode != 1)) return cudaErrorInvalidValue;
  const size_t smem = size_t(3) * kPcaMax * kPcaMax * sizeof(double) + size_t(kPcaMax) * kPcaMax * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(spectral_mds_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  spectral_mds_kernel<<<1, 256, smem, s>>>(x, n, d, ncomp, mode, out);
  return cudaGetLastError();
}

cudaError_t launch_unit_rows(float* r, int64_t n, int ncomp, cudaStream_t s) {
  unit_rows_kernel<<<grid_for(n, 256, 4096), 256, 0, s>>>(r, n, ncomp);
  return cudaGetLastError();
}

cudaError_t launch_upscale(float* result, const int32_t* part, const float* layout, const float* noise, int64_t n,
                           int ncomp, int jitter, cudaStream_t s) {
  upscale_kernel<<<grid_for(n * ncomp, 256, 4096), 256, 0, s>>>(result, part, layout, noise, n, ncomp, jitter);
  return cudaGetLastError();
}

cudaError_t launch_ne_schedule(const float* w, int64_t m, int32_t n_epochs, float negative_sample_rate,
                               float neg_scale, float* eps, float* epns, float* eonn, float* eons, float* max_w,
                               cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(max_w, 0, 4, s);
  if (e != cudaSuccess || m == 0) return e;
  ne_maxw_kernel<<<grid_for(m, 256, 4096), 256, 0, s>>>(w, m, max_w);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  ne_schedule_kernel<<<grid_for(m, 256, 4096), 256, 0, s>>>(w, m, (float)n_epochs, negative_sample_rate, neg_scale,
                                                           max_w, eps, epns, eonn, eons);
  return cudaGetLastError();
}

cudaError_t launch_ne_block(const Csr& g, float* emb, float* upd, const uint32_t* order, int64_t bs, int64_t be,
                            const float* eps, const float* epns, float* eonn, float* eons, uint32_t rng_state,
                            int ncomp, float alpha, uint8_t epoch, float noise, float gamma, float decay,
                            int apply_decay, int64_t heavy_deg, uint32_t* heavy_rows, int32_t* heavy_count, int sms,
                            cudaStream_t s) {
  const int64_t warps = be - bs;
  if (warps <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(heavy_count, 0, 4, s);
  if (e != cudaSuccess) return e;
  const HeavyRows heavy{heavy_deg, heavy_rows, heavy_count};
  const int grid = (int)std::min<int64_t>((warps + kNeWarps - 1) / kNeWarps, 1 << 20);
  const size_t smem = size_t(kNeWarps) * ne_stage_floats(ncomp) * sizeof(float);
  const size_t hsmem = heavy_smem_bytes(ncomp);
  auto run = [&](auto block_kernel, auto heavy_kernel) -> cudaError_t {
    cudaError_t err = cudaFuncSetAttribute(block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    block_kernel<<<grid, kNeWarps * 32, smem, s>>>(g, emb, upd, order, bs, be, eps, epns, eonn, eons, rng_state, ncomp,
                                                   alpha, epoch, noise, gamma, decay, apply_decay, heavy);
    if ((err = cudaGetLastError()) != cudaSuccess) return err;
    if ((err = cudaFuncSetAttribute(heavy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsmem)))
      return err;
    heavy_kernel<<<sms * 2, kHeavyWarps * 32, hsmem, s>>>(g, emb, upd, order, eps, epns, eonn, eons, rng_state, ncomp,
                                                          alpha, epoch, noise, gamma, decay, apply_decay, heavy);
    return cudaGetLastError();
  };
  // narrow rows: more warps per SM (64 registers); wider rows keep their values in registers
  if (ncomp <= 8) return run(ne_block_kernel<8, 8>, ne_heavy_kernel<8, 2>);
  if (ncomp <= 16) return run(ne_block_kernel<16, 1>, ne_heavy_kernel<16, 1>);
  return run(ne_block_kernel<32, 1>, ne_heavy_kernel<32, 1>);
}

cudaError_t launch_edge_head(const int64_t* indptr, int64_t n, uint32_t* head, cudaStream_t s) {
  edge_head_kernel<<<grid_for(n, 256, 4096), 256, 0, s>>>(indptr, n, head);
  return cudaGetLastError();
}

cudaError_t launch_ne_hogwild(const Csr& g, const uint32_t* head, float* emb, const float* eps, const float* epns,
                              float* eonn, float* eons, uint32_t rng_state, int ncomp, float alpha, uint8_t epoch,
                              float noise, int sms, cudaStream_t s) {
  const int grid = grid_for(g.nnz, 256, sms * 32);
  if (ncomp <= 8)
    ne_hogwild_kernel<8><<<grid, 256, 0, s>>>(g, head, emb, eps, epns, eonn, eons, rng_state, ncomp, alpha, epoch,
                                              noise);
  else if (ncomp <= 16)
    ne_hogwild_kernel<16><<<grid, 256, 0, s>>>(g, head, emb, eps, epns, eonn, eons, rng_state, ncomp, alpha, epoch,
                                               noise);
  else
    ne_hogwild_kernel<32><<<grid, 256, 0, s>>>(g, head, emb, eps, epns, eonn, eons, rng_state, ncomp, alpha, epoch,
                                               noise);
  return cudaGetLastError();
}

cudaError_t launch_ne_apply(float* emb, const float* upd, const uint32_t* order, int64_t bs, int64_t be, int64_t nv,
                            int ncomp, cudaStream_t s) {
  ne_apply_kernel<<<grid_for((be - bs) * ncomp, 256, 4096), 256, 0, s>>>(emb, upd, order, bs, be, (uint64_t)nv,
                                                                         ncomp);
  return cudaGetLastError();
}

}  // namespace lp
}  // namespace evoc
