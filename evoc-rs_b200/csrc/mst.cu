// Borůvka minimum spanning tree under mutual-reachability distance, with the
// core distances, on the GPU.
//
// Replaces build_kdtree (src/kdtree.rs:367-413), parallel_tree_query
// (src/kdtree.rs:592-629), initialize_boruvka_from_knn and parallel_boruvka
// with reproducible = false (src/boruvka.rs:437-593): the MST that
// build_cluster_layers (src/clustering.rs:50-110) condenses into the cluster
// hierarchy, over the node embedding (n points of 4..15 dimensions there).
//
//   rdist(a, b)   squared Euclidean distance, summed serially over the
//                 dimensions in f32 without contraction (src/kdtree.rs:415-423)
//   core[i]       rdist to the (min_samples + 1)-th nearest point, the point
//                 itself included (parallel_tree_query with output_rdist)
//   mr(i, j)      max(rdist(i, j), core[i], core[j])
//   edges         n - 1 rows (from, to, sqrt(mr)) as f32, in the order found
//
// Tree.  The reference's balanced KD-tree: node i has children 2i+1 and 2i+2,
// n_levels = floor(log2(max(n-1, 1) / leaf_size)) + 1, and every node's
// positions are fixed by halving -- [s, e) splits at s + (e-s)/2 -- so only
// which points fill a range depends on the data.  It is built level by level:
// each node's bounds (block per node), its split dimension (largest spread,
// first on ties, src/kdtree.rs:232-257), then one stable radix sort of
// (node, coordinate on the node's split dimension) keys puts every node's
// lower half left of its median, as the reference's introselect does (the
// order inside the halves may differ; the tree's geometry does not).  Points
// are then stored in tree order, so a leaf is a contiguous run.
//
// Queries.  One thread per point (in tree order, so neighbouring threads walk
// similar paths) with an explicit stack that visits the nearer child first,
// as the reference's recursion does, and prunes on the node lower bound
// (point_to_node_lower_bound_rdist, src/kdtree.rs:425-447).  The k-NN query
// keeps a min_samples+1 max-heap with the reference's push (simple_heap_push,
// src/kdtree.rs:449-501).
//
// Borůvka.  Components live in a lock-free union-find over tree positions.
// The kNN initialisation takes, for each point, the first of its sorted
// neighbours j >= 1 with core[i] >= core[j] (src/boruvka.rs:437-477).  Each
// round every point searches for its nearest point in another component under
// mr, pruning nodes whose points all share its component (node components,
// src/boruvka.rs:88-127), nodes farther than its best so far, and nodes
// farther than its component's shared bound (an atomic minimum, as the
// non-reproducible reference keeps it, src/boruvka.rs:262-318).  Each
// component's candidate is the smallest (mr, point) key of its points -- the
// lowest point among equal distances, as merge_components keeps the first --
// and components are joined by CAS union; an edge is kept only when its union
// links two roots.  A cycle among the components' choices can only join
// edges of one equal weight, so dropping the closing edge keeps an MST: the
// result has the reference's total weight and the same sorted weights; edges
// can differ only among equal weights.  The reproducible mode
// (boruvka_tree_query_reproducible) freezes component bounds block by block in
// point order and is serial at the block level; it is not built here.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/evoc_gpu.h"
#include "common.cuh"
#include "ctx.h"

namespace evoc {
namespace mst {

constexpr int kMaxStack = 64;  // > 2 * levels: a visit pushes two children and pops one
constexpr int kMaxKnn = 32;    // min_samples + 1
constexpr int kLeafSize = 40;  // build_cluster_layers' leaf size (src/clustering.rs:63)
constexpr uint32_t kInfBits = 0x7f800000u;

struct TreeView {
  int64_t n;
  int n_nodes;
  const int32_t* order;  // tree position -> point index
  const float* pts;      // points in tree order, P floats each (zero padded)
  const int32_t* nstart;
  const int32_t* nend;
  const uint8_t* leaf;
  const float* lo;       // per node, P floats
  const float* hi;
};

template <int P>
__device__ __forceinline__ void load_point(const float* __restrict__ src, float (&q)[P]) {
  const float4* s4 = reinterpret_cast<const float4*>(src);
#pragma unroll
  for (int c = 0; c < P / 4; c++) {
    const float4 v = s4[c];
    q[4 * c] = v.x;
    q[4 * c + 1] = v.y;
    q[4 * c + 2] = v.z;
    q[4 * c + 3] = v.w;
  }
}

// rdist in the reference's order; zero-padded dimensions add +0.0 exactly.
template <int P>
__device__ __forceinline__ float rdist(const float (&q)[P], const float* __restrict__ y) {
  float y4[P];
  load_point<P>(y, y4);
  float r = 0.0f;
#pragma unroll
  for (int c = 0; c < P; c++) {
    const float d = __fsub_rn(q[c], y4[c]);
    r = __fadd_rn(r, __fmul_rn(d, d));
  }
  return r;
}

template <int P>
__device__ __forceinline__ float node_lower_bound(const float (&q)[P], const float* __restrict__ lo,
                                                  const float* __restrict__ hi) {
  float r = 0.0f;
#pragma unroll
  for (int c = 0; c < P; c++) {
    const float dl = lo[c] > q[c] ? __fsub_rn(lo[c], q[c]) : 0.0f;
    const float dh = q[c] > hi[c] ? __fsub_rn(q[c], hi[c]) : 0.0f;
    const float d = __fadd_rn(dl, dh);
    r = __fadd_rn(r, __fmul_rn(d, d));
  }
  return r;
}

// ------------------------------------------------------------------ tree build

__global__ void pad_points_kernel(const float* __restrict__ X, int64_t n, int dim, int64_t ldx, float* __restrict__ Xp,
                                  int P) {
  const int64_t total = n * P;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e / P;
    const int c = int(e % P);
    Xp[e] = c < dim ? X[i * ldx + c] : 0.0f;
  }
}

__global__ void iota_kernel(int32_t* __restrict__ a, int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    a[i] = int32_t(i);
}

// Bounds of nodes first .. first+count-1 (block per node) and, with `split`,
// each node's split dimension: the largest spread, the first on ties.
template <int P>
__global__ void __launch_bounds__(256) node_bounds_kernel(const float* __restrict__ Xp,
                                                          const int32_t* __restrict__ order,
                                                          const int32_t* __restrict__ nstart,
                                                          const int32_t* __restrict__ nend, int first, int count,
                                                          int dim, float* __restrict__ lo, float* __restrict__ hi,
                                                          int32_t* __restrict__ split) {
  __shared__ float smin[8][P], smax[8][P];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int b = blockIdx.x; b < count; b += gridDim.x) {
    const int node = first + b;
    const int32_t s = nstart[node], e = nend[node];
    float mn[P], mx[P];
#pragma unroll
    for (int c = 0; c < P; c++) {
      mn[c] = __int_as_float(0x7f800000);
      mx[c] = __int_as_float(0xff800000);
    }
    for (int32_t p = s + threadIdx.x; p < e; p += blockDim.x) {
      float v[P];
      load_point<P>(Xp + int64_t(order[p]) * P, v);
#pragma unroll
      for (int c = 0; c < P; c++) {
        mn[c] = fminf(mn[c], v[c]);
        mx[c] = fmaxf(mx[c], v[c]);
      }
    }
#pragma unroll
    for (int c = 0; c < P; c++) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        mn[c] = fminf(mn[c], __shfl_xor_sync(0xffffffffu, mn[c], o));
        mx[c] = fmaxf(mx[c], __shfl_xor_sync(0xffffffffu, mx[c], o));
      }
    }
    if (lane == 0)
#pragma unroll
      for (int c = 0; c < P; c++) {
        smin[warp][c] = mn[c];
        smax[warp][c] = mx[c];
      }
    __syncthreads();
    if (threadIdx.x < P) {
      const int c = threadIdx.x;
      float a = smin[0][c], z = smax[0][c];
      for (int w = 1; w < int(blockDim.x >> 5); w++) {
        a = fminf(a, smin[w][c]);
        z = fmaxf(z, smax[w][c]);
      }
      lo[int64_t(node) * P + c] = a;
      hi[int64_t(node) * P + c] = z;
      smin[0][c] = a;
      smax[0][c] = z;
    }
    __syncthreads();
    if (split && threadIdx.x == 0) {
      int best = 0;
      float spread_max = 0.0f;
      for (int c = 0; c < dim; c++) {
        const float spread = __fsub_rn(smax[0][c], smin[0][c]);
        if (spread > spread_max) {
          spread_max = spread;
          best = c;
        }
      }
      split[node] = best;
    }
    __syncthreads();
  }
}

// Sort keys of one level: (node within the level, coordinate on its split dimension).
__global__ void split_keys_kernel(const float* __restrict__ Xp, int P, const int32_t* __restrict__ order, int64_t n,
                                  const int32_t* __restrict__ nstart, int first, int count,
                                  const int32_t* __restrict__ split, uint64_t* __restrict__ keys) {
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n; p += int64_t(gridDim.x) * blockDim.x) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {  // last node of the level starting at or before p
      const int mid = (lo + hi + 1) >> 1;
      if (nstart[first + mid] <= p) lo = mid;
      else hi = mid - 1;
    }
    const float v = Xp[int64_t(order[p]) * P + split[first + lo]];
    keys[p] = (uint64_t(uint32_t(lo)) << 32) | uint64_t(orderable(v));
  }
}

template <int P>
__global__ void gather_points_kernel(const float* __restrict__ Xp, const int32_t* __restrict__ order, int64_t n,
                                     float* __restrict__ out) {
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n; p += int64_t(gridDim.x) * blockDim.x) {
    const float4* s = reinterpret_cast<const float4*>(Xp + int64_t(order[p]) * P);
    float4* d = reinterpret_cast<float4*>(out + p * P);
#pragma unroll
    for (int c = 0; c < P / 4; c++) d[c] = s[c];
  }
}

// ------------------------------------------------------------------ k-NN query (core distances)

// simple_heap_push (src/kdtree.rs:449-501) on a max-heap of `size`.
__device__ __forceinline__ void heap_push(float* hp, int32_t* hi, int size, float p, int32_t n) {
  if (p >= hp[0]) return;
  int i = 0;
  for (;;) {
    const int c1 = 2 * i + 1, c2 = c1 + 1;
    if (c1 >= size) break;
    int sw;
    if (c2 >= size) {
      if (hp[c1] > p) sw = c1;
      else break;
    } else if (hp[c1] >= hp[c2]) {
      if (p < hp[c1]) sw = c1;
      else break;
    } else if (p < hp[c2]) {
      sw = c2;
    } else {
      break;
    }
    hp[i] = hp[sw];
    hi[i] = hi[sw];
    i = sw;
  }
  hp[i] = p;
  hi[i] = n;
}

// Thread per tree position: the kq nearest positions (self included), sorted
// by (rdist, position); core = the kq-th rdist.
template <int P>
__global__ void __launch_bounds__(128) knn_kernel(TreeView t, int kq, float* __restrict__ core,
                                                  int32_t* __restrict__ knn_pos, float* __restrict__ knn_d,
                                                  int* __restrict__ status) {
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < t.n; p += int64_t(gridDim.x) * blockDim.x) {
    float q[P];
    load_point<P>(t.pts + p * P, q);
    float hp[kMaxKnn];
    int32_t hi[kMaxKnn];
    for (int j = 0; j < kq; j++) {
      hp[j] = __int_as_float(0x7f800000);
      hi[j] = -1;
    }
    int sn[kMaxStack];
    float sl[kMaxStack];
    int sp = 0;
    sn[sp] = 0;
    sl[sp++] = node_lower_bound<P>(q, t.lo, t.hi);
    while (sp > 0) {
      const int node = sn[--sp];
      const float lb = sl[sp];
      if (lb > hp[0]) continue;
      if (t.leaf[node]) {
        for (int32_t s = t.nstart[node]; s < t.nend[node]; s++) {
          const float d = rdist<P>(q, t.pts + int64_t(s) * P);
          if (d < hp[0]) heap_push(hp, hi, kq, d, s);
        }
      } else {
        const int l = 2 * node + 1, r = l + 1;
        const float bl = node_lower_bound<P>(q, t.lo + int64_t(l) * P, t.hi + int64_t(l) * P);
        const float br = node_lower_bound<P>(q, t.lo + int64_t(r) * P, t.hi + int64_t(r) * P);
        if (sp + 2 > kMaxStack) {  // cannot happen for the checked depths; stop rather than overrun
          atomicCAS(status, 0, 1);
          break;
        }
        // the nearer child is visited first (pushed last)
        if (bl <= br) {
          sn[sp] = r;
          sl[sp++] = br;
          sn[sp] = l;
          sl[sp++] = bl;
        } else {
          sn[sp] = l;
          sl[sp++] = bl;
          sn[sp] = r;
          sl[sp++] = br;
        }
      }
    }
    core[p] = hp[0];
    // sort ascending by (rdist, position)
    for (int a = 1; a < kq; a++) {
      const float dv = hp[a];
      const int32_t iv = hi[a];
      int b = a - 1;
      while (b >= 0 && (hp[b] > dv || (hp[b] == dv && uint32_t(hi[b]) > uint32_t(iv)))) {
        hp[b + 1] = hp[b];
        hi[b + 1] = hi[b];
        b--;
      }
      hp[b + 1] = dv;
      hi[b + 1] = iv;
    }
    for (int j = 0; j < kq; j++) {
      knn_pos[p * kq + j] = hi[j];
      knn_d[p * kq + j] = hp[j];
    }
  }
}

// ------------------------------------------------------------------ union-find over tree positions

__device__ __forceinline__ int32_t uf_find(int32_t* parent, int32_t x) {
  for (;;) {
    const int32_t p = reinterpret_cast<volatile int32_t*>(parent)[x];
    const int32_t g = reinterpret_cast<volatile int32_t*>(parent)[p];
    if (p == g) return p;
    atomicCAS(&parent[x], p, g);  // path halving
    x = g;
  }
}

// Links the roots of a and b (larger under smaller); false when already joined.
__device__ __forceinline__ bool uf_unite(int32_t* parent, int32_t a, int32_t b) {
  for (;;) {
    a = uf_find(parent, a);
    b = uf_find(parent, b);
    if (a == b) return false;
    if (a < b) {
      const int32_t t = a;
      a = b;
      b = t;
    }
    if (atomicCAS(&parent[a], a, b) == a) return true;
  }
}

__device__ __forceinline__ void add_edge(int32_t a, int32_t b, float w, int32_t* __restrict__ e_from,
                                         int32_t* __restrict__ e_to, float* __restrict__ e_w, int32_t* count,
                                         int64_t cap) {
  const int32_t slot = atomicAdd(count, 1);
  if (slot < cap) {
    e_from[slot] = a;
    e_to[slot] = b;
    e_w[slot] = w;
  }
}

// initialize_boruvka_from_knn (src/boruvka.rs:437-477): each point's first
// sorted neighbour j >= 1 with core[i] >= core[j], joined when it links two
// components.  (The reference joins them serially in point order; any
// spanning forest of these edges has the same weight: each is a minimum
// mutual-reachability edge of its point, and a cycle among them has equal
// weights.)
__global__ void knn_init_kernel(int64_t n, int kq, const float* __restrict__ core, const int32_t* __restrict__ knn_pos,
                                const float* __restrict__ knn_d, int32_t* __restrict__ parent,
                                int32_t* __restrict__ e_from, int32_t* __restrict__ e_to, float* __restrict__ e_w,
                                int32_t* count, int64_t cap) {
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n; p += int64_t(gridDim.x) * blockDim.x) {
    for (int j = 1; j < kq; j++) {
      const int32_t nb = knn_pos[p * kq + j];
      if (nb < 0) break;
      if (core[p] >= core[nb]) {
        const float w = fmaxf(core[p], knn_d[p * kq + j]);
        if (uf_unite(parent, int32_t(p), nb)) add_edge(int32_t(p), nb, w, e_from, e_to, e_w, count, cap);
        break;
      }
    }
  }
}

__global__ void components_kernel(int64_t n, int32_t* __restrict__ parent, int32_t* __restrict__ comp) {
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n; p += int64_t(gridDim.x) * blockDim.x) {
    const int32_t r = uf_find(parent, int32_t(p));
    comp[p] = r;
    parent[p] = r;
  }
}

// Node components (src/boruvka.rs:101-126): a leaf whose points share one
// component has it, an internal node whose children have the same value has
// it, else -1.  Leaves first, then each level bottom-up.
__global__ void leaf_components_kernel(TreeView t, int first, int count, const int32_t* __restrict__ comp,
                                       int32_t* __restrict__ node_comp) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < count; b += gridDim.x * blockDim.x) {
    const int node = first + b;
    if (!t.leaf[node]) continue;  // internal nodes take their children's value
    const int32_t s = t.nstart[node], e = t.nend[node];
    int32_t c = s < e ? comp[s] : -1;
    for (int32_t p = s + 1; p < e && c >= 0; p++)
      if (comp[p] != c) c = -1;
    node_comp[node] = c;
  }
}

__global__ void inner_components_kernel(TreeView t, int first, int count, int32_t* __restrict__ node_comp) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < count; b += gridDim.x * blockDim.x) {
    const int node = first + b;
    if (t.leaf[node]) continue;  // a leaf above the last level (fewer than two points) was set already
    const int32_t l = node_comp[2 * node + 1], r = node_comp[2 * node + 2];
    node_comp[node] = l == r ? l : -1;
  }
}

__global__ void reset_round_kernel(int64_t n, uint32_t* __restrict__ bound, unsigned long long* __restrict__ best) {
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n; p += int64_t(gridDim.x) * blockDim.x) {
    bound[p] = kInfBits;
    best[p] = ~0ull;
  }
}

// One Borůvka round's search: thread per position, the nearest position of
// another component under mutual reachability (component_aware_query_recursion,
// src/boruvka.rs:131-253), with the component's shared bound.
template <int P>
__global__ void __launch_bounds__(128) boruvka_query_kernel(TreeView t, const float* __restrict__ core,
                                                            const int32_t* __restrict__ comp,
                                                            const int32_t* __restrict__ node_comp,
                                                            uint32_t* __restrict__ bound,
                                                            unsigned long long* __restrict__ best,
                                                            int32_t* __restrict__ cand, int* __restrict__ status) {
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < t.n; p += int64_t(gridDim.x) * blockDim.x) {
    const int32_t c = comp[p];
    const float cp = core[p];
    float cbound = __uint_as_float(reinterpret_cast<volatile uint32_t*>(bound)[c]);
    if (cp > cbound) continue;
    float q[P];
    load_point<P>(t.pts + p * P, q);
    float bd = __int_as_float(0x7f800000);
    int32_t bj = -1;
    int sn[kMaxStack];
    float sl[kMaxStack];
    int sp = 0;
    sn[sp] = 0;
    sl[sp++] = node_lower_bound<P>(q, t.lo, t.hi);
    while (sp > 0) {
      const int node = sn[--sp];
      const float lb = sl[sp];
      if (lb > bd || lb > cbound || cp > cbound) continue;
      if (node_comp[node] == c) continue;
      if (t.leaf[node]) {
        // another thread may have lowered the component's bound meanwhile
        cbound = fminf(cbound, __uint_as_float(reinterpret_cast<volatile uint32_t*>(bound)[c]));
        for (int32_t s = t.nstart[node]; s < t.nend[node]; s++) {
          if (comp[s] == c || !(core[s] < cbound)) continue;
          const float d = fmaxf(fmaxf(rdist<P>(q, t.pts + int64_t(s) * P), cp), core[s]);
          if (d < bd) {
            bd = d;
            bj = s;
            if (d < cbound) cbound = d;
          }
        }
      } else {
        const int l = 2 * node + 1, r = l + 1;
        const float bl = node_lower_bound<P>(q, t.lo + int64_t(l) * P, t.hi + int64_t(l) * P);
        const float br = node_lower_bound<P>(q, t.lo + int64_t(r) * P, t.hi + int64_t(r) * P);
        if (sp + 2 > kMaxStack) {
          atomicCAS(status, 0, 1);
          break;
        }
        if (bl <= br) {
          sn[sp] = r;
          sl[sp++] = br;
          sn[sp] = l;
          sl[sp++] = bl;
        } else {
          sn[sp] = l;
          sl[sp++] = bl;
          sn[sp] = r;
          sl[sp++] = br;
        }
      }
    }
    if (bj >= 0) {
      cand[p] = bj;
      atomicMin(&bound[c], __float_as_uint(bd));  // non-negative floats order as their bits
      atomicMin(&best[c], (static_cast<unsigned long long>(__float_as_uint(bd)) << 32) | uint32_t(p));
    }
  }
}

// Each component joins along its smallest (mr, position) candidate.
__global__ void boruvka_merge_kernel(int64_t n, const int32_t* __restrict__ comp,
                                     const unsigned long long* __restrict__ best, const int32_t* __restrict__ cand,
                                     int32_t* __restrict__ parent, int32_t* __restrict__ e_from,
                                     int32_t* __restrict__ e_to, float* __restrict__ e_w, int32_t* count, int64_t cap) {
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n; p += int64_t(gridDim.x) * blockDim.x) {
    if (comp[p] != p) continue;  // one thread per component: its root
    const unsigned long long key = best[p];
    if (key == ~0ull) continue;
    const int32_t src = int32_t(uint32_t(key));
    const int32_t dst = cand[src];
    const float w = __uint_as_float(uint32_t(key >> 32));
    if (uf_unite(parent, src, dst)) add_edge(src, dst, w, e_from, e_to, e_w, count, cap);
  }
}

// (from, to, sqrt(mr)) rows in point indices; core distances in point order.
__global__ void emit_edges_kernel(int64_t m, const int32_t* __restrict__ order, const int32_t* __restrict__ e_from,
                                  const int32_t* __restrict__ e_to, const float* __restrict__ e_w,
                                  float* __restrict__ out) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
    out[3 * i] = float(order[e_from[i]]);
    out[3 * i + 1] = float(order[e_to[i]]);
    out[3 * i + 2] = __fsqrt_rn(e_w[i]);
  }
}

__global__ void scatter_core_kernel(int64_t n, const int32_t* __restrict__ order, const float* __restrict__ core_t,
                                    float* __restrict__ core) {
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n; p += int64_t(gridDim.x) * blockDim.x)
    core[order[p]] = core_t[p];
}

// ------------------------------------------------------------------ host

struct Arena {
  cudaStream_t s;
  cudaMemPool_t pool;
  std::vector<void*> ptrs;
  Arena(cudaStream_t st, cudaMemPool_t pl) : s(st), pool(pl) {}
  ~Arena() {
    for (void* p : ptrs) cudaFreeAsync(p, s);
  }
  template <class T>
  cudaError_t get(T** out, size_t count) {
    void* p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, std::max<size_t>(count, 1) * sizeof(T), pool, s);
    if (e != cudaSuccess) return e;
    ptrs.push_back(p);
    *out = static_cast<T*>(p);
    return cudaSuccess;
  }
};

template <int P>
int run(evoc_gpu_ctx* ctx, Arena& A, const float* d_x, int64_t n, int dim, int64_t ldx, int min_samples,
        float* d_edges, float* d_core, int64_t* n_edges) {
  cudaStream_t st = ctx->stream;
  const int sms = ctx->sms;
  // Node ranges, leaf flags (host): the reference's layout.
  int n_levels = int(std::floor(std::log2(double(std::max<int64_t>(n - 1, 1)) / double(kLeafSize)))) + 1;
  if (n_levels < 1) n_levels = 1;
  if (n_levels > 28) return fail(ctx, EVOC_ERR_ARG, "too many points for the tree (levels > 28)");
  const int n_nodes = (1 << n_levels) - 1;
  std::vector<int32_t> hs(static_cast<size_t>(n_nodes)), he(static_cast<size_t>(n_nodes));
  std::vector<uint8_t> hl(static_cast<size_t>(n_nodes));
  hs[0] = 0;
  he[0] = int32_t(n);
  for (int i = 0; i < n_nodes; i++) {
    hl[size_t(i)] = (2 * i + 1 >= n_nodes || he[size_t(i)] - hs[size_t(i)] < 2) ? 1 : 0;
    if (2 * i + 2 < n_nodes) {
      const int32_t s = hs[size_t(i)], e = he[size_t(i)], mid = s + (e - s) / 2;
      hs[size_t(2 * i + 1)] = s;
      he[size_t(2 * i + 1)] = mid;
      hs[size_t(2 * i + 2)] = mid;
      he[size_t(2 * i + 2)] = e;
    }
  }
  float *Xp, *pts, *lo, *hi, *core, *knn_d, *e_w;
  int32_t *order, *order2, *nstart, *nend, *split, *knn_pos, *parent, *comp, *node_comp, *cand, *e_from, *e_to,
      *counters;
  uint8_t* leaf;
  uint64_t *keys, *keys2;
  uint32_t* bound;
  unsigned long long* best;
  const int kq = min_samples > 1 ? min_samples + 1 : 2;
  const int64_t cap = n - 1;
  EVOC_TRY(A.get(&Xp, size_t(n) * P), "alloc points");
  EVOC_TRY(A.get(&pts, size_t(n) * P), "alloc points");
  EVOC_TRY(A.get(&lo, size_t(n_nodes) * P), "alloc bounds");
  EVOC_TRY(A.get(&hi, size_t(n_nodes) * P), "alloc bounds");
  EVOC_TRY(A.get(&order, size_t(n)), "alloc order");
  EVOC_TRY(A.get(&order2, size_t(n)), "alloc order");
  EVOC_TRY(A.get(&keys, size_t(n)), "alloc keys");
  EVOC_TRY(A.get(&keys2, size_t(n)), "alloc keys");
  EVOC_TRY(A.get(&nstart, size_t(n_nodes)), "alloc nodes");
  EVOC_TRY(A.get(&nend, size_t(n_nodes)), "alloc nodes");
  EVOC_TRY(A.get(&split, size_t(n_nodes)), "alloc nodes");
  EVOC_TRY(A.get(&leaf, size_t(n_nodes)), "alloc nodes");
  EVOC_TRY(A.get(&node_comp, size_t(n_nodes)), "alloc nodes");
  EVOC_TRY(A.get(&core, size_t(n)), "alloc core");
  EVOC_TRY(A.get(&knn_pos, size_t(n) * kq), "alloc knn");
  EVOC_TRY(A.get(&knn_d, size_t(n) * kq), "alloc knn");
  EVOC_TRY(A.get(&parent, size_t(n)), "alloc components");
  EVOC_TRY(A.get(&comp, size_t(n)), "alloc components");
  EVOC_TRY(A.get(&cand, size_t(n)), "alloc components");
  EVOC_TRY(A.get(&bound, size_t(n)), "alloc components");
  EVOC_TRY(A.get(&best, size_t(n)), "alloc components");
  EVOC_TRY(A.get(&e_from, size_t(cap)), "alloc edges");
  EVOC_TRY(A.get(&e_to, size_t(cap)), "alloc edges");
  EVOC_TRY(A.get(&e_w, size_t(cap)), "alloc edges");
  EVOC_TRY(A.get(&counters, 16), "alloc counters");
  EVOC_TRY(cudaMemcpyAsync(nstart, hs.data(), hs.size() * 4, cudaMemcpyHostToDevice, st), "upload nodes");
  EVOC_TRY(cudaMemcpyAsync(nend, he.data(), he.size() * 4, cudaMemcpyHostToDevice, st), "upload nodes");
  EVOC_TRY(cudaMemcpyAsync(leaf, hl.data(), hl.size(), cudaMemcpyHostToDevice, st), "upload nodes");
  EVOC_TRY(cudaMemsetAsync(counters, 0, 64, st), "clear counters");
  int32_t* status = counters + 1;
  const int grid = sms * 8;
  {
    Stage s(ctx, "mst_tree");
    pad_points_kernel<<<grid, 256, 0, st>>>(d_x, n, dim, ldx, Xp, P);
    iota_kernel<<<grid, 256, 0, st>>>(order, n);
    EVOC_TRY(cudaGetLastError(), "pad points");
    ctx->launches += 2;
    size_t tmp_bytes = 0;
    EVOC_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys2, order, order2, int(n), 0, 64, st),
             "sort size");
    void* tmp = nullptr;
    EVOC_TRY(A.get(reinterpret_cast<uint8_t**>(&tmp), tmp_bytes), "alloc sort");
    for (int l = 0; l < n_levels; l++) {
      const int first = (1 << l) - 1, count = 1 << l;
      const bool last = l == n_levels - 1;
      node_bounds_kernel<P><<<std::min(count, sms * 16), 256, 0, st>>>(Xp, order, nstart, nend, first, count, dim,
                                                                       lo, hi, last ? nullptr : split);
      EVOC_TRY(cudaGetLastError(), "node bounds");
      ctx->launches += 1;
      if (last) break;
      split_keys_kernel<<<grid, 256, 0, st>>>(Xp, P, order, n, nstart, first, count, split, keys);
      int end_bit = 32;
      while ((1 << (end_bit - 32)) < count) end_bit++;
      EVOC_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys2, order, order2, int(n), 0, end_bit, st),
               "split sort");
      std::swap(order, order2);
      ctx->launches += 2;
    }
    gather_points_kernel<P><<<grid, 256, 0, st>>>(Xp, order, n, pts);
    EVOC_TRY(cudaGetLastError(), "gather points");
    ctx->launches += 1;
  }
  const TreeView tv{n, n_nodes, order, pts, nstart, nend, leaf, lo, hi};
  const int qgrid = int(std::min<int64_t>((n + 127) / 128, int64_t(sms) * 64));
  {
    Stage s(ctx, "mst_core");
    knn_kernel<P><<<qgrid, 128, 0, st>>>(tv, kq, core, knn_pos, knn_d, status);
    EVOC_TRY(cudaGetLastError(), "core distances");
    ctx->launches += 1;
  }
  if (min_samples <= 1) EVOC_TRY(cudaMemsetAsync(core, 0, size_t(n) * 4, st), "zero core");
  int32_t* e_count = counters;
  {
    Stage s(ctx, "mst_init");
    iota_kernel<<<grid, 256, 0, st>>>(parent, n);
    knn_init_kernel<<<grid, 256, 0, st>>>(n, kq, core, knn_pos, knn_d, parent, e_from, e_to, e_w, e_count, cap);
    EVOC_TRY(cudaGetLastError(), "knn init");
    ctx->launches += 2;
  }
  int32_t h[2] = {0, 0};
  Stage rounds(ctx, "mst_rounds");
  for (int round = 0;; round++) {
    EVOC_TRY(cudaMemcpyAsync(h, counters, 8, cudaMemcpyDeviceToHost, st), "read edge count");
    EVOC_TRY(cudaStreamSynchronize(st), "mst round");
    if (h[1] != 0) return fail(ctx, EVOC_ERR_CUDA, "tree traversal stack overflow");
    if (h[0] >= cap) break;
    if (round > 64) return fail(ctx, EVOC_ERR_CUDA, "Boruvka did not converge");
    const int32_t before = h[0];
    components_kernel<<<grid, 256, 0, st>>>(n, parent, comp);
    const int leaf_first = (1 << (n_levels - 1)) - 1;
    leaf_components_kernel<<<(leaf_first + 1 + 255) / 256, 256, 0, st>>>(tv, leaf_first, leaf_first + 1, comp,
                                                                          node_comp);
    for (int l = n_levels - 2; l >= 0; l--) {
      const int first = (1 << l) - 1, count = 1 << l;
      // leaves above the last level (ranges of fewer than two points) first
      leaf_components_kernel<<<(count + 255) / 256, 256, 0, st>>>(tv, first, count, comp, node_comp);
      inner_components_kernel<<<(count + 255) / 256, 256, 0, st>>>(tv, first, count, node_comp);
    }
    reset_round_kernel<<<grid, 256, 0, st>>>(n, bound, best);
    boruvka_query_kernel<P><<<qgrid, 128, 0, st>>>(tv, core, comp, node_comp, bound, best, cand, status);
    boruvka_merge_kernel<<<grid, 256, 0, st>>>(n, comp, best, cand, parent, e_from, e_to, e_w, e_count, cap);
    EVOC_TRY(cudaGetLastError(), "boruvka round");
    ctx->launches += 5 + 2 * (n_levels - 1);
    EVOC_TRY(cudaMemcpyAsync(h, counters, 8, cudaMemcpyDeviceToHost, st), "read edge count");
    EVOC_TRY(cudaStreamSynchronize(st), "mst round");
    if (h[0] == before && h[0] < cap) return fail(ctx, EVOC_ERR_CUDA, "a Boruvka round joined no components");
  }
  rounds.end();
  *n_edges = cap;
  emit_edges_kernel<<<grid, 256, 0, st>>>(cap, order, e_from, e_to, e_w, d_edges);
  if (d_core) scatter_core_kernel<<<grid, 256, 0, st>>>(n, order, core, d_core);
  EVOC_TRY(cudaGetLastError(), "emit edges");
  ctx->launches += d_core ? 2 : 1;
  return EVOC_OK;
}

int boruvka_impl(evoc_gpu_ctx* ctx, const float* data, int64_t n, int32_t dim, int32_t min_samples, int32_t on_dev,
                 float* out_edges, float* out_core, int64_t* n_edges) {
  if (!ctx) return EVOC_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  ctx->err.clear();
  ctx->n_stages = 0;
  ctx->launches = 0;
  if (n_edges) *n_edges = 0;
  if (n <= 0) return fail(ctx, EVOC_ERR_EMPTY, "no points");
  if (!data || (n > 1 && !out_edges)) return fail(ctx, EVOC_ERR_ARG, "null data or out_edges");
  if (dim < 1 || dim > 32) return fail(ctx, EVOC_ERR_ARG, "dim must be in 1..32");
  if (min_samples < 0 || min_samples + 1 > kMaxKnn) return fail(ctx, EVOC_ERR_ARG, "min_samples must be in 0..31");
  if (n >= (int64_t(1) << 31) - 1) return fail(ctx, EVOC_ERR_ARG, "n exceeds the int32 index range");
  const int kq = min_samples > 1 ? min_samples + 1 : 2;
  if (n < kq) return fail(ctx, EVOC_ERR_ARG, "need more than min_samples points (the core distance is undefined)");
  EVOC_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
  if (!ctx->lp_pool) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = ctx->device;
    EVOC_TRY(cudaMemPoolCreate(&ctx->lp_pool, &props), "memory pool");
    uint64_t keep = UINT64_MAX;
    EVOC_TRY(cudaMemPoolSetAttribute(ctx->lp_pool, cudaMemPoolAttrReleaseThreshold, &keep), "memory pool");
  }
  Stage total(ctx, "total");
  int rc = EVOC_OK;
  {
    Arena A(ctx->stream, ctx->lp_pool);
    const float* d_x = data;
    float *d_edges = out_edges, *d_core = out_core;
    if (!on_dev) {
      float* xs;
      EVOC_TRY(A.get(&xs, size_t(n) * size_t(dim)), "alloc points");
      EVOC_TRY(cudaMemcpyAsync(xs, data, size_t(n) * size_t(dim) * 4, cudaMemcpyHostToDevice, ctx->stream),
               "upload points");
      d_x = xs;
      EVOC_TRY(A.get(&d_edges, size_t(std::max<int64_t>(n - 1, 1)) * 3), "alloc edges");
      d_core = nullptr;
      if (out_core) EVOC_TRY(A.get(&d_core, size_t(n)), "alloc core");
    }
    int64_t ne = 0;
    if (n == 1) {
      if (d_core) EVOC_TRY(cudaMemsetAsync(d_core, 0, 4, ctx->stream), "core");
    } else if (dim <= 4) {
      rc = run<4>(ctx, A, d_x, n, dim, dim, min_samples, d_edges, d_core, &ne);
    } else if (dim <= 8) {
      rc = run<8>(ctx, A, d_x, n, dim, dim, min_samples, d_edges, d_core, &ne);
    } else if (dim <= 16) {
      rc = run<16>(ctx, A, d_x, n, dim, dim, min_samples, d_edges, d_core, &ne);
    } else {
      rc = run<32>(ctx, A, d_x, n, dim, dim, min_samples, d_edges, d_core, &ne);
    }
    if (rc) return rc;
    if (!on_dev) {
      if (ne > 0)
        EVOC_TRY(cudaMemcpyAsync(out_edges, d_edges, size_t(ne) * 12, cudaMemcpyDeviceToHost, ctx->stream),
                 "download edges");
      if (out_core)
        EVOC_TRY(cudaMemcpyAsync(out_core, d_core, size_t(n) * 4, cudaMemcpyDeviceToHost, ctx->stream),
                 "download core");
    }
    if (n_edges) *n_edges = ne;
  }
  total.end();
  EVOC_TRY(cudaStreamSynchronize(ctx->stream), "boruvka");
  return EVOC_OK;
}

}  // namespace mst
}  // namespace evoc

extern "C" int evoc_gpu_boruvka_mst(evoc_gpu_ctx* ctx, const float* data, int64_t n, int32_t dim,
                                    int32_t min_samples, int32_t buffers_on_device, float* out_edges,
                                    float* out_core, int64_t* n_edges) {
  return evoc::mst::boruvka_impl(ctx, data, n, dim, min_samples, buffers_on_device, out_edges, out_core, n_edges);
}
