// Shared device/host helpers for the evoc kNN-graph engine (sm_100a).
//
// Distance conventions follow the evoc-rs kNN path:
//   f32  raw = -dot if dot > 0 else f32::MIN_POSITIVE        src/fast_cosine.rs:33-45
//   i8   raw = -(dot_i32 as f32)                               src/nndescent/int8.rs:15-21
//   u8   raw = -(inter/union) (f32 div), 0.0 if union == 0     src/nndescent/uint8.rs:21-35
//   self raw = -1.0 (leaf-init rule)                           src/nndescent/float.rs:209-215
// Rows are ranked by the total order (raw, index) with f32 equality
// (-0.0 == +0.0), smallest first.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace evoc {

constexpr float kMinPositive = 1.17549435e-38f;  // f32::MIN_POSITIVE
constexpr float kHeapInf = 3.40282347e+38f;      // f32::MAX, heap.rs:8
constexpr uint64_t kKeyInf = ~0ull;

// Codes of a request's device status word (0 = ok).  1..3: a pipeline wait of
// the tensor-core scan ran out (producer, MMA issuer, epilogue); 16, 17: a
// self-check found a malformed row order or a candidate index out of range
// and skipped it.
constexpr int kStatusBadOrder = 16;
constexpr int kStatusBadCandidate = 17;

// Order-preserving map f32 -> u32 (after folding -0.0 onto +0.0).
__device__ __forceinline__ uint32_t orderable(float f) {
  f = f + 0.0f;  // -0.0 + 0.0 == +0.0 under round-to-nearest
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float from_orderable(uint32_t o) {
  uint32_t u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
  return __uint_as_float(u);
}

__device__ __forceinline__ uint64_t make_key(float raw, int32_t idx) {
  return (uint64_t(orderable(raw)) << 32) | uint32_t(idx);
}

__host__ __device__ __forceinline__ int32_t key_index(uint64_t key) { return int32_t(uint32_t(key)); }

__device__ __forceinline__ float raw_cosine(float dot) { return dot > 0.0f ? -dot : kMinPositive; }

__device__ __forceinline__ float raw_int8(int32_t dot) { return -__int2float_rn(dot); }

__device__ __forceinline__ float raw_jaccard(uint32_t inter, uint32_t uni) {
  return uni > 0 ? -__fdiv_rn(__uint2float_rn(inter), __uint2float_rn(uni)) : 0.0f;
}

// Ordering keys fold -0.0 onto +0.0.  An int8 dissimilarity of zero is
// -(0 as f32) = -0.0 in the reference, so the writer restores that sign.
__device__ __forceinline__ float int8_raw_from_key(float r) { return r == 0.0f ? -0.0f : r; }

// Distance transforms, src/knn.rs:156-187 (f64 log2 for f32/u8, f32 division for i8).
__device__ __forceinline__ float transform_raw(int dtype, float d) {
  if (dtype == 0) {
    if (d >= 0.0f) return 0.0f;
    double sim = double(-d);
    if (sim >= 1.0) return 0.0f;
    return float(fmax(-log2(sim), 0.0));
  } else if (dtype == 1) {
    return d >= 0.0f ? 0.0f : __fdiv_rn(1.0f, -d);
  } else {
    return d >= 0.0f ? 0.0f : float(-log2(double(-d)));
  }
}

// ---------------------------------------------------------------------------
// Thread-private candidate buffer: one owner thread per query row appends
// keys that beat its current threshold; when the buffer is full it keeps the
// k smallest (nth-element) and the k-th becomes the new threshold.  The final
// answer depends only on the set of keys offered, so it is deterministic.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void kswap(uint64_t* a, int i, int j) {
  uint64_t t = a[i];
  a[i] = a[j];
  a[j] = t;
}

// Rearranges buf[0..cnt) so that buf[0..k) hold the k smallest keys and
// buf[k-1] is the largest of them.  Requires 1 <= k <= cnt.
__device__ inline void nth_smallest(uint64_t* buf, int cnt, int k) {
  int lo = 0, hi = cnt - 1;
  const int target = k - 1;
  while (hi > lo) {
    int mid = lo + ((hi - lo) >> 1);
    // median-of-three pivot into buf[hi]
    if (buf[mid] < buf[lo]) kswap(buf, mid, lo);
    if (buf[hi] < buf[lo]) kswap(buf, hi, lo);
    if (buf[mid] < buf[hi]) kswap(buf, mid, hi);
    uint64_t pivot = buf[hi];
    int store = lo;
    for (int i = lo; i < hi; i++) {
      uint64_t v = buf[i];
      if (v < pivot) {
        buf[i] = buf[store];
        buf[store] = v;
        store++;
      }
    }
    kswap(buf, store, hi);
    if (store == target) return;
    if (store < target) lo = store + 1;
    else hi = store - 1;
  }
}

__device__ inline void sort_keys(uint64_t* buf, int cnt) {
  for (int i = 1; i < cnt; i++) {
    uint64_t v = buf[i];
    int j = i - 1;
    while (j >= 0 && buf[j] > v) {
      buf[j + 1] = buf[j];
      j--;
    }
    buf[j + 1] = v;
  }
}

struct RowTopK {
  uint64_t* buf;  // CAP entries, private to the owner thread
  int cnt;
  int k;
  int cap;
  uint64_t thr;   // keys >= thr cannot enter
  float thr_raw;  // raw part of thr (quick reject)

  __device__ __forceinline__ void init(uint64_t* b, int kk, int capacity) {
    buf = b;
    cnt = 0;
    k = kk;
    cap = capacity;
    thr = kKeyInf;
    thr_raw = __int_as_float(0x7f800000);  // +inf
  }

  __device__ __forceinline__ void compact() {
    nth_smallest(buf, cnt, k);
    cnt = k;
    thr = buf[k - 1];
    thr_raw = from_orderable(uint32_t(thr >> 32));
  }

  // Offer (raw, idx).  raw must not be NaN.
  __device__ __forceinline__ void offer(float raw, int32_t idx) {
    if (raw > thr_raw) return;
    uint64_t key = make_key(raw, idx);
    if (key >= thr) return;
    buf[cnt++] = key;
    if (cnt == cap) compact();
  }

  // Sorts and returns the number of valid entries (min(cnt, k)).
  __device__ __forceinline__ int finish() {
    if (cnt > k) compact();
    sort_keys(buf, cnt);
    return cnt;
  }
};

}  // namespace evoc

namespace evoc {

// ---------------------------------------------------------------------------
// Thread-private bounded max-heap of ordering keys (one owner thread per query
// row).  Holds the `cap` smallest keys offered so far; its root is the exact
// cap-th best, so it is also the admission threshold.  The storage may be
// shared memory (row stride chosen odd in 8-byte words, so the 32 owners of a
// warp touching the same slot hit distinct banks) or global memory.
// ---------------------------------------------------------------------------
struct KeyHeap {
  uint64_t* h;
  int size;
  int cap;

  __device__ __forceinline__ void init(uint64_t* storage, int capacity) {
    h = storage;
    size = 0;
    cap = capacity;
  }

  __device__ __forceinline__ uint64_t threshold() const { return size < cap ? kKeyInf : h[0]; }

  __device__ inline void sift_down(int e) {
    const uint64_t v = h[e];
    for (;;) {
      int c = 2 * e + 1;
      if (c >= cap) break;
      uint64_t cv = h[c];
      if (c + 1 < cap) {
        const uint64_t r = h[c + 1];
        if (r > cv) {
          cv = r;
          c++;
        }
      }
      if (cv <= v) break;
      h[e] = cv;
      e = c;
    }
    h[e] = v;
  }

  // Keys are unique (they embed the row index), so a strict compare suffices.
  __device__ inline void offer(uint64_t key) {
    if (size < cap) {
      h[size++] = key;
      if (size == cap)
        for (int e = cap / 2 - 1; e >= 0; e--) sift_down(e);
      return;
    }
    if (key >= h[0]) return;
    h[0] = key;
    sift_down(0);
  }

  // Sorts ascending in place (insertion sort; cap is small) and returns the count.
  __device__ inline int finish() {
    sort_keys(h, size);
    return size;
  }
};

}  // namespace evoc
