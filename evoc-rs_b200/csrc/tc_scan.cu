// Tensor-core exact scan with the top-k selection fused into the epilogue.
//
// One persistent CTA per SM walks 128-row query blocks; for each it streams
// every 256-row key tile through a 4-stage shared-memory pipeline and
// multiplies on the 5th-generation tensor cores (tcgen05.mma, M=128, N=256,
// FP16 or BF16 -> F32, or S8 -> S32), accumulating in TMEM.  Two accumulators let the
// epilogue read tile t while the MMAs of tile t+1 run.  Nothing of the n x n
// score matrix is written to HBM: each epilogue thread owns one query row,
// reads its 256 scores straight from TMEM and offers the few that beat its
// row threshold to a thread-private candidate buffer (common.cuh).
//
// Warp roles (192 threads):
//   warp 0      TMA producer (one elected lane, no multicast)
//   warp 1      TMEM allocator + MMA issuer (one elected lane)
//   warps 2..5  epilogue; warp w reads TMEM lanes 32*(w%4) .. +31
//
// CTA-pair variants (cluster of 2, tcgen05 cta_group::2): the two CTAs take
// two neighbouring query blocks (256 rows) through one M = 256 MMA per key
// tile.  Each CTA loads its own 128 query rows and half of the 256-row key
// tile (128 rows) -- 32 KB per pipeline stage instead of 48 KB, a third less
// L2-to-SM traffic per product -- and the leader CTA issues the MMAs, whose
// 256 x 256 product lands as 128 x 256 in each CTA's TMEM.  Both CTAs'
// loads complete on the leader's stage barrier; the leader's commits arrive
// on both CTAs' stage-free and accumulator-ready barriers; both CTAs'
// epilogues arrive on the leader's accumulator-free barrier.
//
// Symmetric mode (opt-in; sym.cu has the pre-scan, thresholds and merge):
// all rows are queries and keys, in a permuted order (pivot groups side by
// side); query block b multiplies only the key tiles from its own rows on,
// its own tile first and then the rest from the last tile down.  A score for
// a key row past the block also counts for that row: if it reaches the row's
// mailbox threshold it is staged in shared memory and appended to the row's
// mailbox in HBM, 64 keys per warp at a time.
//
// Three score modes share the kernel: 16-bit float dot products (cosine; FP16
// or BF16 operands, the same instruction and rate), int8 dot products, and
// binary Jaccard, where the packed bits are expanded to 0/1
// int8 rows so that the intersection popcount is an exact s8 x s8 -> s32
// contraction; the epilogue then forms -(inter / union) with union =
// |a| + |b| - inter from per-row popcounts, as the reference does
// (src/nndescent/uint8.rs:21-35).
//
// Replaces the distance evaluations of the reference's NN-descent local join
// (src/nndescent/float.rs:552-660 with fast_cosine, src/fast_cosine.rs:33-45;
// src/nndescent/int8.rs:15-21 for the int8 dissimilarity).
#include <algorithm>
#include <cstring>
#include <cuda.h>
#include <cudaTypedefs.h>

#include "batch.h"
#include "common.cuh"
#include "kernels.h"
#include "sm100.cuh"

namespace evoc {

namespace {
constexpr int BM = 128;              // query rows per block (TMEM lanes)
constexpr int BN = 256;              // key rows per tile (accumulator columns)
constexpr int KCB = 128;             // bytes of K per pipeline stage (one 128B swizzle span)
constexpr int A_BYTES = BM * KCB;    // 16 KB
constexpr int B_BYTES = BN * KCB;    // 32 KB
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int PAIR_STAGE_BYTES = A_BYTES + B_BYTES / 2;  // a CTA of a pair: its query rows and half the key tile
constexpr int TMEM_COLS = 2 * BN;    // two f32/s32 accumulators
constexpr size_t SMEM_LIMIT = 232448;      // 227 KB opt-in maximum per block
constexpr size_t SMEM_FIXED = 1024 /*align*/ + 256 /*barriers*/;
constexpr uint64_t kDrainNs = 4000000000ull;  // limit of the drain waits whatever the pipeline limit

// Shared memory for a pipeline depth, a number of epilogue warp groups (each
// with one heap per row) and a heap stride (0: heaps in global memory).
constexpr size_t smem_bytes(int stages, int groups, int heap_stride, bool pair = false) {
  return size_t(stages) * (pair ? PAIR_STAGE_BYTES : STAGE_BYTES) + size_t(groups) * BM * size_t(heap_stride) * 8 +
         SMEM_FIXED;
}
}  // namespace

struct ScanParams {
  int64_t n_q, n_k;  // query rows taken (starting at q_row0 of Q), key rows
  int64_t q_row0;    // first query row; query i is row q_row0 + i of Q (and key q_row0 + i)
  int n_kchunks;     // 128-byte K chunks per row
  int keep;          // entries kept per query row (the heap size)
  int heap_stride;   // 8-byte words between rows' heaps (odd when heaps are in shared memory)
  uint64_t* scratch; // gridDim.x * BM * keep keys, used when heaps are in global memory
  int self_mode;     // 1: query row i is key row i (offer self with raw -1.0, skip it in the scan)
  int final_mode;    // 1: write sorted idx/raw/transformed dist; 0: write candidates (idx, raw)
  int dtype;         // distance transform for final_mode
  int32_t* out_idx;
  float* out_raw;
  float* out_dist;
  int* status;       // 0 ok; set non-zero by the first role that gives up
  uint64_t timeout_ns;  // limit of each pipeline wait (settable per context)
  uint64_t drain_ns;    // limit of the waits for loads and MMAs already issued (never shorter than 4 s)
  uint64_t delay_ns;    // tests of the timeout path: the producer starts this late (0 in normal use)
  const int32_t* pc; // Jaccard mode: popcount of every row (queries and keys)
  int half_type;     // 16-bit mode: kHalfF16 or kHalfBf16 operands
  const int32_t* q_self;  // optional: key index of query i is q_self_base + q_self[i] (gathered query rows)
  int64_t q_self_base;
  float* out_bound;  // optional: raw value of the keep-th kept key of each query
  // Symmetric mode (queries = keys = all rows, self rule): query block b
  // multiplies only key tiles from its own rows on; a score counts for its
  // query row (own side) and, for key rows past the block, for the key row
  // too (mirror side): a score reaching sym_thr[key] is appended to the key
  // row's mailbox, which a merge folds into the row's kept keys afterwards.
  const float* sym_thr;   // per key row, padded to whole tiles with +inf: the mirror side's score threshold
  const float* sym_umin;  // per 32 key rows: the smallest of their thresholds (quick reject)
  int32_t* sym_count;     // per row: mirror keys offered (beyond sym_cap the row's mailbox overflowed)
  uint64_t* sym_mail;     // per row: sym_cap keys
  int sym_cap;
  // The rows are scanned in a permuted order (rows of one pivot group side by
  // side, so that a chunk's key rows have similar thresholds and the quick
  // reject works): scanned row i is row sym_perm[i] of the data set (padded
  // to whole tiles).  Keys, outputs and mailboxes use data-set rows;
  // sym_thr / sym_umin follow the scanned order.
  const int32_t* sym_perm;
  // Batch mode: the work-list of (request, query block) items and the
  // requests' tensor maps and parameters, all in device memory.
  const ScanJob* jobs;
  const ScanItem* items;
  const int32_t* n_items;
};

namespace {

__device__ __forceinline__ void set_status(int* status, int code) { atomicCAS(status, 0, code); }

constexpr int kModeHalf = 0;     // FP16 / BF16 dot products, cosine dissimilarity
constexpr int kModeInt8 = 1;     // int8 dot products, -(dot as f32)
constexpr int kModeJaccard = 2;  // 0/1 int8 rows: intersection counts, -(inter / union)

// Quick-reject threshold as the raw 32-bit score pattern the accumulator holds:
// a score below it cannot enter the heap.  For int8 it is an s32 lower bound
// (exact while |dot| < 2^24, loosened by 256 beyond, where f32 rounds); for
// 16-bit float operands it is an f32.  For Jaccard it is a lower bound on the intersection:
// J = inter / (pa + pb - inter) <= inter / pa, so a key reaching the heap's
// similarity t needs inter >= t * pa (taken 1e-6 looser so f32 rounding of J
// never rejects a key the exact compare would admit).  Passing scores are
// re-checked exactly by the key compare.
// Integer scores are below 2^29 in magnitude (int8 dots for rows of fewer than
// 33,000 bytes, intersection counts), so the "admit everything" threshold
// -2^30 keeps score - threshold free of overflow.
constexpr int32_t kIntOpen = -(1 << 30);

template <int MODE>
__device__ __forceinline__ uint32_t pass_threshold(const KeyHeap& heap, int32_t pa) {
  const uint64_t t = heap.threshold();
  if (MODE == kModeInt8) {
    if (t == kKeyInf) return uint32_t(kIntOpen);
    const float ts = -from_orderable(uint32_t(t >> 32));  // raw = -score
    int32_t ti = int32_t(ts);
    if (!(fabsf(ts) < 16777216.0f)) ti -= 256;
    return uint32_t(ti);
  }
  if (MODE == kModeJaccard) {
    if (t == kKeyInf) return uint32_t(kIntOpen);
    const float sim = -from_orderable(uint32_t(t >> 32));  // raw = -J (or +0.0 for J = 0)
    if (!(sim > 0.0f)) return uint32_t(kIntOpen);
    return uint32_t(int32_t(floorf(sim * float(pa) * (1.0f - 1e-6f))));
  }
  const uint32_t NEG_INF = 0xff800000u;
  if (t == kKeyInf) return NEG_INF;
  const float raw = from_orderable(uint32_t(t >> 32));
  return raw < 0.0f ? __float_as_uint(-raw) : NEG_INF;  // raw = -score, or MIN_POSITIVE for scores <= 0
}

// The threshold with a row's seed (16-bit scores only; -inf: none): a score
// below the seed provably cannot be among the row's kept keys, so the heap
// admits only scores reaching both.
template <int MODE>
__device__ __forceinline__ uint32_t seeded(uint32_t thr, float seed) {
  return MODE == kModeHalf ? __float_as_uint(fmaxf(__uint_as_float(thr), seed)) : thr;
}

template <int MODE>
__device__ __forceinline__ bool passes(uint32_t v, uint32_t thr) {
  return MODE != kModeHalf ? (int32_t(v) >= int32_t(thr)) : (__uint_as_float(v) >= __uint_as_float(thr));
}

// Jaccard dissimilarity from exact counts, as the reference computes it.
__device__ __forceinline__ float jaccard_raw_counts(int32_t inter, int32_t uni) {
  return uni > 0 ? -__fdiv_rn(__int2float_rn(inter), __int2float_rn(uni)) : 0.0f;
}

// Column j of a chunk's 32 values: a five-level select tree (31 selects,
// dependency depth 5) instead of a 32-deep chain.
__device__ __forceinline__ uint32_t pick(const uint32_t (&v)[32], int j) {
  uint32_t s[16];
#pragma unroll
  for (int i = 0; i < 16; i++) s[i] = (j & 16) ? v[i + 16] : v[i];
#pragma unroll
  for (int i = 0; i < 8; i++) s[i] = (j & 8) ? s[i + 8] : s[i];
#pragma unroll
  for (int i = 0; i < 4; i++) s[i] = (j & 4) ? s[i + 4] : s[i];
#pragma unroll
  for (int i = 0; i < 2; i++) s[i] = (j & 2) ? s[i + 2] : s[i];
  return (j & 1) ? s[1] : s[0];
}

// Offers the scores of one 32-column chunk that beat the threshold.  The
// chunk's values stay in registers; a survivor's value is picked by a select
// tree (survivors are rare once the heap is full).  Bit 31 - j of `mask`
// stands for column j (the order chunk_mask builds).
template <int MODE>
__device__ __forceinline__ void offer_chunk(const uint32_t (&v)[32], uint32_t mask, int64_t col0, int64_t n_k,
                                            bool self_mode, int64_t q, KeyHeap& heap, uint32_t& thr, int32_t pa,
                                            const int32_t* __restrict__ pc, const int32_t* ids = nullptr,
                                            float seed = -__builtin_huge_valf()) {
  while (mask) {
    const int j = __clz(mask);
    mask &= ~(0x80000000u >> j);
    const uint32_t bits = pick(v, j);
    if (!passes<MODE>(bits, thr)) continue;  // threshold may have moved
    const int64_t key = col0 + j;
    if (key >= n_k || (self_mode && key == q)) continue;
    float raw;
    if (MODE == kModeJaccard) {
      const int32_t inter = int32_t(bits);
      raw = jaccard_raw_counts(inter, pa + pc[key] - inter);
    } else {
      raw = MODE == kModeInt8 ? -__int2float_rn(int32_t(bits)) : raw_cosine(__uint_as_float(bits));
    }
    heap.offer(make_key(raw, ids ? ids[j] : int32_t(key)));  // ids: the chunk's row indices of the data set
    thr = seeded<MODE>(pass_threshold<MODE>(heap, pa), seed);
  }
}

// Pass mask of a 32-column chunk, bit 31 - j for column j.  Two instructions
// per score: the sign of (score - threshold) -- an integer subtraction, or an
// f32 subtraction on the FMA pipe for BF16 -- is funnel-shifted into one of
// four independent accumulators (short dependency chains), then inverted.
// Equal scores pass (their difference is +0), as `passes` admits them.
// Largest of 32 signed integers by three-input max (16 instructions).
__device__ __forceinline__ int32_t max32_s32(const uint32_t (&v)[32]) {
  int32_t m[11];
#pragma unroll
  for (int i = 0; i < 10; i++) m[i] = __vimax3_s32(int32_t(v[3 * i]), int32_t(v[3 * i + 1]), int32_t(v[3 * i + 2]));
  m[10] = max(int32_t(v[30]), int32_t(v[31]));
  const int32_t a = __vimax3_s32(m[0], m[1], m[2]), b = __vimax3_s32(m[3], m[4], m[5]),
                c = __vimax3_s32(m[6], m[7], m[8]), d = max(m[9], m[10]);
  return max(__vimax3_s32(a, b, c), d);
}

// Whether any score of the chunk passes: a max tree (independent at each
// level) and one compare.  Once a row's heap is full most chunks fail here
// and skip the per-column mask.  Not for Jaccard: its intersection bound is
// loose enough that the pre-check passes too often to pay for itself.
template <int MODE>
__device__ __forceinline__ bool chunk_any(const uint32_t (&v)[32], uint32_t thr) {
  if (MODE == kModeJaccard) return true;
  if (MODE != kModeHalf) return max32_s32(v) >= int32_t(thr);
  // 16-bit float scores: against a positive threshold the bit patterns as
  // signed integers order as the floats do (a negative score is a negative
  // integer, below any positive threshold), so the integer max tree serves.
  if (int32_t(thr) > 0) return max32_s32(v) >= int32_t(thr);
  float m[16];
#pragma unroll
  for (int j = 0; j < 16; j++) m[j] = fmaxf(__uint_as_float(v[j]), __uint_as_float(v[j + 16]));
#pragma unroll
  for (int w = 8; w > 0; w >>= 1)
#pragma unroll
    for (int j = 0; j < w; j++) m[j] = fmaxf(m[j], m[j + w]);
  return m[0] >= __uint_as_float(thr);
}

template <int MODE>
__device__ __forceinline__ uint32_t chunk_mask(const uint32_t (&v)[32], uint32_t thr) {
  uint32_t f[4] = {0u, 0u, 0u, 0u};  // fail bits
#pragma unroll
  for (int j = 0; j < 32; j++) {
    const uint32_t d = MODE != kModeHalf ? uint32_t(int32_t(v[j]) - int32_t(thr))
                                         : __float_as_uint(__uint_as_float(v[j]) - __uint_as_float(thr));
    f[j >> 3] = __funnelshift_l(d, f[j >> 3], 1);  // (f << 1) | sign(d)
  }
  return ~((f[0] << 24) | (f[1] << 16) | (f[2] << 8) | f[3]);
}

// Symmetric mode, mirror side.  The keys for later rows wait in a per-warp
// shared-memory stage and go to the mailboxes kMirrorStage at a time: one
// round trip of the global atomics per flush, both halves' atomics issued
// before either store, instead of one per chunk.
constexpr int kMirrorStage = 64;
constexpr size_t kMirrorStageBytes = size_t(kMirrorStage) * 12;  // keys, then rows
// Each epilogue warp also holds two tiles' mailbox thresholds (256), their
// per-32 minima (8) and the data-set rows of the tile's keys (256), copied
// one tile ahead by cp.async: a global load inside the chunk loop would stall
// the warp for an L2 round trip.
constexpr int kTileThr = BN + BN / 32 + BN;
constexpr int kTileIds = BN + BN / 32;  // offset of the row ids in a tile buffer (words)
constexpr size_t kMirrorWarpBytes = kMirrorStageBytes + 2 * kTileThr * 4;

struct MirrorStage {
  uint64_t* key;
  int32_t* row;
  int n;
};

__device__ __forceinline__ void mirror_flush(MirrorStage& st, int lane, const ScanParams& p) {
  int s0 = -1, s1 = -1;
  int32_t c0 = 0, c1 = 0;
  if (lane < st.n) {
    c0 = st.row[lane];
    s0 = atomicAdd(p.sym_count + c0, 1);
  }
  if (lane + 32 < st.n) {
    c1 = st.row[lane + 32];
    s1 = atomicAdd(p.sym_count + c1, 1);
  }
  if (s0 >= 0 && s0 < p.sym_cap) p.sym_mail[int64_t(c0) * p.sym_cap + s0] = st.key[lane];
  if (s1 >= 0 && s1 < p.sym_cap) p.sym_mail[int64_t(c1) * p.sym_cap + s1] = st.key[lane + 32];
  __syncwarp();
  st.n = 0;
}

// One 32-column chunk of query row r (warp-collective: every lane of the warp
// calls it, rows past n_q with valid = false).  Scores reaching their key
// rows' thresholds (th) are staged for those rows (ids: data-set rows; r is
// one too).  mx is the chunk's largest score as a
// signed integer (against a positive threshold the float bit patterns order
// as integers); umin the loosest threshold of the chunk's key rows.
__device__ __forceinline__ void mirror_chunk(const uint32_t (&v)[32], int32_t mx, float umin, const float* th,
                                             const int32_t* ids, int64_t col, int64_t n_k, int32_t r, bool valid,
                                             MirrorStage& st, int lane, const ScanParams& p) {
  const bool maybe = valid && !(umin > 0.0f && mx < __float_as_int(umin));
  if (!__any_sync(0xffffffffu, maybe)) return;
  uint32_t mask = 0;
  if (maybe) {
    const float4* t4 = reinterpret_cast<const float4*>(th);  // the chunk's 32 thresholds (shared memory)
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const float4 t = t4[i];
      mask |= (__uint_as_float(v[4 * i]) >= t.x ? 1u : 0u) << (4 * i);
      mask |= (__uint_as_float(v[4 * i + 1]) >= t.y ? 1u : 0u) << (4 * i + 1);
      mask |= (__uint_as_float(v[4 * i + 2]) >= t.z ? 1u : 0u) << (4 * i + 2);
      mask |= (__uint_as_float(v[4 * i + 3]) >= t.w ? 1u : 0u) << (4 * i + 3);
    }
    if (col + 32 > n_k) mask &= col >= n_k ? 0u : (1u << (n_k - col)) - 1u;  // padding thresholds are +inf anyway
  }
  const int cnt = __popc(mask);
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  const int total = __shfl_sync(0xffffffffu, incl, 31);
  if (total == 0) return;
  if (total > kMirrorStage) {  // more than a stage at once (many near-duplicate rows): straight to the mailboxes
    while (mask) {
      const int j = __ffs(mask) - 1;
      mask &= mask - 1;
      const int64_t c = ids[j];
      const uint64_t key = make_key(raw_cosine(__uint_as_float(pick(v, j))), r);
      const int slot = atomicAdd(p.sym_count + c, 1);
      if (slot < p.sym_cap) p.sym_mail[c * p.sym_cap + slot] = key;
    }
    __syncwarp();
    return;
  }
  if (st.n + total > kMirrorStage) mirror_flush(st, lane, p);
  int at = st.n + incl - cnt;
  while (mask) {
    const int j = __ffs(mask) - 1;
    mask &= mask - 1;
    st.key[at] = make_key(raw_cosine(__uint_as_float(pick(v, j))), r);
    st.row[at] = ids[j];
    at++;
  }
  __syncwarp();
  st.n += total;
}

// One work item as every role sees it: a 128-row query block of one request.
struct ItemView {
  const CUtensorMap* ma;
  const CUtensorMap* mb;
  int64_t qb, n_q, n_k, q_row0, n_ktiles;
  int64_t kt0;  // first key tile (symmetric mode: the tile holding the block's own rows)
  int n_kchunks, keep, self_mode, final_mode, dtype;
  int32_t* out_idx;
  float* out_raw;
  float* out_dist;
  const int32_t* pc;
  const int32_t* q_self;
  int64_t q_self_base;
  float* out_bound;
};

// Symmetric mode: block b multiplies n_ktiles - b/2 key tiles, so the work
// shrinks with b.  Items are dealt to the CTAs in rounds of gridDim.x, every
// other full round in reverse, so that each CTA's pair of rounds sums to the
// same work.
__device__ __forceinline__ int64_t sym_block(int64_t it, int64_t n_blocks) {
  const int64_t g = gridDim.x, round = it / g, pos = it % g;
  if ((round & 1) && (round + 1) * g <= n_blocks) return round * g + (g - 1 - pos);
  return it;
}

template <bool kBatch, bool kSym = false>
__device__ __forceinline__ ItemView item_view(const ScanParams& p, const CUtensorMap* tmA, const CUtensorMap* tmB,
                                              int64_t it) {
  ItemView v;
  if (kBatch) {
    const ScanItem si = p.items[it];
    const ScanJob* J = p.jobs + si.job;
    v.ma = &J->ma;
    v.mb = &J->mb;
    v.qb = si.qb;
    v.n_q = J->n_q;
    v.n_k = J->n_k;
    v.q_row0 = J->q_row0;
    v.n_kchunks = J->n_kchunks;
    v.keep = J->keep;
    v.self_mode = J->self_mode;
    v.final_mode = J->final_mode;
    v.dtype = J->dtype;
    v.out_idx = J->out_idx;
    v.out_raw = J->out_raw;
    v.out_dist = J->out_dist;
    v.pc = J->pc;
    v.q_self = nullptr;
    v.q_self_base = 0;
    v.out_bound = J->out_bound;
  } else {
    v.ma = tmA;
    v.mb = tmB;
    v.qb = kSym ? sym_block(it, (p.n_q + BM - 1) / BM) : it;
    v.n_q = p.n_q;
    v.n_k = p.n_k;
    v.q_row0 = p.q_row0;
    v.n_kchunks = p.n_kchunks;
    v.keep = p.keep;
    v.self_mode = p.self_mode;
    v.final_mode = p.final_mode;
    v.dtype = p.dtype;
    v.out_idx = p.out_idx;
    v.out_raw = p.out_raw;
    v.out_dist = p.out_dist;
    v.pc = p.pc;
    v.q_self = p.q_self;
    v.q_self_base = p.q_self_base;
    v.out_bound = p.out_bound;
  }
  v.n_ktiles = (v.n_k + BN - 1) / BN;
  v.kt0 = kSym ? v.qb * BM / BN : 0;
  return v;
}

// Tile ti of an item's sequence.  Symmetric mode: the tile of the block's
// own rows first (its nearest keys, so the heap's threshold tightens at
// once), then the rest from the last tile down: the CTAs of a round of items
// all start at the top and stream the same key tiles nearly in step, as in
// the plain scan, so each tile is read from HBM once and then from L2.
template <bool kSym>
__device__ __forceinline__ int64_t tile_at(const ItemView& v, int64_t ti) {
  return (kSym && ti > 0) ? v.n_ktiles - ti : v.kt0 + ti;
}

// A tensor map in global memory written before the launch: order the
// tensor-map proxy's reads after it.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(map))
               : "memory");
}

__device__ __forceinline__ void epilogue_sync(int nthreads) {
  asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

// Whether every epilogue thread finished the block (a barrier with an AND
// reduction over the same named barrier): the groups then stop, or fold their
// heaps, together.  Without it a warp that gave up on a wait could skip the
// fold barrier another group's warps wait at, and those would never return.
__device__ __forceinline__ bool epilogue_vote(int nthreads, bool ok) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.and.pred p, 1, %2, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(r)
      : "r"(uint32_t(ok ? 1 : 0)), "r"(nthreads)
      : "memory");
  return r != 0;
}

}  // namespace

template <int MODE, int STAGES, int GROUPS, bool kSmemHeap, bool kBatch, bool kPair = false, bool kSym = false>
__global__ void __launch_bounds__(64 + GROUPS * 128, 1)
tc_scan_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, const ScanParams p) {
  using namespace sm100;
  static_assert(!(kPair && kBatch), "CTA pairs run single requests");
  static_assert(!kSym || (MODE == kModeHalf && !kBatch && !kPair), "symmetric mode: 16-bit single requests");
  constexpr int SB = kPair ? PAIR_STAGE_BYTES : STAGE_BYTES;  // bytes of one stage in this CTA
  extern __shared__ uint8_t smem_dyn[];
  const uint32_t pad = (1024u - (smem_addr(smem_dyn) & 1023u)) & 1023u;
  uint8_t* smem = smem_dyn + pad;
  uint64_t* heaps = reinterpret_cast<uint64_t*>(smem + STAGES * SB);
  // Barriers follow every group's heaps (GROUPS x BM rows of heap_stride words).
  uint64_t* bars = kSmemHeap ? heaps + GROUPS * BM * p.heap_stride : heaps;
  uint64_t* full = bars;
  uint64_t* empty = bars + STAGES;
  uint64_t* tfull = bars + 2 * STAGES;
  uint64_t* tempty = bars + 2 * STAGES + 2;
  uint64_t* mma_done = bars + 2 * STAGES + 4;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 5);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = kPair ? cluster_rank() : 0u;  // 0: the leader (it issues the pair's MMAs)
  const bool leader = rank == 0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; a++) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], (kPair ? 2 : 1) * GROUPS * 128);  // a pair: both CTAs' epilogue threads
    }
    mbar_init(mma_done, 1);
    fence_barrier_init();
  }
  if (!kBatch && warp == 0 && lane == 0) {
    prefetch_tmap(&tmA);
    prefetch_tmap(&tmB);
  }
  if (warp == 1) {
    if (kPair) {
      tmem_alloc_pair(tmem_slot, TMEM_COLS);
      tmem_relinquish_pair();
    } else {
      tmem_alloc(tmem_slot, TMEM_COLS);
      tmem_relinquish();
    }
  }
  tc_fence_before();
  __syncthreads();
  if (kPair) cluster_sync();  // both CTAs' barriers are initialised before either signals the other's
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  constexpr bool kInt8 = MODE != kModeHalf;
  // Work items: query blocks (a pair: pairs of neighbouring blocks), strided
  // over the CTAs (the clusters).
  const int64_t n_blocks = kBatch ? int64_t(*p.n_items) : (p.n_q + BM - 1) / BM;
  const int64_t n_items = kPair ? (n_blocks + 1) / 2 : n_blocks;
  const int64_t item0 = kPair ? int64_t(blockIdx.x >> 1) : int64_t(blockIdx.x);
  const int64_t item_step = kPair ? int64_t(gridDim.x >> 1) : int64_t(gridDim.x);
  const volatile int* abort = p.status;
  constexpr int KC_ELEMS = kInt8 ? KCB : KCB / 2;
  constexpr int MM = kPair ? 2 * BM : BM;  // rows of one MMA
  const uint32_t IDESC = kInt8 ? idesc_s8_s32(MM, BN)
                               : (p.half_type == kHalfBf16 ? idesc_bf16_f32(MM, BN) : idesc_f16_f32(MM, BN));

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      if (p.delay_ns) {  // bounded: the host caps it
        const uint64_t t0 = globaltimer_ns();
        while (globaltimer_ns() - t0 < p.delay_ns) __nanosleep(1000);
      }
      uint32_t it = 0;
      bool ok = true;
      for (int64_t itm = item0; ok && itm < n_items; itm += item_step) {
        const ItemView v = item_view<kBatch, kSym>(p, &tmA, &tmB, kPair ? 2 * itm + rank : itm);
        if (kBatch) {
          tensormap_acquire(v.ma);
          tensormap_acquire(v.mb);
        }
        for (int64_t ti = 0; ok && ti < v.n_ktiles - v.kt0; ti++) {
          const int64_t kt = tile_at<kSym>(v, ti);
          for (int kc = 0; kc < v.n_kchunks; kc++) {
            const uint32_t s = it % STAGES, ph = (it / STAGES) & 1u;
            if (!mbar_wait(&empty[s], ph ^ 1u, abort, p.timeout_ns)) {
              set_status(p.status, 1);
              ok = false;
              break;
            }
            uint8_t* a_dst = smem + s * SB;
            if (kPair) {
              // both CTAs' bytes complete on the leader's barrier, armed by the leader for the two
              const uint32_t bar = mapa_shared(smem_addr(&full[s]), 0);
              if (leader) mbar_arrive_expect_tx(&full[s], 2 * SB);
              tma_load_2d_pair(a_dst, v.ma, bar, kc * KC_ELEMS, int32_t(v.q_row0 + v.qb * BM));
              tma_load_2d_pair(a_dst + A_BYTES, v.mb, bar, kc * KC_ELEMS, int32_t(kt * BN + rank * BM));
            } else {
              mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
              tma_load_2d(a_dst, v.ma, &full[s], kc * KC_ELEMS, int32_t(v.q_row0 + v.qb * BM));
              tma_load_2d(a_dst + A_BYTES, v.mb, &full[s], kc * KC_ELEMS, int32_t(kt * BN));
            }
            it++;
          }
        }
      }
      // Let the last loads land before the CTA can exit (full-length limit:
      // these loads were issued and complete on their own).  A pair's second
      // CTA cannot see the leader's barrier: it waits for the MMAs to release
      // its last stages instead, which they do only after reading them.
      for (uint32_t j = (it > STAGES ? it - STAGES : 0); j < it; j++) {
        if (!kPair || leader) mbar_wait(&full[j % STAGES], (j / STAGES) & 1u, nullptr, p.drain_ns);
        else mbar_wait(&empty[j % STAGES], (j / STAGES) & 1u, nullptr, p.drain_ns);
      }
    }
  } else if (warp == 1) {
    // ----------------------------------------------------------- MMA issuer
    if (lane == 0 && leader) {
      uint32_t it = 0, tile = 0;
      bool ok = true;
      for (int64_t itm = item0; ok && itm < n_items; itm += item_step) {
        const ItemView v = item_view<kBatch, kSym>(p, &tmA, &tmB, kPair ? 2 * itm : itm);
        for (int64_t ti = 0; ok && ti < v.n_ktiles - v.kt0; ti++, tile++) {
          const uint32_t a = tile & 1u, tph = (tile >> 1) & 1u;
          if (!mbar_wait(&tempty[a], tph ^ 1u, abort, p.timeout_ns)) {
            set_status(p.status, 2);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d_tmem = tmem_base + a * BN;
          for (int kc = 0; kc < v.n_kchunks; kc++) {
            const uint32_t s = it % STAGES, ph = (it / STAGES) & 1u;
            if (!mbar_wait(&full[s], ph, abort, p.timeout_ns)) {
              set_status(p.status, 2);
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t a_addr = smem_addr(smem + s * SB);
            const uint64_t adesc = sw128_kmajor_desc(a_addr);
            const uint64_t bdesc = sw128_kmajor_desc(a_addr + A_BYTES);
#pragma unroll
            for (int j = 0; j < KCB / 32; j++) {  // 32 bytes of K per instruction
              const uint32_t acc = (kc > 0 || j > 0) ? 1u : 0u;
              if (kPair) {
                if (kInt8) mma_i8_pair(d_tmem, adesc + 2 * j, bdesc + 2 * j, IDESC, acc);
                else mma_f16_pair(d_tmem, adesc + 2 * j, bdesc + 2 * j, IDESC, acc);
              } else {
                if (kInt8) mma_i8(d_tmem, adesc + 2 * j, bdesc + 2 * j, IDESC, acc);
                else mma_f16(d_tmem, adesc + 2 * j, bdesc + 2 * j, IDESC, acc);
              }
            }
            // stage is free (in both CTAs of a pair) once these MMAs have read it
            if (kPair) mma_commit_pair_mc(&empty[s], 3);
            else mma_commit(&empty[s]);
            it++;
          }
          if (!ok) break;
          // accumulator ready for the epilogue (both CTAs' TMEM)
          if (kPair) mma_commit_pair_mc(&tfull[a], 3);
          else mma_commit(&tfull[a]);
        }
      }
      // every MMA issued completes before TMEM is freed
      if (kPair) mma_commit_pair_mc(mma_done, 1);
      else mma_commit(mma_done);
      mbar_wait(mma_done, 0, nullptr, p.drain_ns);
    }
  } else {
    // -------------------------------------------------------------- epilogue
    // Epilogue warp e = warp - 2 reads TMEM lanes 32*(warp%4).. (its row
    // quadrant) and columns [group*BN/GROUPS, (group+1)*BN/GROUPS) of every tile.
    const int quad = warp & 3;
    const int group = (warp - 2) / 4;
    const int row_local = quad * 32 + lane;
    constexpr int NCH = BN / GROUPS / 32;  // 32-column chunks per tile per group
    const int col_base = group * (BN / GROUPS);
    const int heap_slot = group * BM + row_local;
    uint64_t* hstore = kSmemHeap ? heaps + int64_t(heap_slot) * p.heap_stride
                                 : p.scratch + (int64_t(blockIdx.x) * GROUPS * BM + heap_slot) * p.heap_stride;
    // a pair's second CTA frees the accumulator on the leader's barrier
    const uint32_t tempty_c0 = kPair ? mapa_shared(smem_addr(&tempty[0]), 0) : 0u;
    const uint32_t tempty_c1 = kPair ? mapa_shared(smem_addr(&tempty[1]), 0) : 0u;
    // symmetric mode: this warp's stage of mirror keys, after the barriers
    MirrorStage mst{nullptr, nullptr, 0};
    float* sthr = nullptr;  // two tiles' thresholds, minima and row ids (tile ti of an item in buffer ti & 1)
    if (kSym) {
      uint8_t* sb = reinterpret_cast<uint8_t*>(bars) + 256 + size_t(warp - 2) * kMirrorWarpBytes;
      mst.key = reinterpret_cast<uint64_t*>(sb);
      mst.row = reinterpret_cast<int32_t*>(sb + kMirrorStage * 8);
      sthr = reinterpret_cast<float*>(sb + kMirrorStageBytes);
    }
    // copy tile t's thresholds (64 x 16 bytes), minima (2 x 16 bytes) and row ids (64 x 16 bytes) to buffer b
    auto fetch_thr = [&](int64_t t, int64_t b) {
      float* dst = sthr + b * kTileThr;
      cp_async16(dst + lane * 4, p.sym_thr + t * BN + lane * 4);
      cp_async16(dst + 128 + lane * 4, p.sym_thr + t * BN + 128 + lane * 4);
      if (lane < 2) cp_async16(dst + BN + lane * 4, p.sym_umin + t * (BN / 32) + lane * 4);
      int32_t* ids = reinterpret_cast<int32_t*>(dst + kTileIds);
      cp_async16(ids + lane * 4, p.sym_perm + t * BN + lane * 4);
      cp_async16(ids + 128 + lane * 4, p.sym_perm + t * BN + 128 + lane * 4);
    };
    uint32_t tile = 0;
    bool ok = true;
    for (int64_t itm = item0; ok && itm < n_items; itm += item_step) {
      const ItemView v = item_view<kBatch, kSym>(p, &tmA, &tmB, kPair ? 2 * itm + rank : itm);
      const int64_t q = v.qb * BM + row_local;  // output row
      const bool valid = q < v.n_q;
      // row of the data set (its key index for the self rule)
      const int64_t qg = v.q_self ? (valid ? v.q_self_base + v.q_self[q] : -1) : v.q_row0 + q;
      // symmetric mode: qg is the scanned row, qd its row of the data set (keys and outputs)
      const int32_t qd = kSym ? (valid ? p.sym_perm[q] : -1) : int32_t(qg);
      KeyHeap heap;
      heap.init(hstore, v.keep);
      if (valid && v.self_mode && group == 0) heap.offer(make_key(-1.0f, qd));
      const int32_t pa = (MODE == kModeJaccard && valid) ? v.pc[qg] : 0;
      // symmetric mode: the row's mailbox threshold also bounds its own side (a score
      // below it cannot be among the row's C best over all keys)
      const float seed = kSym && valid ? p.sym_thr[q] : -__builtin_huge_valf();
      uint32_t thr = seeded<MODE>(pass_threshold<MODE>(heap, pa), seed);
      for (int64_t ti = 0; ti < v.n_ktiles - v.kt0; ti++, tile++) {
        const int64_t kt = tile_at<kSym>(v, ti);
        const uint32_t a = tile & 1u, tph = (tile >> 1) & 1u;
        int got = 1;
        if (lane == 0) got = mbar_wait(&tfull[a], tph, abort, p.timeout_ns) ? 1 : 0;
        got = __shfl_sync(0xffffffffu, got, 0);
        if (!got) {
          set_status(p.status, 3);
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t tbase = tmem_base + (uint32_t(quad * 32) << 16) + a * BN + col_base;
        const int64_t k0 = kt * BN + col_base;
        const float* tth = nullptr;  // this tile's thresholds, then minima, for this group's columns
        if (kSym) {
          // this tile's copy was issued with the tile before (the first of an item: now); the next tile's goes now
          if (ti == 0) fetch_thr(kt, 0);
          cp_async_commit();
          if (ti + 1 < v.n_ktiles - v.kt0) fetch_thr(tile_at<kSym>(v, ti + 1), (ti + 1) & 1);
          cp_async_commit();
          cp_async_wait<1>();
          __syncwarp();
          tth = sthr + (ti & 1) * kTileThr;
        }
        uint32_t va[32], vb[32];
        tmem_ld_32x32b_x32(tbase, va);
        // One chunk of 32 columns.  Symmetric mode: key rows before the
        // block's own (the first tile of an odd block) belong to the block
        // before; those past the block also feed their own rows' mailboxes.
        auto chunk = [&](const uint32_t(&vv)[32], int c, float um) {
          const int64_t col = k0 + c * 32;
          if (kSym) {
            if (col < v.qb * BM) return;  // warp-uniform
            const int32_t mx = max32_s32(vv);
            const int32_t* ids = reinterpret_cast<const int32_t*>(tth + kTileIds) + col_base + c * 32;
            if (valid && (int32_t(thr) > 0 ? mx >= int32_t(thr) : chunk_any<MODE>(vv, thr)))
              offer_chunk<MODE>(vv, chunk_mask<MODE>(vv, thr), col, v.n_k, v.self_mode, qg, heap, thr, pa, v.pc,
                                ids, seed);
            if (col >= (v.qb + 1) * BM)
              mirror_chunk(vv, mx, um, tth + (col_base + c * 32), ids, col, v.n_k, qd, valid, mst, lane, p);
          } else if (valid && chunk_any<MODE>(vv, thr)) {
            offer_chunk<MODE>(vv, chunk_mask<MODE>(vv, thr), col, v.n_k, v.self_mode, qg, heap, thr, pa, v.pc);
          }
        };
#pragma unroll 1
        for (int c = 0; c < NCH; c += 2) {
          float um0 = 0.0f, um1 = 0.0f;
          if (kSym) {
            um0 = tth[BN + col_base / 32 + c];
            um1 = tth[BN + col_base / 32 + c + 1];
          }
          tmem_ld_wait();
          tmem_ld_32x32b_x32(tbase + (c + 1) * 32, vb);
          chunk(va, c, um0);
          tmem_ld_wait();
          if (c + 2 < NCH) tmem_ld_32x32b_x32(tbase + (c + 2) * 32, va);
          chunk(vb, c + 1, um1);
        }
        tc_fence_before();
        if (kPair && !leader) mbar_arrive_cluster(a ? tempty_c1 : tempty_c0);
        else mbar_arrive(&tempty[a]);
      }
      if (GROUPS > 1) ok = epilogue_vote(GROUPS * 128, ok);
      if (!ok) break;
      if (GROUPS > 1) {
        // Fold the other groups' heaps for this row into group 0's.  Unused
        // slots of a heap that never filled are marked empty first.
        if (group > 0)
          for (int j = heap.size; j < v.keep; j++) heap.h[j] = kKeyInf;
        epilogue_sync(GROUPS * 128);
        if (group == 0 && valid) {
          for (int g = 1; g < GROUPS; g++) {
            const uint64_t* other = kSmemHeap ? heaps + int64_t(g * BM + row_local) * p.heap_stride
                                              : p.scratch + (int64_t(blockIdx.x) * GROUPS * BM + g * BM + row_local) *
                                                                p.heap_stride;
            for (int j = 0; j < v.keep; j++) {
              const uint64_t kv = other[j];
              if (kv != kKeyInf) heap.offer(kv);
            }
          }
        }
      }
      if (group == 0 && valid) {
        const int got = heap.finish();
        const int64_t orow = (kSym ? int64_t(qd) : q) * v.keep;  // symmetric mode: rows of the data set
        for (int j = 0; j < v.keep; j++) {
          float raw = kHeapInf;
          int32_t idx = -1;
          if (j < got) {
            raw = from_orderable(uint32_t(heap.h[j] >> 32));
            idx = key_index(heap.h[j]);
            // Keys fold -0.0 onto +0.0; restore the reference's sign: an int8
            // zero dot is -0.0; a Jaccard zero is +0.0 only for two empty rows.
            if (MODE == kModeInt8) raw = int8_raw_from_key(raw);
            if (MODE == kModeJaccard && raw == 0.0f) raw = (pa + v.pc[idx] == 0) ? 0.0f : -0.0f;
          }
          v.out_idx[orow + j] = idx;
          if (v.out_raw) v.out_raw[orow + j] = raw;
          if (v.final_mode && v.out_dist) v.out_dist[orow + j] = transform_raw(v.dtype, raw);
          if (v.out_bound && j == v.keep - 1) v.out_bound[q] = raw;
        }
      }
      if (GROUPS > 1) epilogue_sync(GROUPS * 128);  // heaps are reused by the next block
    }
    if (kSym) mirror_flush(mst, lane, p);  // the keys still staged
  }

  tc_fence_before();
  __syncthreads();
  // A pair's CTAs leave together: the leader's MMAs have read the peer's
  // stages, the peer's arrivals and loads have reached the leader's barriers.
  if (kPair) cluster_sync();
  if (warp == 1) {
    tc_fence_after();
    if (kPair) tmem_dealloc_pair(tmem_base, TMEM_COLS);
    else tmem_dealloc(tmem_base, TMEM_COLS);
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace {

// Looked up once per process; the initialisation of a local static is
// thread-safe, so serving lanes may make their first scans concurrently.
PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    return nullptr;
  }();
  return fn;
}

// 2-D map over `rows` rows of `row_bytes` (a multiple of 128); box = 128 bytes x box_rows.
bool make_map(CUtensorMap* m, const void* base, int64_t rows, int64_t row_bytes, int elem_bytes, int box_rows,
              int half_type = kHalfF16) {
  auto enc = get_encode();
  if (!enc) return false;
  const cuuint64_t dims[2] = {cuuint64_t(row_bytes / elem_bytes), cuuint64_t(rows)};
  const cuuint64_t strides[1] = {cuuint64_t(row_bytes)};
  const cuuint32_t box[2] = {cuuint32_t(KCB / elem_bytes), cuuint32_t(box_rows)};
  const cuuint32_t estr[2] = {1, 1};
  const CUtensorMapDataType dt = elem_bytes == 1          ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                 : half_type == kHalfBf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                          : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
  CUresult r = enc(m, dt, 2,
                   const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace

size_t tc_scan_smem_bytes() { return smem_bytes(4, 1, 0); }

namespace {
template <int MODE, int STAGES, int GROUPS, bool kSmemHeap, bool kBatch = false>
cudaError_t launch_variant(const CUtensorMap& ma, const CUtensorMap& mb, const ScanParams& p, int grid, size_t smem,
                           cudaStream_t stream) {
  auto kern = tc_scan_kernel<MODE, STAGES, GROUPS, kSmemHeap, kBatch>;
  // The opt-in limit, not `smem`: the launch's shared memory varies with keep,
  // and concurrent callers (serving lanes) must not lower each other's limit
  // between this call and their launch.
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_LIMIT));
  if (e != cudaSuccess) return e;
  kern<<<grid, 64 + GROUPS * 128, smem, stream>>>(ma, mb, p);
  return cudaGetLastError();
}

// CTA-pair variants: clusters of two, at most as many as the GPU holds at
// once (neighbouring SMs of a GPC pair up; one CTA per SM), a pair of query
// blocks per cluster and item.  `grid` is the caller's CTA budget.
template <int MODE, int STAGES, int GROUPS>
cudaError_t launch_pair(const CUtensorMap& ma, const CUtensorMap& mb, const ScanParams& p, int grid, size_t smem,
                        cudaStream_t stream) {
  auto kern = tc_scan_kernel<MODE, STAGES, GROUPS, true, false, true>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_LIMIT));
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(64 + GROUPS * 128);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // Clusters resident at once, for this instantiation at the largest shared
  // memory any launch of it asks for (one CTA per SM); looked up once, the
  // initialisation of a local static being thread-safe for serving lanes.
  static const int max_clusters = [&]() {
    cudaLaunchConfig_t c = cfg;
    c.gridDim = dim3(2);
    c.dynamicSmemBytes = SMEM_LIMIT;
    int m = 0;
    if (cudaOccupancyMaxActiveClusters(&m, kern, &c) != cudaSuccess) {
      cudaGetLastError();
      m = 0;
    }
    return m > 0 ? m : 1;
  }();
  const int64_t items = (p.n_q + 2 * BM - 1) / (2 * BM);
  int64_t clusters = std::min<int64_t>({items, int64_t(grid + 1) / 2, int64_t(max_clusters)});
  if (clusters < 1) clusters = 1;
  cfg.gridDim = dim3(unsigned(2 * clusters));
  e = cudaLaunchKernelEx(&cfg, kern, ma, mb, p);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

// The kernel variants an autotuner may choose between: pipeline stages,
// epilogue warp groups, heaps in shared (1) or global (0) memory, CTA pair (1).
constexpr int kVariantCfg[kScanVariants][4] = {{4, 2, 1, 0}, {3, 2, 1, 0}, {4, 1, 1, 0}, {3, 1, 1, 0},
                                               {4, 1, 0, 0}, {2, 2, 1, 0}, {4, 2, 1, 1}, {4, 1, 1, 1},
                                               {6, 1, 1, 1}, {3, 2, 1, 1}, {3, 4, 1, 0}, {2, 4, 1, 0},
                                               {5, 1, 1, 1}, {2, 2, 1, 1}, {2, 1, 1, 0}};

bool variant_feasible(int v, int keep, bool has_scratch) {
  if (v < 0 || v >= kScanVariants) return false;
  if (kVariantCfg[v][2] == 0) return has_scratch;
  return smem_bytes(kVariantCfg[v][0], kVariantCfg[v][1], keep | 1, kVariantCfg[v][3] != 0) <= SMEM_LIMIT;
}

template <int MODE>
cudaError_t launch_forced(const CUtensorMap& ma, const CUtensorMap& mb, ScanParams p, int grid, int v,
                          cudaStream_t stream) {
  const int odd = p.keep | 1;
  p.heap_stride = odd;
  switch (v) {
    case 0: return launch_variant<MODE, 4, 2, true>(ma, mb, p, grid, smem_bytes(4, 2, odd), stream);
    case 1: return launch_variant<MODE, 3, 2, true>(ma, mb, p, grid, smem_bytes(3, 2, odd), stream);
    case 2: return launch_variant<MODE, 4, 1, true>(ma, mb, p, grid, smem_bytes(4, 1, odd), stream);
    case 3: return launch_variant<MODE, 3, 1, true>(ma, mb, p, grid, smem_bytes(3, 1, odd), stream);
    case 5: return launch_variant<MODE, 2, 2, true>(ma, mb, p, grid, smem_bytes(2, 2, odd), stream);
    case 6: return launch_pair<MODE, 4, 2>(ma, mb, p, grid, smem_bytes(4, 2, odd, true), stream);
    case 7: return launch_pair<MODE, 4, 1>(ma, mb, p, grid, smem_bytes(4, 1, odd, true), stream);
    case 8: return launch_pair<MODE, 6, 1>(ma, mb, p, grid, smem_bytes(6, 1, odd, true), stream);
    case 9: return launch_pair<MODE, 3, 2>(ma, mb, p, grid, smem_bytes(3, 2, odd, true), stream);
    case 10: return launch_variant<MODE, 3, 4, true>(ma, mb, p, grid, smem_bytes(3, 4, odd), stream);
    case 11: return launch_variant<MODE, 2, 4, true>(ma, mb, p, grid, smem_bytes(2, 4, odd), stream);
    case 12: return launch_pair<MODE, 5, 1>(ma, mb, p, grid, smem_bytes(5, 1, odd, true), stream);
    case 13: return launch_pair<MODE, 2, 2>(ma, mb, p, grid, smem_bytes(2, 2, odd, true), stream);
    case 14: return launch_variant<MODE, 2, 1, true>(ma, mb, p, grid, smem_bytes(2, 1, odd), stream);
    default:
      p.heap_stride = p.keep;
      return launch_variant<MODE, 4, 1, false>(ma, mb, p, grid, smem_bytes(4, 1, 0), stream);
  }
}

template <int MODE>
cudaError_t launch_mode(const CUtensorMap& ma, const CUtensorMap& mb, ScanParams p, int grid, int variant,
                        cudaStream_t stream) {
  if (variant >= 0 && variant_feasible(variant, p.keep, p.scratch != nullptr))
    return launch_forced<MODE>(ma, mb, p, grid, variant, stream);
  const int odd = p.keep | 1;
  p.heap_stride = odd;
  // int8 dot products with small keep: four epilogue groups.  Measured at
  // full size (2M x 384, k = 15), they beat two groups by 18 %: the scan is
  // epilogue-paced and the wider epilogue also draws less power, so the
  // clocks under the power cap rise (1,642 vs 1,125 MHz).  Short tuning runs
  // do not see that, so it is the automatic choice rather than the tuner's.
  if (MODE == kModeInt8 && smem_bytes(3, 4, odd) <= SMEM_LIMIT)
    return launch_variant<MODE, 3, 4, true>(ma, mb, p, grid, smem_bytes(3, 4, odd), stream);
  // Otherwise prefer two epilogue groups (more warps to hide TMEM/issue
  // latency), then the deeper pipeline; heaps fall back to global memory for
  // very large keep.  (Jaccard at 4M x 1,024 bits: two groups with four
  // stages beat four groups with three by 8 % at full size.)
  if (smem_bytes(4, 2, odd) <= SMEM_LIMIT)
    return launch_variant<MODE, 4, 2, true>(ma, mb, p, grid, smem_bytes(4, 2, odd), stream);
  if (smem_bytes(3, 2, odd) <= SMEM_LIMIT)
    return launch_variant<MODE, 3, 2, true>(ma, mb, p, grid, smem_bytes(3, 2, odd), stream);
  if (smem_bytes(4, 1, odd) <= SMEM_LIMIT)
    return launch_variant<MODE, 4, 1, true>(ma, mb, p, grid, smem_bytes(4, 1, odd), stream);
  if (smem_bytes(3, 1, odd) <= SMEM_LIMIT)
    return launch_variant<MODE, 3, 1, true>(ma, mb, p, grid, smem_bytes(3, 1, odd), stream);
  // heaps in shared memory beside two stages beat heaps in global memory by
  // far (each heap insert is a chain of dependent loads)
  if (smem_bytes(2, 1, odd) <= SMEM_LIMIT)
    return launch_variant<MODE, 2, 1, true>(ma, mb, p, grid, smem_bytes(2, 1, odd), stream);
  if (!p.scratch) return cudaErrorInvalidValue;
  p.heap_stride = p.keep;
  return launch_variant<MODE, 4, 1, false>(ma, mb, p, grid, smem_bytes(4, 1, 0), stream);
}
}  // namespace

cudaError_t launch_tc_scan(int mode, const void* Q, int64_t q_rows, int64_t q_row0, int64_t n_q, const void* K,
                           int64_t k_rows, int64_t n_k, int64_t row_bytes, int keep, uint64_t* scratch, int grid,
                           int self_mode, int final_mode, int dtype, int32_t* out_idx, float* out_raw, float* out_dist,
                           int* status, uint64_t timeout_ns, const int32_t* pc, cudaStream_t stream,
                           int variant, int half_type, const int32_t* q_self, float* out_bound,
                           int64_t q_self_base, uint64_t delay_ns) {
  // q_rows / k_rows: rows present in memory (multiples of the box heights);
  // n_q / n_k: rows that take part.  Rows past n are zero and never offered.
  if (row_bytes % KCB != 0 || n_q <= 0 || n_k <= 0 || keep < 1) return cudaErrorInvalidValue;
  if (q_row0 < 0 || q_rows < q_row0 + n_q || k_rows < n_k || q_rows % BN != 0 || k_rows % BN != 0)
    return cudaErrorInvalidValue;
  if ((reinterpret_cast<uintptr_t>(Q) & 15) || (reinterpret_cast<uintptr_t>(K) & 15)) return cudaErrorInvalidValue;
  if (mode < kModeHalf || mode > kModeJaccard) return cudaErrorInvalidValue;
  // Jaccard reads one popcount per query row and key row: queries are keys.
  if (mode == kModeJaccard && (!pc || !self_mode || Q != K)) return cudaErrorInvalidValue;
  if (half_type != kHalfF16 && half_type != kHalfBf16) return cudaErrorInvalidValue;
  if (q_self && q_row0 != 0) return cudaErrorInvalidValue;
  const int eb = mode == kModeHalf ? 2 : 1;
  // A CTA pair loads half of each key tile per CTA: 128-row boxes (the
  // variant launch_mode takes, a forced one when it is feasible).
  const bool pair = variant >= 0 && variant_feasible(variant, keep, scratch != nullptr) && kVariantCfg[variant][3];
  alignas(64) CUtensorMap ma, mb;
  if (!make_map(&ma, Q, q_rows, row_bytes, eb, BM, half_type) ||
      !make_map(&mb, K, k_rows, row_bytes, eb, pair ? BM : BN, half_type))
    return cudaErrorInvalidValue;
  ScanParams p{};
  p.n_q = n_q;
  p.n_k = n_k;
  p.q_row0 = q_row0;
  p.n_kchunks = int(row_bytes / KCB);
  p.keep = keep;
  p.scratch = scratch;
  p.self_mode = self_mode;
  p.final_mode = final_mode;
  p.dtype = dtype;
  p.out_idx = out_idx;
  p.out_raw = out_raw;
  p.out_dist = out_dist;
  p.status = status;
  p.timeout_ns = timeout_ns;
  p.drain_ns = timeout_ns > kDrainNs ? timeout_ns : kDrainNs;
  p.delay_ns = delay_ns;
  p.pc = pc;
  p.half_type = half_type;
  p.q_self = q_self;
  p.q_self_base = q_self_base;
  p.out_bound = out_bound;
  if (mode == kModeInt8) return launch_mode<kModeInt8>(ma, mb, p, grid, variant, stream);
  if (mode == kModeJaccard) return launch_mode<kModeJaccard>(ma, mb, p, grid, variant, stream);
  return launch_mode<kModeHalf>(ma, mb, p, grid, variant, stream);
}

namespace {
// A symmetric variant also holds each epilogue warp's stage of mirror keys.
constexpr size_t sym_smem_bytes(int stages, int groups, int heap_stride) {
  return smem_bytes(stages, groups, heap_stride) + size_t(groups) * 4 * kMirrorWarpBytes;
}

template <int STAGES, int GROUPS>
cudaError_t launch_sym_variant(const CUtensorMap& ma, const CUtensorMap& mb, const ScanParams& p, int grid,
                               cudaStream_t stream) {
  auto kern = tc_scan_kernel<kModeHalf, STAGES, GROUPS, true, false, false, true>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_LIMIT));
  if (e != cudaSuccess) return e;
  kern<<<grid, 64 + GROUPS * 128, sym_smem_bytes(STAGES, GROUPS, p.heap_stride), stream>>>(ma, mb, p);
  return cudaGetLastError();
}
}  // namespace

bool tc_scan_sym_feasible(int keep) { return sym_smem_bytes(2, 1, keep | 1) <= SMEM_LIMIT; }

cudaError_t launch_tc_scan_sym(const void* X, int64_t rows, int64_t n, int64_t row_bytes, int keep, int grid,
                               int32_t* out_idx, float* out_raw, int* status, uint64_t timeout_ns,
                               cudaStream_t stream, int half_type, const float* thr, const float* umin,
                               const int32_t* perm, int32_t* count, uint64_t* mail, int cap, uint64_t delay_ns) {
  if (row_bytes % KCB != 0 || n <= 0 || keep < 1 || rows < n || rows % BN != 0 || cap < 1) return cudaErrorInvalidValue;
  // the tile copies (cp.async, 16 bytes) read thr, umin and perm in whole tiles
  if ((reinterpret_cast<uintptr_t>(X) & 15) || (reinterpret_cast<uintptr_t>(thr) & 15) ||
      (reinterpret_cast<uintptr_t>(umin) & 15) || (reinterpret_cast<uintptr_t>(perm) & 15) || !count || !mail)
    return cudaErrorInvalidValue;
  if (half_type != kHalfF16 && half_type != kHalfBf16) return cudaErrorInvalidValue;
  if (!tc_scan_sym_feasible(keep)) return cudaErrorInvalidValue;
  // the same rows as queries (128-row boxes) and keys (256-row boxes)
  alignas(64) CUtensorMap ma, mb;
  if (!make_map(&ma, X, rows, row_bytes, 2, BM, half_type) || !make_map(&mb, X, rows, row_bytes, 2, BN, half_type))
    return cudaErrorInvalidValue;
  ScanParams p{};
  p.n_q = n;
  p.n_k = n;
  p.n_kchunks = int(row_bytes / KCB);
  p.keep = keep;
  p.heap_stride = keep | 1;
  p.self_mode = 1;
  p.out_idx = out_idx;
  p.out_raw = out_raw;
  p.status = status;
  p.timeout_ns = timeout_ns;
  p.drain_ns = timeout_ns > kDrainNs ? timeout_ns : kDrainNs;
  p.delay_ns = delay_ns;
  p.half_type = half_type;
  p.sym_thr = thr;
  p.sym_umin = umin;
  p.sym_count = count;
  p.sym_mail = mail;
  p.sym_cap = cap;
  p.sym_perm = perm;
  const int odd = keep | 1;
  if (sym_smem_bytes(4, 2, odd) <= SMEM_LIMIT) return launch_sym_variant<4, 2>(ma, mb, p, grid, stream);
  if (sym_smem_bytes(3, 2, odd) <= SMEM_LIMIT) return launch_sym_variant<3, 2>(ma, mb, p, grid, stream);
  if (sym_smem_bytes(4, 1, odd) <= SMEM_LIMIT) return launch_sym_variant<4, 1>(ma, mb, p, grid, stream);
  if (sym_smem_bytes(3, 1, odd) <= SMEM_LIMIT) return launch_sym_variant<3, 1>(ma, mb, p, grid, stream);
  return launch_sym_variant<2, 1>(ma, mb, p, grid, stream);
}

bool tc_scan_variant_feasible(int variant, int keep, bool has_scratch) {
  return variant_feasible(variant, keep, has_scratch);
}

bool tc_scan_uses_global_heaps(int variant, int keep) {
  if (variant >= 0 && variant_feasible(variant, keep, true)) return kVariantCfg[variant][2] == 0;
  return smem_bytes(2, 1, keep | 1) > SMEM_LIMIT;  // the automatic choice: no shared-memory variant fits
}

int tc_scan_automatic_variant(int mode, int keep) {
  const int odd = keep | 1;
  if (mode == kModeInt8 && smem_bytes(3, 4, odd) <= SMEM_LIMIT) return 10;
  if (smem_bytes(4, 2, odd) <= SMEM_LIMIT) return 0;
  if (smem_bytes(3, 2, odd) <= SMEM_LIMIT) return 1;
  if (smem_bytes(4, 1, odd) <= SMEM_LIMIT) return 2;
  if (smem_bytes(3, 1, odd) <= SMEM_LIMIT) return 3;
  if (smem_bytes(2, 1, odd) <= SMEM_LIMIT) return 14;
  return 4;
}

const char* tc_scan_variant_name(int variant) {
  static const char* names[kScanVariants] = {"4 stages, 2 epilogue groups, shared-memory heaps",
                                             "3 stages, 2 epilogue groups, shared-memory heaps",
                                             "4 stages, 1 epilogue group, shared-memory heaps",
                                             "3 stages, 1 epilogue group, shared-memory heaps",
                                             "4 stages, 1 epilogue group, global-memory heaps",
                                             "2 stages, 2 epilogue groups, shared-memory heaps",
                                             "CTA pair, 4 stages, 2 epilogue groups, shared-memory heaps",
                                             "CTA pair, 4 stages, 1 epilogue group, shared-memory heaps",
                                             "CTA pair, 6 stages, 1 epilogue group, shared-memory heaps",
                                             "CTA pair, 3 stages, 2 epilogue groups, shared-memory heaps",
                                             "3 stages, 4 epilogue groups, shared-memory heaps",
                                             "2 stages, 4 epilogue groups, shared-memory heaps",
                                             "CTA pair, 5 stages, 1 epilogue group, shared-memory heaps",
                                             "CTA pair, 2 stages, 2 epilogue groups, shared-memory heaps",
                                             "2 stages, 1 epilogue group, shared-memory heaps"};
  return variant >= 0 && variant < kScanVariants ? names[variant] : "automatic";
}

// ---------------------------------------------------------------------------
// Batches: one persistent launch over the work-list of many requests.
// ---------------------------------------------------------------------------
bool encode_scan_job(ScanJob* sj, int mode, const void* rows, int64_t rows_mem, int64_t n, int64_t row_bytes,
                     int keep, int final_mode, int dtype, int32_t* out_idx, float* out_raw, float* out_dist,
                     float* out_bound, int half_type) {
  if (mode != kModeHalf && mode != kModeInt8) return false;
  if (row_bytes % KCB != 0 || n <= 0 || keep < 1 || rows_mem < n || rows_mem % BN != 0) return false;
  if (reinterpret_cast<uintptr_t>(rows) & 15) return false;
  const int eb = mode == kModeHalf ? 2 : 1;
  if (!make_map(&sj->ma, rows, rows_mem, row_bytes, eb, BM, half_type) ||
      !make_map(&sj->mb, rows, rows_mem, row_bytes, eb, BN, half_type))
    return false;
  sj->n_q = n;
  sj->n_k = n;
  sj->q_row0 = 0;
  sj->n_kchunks = int(row_bytes / KCB);
  sj->keep = keep;
  sj->self_mode = 1;
  sj->final_mode = final_mode;
  sj->dtype = dtype;
  sj->pad_ = 0;
  sj->out_idx = out_idx;
  sj->out_raw = out_raw;
  sj->out_dist = out_dist;
  sj->pc = nullptr;
  sj->out_bound = out_bound;
  return true;
}

namespace {
// The batch variants: shared-memory heaps only (keep stays small for batched
// requests), chosen by the largest keep in the batch as launch_mode chooses.
template <int MODE>
int batch_variant(int max_keep, size_t* smem) {
  const int odd = max_keep | 1;
  const int cfg[4][2] = {{4, 2}, {3, 2}, {4, 1}, {3, 1}};
  for (int i = 0; i < 4; i++)
    if (smem_bytes(cfg[i][0], cfg[i][1], odd) <= SMEM_LIMIT) {
      *smem = smem_bytes(cfg[i][0], cfg[i][1], odd);
      return i;
    }
  return -1;
}

template <int MODE>
cudaError_t set_batch_attr(int v) {
  const void* kerns[4] = {reinterpret_cast<const void*>(tc_scan_kernel<MODE, 4, 2, true, true>),
                          reinterpret_cast<const void*>(tc_scan_kernel<MODE, 3, 2, true, true>),
                          reinterpret_cast<const void*>(tc_scan_kernel<MODE, 4, 1, true, true>),
                          reinterpret_cast<const void*>(tc_scan_kernel<MODE, 3, 1, true, true>)};
  return cudaFuncSetAttribute(kerns[v], cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_LIMIT));
}

template <int MODE>
cudaError_t launch_batch_mode(const ScanParams& p, int max_keep, int grid, cudaStream_t stream) {
  size_t smem = 0;
  const int v = batch_variant<MODE>(max_keep, &smem);
  if (v < 0) return cudaErrorInvalidValue;
  CUtensorMap none;
  std::memset(&none, 0, sizeof(none));  // unused in batch mode: every item names its request's maps
  switch (v) {
    case 0:
      tc_scan_kernel<MODE, 4, 2, true, true><<<grid, 64 + 2 * 128, smem, stream>>>(none, none, p);
      break;
    case 1:
      tc_scan_kernel<MODE, 3, 2, true, true><<<grid, 64 + 2 * 128, smem, stream>>>(none, none, p);
      break;
    case 2:
      tc_scan_kernel<MODE, 4, 1, true, true><<<grid, 64 + 1 * 128, smem, stream>>>(none, none, p);
      break;
    default:
      tc_scan_kernel<MODE, 3, 1, true, true><<<grid, 64 + 1 * 128, smem, stream>>>(none, none, p);
  }
  return cudaGetLastError();
}
}  // namespace

cudaError_t prepare_tc_scan_batch(int mode, int max_keep) {
  size_t smem = 0;
  if (mode == kModeHalf) {
    const int v = batch_variant<kModeHalf>(max_keep, &smem);
    return v < 0 ? cudaErrorInvalidValue : set_batch_attr<kModeHalf>(v);
  }
  if (mode == kModeInt8) {
    const int v = batch_variant<kModeInt8>(max_keep, &smem);
    return v < 0 ? cudaErrorInvalidValue : set_batch_attr<kModeInt8>(v);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_tc_scan_batch(int mode, BatchHeader* hdr, const ScanJob* jobs, const ScanItem* items,
                                 int max_keep, int grid, uint64_t timeout_ns, cudaStream_t stream, int half_type) {
  ScanParams p{};
  p.half_type = half_type;
  p.heap_stride = max_keep | 1;
  p.status = &hdr->status;
  p.timeout_ns = timeout_ns;
  p.drain_ns = timeout_ns > kDrainNs ? timeout_ns : kDrainNs;
  p.jobs = jobs;
  p.items = items;
  p.n_items = &hdr->n_items;
  if (mode == kModeHalf) return launch_batch_mode<kModeHalf>(p, max_keep, grid, stream);
  if (mode == kModeInt8) return launch_batch_mode<kModeInt8>(p, max_keep, grid, stream);
  return cudaErrorInvalidValue;
}

}  // namespace evoc
