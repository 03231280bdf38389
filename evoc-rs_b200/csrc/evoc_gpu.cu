// C ABI of the evoc kNN-graph engine: argument checks, reference defaults,
// device buffers, and dispatch to the kernels of each form.
//
// The host logic restates knn_graph_impl (src/knn.rs:377-454): the error
// order (k == 0 before n == 0), the k clamp max(1, min(k, n-1)), f32
// renormalisation (prepare_float), then the search and the per-dtype distance
// transform (fused into the kernels' epilogues).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include "../../include/evoc_gpu.h"
#include "batch.h"
#include "common.cuh"
#include "ctx.h"
#include "ctx_plan.h"
#include "kernels.h"

using evoc::cuda_fail;
using evoc::DevBuf;
using evoc::fail;
using evoc::Stage;
using evoc::StageRec;

namespace {

inline int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// The form a request runs.  NN-descent keeps a row's list in a warp's
// registers, two keys per lane, so above k = 64 the request takes the dtype's
// exact form instead (exact neighbour sets, at least the NN-descent recall).
int resolve_form(int32_t dtype, int32_t form, int64_t keff = 0) {
  const int exact = dtype == EVOC_DTYPE_F32 ? EVOC_FORM_BF16_RERANK : EVOC_FORM_EXACT_INT;
  if (form == EVOC_FORM_AUTO) return exact;
  if (form == EVOC_FORM_NNDESCENT && keff > 64) return exact;
  return form;
}

// Copies the caller's rows into a zero-padded device matrix of `ld_bytes` per
// row.  Rows past n (up to padded_rows(n)) are zero.
int stage_rows(evoc_gpu_ctx* ctx, const void* data, int64_t n, int64_t row_bytes, int64_t ld_bytes, bool on_device) {
  Stage st(ctx, on_device ? "copy_rows" : "h2d_rows");
  const int64_t rows = evoc::padded_rows(n);
  EVOC_TRY(ctx->x.ensure(size_t(rows * ld_bytes)), "alloc rows");
  if (on_device) {
    // One SM pass copies, pads and zero-fills (the copy engines may be busy
    // with other streams' host transfers).
    EVOC_TRY(evoc::launch_copy_rows(data, n, row_bytes, ctx->x.p, rows, ld_bytes, ctx->sms, ctx->stream),
             "copy rows");
    ctx->launches += 1;
    return EVOC_OK;
  }
  if (ld_bytes != row_bytes)
    EVOC_TRY(cudaMemsetAsync(ctx->x.p, 0, size_t(rows * ld_bytes), ctx->stream), "memset rows");
  else if (rows > n)
    EVOC_TRY(cudaMemsetAsync(ctx->x.as<uint8_t>() + n * ld_bytes, 0, size_t((rows - n) * ld_bytes), ctx->stream),
             "memset pad rows");
  EVOC_TRY(cudaMemcpy2DAsync(ctx->x.p, size_t(ld_bytes), data, size_t(row_bytes), size_t(row_bytes), size_t(n),
                             cudaMemcpyHostToDevice, ctx->stream),
           "upload rows");
  return EVOC_OK;
}

int ilog2(int64_t v) {
  int l = 0;
  while (v > 1) {
    v >>= 1;
    l++;
  }
  return l;
}

// The autotuned scan variant for this shape, or -1 (automatic).
int tuned_variant(const evoc_gpu_ctx* ctx, int mode, int keep, int64_t row_bytes, int64_t n) {
  auto it = ctx->tune.find(std::make_tuple(mode, keep, row_bytes, ilog2(n)));
  return it == ctx->tune.end() ? -1 : it->second;
}

int scan_grid(const evoc_gpu_ctx* ctx, int64_t n_q) {
  const int64_t qblocks = (n_q + 127) / 128;
  return int(qblocks < ctx->sms ? qblocks : ctx->sms);
}

// Grid of a request's main scan.  Persistent by default (a CTA per SM walking
// many query blocks); a context with scan_per_block (a serving lane running a
// big request) launches a CTA per query block instead, so SMs come free block
// by block -- every few ms -- for other streams' kernels, high-priority ones
// first.  Global-memory heaps are sized for the persistent grid, so a launch
// that uses them stays persistent.
int main_scan_grid(const evoc_gpu_ctx* ctx, int64_t n_q, int keep, int variant) {
  const int persistent = scan_grid(ctx, n_q);
  if (!ctx->scan_per_block || evoc::tc_scan_uses_global_heaps(variant, keep)) return persistent;
  return int(std::min<int64_t>((n_q + 127) / 128, int64_t(1) << 30));
}

// One kNN request: all n rows are keys; query rows r0 .. r0+nq-1 are output rows 0 .. nq-1.
struct Job {
  int64_t n, r0, nq;
  int keff;
  int32_t* idx;
  float* raw;
  float* dist;
  int* status;
};

int run_fp32(evoc_gpu_ctx* ctx, const Job& j, int ld) {
  Stage st(ctx, "fp32_scan");
  const int cap = evoc::topk_capacity(j.keff);
  const int64_t qblocks = (j.nq + 127) / 128;
  const int grid = int(qblocks < int64_t(ctx->sms) * 2 ? qblocks : int64_t(ctx->sms) * 2);
  EVOC_TRY(ctx->scratch.ensure(size_t(grid) * 128 * size_t(cap) * 8), "alloc scratch");
  if (j.r0 % 4 == 0) {
    // k-major copy of the rows in the (otherwise unused) 16-bit row buffer
    EVOC_TRY(ctx->xb.ensure(size_t(evoc::knn_f32_kt_cols(j.n)) * size_t(ld) * 4), "alloc k-major rows");
    EVOC_TRY(evoc::launch_knn_f32_kt(ctx->x.as<float>(), j.n, ld, ctx->xb.as<float>(), j.keff, cap,
                                     ctx->scratch.as<uint64_t>(), grid, j.idx, j.raw, j.dist, j.r0, j.r0 + j.nq,
                                     ctx->sms, ctx->stream),
             "knn_f32_kt");
    ctx->launches += 2;
    return EVOC_OK;
  }
  EVOC_TRY(evoc::launch_knn_f32_simt(ctx->x.as<float>(), j.n, ld, j.keff, cap, ctx->scratch.as<uint64_t>(), grid,
                                     j.idx, j.raw, j.dist, j.r0, j.r0 + j.nq, ctx->stream),
           "knn_f32_simt");
  ctx->launches += 1;
  return EVOC_OK;
}

// Query rows grouped by nearest pivot so that concurrently reranked rows share
// candidates in L2.  Leaves ctx->order holding a permutation of 0..nq-1.
int64_t pivot_count(int64_t n) {
  int64_t n_piv = n / 256;
  if (n_piv > 4096) n_piv = 4096;
  if (n_piv < 2) n_piv = 2;
  return n_piv;
}

int locality_order(evoc_gpu_ctx* ctx, const Job& j, const void* rows, int64_t row_bytes, bool int8,
                   bool sorted_cells, int half_type = evoc::kHalfF16) {
  Stage st(ctx, "pivot_order");
  const int64_t n_piv = pivot_count(j.n);
  const int64_t piv_rows = evoc::padded_rows(n_piv);
  EVOC_TRY(ctx->pivots.ensure(size_t(piv_rows * row_bytes)), "alloc pivots");
  EVOC_TRY(cudaMemsetAsync(ctx->pivots.p, 0, size_t(piv_rows * row_bytes), ctx->stream), "clear pivots");
  EVOC_TRY(evoc::launch_gather_pivots(rows, row_bytes, j.n, n_piv, ctx->pivots.p, ctx->sms, ctx->stream),
           "gather pivots");
  const int grid = scan_grid(ctx, j.nq);
  EVOC_TRY(ctx->labels.ensure(size_t(j.nq) * 4), "alloc labels");
  EVOC_TRY(evoc::launch_tc_scan(int8 ? evoc::kScanInt8 : evoc::kScanHalf, rows, evoc::padded_rows(j.n), j.r0, j.nq,
                                ctx->pivots.p, piv_rows, n_piv,
                                row_bytes, 1, nullptr, grid, 0, 0, 0, ctx->labels.as<int32_t>(), nullptr, nullptr,
                                j.status, ctx->timeout_ns, nullptr, ctx->stream, -1, half_type),
           "pivot scan");
  EVOC_TRY(ctx->order.ensure(size_t(j.nq) * 4), "alloc order");
  EVOC_TRY(ctx->hist.ensure(size_t(n_piv) * 4), "alloc hist");
  EVOC_TRY(ctx->cursor.ensure(size_t(n_piv) * 4), "alloc cursor");
  EVOC_TRY(evoc::launch_order_by_label(ctx->labels.as<int32_t>(), j.nq, int(n_piv), ctx->hist.as<int32_t>(),
                                       ctx->cursor.as<int32_t>(), ctx->order.as<int32_t>(), sorted_cells, ctx->sms,
                                       ctx->stream),
           "order by pivot");
  ctx->launches += sorted_cells ? 6 : 5;
  return EVOC_OK;
}

// Rows the certificate's rescans take per pass (bounds their arena; 128
// query blocks, one wave of the scan).
constexpr int64_t kRepairChunk = 16384;

// Candidates kept per row by the 16-bit scan: oversample * k; automatic:
// 2k from 500,000 rows (the scan's epilogue costs grow with the kept count,
// and the few rows that then fail the certificate are rescanned cheaply),
// ceil(2.5 k) below (fewer rescans, which small requests cannot amortise);
// within [k, n].
int64_t bf16_candidates(const evoc_gpu_opts& opts, int64_t n, int keff) {
  int64_t C = opts.oversample > 0 ? int64_t(opts.oversample) * keff
              : (n >= 500000 ? int64_t(2) * keff : (int64_t(5) * keff + 1) / 2);
  if (C > n) C = n;
  if (C < keff) C = keff;
  return C;
}

// Certificate buffer of the 16-bit form (one allocation, parts 256-byte
// aligned): residual and operand norms of the n rows, their two maxima, the
// scan's C-th kept value per query row (first and second pass), the failed-row
// counters and lists.  The second pass's lists are indexed by chunk item.
struct CertLayout {
  size_t rnorm, hnorm, maxes, bound, bound2, counts, fail1, fail2, total;
};

CertLayout cert_layout(int64_t n, int64_t nq) {
  CertLayout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off += (bytes + 255) / 256 * 256;
    return at;
  };
  L.rnorm = take(size_t(n) * 4);
  L.hnorm = take(size_t(n) * 4);
  L.maxes = take(8);
  L.bound = take(size_t(nq) * 4);
  L.bound2 = take(size_t(kRepairChunk) * 4);
  L.counts = take(8);
  L.fail1 = take(size_t(nq) * 4);
  L.fail2 = take(size_t(nq) * 4);
  L.total = off;
  return L;
}

// Rescan arena for at most kRepairChunk rows: gathered 16-bit query rows,
// their candidates, and gathered f32 query rows for the exact pass.
struct RepairLayout {
  size_t qh, cand2, qf, part, total;
};

RepairLayout repair_layout(int64_t nq, int64_t ld, int64_t ldb, int64_t C2, int64_t keff) {
  const int64_t R = std::min<int64_t>(nq, kRepairChunk);
  RepairLayout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off += (bytes + 255) / 256 * 256;
    return at;
  };
  L.qh = take(size_t(evoc::padded_rows(R) * ldb * 2));
  L.cand2 = take(size_t(R * C2) * 4);
  L.qf = take(size_t(R * ld) * 4);
  L.part = take(size_t(evoc::kSplitRowsMax) * size_t(keff) * 8);  // key-split partial lists of the exact pass
  L.total = off;
  return L;
}

// Candidates of the second certificate pass: 120 when the first pass kept
// fewer (heaps of 120 fit shared memory beside two pipeline stages), else 256
// (the rerank's limit); at most n.
int64_t second_pass_candidates(int64_t n, int64_t C) { return std::min<int64_t>(C < 120 ? 120 : 256, n); }

// Scratch of the scan for `rows` query rows keeping C candidates.
size_t scan_scratch_bytes(const evoc_gpu_ctx* ctx, int64_t rows, int64_t C) {
  return size_t(scan_grid(ctx, rows)) * 256 * size_t(C) * 8;
}

// One request's data as the certificate's rescans see it: its f32 rows and
// 16-bit rows (n keys, `rows` padded), query rows r0 .. r0+nq-1 written to
// output rows 0 .. nq-1, the first pass's candidate count, and the
// certificate's norms.
struct RescanJob {
  const float* x;
  int ld, d;
  const void* xh;
  int64_t ldb, rows, n, r0, nq;
  int keff, half;
  int64_t C;
  int32_t* idx;
  float* raw;
  float* dist;
  int* status;
  evoc::CertArgs cert;  // rnorm, hnorm, maxes, half_len of the request
};

// Key splits of the exact pass over `count` rows: enough work items for two
// CTAs per SM, at least four 128-row key tiles per split, and the partial
// lists within the arena (n_splits * count <= kSplitRowsMax).
int exact_splits(const evoc_gpu_ctx* ctx, int64_t count, int64_t n) {
  const int64_t qblocks = (count + 127) / 128;
  int64_t s = int64_t(ctx->sms) * 2 / std::max<int64_t>(qblocks, 1);
  s = std::min(s, ((n + 127) / 128) / 4);
  s = std::min(s, evoc::kSplitRowsMax / std::max<int64_t>(count, 1));
  return int(std::max<int64_t>(s, 1));
}

// The exact FP32 pass over rows listed on the device (output rows of j).
// part: the arena's split lists (kSplitRowsMax x keff keys).
int exact_rows(evoc_gpu_ctx* ctx, const RescanJob& j, const int32_t* list, int64_t count, float* qf,
               uint64_t* part) {
  const int cap = evoc::topk_capacity(j.keff);
  const int64_t qblocks = (count + 127) / 128;
  const int splits = exact_splits(ctx, count, j.n);
  const int grid = int(std::min<int64_t>(qblocks * splits, int64_t(ctx->sms) * 2));
  EVOC_TRY(evoc::launch_gather_rows_list(j.x, int64_t(j.ld) * 4, j.r0, list, count, count, qf, ctx->sms,
                                         ctx->stream),
           "gather rows");
  EVOC_TRY(ctx->scratch.ensure(size_t(grid) * 128 * size_t(cap) * 8), "alloc scratch");
  EVOC_TRY(evoc::launch_knn_f32_simt(j.x, j.n, j.ld, j.keff, cap, ctx->scratch.as<uint64_t>(), grid, j.idx, j.raw,
                                     j.dist, 0, count, ctx->stream, qf, list, j.r0, splits, part),
           "exact rescan");
  ctx->launches += 2;
  if (splits > 1) {
    EVOC_TRY(evoc::launch_merge_key_splits(part, count, j.keff, splits, list, j.idx, j.raw, j.dist, ctx->sms,
                                           ctx->stream),
             "merge key splits");
    ctx->launches += 1;
  }
  return EVOC_OK;
}

int32_t read_count(evoc_gpu_ctx* ctx, const int32_t* d_count, int* rc) {
  int32_t v = 0;
  cudaError_t e = cudaMemcpyAsync(&v, d_count, 4, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) *rc = cuda_fail(ctx, e, "read certificate count");
  return v;
}

// Whether `rows` failed rows take the exact FP32 pass directly.  The 16-bit
// rescan runs a CTA per 128 query rows over every key (a handful of rows
// leave most SMs idle) and is paced by its epilogue: ~2 TFLOP/s per CTA
// measured with 256-entry heaps in global memory, taken as ~5 with 120-entry
// heaps in shared memory; the exact pass splits the keys over all SMs at the
// FP32 rate (~48 TFLOP/s measured).  Estimated costs: 16-bit waves x
// 128 n d 2 FLOP / per-CTA rate against rows n d 2 FLOP / 45e12.
bool exact_first(const evoc_gpu_ctx* ctx, int64_t rows, int64_t n, int d, int64_t C2) {
  const double work = double(n) * double(d) * 2.0;
  const double waves = std::ceil(double((rows + 127) / 128) / double(ctx->sms));
  const double half_ms = waves * 128.0 * work / (C2 <= 120 ? 5e12 : 2e12) * 1e3;
  const double exact_ms = double(rows) * work / 45e12 * 1e3;
  return exact_ms <= half_ms;
}

// Rows of j (output rows listed in fail1, `failed1` of them) that failed the
// first certificate: the 16-bit scan again over those rows, gathered, keeping
// 256 candidates, the rerank with the certificate; rows failing again (listed
// in fail2 through count2, whose C-th bounds go to bound2) get the exact FP32
// scan.  *second / *exact: rows of each rescan.
int certify_rescan(evoc_gpu_ctx* ctx, const RescanJob& j, int32_t* fail1, int64_t failed1, int32_t* fail2,
                   float* bound2, int32_t* count2, int64_t* second, int64_t* exact) {
  Stage st(ctx, "certify_rescan");
  const int64_t C2 = second_pass_candidates(j.n, j.C);
  const RepairLayout RL = repair_layout(std::min<int64_t>(failed1, kRepairChunk), j.ld, j.ldb, C2, j.keff);
  EVOC_TRY(ctx->repair.ensure(RL.total), "alloc rescan arena");
  uint8_t* rb = ctx->repair.as<uint8_t>();
  float* qf = reinterpret_cast<float*>(rb + RL.qf);
  uint64_t* part = reinterpret_cast<uint64_t*>(rb + RL.part);
  int64_t failed2 = 0;
  int rc = EVOC_OK;
  *second = failed1;
  if (C2 > j.C && !exact_first(ctx, failed1, j.n, j.d, C2)) {
    void* qh = rb + RL.qh;
    int32_t* cand2 = reinterpret_cast<int32_t*>(rb + RL.cand2);
    EVOC_TRY(ctx->scratch.ensure(scan_scratch_bytes(ctx, std::min<int64_t>(failed1, kRepairChunk), C2)),
             "alloc scratch");
    EVOC_TRY(cudaMemsetAsync(count2, 0, 4, ctx->stream), "clear certificate count");
    evoc::CertArgs c2 = j.cert;
    c2.bound = bound2;
    c2.fail_list = fail2;
    c2.fail_count = count2;
    c2.fail_cap = failed1;
    for (int64_t c0 = 0; c0 < failed1; c0 += kRepairChunk) {
      const int64_t cnt = std::min<int64_t>(kRepairChunk, failed1 - c0);
      const int64_t qrows = evoc::padded_rows(cnt);
      // the list holds output rows; the scan's self rule takes r0 + list[i]
      EVOC_TRY(evoc::launch_gather_rows_list(j.xh, j.ldb * 2, j.r0, fail1 + c0, cnt, qrows, qh, ctx->sms,
                                             ctx->stream),
               "gather 16-bit rows");
      EVOC_TRY(evoc::launch_tc_scan(evoc::kScanHalf, qh, qrows, 0, cnt, j.xh, j.rows, j.n, j.ldb * 2, int(C2),
                                    ctx->scratch.as<uint64_t>(), scan_grid(ctx, cnt), 1, 0, 0, cand2, nullptr, nullptr,
                                    j.status, ctx->timeout_ns, nullptr, ctx->stream, -1, j.half, fail1 + c0, bound2,
                                    j.r0),
               "16-bit rescan");
      EVOC_TRY(evoc::launch_rerank_f32(j.x, j.ld, j.d, cnt, j.n, j.r0, cand2, int(C2), j.keff, fail1 + c0, j.idx,
                                       j.raw, j.dist, j.status, ctx->sms, ctx->stream, &c2, true, j.nq),
               "rescan rerank");
      ctx->launches += 3;
    }
    failed2 = read_count(ctx, count2, &rc);
    if (rc) return rc;
  } else {
    // no larger candidate set exists, or the rows are few enough that the
    // exact pass over key splits is the cheaper: every failed row goes there
    fail2 = fail1;
    failed2 = failed1;
  }
  *exact = failed2;
  for (int64_t c0 = 0; c0 < failed2; c0 += kRepairChunk) {
    const int64_t cnt = std::min<int64_t>(kRepairChunk, failed2 - c0);
    rc = exact_rows(ctx, j, fail2 + c0, cnt, qf, part);
    if (rc) return rc;
  }
  return EVOC_OK;
}

// Symmetric scan (sym.cu): a self-join computes only the key tiles from each
// query block on, and scores for later rows reach them through mailboxes
// filtered by thresholds from a pre-scan of every row against a strided
// sample of n / kSymSampleStride rows.  The sample's (C+1)-th best is at
// about rank (C+1) * stride among all keys (for any data), so a row collects
// about that many mailbox keys plus the few within the threshold's rounding
// slack: kSymCap gives it twice that and 256 more (a row that overflows is
// rescanned, so the capacity only matters for speed).
constexpr int64_t kSymSampleStride = 16;

int64_t sym_cap(int64_t C) { return round_up(2 * (C + 1) * kSymSampleStride + 256, 256); }

struct SymLayout {
  size_t thr, umin, perm, count, bound, own_raw, stats, rows, sample, mail, total;
  int64_t m, m_pad, n_pad, cap;
};

SymLayout sym_layout(int64_t n, int64_t C, int64_t ldb) {
  SymLayout L{};
  L.m = n / kSymSampleStride;
  L.m_pad = round_up(L.m, 256);
  L.n_pad = round_up(n, 256);
  L.cap = sym_cap(C);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off += (bytes + 255) / 256 * 256;
    return at;
  };
  L.thr = take(size_t(L.n_pad) * 4);
  L.umin = take(size_t(L.n_pad / 32) * 4);
  L.perm = take(size_t(L.n_pad) * 4);  // scanned row -> data-set row
  L.count = take(size_t(n) * 4);
  L.bound = take(size_t(n) * 4);  // the pre-scan's (C+1)-th raw values
  L.own_raw = take(size_t(n * C) * 4);
  L.stats = take(8);
  L.rows = take(size_t(evoc::padded_rows(n) * ldb) * 2);  // the 16-bit rows in scanned order
  L.sample = take(size_t(L.m_pad * ldb) * 2);
  // the pre-scan's candidate output is written there too, before the mailboxes
  L.mail = take(std::max(size_t(n) * size_t(L.cap) * 8, size_t(n * (C + 1)) * 4));
  L.total = off;
  return L;
}

// Whether a 16-bit form request takes the symmetric scan: certified (an
// overflowed row is repaired by the certificate's rescan), all rows as
// queries, a persistent grid (not a serving lane's per-block launch), and a
// sample large enough for its (C+1)-th best to mean something.
bool use_symmetric(const evoc_gpu_ctx* ctx, bool certify, int64_t n, int64_t r0, int64_t nq, int64_t C) {
  return certify && !ctx->scan_per_block && ctx->sym_min_rows > 0 && n >= ctx->sym_min_rows && r0 == 0 &&
         nq == n && n / kSymSampleStride >= 4 * (C + 1) && evoc::tc_scan_sym_feasible(int(C));
}

// The symmetric scan of all rows: candidates into ctx->cand, the certificate's
// bound (C-th kept raw value) into `bound`.  The rows are scanned grouped by
// nearest pivot (ctx->order, which the rerank then reuses): the 32 key rows
// of a chunk mostly share a cluster, so their mailbox thresholds are alike
// and a query row of another cluster falls below all of them, which one
// compare with their minimum shows.
int symmetric_scan(evoc_gpu_ctx* ctx, const Job& j, int half, int64_t ldb, int64_t rows, int64_t C, float* bound,
                   const float* hnorm, const unsigned int* maxes) {
  const SymLayout S = sym_layout(j.n, C, ldb);
  EVOC_TRY(ctx->sym.ensure(S.total), "alloc symmetric scan");
  uint8_t* b = ctx->sym.as<uint8_t>();
  float* thr = reinterpret_cast<float*>(b + S.thr);
  float* umin = reinterpret_cast<float*>(b + S.umin);
  int32_t* count = reinterpret_cast<int32_t*>(b + S.count);
  float* T = reinterpret_cast<float*>(b + S.bound);
  float* own_raw = reinterpret_cast<float*>(b + S.own_raw);
  int32_t* stats = reinterpret_cast<int32_t*>(b + S.stats);
  int32_t* perm = reinterpret_cast<int32_t*>(b + S.perm);
  void* xs = b + S.rows;
  void* sample = b + S.sample;
  uint64_t* mail = reinterpret_cast<uint64_t*>(b + S.mail);
  int rc = locality_order(ctx, j, ctx->xb.p, ldb * 2, false, false, half);
  if (rc) return rc;
  {
    Stage st(ctx, "sym_sample");
    const int32_t* order = ctx->order.as<int32_t>();
    EVOC_TRY(cudaMemcpyAsync(perm, order, size_t(j.n) * 4, cudaMemcpyDeviceToDevice, ctx->stream), "copy order");
    EVOC_TRY(cudaMemsetAsync(perm + j.n, 0, size_t(S.n_pad - j.n) * 4, ctx->stream), "pad order");
    EVOC_TRY(evoc::launch_gather_rows_list(ctx->xb.p, ldb * 2, 0, order, j.n, rows, xs, ctx->sms, ctx->stream),
             "rows in scanned order");
    EVOC_TRY(evoc::launch_gather_strided_rows(xs, ldb * 2, kSymSampleStride, S.m, S.m_pad, sample, ctx->sms,
                                              ctx->stream),
             "gather sample rows");
    EVOC_TRY(ctx->scratch.ensure(scan_scratch_bytes(ctx, j.n, C + 1)), "alloc scratch");
    EVOC_TRY(evoc::launch_tc_scan(evoc::kScanHalf, xs, rows, 0, j.n, sample, S.m_pad, S.m, ldb * 2,
                                  int(C + 1), ctx->scratch.as<uint64_t>(), scan_grid(ctx, j.n), 0, 0, 0,
                                  reinterpret_cast<int32_t*>(mail), nullptr, nullptr, j.status, ctx->timeout_ns,
                                  nullptr, ctx->stream, -1, half, nullptr, T),
             "sample pre-scan");
    EVOC_TRY(evoc::launch_sym_thresholds(j.n, S.n_pad, T, hnorm, perm, maxes, int(ldb), thr, umin, count, ctx->sms,
                                         ctx->stream),
             "mailbox thresholds");
    EVOC_TRY(cudaMemsetAsync(stats, 0, 8, ctx->stream), "clear merge statistics");
    ctx->launches += 4;
  }
  {
    Stage st(ctx, "bf16_scan");
    EVOC_TRY(evoc::launch_tc_scan_sym(xs, rows, j.n, ldb * 2, int(C), scan_grid(ctx, j.n), ctx->cand.as<int32_t>(),
                                      own_raw, j.status, ctx->timeout_ns, ctx->stream, half, thr, umin, perm, count,
                                      mail, int(S.cap), ctx->delay_ns),
             "symmetric 16-bit scan");
    ctx->launches += 1;
  }
  {
    Stage st(ctx, "sym_merge");
    EVOC_TRY(evoc::launch_sym_merge(j.n, int(C), ctx->cand.as<int32_t>(), own_raw, count, mail, int(S.cap), bound,
                                    stats, ctx->sms, ctx->stream),
             "merge mailboxes");
    ctx->launches += 1;
  }
  ctx->sym_sample = S.m;
  ctx->sym_cap = S.cap;
  return EVOC_OK;
}

// The 16-bit form: FP16 (or BF16) tensor-core scan keeping C candidates per
// row, FP32 rerank with the per-row certificate (rerank.cu), then for rows
// that fail it a second scan keeping 256 candidates, and for rows that fail
// again an exact FP32 scan.  Every returned row is either certified or exact.
// Beyond 256 candidates per row (the rerank's shared-memory limit) every row
// takes the exact FP32 scan directly.
int run_bf16_rerank(evoc_gpu_ctx* ctx, const evoc_gpu_opts& opts, const Job& j, int ld, int d) {
  const int64_t C = bf16_candidates(opts, j.n, j.keff);
  if (C > 256) return run_fp32(ctx, j, ld);
  if (opts.scan_type != evoc::kHalfF16 && opts.scan_type != evoc::kHalfBf16)
    return fail(ctx, EVOC_ERR_ARG, "scan_type must be 0 (FP16) or 1 (BF16)");
  const int half = opts.scan_type;
  const bool certify = opts.certify != 0;
  const int64_t ldb = round_up(d, 64);
  const int64_t rows = evoc::padded_rows(j.n);
  const CertLayout CL = cert_layout(j.n, j.nq);
  uint8_t* cb = nullptr;
  if (certify) {
    EVOC_TRY(ctx->cert.ensure(CL.total), "alloc certificate");
    cb = ctx->cert.as<uint8_t>();
  }
  auto cf = [&](size_t off) { return reinterpret_cast<float*>(cb + off); };
  auto ci = [&](size_t off) { return reinterpret_cast<int32_t*>(cb + off); };
  unsigned int* maxes = certify ? reinterpret_cast<unsigned int*>(cb + CL.maxes) : nullptr;
  {
    Stage st(ctx, "to_half");
    EVOC_TRY(ctx->xb.ensure(size_t(rows * ldb * 2)), "alloc 16-bit rows");
    EVOC_TRY(evoc::launch_to_half(ctx->x.as<float>(), rows, j.n, ld, d, ctx->xb.p, int(ldb), half,
                                  certify ? cf(CL.rnorm) : nullptr, certify ? cf(CL.hnorm) : nullptr, maxes, ctx->sms,
                                  ctx->stream),
             "to 16-bit");
    ctx->launches += 1;
  }
  const int variant = tuned_variant(ctx, evoc::kScanHalf, int(C), ldb * 2, j.n);
  const int grid = main_scan_grid(ctx, j.nq, int(C), variant);
  EVOC_TRY(ctx->cand.ensure(size_t(j.nq * C) * 4), "alloc candidates");
  const bool sym = use_symmetric(ctx, certify, j.n, j.r0, j.nq, C);
  if (sym) {
    int rc = symmetric_scan(ctx, j, half, ldb, rows, C, cf(CL.bound), cf(CL.hnorm), maxes);
    if (rc) return rc;
  } else {
    Stage st(ctx, "bf16_scan");
    EVOC_TRY(ctx->scratch.ensure(scan_scratch_bytes(ctx, j.nq, C)), "alloc scratch");
    EVOC_TRY(evoc::launch_tc_scan(evoc::kScanHalf, ctx->xb.p, rows, j.r0, j.nq, ctx->xb.p, rows, j.n, ldb * 2, int(C),
                                  ctx->scratch.as<uint64_t>(), grid, 1, 0, 0, ctx->cand.as<int32_t>(), nullptr,
                                  nullptr, j.status, ctx->timeout_ns, nullptr, ctx->stream, variant, half, nullptr,
                                  certify ? cf(CL.bound) : nullptr, 0, ctx->delay_ns),
             "16-bit scan");
    ctx->launches += 1;
  }
  const int32_t* order = nullptr;
  if (j.nq >= 65536) {
    // the order only schedules the rerank (the symmetric scan computed it already)
    if (!sym) {
      int rc = locality_order(ctx, j, ctx->xb.p, ldb * 2, false, false, half);
      if (rc) return rc;
    }
    order = ctx->order.as<int32_t>();
  }
  int32_t* counts = certify ? ci(CL.counts) : nullptr;
  evoc::CertArgs ca{};
  if (certify) {
    EVOC_TRY(cudaMemsetAsync(counts, 0, 8, ctx->stream), "clear certificate counts");
    ca = evoc::CertArgs{cf(CL.bound), cf(CL.rnorm), cf(CL.hnorm), maxes, int(ldb), ci(CL.fail1), counts, j.nq};
  }
  {
    Stage st(ctx, "rerank");
    EVOC_TRY(evoc::launch_rerank_f32(ctx->x.as<float>(), ld, d, j.nq, j.n, j.r0, ctx->cand.as<int32_t>(), int(C),
                                     j.keff, order, j.idx, j.raw, j.dist, j.status, ctx->sms, ctx->stream,
                                     certify ? &ca : nullptr),
             "rerank");
    ctx->launches += 1;
  }
  ctx->cert_checked = certify ? j.nq : 0;
  if (!certify) return EVOC_OK;
  int rc = EVOC_OK;
  const int64_t failed1 = read_count(ctx, counts, &rc);
  if (rc) return rc;
  if (sym) {
    const int32_t* stats = reinterpret_cast<const int32_t*>(ctx->sym.as<uint8_t>() + sym_layout(j.n, C, ldb).stats);
    ctx->sym_overflow = read_count(ctx, stats, &rc);
    if (rc == EVOC_OK) ctx->sym_max_offers = read_count(ctx, stats + 1, &rc);
    if (rc) return rc;
  }
  if (failed1 == 0) return EVOC_OK;
  RescanJob rj{ctx->x.as<float>(), ld, d, ctx->xb.p, ldb, rows, j.n, j.r0, j.nq, j.keff, half, C, j.idx, j.raw,
               j.dist, j.status, ca};
  int64_t second = 0, exact = 0;
  rc = certify_rescan(ctx, rj, ci(CL.fail1), failed1, ci(CL.fail2), cf(CL.bound2), counts + 1, &second, &exact);
  ctx->cert_second = second;
  ctx->cert_exact = exact;
  return rc;
}

int run_int8(evoc_gpu_ctx* ctx, const Job& j, int64_t ldb) {
  Stage st(ctx, "int8_scan");
  const int variant = tuned_variant(ctx, evoc::kScanInt8, j.keff, ldb, j.n);
  const int grid = main_scan_grid(ctx, j.nq, j.keff, variant);
  const int64_t rows = evoc::padded_rows(j.n);
  EVOC_TRY(ctx->scratch.ensure(size_t(scan_grid(ctx, j.nq)) * 256 * size_t(j.keff) * 8), "alloc scratch");
  EVOC_TRY(evoc::launch_tc_scan(evoc::kScanInt8, ctx->x.p, rows, j.r0, j.nq, ctx->x.p, rows, j.n, ldb, j.keff,
                                ctx->scratch.as<uint64_t>(), grid, 1, 1, EVOC_DTYPE_I8, j.idx, j.raw, j.dist, j.status,
                                ctx->timeout_ns, nullptr, ctx->stream, variant, evoc::kHalfF16, nullptr, nullptr, 0,
                                ctx->delay_ns),
           "int8 scan");
  ctx->launches += 1;
  return EVOC_OK;
}

// Bytes per row of the 0/1 int8 expansion of `nbytes` packed bytes.
int64_t expanded_row_bytes(int64_t nbytes) { return round_up(nbytes * 8, 128); }

// Binary rows on the tensor cores: popcounts and the 0/1 expansion, then the
// int8 scan in Jaccard mode.  ldb: bytes between staged packed rows.
int run_jaccard_tc(evoc_gpu_ctx* ctx, const Job& j, int64_t ldb, int64_t nbytes) {
  const int64_t rows = evoc::padded_rows(j.n);
  const int64_t lde = expanded_row_bytes(nbytes);
  {
    Stage st(ctx, "expand_bits");
    EVOC_TRY(ctx->popc.ensure(size_t(j.n) * 4), "alloc popcounts");
    EVOC_TRY(evoc::launch_popcount_rows(ctx->x.p, j.n, int(ldb / 4), ctx->popc.as<int32_t>(), ctx->sms, ctx->stream),
             "popcounts");
    EVOC_TRY(ctx->xb.ensure(size_t(rows * lde)), "alloc expanded rows");
    EVOC_TRY(evoc::launch_expand_bits(ctx->x.p, j.n, ldb, nbytes, ctx->xb.p, rows, lde, ctx->sms, ctx->stream),
             "expand bits");
    ctx->launches += 2;
  }
  Stage st(ctx, "jaccard_scan");
  const int grid = scan_grid(ctx, j.nq);
  EVOC_TRY(ctx->scratch.ensure(size_t(grid) * 256 * size_t(j.keff) * 8), "alloc scratch");
  EVOC_TRY(evoc::launch_tc_scan(evoc::kScanJaccard, ctx->xb.p, rows, j.r0, j.nq, ctx->xb.p, rows, j.n, lde, j.keff,
                                ctx->scratch.as<uint64_t>(), grid, 1, 1, EVOC_DTYPE_U8, j.idx, j.raw, j.dist, j.status,
                                ctx->timeout_ns, ctx->popc.as<int32_t>(), ctx->stream,
                                tuned_variant(ctx, evoc::kScanJaccard, j.keff, lde, j.n)),
           "jaccard scan");
  ctx->launches += 1;
  return EVOC_OK;
}

int run_jaccard(evoc_gpu_ctx* ctx, const Job& j, int64_t ldb) {
  Stage st(ctx, "jaccard_scan");
  if (evoc::knn_jaccard_smem(j.keff) > 232448) return fail(ctx, EVOC_ERR_UNSUPPORTED, "k too large for this form");
  const int64_t qblocks = (j.nq + 127) / 128;
  const int grid = int(qblocks < ctx->sms ? qblocks : ctx->sms);
  EVOC_TRY(ctx->popc.ensure(size_t(j.n) * 4), "alloc popcounts");
  EVOC_TRY(evoc::launch_knn_jaccard(ctx->x.p, j.n, int(ldb / 4), j.keff, ctx->popc.as<int32_t>(), grid, j.idx, j.raw,
                                    j.dist, j.r0, j.r0 + j.nq, ctx->sms, ctx->stream),
           "jaccard scan");
  ctx->launches += 2;
  return EVOC_OK;
}

// Carves the fuzzy-graph work buffers out of one allocation.
int fuzzy_work(evoc_gpu_ctx* ctx, int64_t n, int k, evoc::FuzzyWork* w) {
  const size_t nk = size_t(n) * size_t(k);
  const size_t sizes[] = {64, 64, nk * 4, nk * 4, size_t(n) * 4, size_t(n) * 4, size_t(n + 1) * 8, size_t(n) * 4,
                          nk * 4, nk * 4, size_t(n) * 4, size_t(n) * 4, 64};
  constexpr int kParts = int(sizeof(sizes) / sizeof(sizes[0]));
  size_t total = 0;
  for (size_t s : sizes) total += (s + 255) / 256 * 256;
  EVOC_TRY(ctx->g_work.ensure(total), "alloc graph work");
  uint8_t* p = ctx->g_work.as<uint8_t>();
  void* ptrs[kParts];
  for (int i = 0; i < kParts; i++) {
    ptrs[i] = p;
    p += (sizes[i] + 255) / 256 * 256;
  }
  w->flags = static_cast<int*>(ptrs[0]);
  w->mean = static_cast<float*>(ptrs[1]);
  w->a_cols = static_cast<int32_t*>(ptrs[2]);
  w->a_vals = static_cast<float*>(ptrs[3]);
  w->a_cnt = static_cast<int32_t*>(ptrs[4]);
  w->indeg = static_cast<int32_t*>(ptrs[5]);
  w->colptr = static_cast<int64_t*>(ptrs[6]);
  w->fill = static_cast<int32_t*>(ptrs[7]);
  w->at_rows = static_cast<int32_t*>(ptrs[8]);
  w->at_vals = static_cast<float*>(ptrs[9]);
  w->row_cnt = static_cast<int32_t*>(ptrs[10]);
  w->big = static_cast<int32_t*>(ptrs[11]);
  w->n_big = static_cast<int32_t*>(ptrs[12]);
  return EVOC_OK;
}

int fuzzy_impl(evoc_gpu_ctx* ctx, const int32_t* idx, const float* dist, int64_t n, int32_t k, float n_neighbors,
               int32_t symmetrize, int32_t on_dev, float* sigma, float* rho, bool graph, int64_t* indptr,
               int32_t* indices, float* data, int64_t cap, int64_t* nnz) {
  if (!ctx) return EVOC_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  ctx->err.clear();
  ctx->n_stages = 0;
  ctx->launches = 0;
  if (n <= 0) return fail(ctx, EVOC_ERR_EMPTY, "empty kNN graph");
  if (k <= 0) return fail(ctx, EVOC_ERR_ARG, "k must be positive");
  if (!dist || (graph && (!idx || !indptr))) return fail(ctx, EVOC_ERR_ARG, "null input or output");
  EVOC_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
  Stage total(ctx, "total");
  const size_t nk = size_t(n) * size_t(k);
  const int32_t* d_idx = idx;
  const float* d_dist = dist;
  if (!on_dev) {
    Stage st(ctx, "h2d_knn");
    EVOC_TRY(ctx->g_dist.ensure(nk * 4), "alloc dist");
    EVOC_TRY(cudaMemcpyAsync(ctx->g_dist.p, dist, nk * 4, cudaMemcpyHostToDevice, ctx->stream), "upload dist");
    d_dist = ctx->g_dist.as<float>();
    if (idx) {
      EVOC_TRY(ctx->g_idx.ensure(nk * 4), "alloc idx");
      EVOC_TRY(cudaMemcpyAsync(ctx->g_idx.p, idx, nk * 4, cudaMemcpyHostToDevice, ctx->stream), "upload idx");
      d_idx = ctx->g_idx.as<int32_t>();
    }
  }
  evoc::FuzzyWork w;
  int rc = fuzzy_work(ctx, n, k, &w);
  if (rc) return rc;
  float* d_sigma = (on_dev && sigma) ? sigma : nullptr;
  float* d_rho = (on_dev && rho) ? rho : nullptr;
  if (!d_sigma) {
    EVOC_TRY(ctx->g_sigma.ensure(size_t(n) * 4), "alloc sigma");
    d_sigma = ctx->g_sigma.as<float>();
  }
  if (!d_rho) {
    EVOC_TRY(ctx->g_rho.ensure(size_t(n) * 4), "alloc rho");
    d_rho = ctx->g_rho.as<float>();
  }
  // Without indices there is no graph: membership rows are still built from a
  // dummy index array so sigma/rho come from the same kernel.
  if (!d_idx) {
    EVOC_TRY(ctx->g_idx.ensure(nk * 4), "alloc idx");
    EVOC_TRY(cudaMemsetAsync(ctx->g_idx.p, 0xff, nk * 4, ctx->stream), "fill idx");
    d_idx = ctx->g_idx.as<int32_t>();
  }
  {
    Stage st(ctx, "smooth_knn_dist");
    EVOC_TRY(evoc::launch_smooth_and_membership(d_idx, d_dist, n, k, n_neighbors, w, d_sigma, d_rho, ctx->sms,
                                                ctx->stream),
             "smooth_knn_dist");
    ctx->launches += 3;
  }
  int64_t total_nnz = 0;
  if (graph) {
    int64_t* d_indptr = on_dev ? indptr : nullptr;
    if (!d_indptr) {
      EVOC_TRY(ctx->g_indptr.ensure(size_t(n + 1) * 8), "alloc indptr");
      d_indptr = ctx->g_indptr.as<int64_t>();
    }
    {
      Stage st(ctx, "union_count");
      EVOC_TRY(evoc::launch_fuzzy_union_count(n, k, symmetrize, w, d_indptr, ctx->sms, ctx->stream), "union count");
      ctx->launches += symmetrize ? 5 : 2;
    }
    EVOC_TRY(cudaMemcpyAsync(&total_nnz, d_indptr + n, 8, cudaMemcpyDeviceToHost, ctx->stream), "read nnz");
    EVOC_TRY(cudaStreamSynchronize(ctx->stream), "union count");
    if (nnz) *nnz = total_nnz;
    if (total_nnz > cap) return fail(ctx, EVOC_ERR_ARG, "cap too small for the graph; *nnz holds the size needed");
    int32_t* d_indices = on_dev ? indices : nullptr;
    float* d_data = on_dev ? data : nullptr;
    if (!on_dev) {
      EVOC_TRY(ctx->g_indices.ensure(size_t(total_nnz > 0 ? total_nnz : 1) * 4), "alloc indices");
      EVOC_TRY(ctx->g_data.ensure(size_t(total_nnz > 0 ? total_nnz : 1) * 4), "alloc data");
      d_indices = ctx->g_indices.as<int32_t>();
      d_data = ctx->g_data.as<float>();
    }
    {
      Stage st(ctx, "union_write");
      EVOC_TRY(evoc::launch_fuzzy_union_write(n, k, symmetrize, w, d_indptr, d_indices, d_data, ctx->sms,
                                              ctx->stream),
               "union write");
      ctx->launches += 1;
    }
    if (!on_dev) {
      EVOC_TRY(cudaMemcpyAsync(indptr, d_indptr, size_t(n + 1) * 8, cudaMemcpyDeviceToHost, ctx->stream), "indptr");
      if (total_nnz > 0) {
        EVOC_TRY(cudaMemcpyAsync(indices, d_indices, size_t(total_nnz) * 4, cudaMemcpyDeviceToHost, ctx->stream),
                 "indices");
        EVOC_TRY(cudaMemcpyAsync(data, d_data, size_t(total_nnz) * 4, cudaMemcpyDeviceToHost, ctx->stream), "data");
      }
    }
  }
  if (!on_dev) {
    if (sigma) EVOC_TRY(cudaMemcpyAsync(sigma, d_sigma, size_t(n) * 4, cudaMemcpyDeviceToHost, ctx->stream), "sigma");
    if (rho) EVOC_TRY(cudaMemcpyAsync(rho, d_rho, size_t(n) * 4, cudaMemcpyDeviceToHost, ctx->stream), "rho");
  }
  total.end();
  EVOC_TRY(cudaStreamSynchronize(ctx->stream), "fuzzy graph");
  return EVOC_OK;
}

// GPU NN-descent over the staged rows (see nndescent.cu).  Row slices are not
// supported: the graph is built for every row.
// `rows` / `row_bytes`: the rows the join reads (FP16 rows for f32 data,
// which the pivot scan also runs on; the int8 rows; the packed bits).
constexpr int kNndParts = 12;

// max_candidates: the option, else min(60, floor(1.5 k)) as the reference
// defaults it (src/knn.rs:410-412), capped at 64.
int nnd_max_candidates(const evoc_gpu_opts& opts, int k) {
  int mc = opts.max_candidates > 0 ? opts.max_candidates : std::min(60, int(float(k) * 1.5f));
  return std::max(1, std::min(mc, 64));
}

// Parts of the NN-descent work buffer (graph keys and newness flags, double
// buffered; reverse-edge counts, offsets, fill cursors, rows; the candidate
// lists; the change counter and the distance sum), each 256-byte aligned.
// Returns the total.
size_t nnd_work_sizes(int64_t n, int k, int mc, size_t* sizes) {
  const size_t nk = size_t(n) * size_t(k);
  const size_t v[kNndParts] = {nk * 8, nk * 8, nk, nk, size_t(n) * 4, size_t(n + 1) * 8, size_t(n) * 4, nk * 4,
                               size_t(n) * size_t(2 * mc) * 4, 64, size_t(1 + evoc::kNndSumParts) * 8, 64};
  size_t total = 0;
  for (int i = 0; i < kNndParts; i++) {
    sizes[i] = v[i];
    total += (v[i] + 255) / 256 * 256;
  }
  return total;
}

int run_nndescent(evoc_gpu_ctx* ctx, const evoc_gpu_opts& opts, const Job& j, int32_t dtype, int64_t row_bytes,
                  const void* rows, int ld_f32, int d, const int64_t* rng_state) {
  if (j.r0 != 0 || j.nq != j.n) return fail(ctx, EVOC_ERR_UNSUPPORTED, "the NN-descent form builds whole graphs only");
  const int64_t n = j.n;
  const int k = j.keff;
  const int mc = nnd_max_candidates(opts, k);
  evoc::NndArgs a{};
  a.X = static_cast<const uint8_t*>(rows);
  a.row_bytes = row_bytes;
  a.n = n;
  a.k = k;
  a.mc = mc;
  a.dtype = dtype;
  a.sms = ctx->sms;
  uint64_t seed = 0x5eed5eedull;
  if (rng_state)
    seed = (uint64_t(rng_state[0]) * 0x9e3779b97f4a7c15ull) ^ (uint64_t(rng_state[1]) << 21) ^ uint64_t(rng_state[2]);
  a.seed = seed;
  if (dtype == EVOC_DTYPE_U8) {
    EVOC_TRY(ctx->popc.ensure(size_t(n) * 4), "alloc popcounts");
    EVOC_TRY(evoc::launch_popcount_rows(rows, n, int(row_bytes / 4), ctx->popc.as<int32_t>(), ctx->sms, ctx->stream),
             "popcounts");
    a.pc = ctx->popc.as<int32_t>();
    ctx->launches += 1;
  } else {
    // Pivot cells seed the graph and fix the visiting order.
    int rc = locality_order(ctx, j, rows, row_bytes, dtype == EVOC_DTYPE_I8, true);
    if (rc) return rc;
    a.order = ctx->order.as<int32_t>();
    a.label = ctx->labels.as<int32_t>();
    a.cell_end = ctx->cursor.as<int32_t>();
    a.cell_cnt = ctx->hist.as<int32_t>();
  }
  const size_t nk = size_t(n) * size_t(k);
  size_t sizes[kNndParts];
  const size_t total = nnd_work_sizes(n, k, mc, sizes);
  EVOC_TRY(ctx->nnd_work.ensure(total), "alloc NN-descent work");
  uint8_t* p = ctx->nnd_work.as<uint8_t>();
  void* ptrs[kNndParts];
  for (int i = 0; i < kNndParts; i++) {
    ptrs[i] = p;
    p += (sizes[i] + 255) / 256 * 256;
  }
  a.keys[0] = static_cast<uint64_t*>(ptrs[0]);
  a.keys[1] = static_cast<uint64_t*>(ptrs[1]);
  a.isnew[0] = static_cast<uint8_t*>(ptrs[2]);
  a.isnew[1] = static_cast<uint8_t*>(ptrs[3]);
  a.rcnt = static_cast<int32_t*>(ptrs[4]);
  a.rptr = static_cast<int64_t*>(ptrs[5]);
  a.rfill = static_cast<int32_t*>(ptrs[6]);
  a.rrows = static_cast<int32_t*>(ptrs[7]);
  a.cand = static_cast<int32_t*>(ptrs[8]);
  a.changes = static_cast<unsigned long long*>(ptrs[9]);
  a.sum = static_cast<double*>(ptrs[10]);
  a.evals = static_cast<unsigned long long*>(ptrs[11]);
  EVOC_TRY(cudaMemsetAsync(a.evals, 0, 8, ctx->stream), "clear evaluation count");
  {
    Stage st(ctx, "nnd_init");
    EVOC_TRY(evoc::launch_nnd_init(a, ctx->stream), "NN-descent init");
    ctx->launches += 1;
  }
  int n_iters = opts.n_iters > 0 ? opts.n_iters : int(std::max(5.0, std::round(std::log2(double(n)))));
  const float delta = opts.delta;
  // c <= (delta * n_neighbors as f32 * n as f32) as u32 (src/nndescent/float.rs:849)
  const double limit = double(uint32_t(delta * float(k) * float(n)));
  double prev_sum = 0.0;
  bool has_prev = false;
  int cur = 0;
  for (int it = 0; it < n_iters; it++) {
    Stage st(ctx, "nnd_iteration");
    EVOC_TRY(cudaMemsetAsync(a.changes, 0, 8, ctx->stream), "clear changes");
    EVOC_TRY(evoc::launch_nnd_iteration(a, cur, it, ctx->stream), "NN-descent iteration");
    ctx->launches += 7;
    cur ^= 1;
    unsigned long long ch = 0;
    double sum = 0.0;
    EVOC_TRY(cudaMemcpyAsync(&ch, a.changes, 8, cudaMemcpyDeviceToHost, ctx->stream), "read changes");
    EVOC_TRY(cudaMemcpyAsync(&sum, a.sum, 8, cudaMemcpyDeviceToHost, ctx->stream), "read distance sum");
    EVOC_TRY(cudaStreamSynchronize(ctx->stream), "NN-descent iteration");
    ctx->nnd_iterations = it + 1;
    if (double(ch) <= limit) break;
    // delta_improv (src/nndescent/float.rs:857-870): relative change of the
    // sum of distances from the previous iteration; <= 0 switches it off
    if (opts.delta_improv > 0.0f) {
      if (has_prev && std::fabs(sum - prev_sum) / std::fabs(prev_sum) < double(opts.delta_improv)) break;
      prev_sum = sum;
      has_prev = true;
    }
  }
  EVOC_TRY(cudaMemcpyAsync(&ctx->nnd_evals, a.evals, 8, cudaMemcpyDeviceToHost, ctx->stream), "read evaluations");
  ctx->nnd_row_bytes = row_bytes;
  Stage st(ctx, "nnd_finish");
  if (dtype == EVOC_DTYPE_F32) {
    EVOC_TRY(ctx->cand.ensure(nk * 4), "alloc candidates");
    EVOC_TRY(evoc::launch_nnd_emit(a, cur, ctx->cand.as<int32_t>(), nullptr, nullptr, ctx->stream), "emit");
    EVOC_TRY(evoc::launch_rerank_f32(ctx->x.as<float>(), ld_f32, d, n, n, 0, ctx->cand.as<int32_t>(), k, k, a.order,
                                     j.idx, j.raw, j.dist, j.status, ctx->sms, ctx->stream),
             "rerank");
    ctx->launches += 2;
  } else {
    EVOC_TRY(evoc::launch_nnd_emit(a, cur, j.idx, j.raw, j.dist, ctx->stream), "emit");
    ctx->launches += 1;
  }
  return EVOC_OK;
}

int knn_impl(evoc_gpu_ctx* ctx, const evoc_gpu_opts* opts_in, int32_t dtype, const void* data, int64_t n,
             int64_t dim, int32_t k, const int64_t* rng_state, int32_t* out_idx, float* out_dist, float* out_raw,
             int32_t* out_k) {
  if (!ctx) return EVOC_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  ctx->err.clear();
  ctx->n_stages = 0;
  ctx->launches = 0;
  ctx->cert_checked = ctx->cert_second = ctx->cert_exact = 0;
  ctx->sym_sample = ctx->sym_cap = ctx->sym_max_offers = ctx->sym_overflow = 0;
  evoc_gpu_opts opts;
  evoc_gpu_default_opts(&opts);
  if (opts_in) {
    if (opts_in->struct_size != sizeof(evoc_gpu_opts)) return fail(ctx, EVOC_ERR_ARG, "opts.struct_size mismatch");
    opts = *opts_in;
  }
  if (k <= 0) return fail(ctx, EVOC_ERR_K, "n_neighbors must be positive");
  if (n <= 0) return fail(ctx, EVOC_ERR_EMPTY, "empty embedding matrix");
  if (!data || !out_idx) return fail(ctx, EVOC_ERR_ARG, "null data or out_idx");
  if (dim <= 0) return fail(ctx, EVOC_ERR_ARG, "dim must be positive");
  if (dtype < EVOC_DTYPE_F32 || dtype > EVOC_DTYPE_U8) return fail(ctx, EVOC_ERR_ARG, "unknown dtype");
  if (n >= (int64_t(1) << 31) - 1) return fail(ctx, EVOC_ERR_ARG, "n exceeds int32 index range");
  int64_t r0 = 0, r1 = n;
  if (opts.row_begin != 0 || opts.row_end != 0) {
    r0 = opts.row_begin;
    r1 = opts.row_end;
    if (r0 < 0 || r1 > n || r0 >= r1) return fail(ctx, EVOC_ERR_ARG, "row_begin/row_end out of range");
  }
  int64_t kk = k < n - 1 ? k : n - 1;
  if (kk < 1) kk = 1;
  const int keff = int(kk);
  if (out_k) *out_k = keff;
  const int form = resolve_form(dtype, opts.form, keff);
  const bool on_dev = opts.buffers_on_device != 0;
  EVOC_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
  Stage total(ctx, "total");

  // Output staging.
  const int64_t nq = r1 - r0;
  const size_t out_elems = size_t(nq) * size_t(keff);
  Job job{n, r0, nq, keff, out_idx, out_raw, out_dist, nullptr};
  if (!on_dev) {
    EVOC_TRY(ctx->out_idx.ensure(out_elems * 4), "alloc out_idx");
    job.idx = ctx->out_idx.as<int32_t>();
    if (out_dist) {
      EVOC_TRY(ctx->out_dist.ensure(out_elems * 4), "alloc out_dist");
      job.dist = ctx->out_dist.as<float>();
    }
    if (out_raw) {
      EVOC_TRY(ctx->out_raw.ensure(out_elems * 4), "alloc out_raw");
      job.raw = ctx->out_raw.as<float>();
    }
  }
  EVOC_TRY(ctx->flag.ensure(64), "alloc flag");
  int* d_flags = ctx->flag.as<int>();  // [0] prepare_float, [1] scan status
  EVOC_TRY(cudaMemsetAsync(d_flags, 0, 64, ctx->stream), "clear flags");
  job.status = d_flags + 1;
  int rc = EVOC_OK;
  // The reference's integer brute-force branch (src/knn.rs:418-421) takes
  // precedence over the form, as it does over NN-descent there.
  const bool brute = dtype != EVOC_DTYPE_F32 && n <= opts.brute_force_max_n;
  if (opts.strict_precision && !brute)
    return fail(ctx, EVOC_ERR_UNSUPPORTED,
                "strict_precision: the Strict backend's results come from its RP-forest NN-descent "
                "(src/knn.rs:423-445), which no GPU form reproduces bit for bit; only i8/u8 data with "
                "n <= brute_force_max_n (the reference's brute-force branch) is bit-identical here. "
                "Set strict_precision = false to take the exact GPU search");
  if (brute) {
    const int64_t ldb = dtype == EVOC_DTYPE_I8 ? round_up(dim, 128) : round_up(dim, 64);
    if (evoc::brute_force_smem_per_warp(ldb, keff) > 200 * 1024)
      return fail(ctx, EVOC_ERR_UNSUPPORTED, "k and row length too large for the brute-force branch");
    rc = stage_rows(ctx, data, n, dim, ldb, on_dev);
    if (rc) return rc;
    Stage st(ctx, "brute_force");
    EVOC_TRY(evoc::launch_brute_force_heap(dtype, ctx->x.p, n, ldb, keff, r0, r1, job.idx, job.raw, job.dist, ctx->sms,
                                           ctx->stream),
             "brute force");
    ctx->launches += 1;
  } else if (dtype == EVOC_DTYPE_F32) {
    if (form != EVOC_FORM_FP32 && form != EVOC_FORM_BF16_RERANK && form != EVOC_FORM_NNDESCENT)
      return fail(ctx, EVOC_ERR_UNSUPPORTED, "form not built for f32 in this library");
    const int ld = int(round_up(dim, 16));
    rc = stage_rows(ctx, data, n, dim * 4, int64_t(ld) * 4, on_dev);
    if (rc) return rc;
    {
      Stage st(ctx, "prepare_float");
      EVOC_TRY(ctx->norms.ensure(size_t(n) * 4), "alloc norms");
      EVOC_TRY(evoc::launch_prepare_float(ctx->x.as<float>(), n, ld, int(dim), ctx->norms.as<float>(), d_flags,
                                          ctx->sms, ctx->stream),
               "prepare_float");
      ctx->launches += 2;
    }
    if (form == EVOC_FORM_FP32) rc = run_fp32(ctx, job, ld);
    else if (form == EVOC_FORM_BF16_RERANK) rc = run_bf16_rerank(ctx, opts, job, ld, int(dim));
    else {
      // The pivot cells come from the FP16 tensor-core scan; the join reads the f32 rows.
      const int64_t ldb = round_up(dim, 64);
      const int64_t rows = evoc::padded_rows(n);
      {
        Stage st(ctx, "to_half");
        EVOC_TRY(ctx->xb.ensure(size_t(rows * ldb * 2)), "alloc 16-bit rows");
        EVOC_TRY(evoc::launch_to_half(ctx->x.as<float>(), rows, n, ld, int(dim), ctx->xb.p, int(ldb), evoc::kHalfF16,
                                      nullptr, nullptr, nullptr, ctx->sms, ctx->stream),
                 "to 16-bit");
        ctx->launches += 1;
      }
      rc = run_nndescent(ctx, opts, job, EVOC_DTYPE_F32, ldb * 2, ctx->xb.p, ld, int(dim), rng_state);
    }
  } else if (dtype == EVOC_DTYPE_I8) {
    if (form != EVOC_FORM_EXACT_INT && form != EVOC_FORM_NNDESCENT)
      return fail(ctx, EVOC_ERR_UNSUPPORTED, "form not built for i8 in this library");
    const int64_t ldb = round_up(dim, 128);
    rc = stage_rows(ctx, data, n, dim, ldb, on_dev);
    if (rc) return rc;
    if (form == EVOC_FORM_EXACT_INT) rc = run_int8(ctx, job, ldb);
    else rc = run_nndescent(ctx, opts, job, EVOC_DTYPE_I8, ldb, ctx->x.p, 0, int(dim), rng_state);
  } else {
    if (form != EVOC_FORM_EXACT_INT && form != EVOC_FORM_POPCOUNT && form != EVOC_FORM_NNDESCENT)
      return fail(ctx, EVOC_ERR_UNSUPPORTED, "form not built for u8 in this library");
    const int64_t ldb = round_up(dim, 64);
    rc = stage_rows(ctx, data, n, dim, ldb, on_dev);
    if (rc) return rc;
    if (form == EVOC_FORM_EXACT_INT) rc = run_jaccard_tc(ctx, job, ldb, dim);
    else if (form == EVOC_FORM_POPCOUNT) rc = run_jaccard(ctx, job, ldb);
    else rc = run_nndescent(ctx, opts, job, EVOC_DTYPE_U8, ldb, ctx->x.p, 0, int(dim), rng_state);
  }
  if (rc) return rc;
  int flags[2] = {0, 0};
  if (!on_dev) {
    Stage st(ctx, "d2h_out");
    EVOC_TRY(cudaMemcpyAsync(out_idx, job.idx, out_elems * 4, cudaMemcpyDeviceToHost, ctx->stream), "download idx");
    if (out_dist)
      EVOC_TRY(cudaMemcpyAsync(out_dist, job.dist, out_elems * 4, cudaMemcpyDeviceToHost, ctx->stream),
               "download dist");
    if (out_raw)
      EVOC_TRY(cudaMemcpyAsync(out_raw, job.raw, out_elems * 4, cudaMemcpyDeviceToHost, ctx->stream), "download raw");
  }
  EVOC_TRY(cudaMemcpyAsync(flags, d_flags, sizeof(flags), cudaMemcpyDeviceToHost, ctx->stream), "read status");
  total.end();
  EVOC_TRY(cudaStreamSynchronize(ctx->stream), "knn_graph");
  if (flags[1] == evoc::kStatusBadOrder || flags[1] == evoc::kStatusBadCandidate)
    return fail(ctx, EVOC_ERR_CUDA, "device self-check failed (code " + std::to_string(flags[1]) + ")");
  if (flags[1] != 0)
    return fail(ctx, EVOC_ERR_TIMEOUT, "a kernel pipeline wait timed out (stage " + std::to_string(flags[1]) + ")");
  return EVOC_OK;
}

// ---------------------------------------------------------------------------
// Batches of small requests (evoc_gpu_knn_graph_batch)
// ---------------------------------------------------------------------------
inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

struct BatchJobPlan {
  int64_t n, dim, rows, ld, ldb;
  int keff, C, keep;
  size_t off_x, off_xb, off_norms, off_cand, off_flag;
  size_t off_rnorm, off_hnorm, off_maxes, off_bound;  // f32 with the certificate
};

struct BatchLayout {
  std::vector<BatchJobPlan> jobs;
  size_t off_fail = 0;  // (request, row) pairs of rows that failed the certificate
  int64_t max_n = 0;
  size_t ws_bytes = 0;
  size_t off_sj = 0, off_rj = 0, off_it = 0, tab_bytes = 0;
  int max_keep = 1;
  int64_t n_items = 0, total_rows = 0, total_blocks = 0;
};

// Largest keep the batch scan supports (its heaps must fit in shared memory).
constexpr int kBatchMaxKeep = 80;
constexpr int32_t kBatchMaxJobs = 4096;

// Sizes and offsets of a batch's arena and tables; the serving planner uses
// the same function, so admission counts exactly what the batch allocates.
int batch_layout(bool f32, const evoc_gpu_opts& opts, int32_t n_jobs, const int64_t* n, const int64_t* dim,
                 int32_t k, BatchLayout* L) {
  L->jobs.resize(size_t(n_jobs));
  size_t ws = 0;
  for (int i = 0; i < n_jobs; i++) {
    BatchJobPlan& J = L->jobs[size_t(i)];
    if (n[i] <= 0) return EVOC_ERR_EMPTY;
    if (dim[i] <= 0) return EVOC_ERR_ARG;
    J.n = n[i];
    J.dim = dim[i];
    J.rows = evoc::padded_rows(J.n);
    J.keff = int(std::max<int64_t>(1, std::min<int64_t>(k, J.n - 1)));
    if (f32) {
      J.ld = round_up(J.dim, 16);
      J.ldb = round_up(J.dim, 64) * 2;
      J.C = int(bf16_candidates(opts, J.n, J.keff));
      J.keep = J.C;
      J.off_x = ws;
      ws += align_up(size_t(J.rows * J.ld * 4), 256);
      J.off_xb = ws;
      ws += align_up(size_t(J.rows * J.ldb), 256);
      J.off_norms = ws;
      ws += align_up(size_t(J.n) * 4, 256);
      J.off_cand = ws;
      ws += align_up(size_t(J.n) * size_t(J.C) * 4, 256);
      J.off_flag = ws;
      ws += 256;
      if (opts.certify) {
        J.off_rnorm = ws;
        ws += align_up(size_t(J.n) * 4, 256);
        J.off_hnorm = ws;
        ws += align_up(size_t(J.n) * 4, 256);
        J.off_maxes = ws;
        ws += 256;
        J.off_bound = ws;
        ws += align_up(size_t(J.n) * 4, 256);
      } else {
        J.off_rnorm = J.off_hnorm = J.off_maxes = J.off_bound = 0;
      }
    } else {
      J.ld = 0;
      J.ldb = round_up(J.dim, 128);
      J.C = J.keff;
      J.keep = J.keff;
      J.off_xb = ws;
      ws += align_up(size_t(J.rows * J.ldb), 256);
      J.off_x = J.off_norms = J.off_cand = J.off_flag = 0;
      J.off_rnorm = J.off_hnorm = J.off_maxes = J.off_bound = 0;
    }
    L->max_n = std::max(L->max_n, J.n);
    L->max_keep = std::max(L->max_keep, J.keep);
    L->n_items += (J.n + 127) / 128;
    L->total_rows += J.n;
    L->total_blocks += (J.n + 127) / 128;
  }
  if (f32 && opts.certify) {
    L->off_fail = ws;
    ws += align_up(size_t(L->total_rows) * 8, 256);
  }
  L->ws_bytes = std::max<size_t>(ws, 256);
  // Fixed offsets (room for the largest batch), so the tables' addresses --
  // which the kernels take as launch parameters -- do not depend on the batch
  // and one captured graph serves every batch on this buffer.
  L->off_sj = 64;
  L->off_rj = align_up(L->off_sj + sizeof(evoc::ScanJob) * size_t(kBatchMaxJobs), 64);
  L->off_it = align_up(L->off_rj + sizeof(evoc::BatchRowJob) * size_t(kBatchMaxJobs), 64);
  L->tab_bytes = align_up(L->off_it + sizeof(evoc::ScanItem) * size_t(L->n_items), 256);
  return EVOC_OK;
}

int knn_batch_impl(evoc_gpu_ctx* ctx, const evoc_gpu_opts* opts_in, int32_t dtype, int32_t n_jobs,
                   const void* const* data, const int64_t* n, const int64_t* dim, int32_t k, int32_t* const* out_idx,
                   float* const* out_dist, float* const* out_raw, int32_t* out_k) {
  if (!ctx) return EVOC_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  ctx->err.clear();
  ctx->n_stages = 0;
  ctx->launches = 0;
  ctx->cert_checked = ctx->cert_second = ctx->cert_exact = 0;
  ctx->sym_sample = ctx->sym_cap = ctx->sym_max_offers = ctx->sym_overflow = 0;
  evoc_gpu_opts opts;
  evoc_gpu_default_opts(&opts);
  if (opts_in) {
    if (opts_in->struct_size != sizeof(evoc_gpu_opts)) return fail(ctx, EVOC_ERR_ARG, "opts.struct_size mismatch");
    opts = *opts_in;
  }
  if (k <= 0) return fail(ctx, EVOC_ERR_K, "n_neighbors must be positive");
  if (n_jobs <= 0 || n_jobs > kBatchMaxJobs || !data || !n || !dim || !out_idx)
    return fail(ctx, EVOC_ERR_ARG, "bad batch arguments (1 <= n_jobs <= 4096, non-null arrays)");
  if (!opts.buffers_on_device) return fail(ctx, EVOC_ERR_ARG, "batches take device buffers (buffers_on_device = 1)");
  if (opts.row_begin != 0 || opts.row_end != 0) return fail(ctx, EVOC_ERR_ARG, "batches build whole graphs");
  const bool f32 = dtype == EVOC_DTYPE_F32;
  const int form = resolve_form(dtype, opts.form);
  if (!((f32 && form == EVOC_FORM_BF16_RERANK) || (dtype == EVOC_DTYPE_I8 && form == EVOC_FORM_EXACT_INT)))
    return fail(ctx, EVOC_ERR_UNSUPPORTED, "batches run the BF16+rerank form (f32) or the exact int8 form (i8)");
  for (int i = 0; i < n_jobs; i++) {
    if (n[i] <= 0) return fail(ctx, EVOC_ERR_EMPTY, "empty embedding matrix in the batch");
    if (n[i] >= (int64_t(1) << 31) - 1) return fail(ctx, EVOC_ERR_ARG, "n exceeds int32 index range");
    if (!data[i] || !out_idx[i]) return fail(ctx, EVOC_ERR_ARG, "null data or out_idx in the batch");
  }
  BatchLayout L;
  int rc = batch_layout(f32, opts, n_jobs, n, dim, k, &L);
  if (rc) return fail(ctx, rc, "bad request in the batch");
  if (L.max_keep > kBatchMaxKeep) return fail(ctx, EVOC_ERR_UNSUPPORTED, "k too large for a batch");
  EVOC_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
  Stage total(ctx, "batch");
  EVOC_TRY(ctx->batch_ws.ensure(L.ws_bytes), "alloc batch arena");
  EVOC_TRY(ctx->batch_tab.ensure(L.tab_bytes), "alloc batch tables");
  if (ctx->batch_host_bytes < L.tab_bytes) {
    if (ctx->batch_host) cudaFreeHost(ctx->batch_host);
    ctx->batch_host = nullptr;
    ctx->batch_host_bytes = 0;
    const size_t want = L.tab_bytes + L.tab_bytes / 4;
    EVOC_TRY(cudaHostAlloc(&ctx->batch_host, want, cudaHostAllocDefault), "alloc pinned batch tables");
    ctx->batch_host_bytes = want;
  }
  // Host tables.
  uint8_t* H = static_cast<uint8_t*>(ctx->batch_host);
  uint8_t* W = ctx->batch_ws.as<uint8_t>();
  uint8_t* T = ctx->batch_tab.as<uint8_t>();
  std::memset(H, 0, L.off_sj);
  auto* hdr = reinterpret_cast<evoc::BatchHeader*>(H);
  hdr->n_jobs = n_jobs;
  hdr->n_items = int32_t(L.n_items);
  hdr->status = 0;
  hdr->fail_count = 0;
  hdr->total_rows = L.total_rows;
  hdr->total_blocks = L.total_blocks;
  const bool certify = f32 && opts.certify != 0;
  hdr->fail_list = certify ? reinterpret_cast<int32_t*>(W + L.off_fail) : nullptr;
  hdr->fail_cap = certify ? L.total_rows : 0;
  if (f32 && opts.scan_type != evoc::kHalfF16 && opts.scan_type != evoc::kHalfBf16)
    return fail(ctx, EVOC_ERR_ARG, "scan_type must be 0 (FP16) or 1 (BF16)");
  auto* sj = reinterpret_cast<evoc::ScanJob*>(H + L.off_sj);
  auto* rj = reinterpret_cast<evoc::BatchRowJob*>(H + L.off_rj);
  auto* it = reinterpret_cast<evoc::ScanItem*>(H + L.off_it);
  int64_t row_base = 0, blk_base = 0;
  for (int i = 0; i < n_jobs; i++) {
    const BatchJobPlan& J = L.jobs[size_t(i)];
    evoc::BatchRowJob& R = rj[i];
    R.n = J.n;
    R.dim = J.dim;
    R.rows = J.rows;
    R.row_bytes = f32 ? J.dim * 4 : J.dim;
    R.ld = J.ld;
    R.ldb = J.ldb;
    R.row_base = row_base;
    R.blk_base = blk_base;
    row_base += J.n;
    blk_base += (J.n + 127) / 128;
    R.src = static_cast<const uint8_t*>(data[i]);
    R.x = f32 ? reinterpret_cast<float*>(W + J.off_x) : nullptr;
    R.xb = W + J.off_xb;
    R.norms = f32 ? reinterpret_cast<float*>(W + J.off_norms) : nullptr;
    R.flag = f32 ? reinterpret_cast<int32_t*>(W + J.off_flag) : nullptr;
    R.cand = f32 ? reinterpret_cast<int32_t*>(W + J.off_cand) : nullptr;
    R.C = J.C;
    R.keff = J.keff;
    R.out_idx = out_idx[i];
    R.out_dist = out_dist ? out_dist[i] : nullptr;
    R.out_raw = out_raw ? out_raw[i] : nullptr;
    R.half_type = f32 ? opts.scan_type : 0;
    R.certify = certify ? 1 : 0;
    R.rnorm = certify ? reinterpret_cast<float*>(W + J.off_rnorm) : nullptr;
    R.hnorm = certify ? reinterpret_cast<float*>(W + J.off_hnorm) : nullptr;
    R.maxes = certify ? reinterpret_cast<unsigned int*>(W + J.off_maxes) : nullptr;
    R.bound = certify ? reinterpret_cast<float*>(W + J.off_bound) : nullptr;
    const bool ok =
        f32 ? evoc::encode_scan_job(&sj[i], evoc::kScanHalf, R.xb, J.rows, J.n, J.ldb, J.C, 0, 0, R.cand, nullptr,
                                    nullptr, R.bound, R.half_type)
            : evoc::encode_scan_job(&sj[i], evoc::kScanInt8, R.xb, J.rows, J.n, J.ldb, J.keff, 1, EVOC_DTYPE_I8,
                                    R.out_idx, R.out_raw, R.out_dist, nullptr, 0);
    if (!ok) return fail(ctx, EVOC_ERR_CUDA, "tensor map encoding failed for a batch request");
    if (out_k) out_k[i] = J.keff;
  }
  // Work-list: the query blocks of the largest requests first, so the
  // persistent CTAs' round-robin share of the items is balanced.
  std::vector<int32_t> by_size(static_cast<size_t>(n_jobs));
  for (int i = 0; i < n_jobs; i++) by_size[size_t(i)] = i;
  std::stable_sort(by_size.begin(), by_size.end(),
                   [&](int32_t a, int32_t b) { return L.jobs[size_t(a)].n > L.jobs[size_t(b)].n; });
  int64_t w = 0;
  for (int32_t i : by_size)
    for (int64_t qb = 0; qb < (L.jobs[size_t(i)].n + 127) / 128; qb++) it[w++] = evoc::ScanItem{i, int32_t(qb)};
  EVOC_TRY(cudaMemcpyAsync(T, H, L.off_sj + sizeof(evoc::ScanJob) * size_t(n_jobs), cudaMemcpyHostToDevice,
                           ctx->stream),
           "upload batch tables");
  EVOC_TRY(cudaMemcpyAsync(T + L.off_rj, H + L.off_rj, sizeof(evoc::BatchRowJob) * size_t(n_jobs),
                           cudaMemcpyHostToDevice, ctx->stream),
           "upload batch tables");
  EVOC_TRY(cudaMemcpyAsync(T + L.off_it, H + L.off_it, sizeof(evoc::ScanItem) * size_t(L.n_items),
                           cudaMemcpyHostToDevice, ctx->stream),
           "upload batch tables");
  auto* d_hdr = reinterpret_cast<evoc::BatchHeader*>(T);
  auto* d_sj = reinterpret_cast<const evoc::ScanJob*>(T + L.off_sj);
  auto* d_rj = reinterpret_cast<const evoc::BatchRowJob*>(T + L.off_rj);
  auto* d_it = reinterpret_cast<const evoc::ScanItem*>(T + L.off_it);
  const int mode = f32 ? evoc::kScanHalf : evoc::kScanInt8;
  EVOC_TRY(evoc::prepare_tc_scan_batch(mode, L.max_keep), "batch scan attributes");
  // Grids sized for this batch (rounded up to a power of two, so few distinct
  // launch configurations occur): a small batch takes a few SMs and runs
  // beside the other lanes' work instead of waiting for every SM.
  auto bucket = [](int64_t v, int64_t cap) {
    int64_t b = 1;
    while (b < v && b < cap) b <<= 1;
    return int(b < cap ? b : cap);
  };
  int64_t words = 0;
  for (const BatchJobPlan& J : L.jobs) words += f32 ? J.rows * J.ld : J.rows * J.ldb / 4;
  const int grids[4] = {bucket((words + 255) / 256, int64_t(ctx->sms) * 8),
                        bucket(L.total_blocks, int64_t(ctx->sms) * 8), bucket(L.n_items, ctx->sms),
                        bucket((L.total_rows + 7) / 8, int64_t(ctx->sms) * 16)};
  // The table offsets are fixed; the graph is keyed on everything else its
  // launch parameters hold.
  const int keep_odd = L.max_keep | 1;
  const int gkey = (certify ? 1 : 0) | (f32 ? opts.scan_type : 0) << 1;  // kernels' per-batch constants
  auto launch_all = [&](cudaStream_t st) -> cudaError_t {
    cudaError_t e = evoc::launch_batch_rows(f32, d_hdr, d_rj, grids[0], grids[1], st);
    if (e == cudaSuccess)
      e = evoc::launch_tc_scan_batch(mode, d_hdr, d_sj, d_it, L.max_keep, grids[2], ctx->timeout_ns, st,
                                     f32 ? opts.scan_type : 0);
    if (e == cudaSuccess && f32) e = evoc::launch_batch_rerank(d_hdr, d_rj, grids[3], st);
    return e;
  };
  ctx->launches += f32 ? 6 : 2;
  if (ctx->use_graphs && !ctx->sync_check) {
    // Drop graphs captured over an older table buffer.
    for (size_t g = 0; g < ctx->batch_graphs.size();) {
      if (ctx->batch_graphs[g].tab != ctx->batch_tab.p) {
        cudaGraphExecDestroy(ctx->batch_graphs[g].exec);
        ctx->batch_graphs.erase(ctx->batch_graphs.begin() + long(g));
      } else {
        g++;
      }
    }
    cudaGraphExec_t exec = nullptr;
    for (const auto& g : ctx->batch_graphs)
      if (g.f32 == f32 && g.keep_odd == keep_odd && g.tab == ctx->batch_tab.p && g.key == gkey &&
          std::equal(grids, grids + 4, g.grids))
        exec = g.exec;
    if (!exec) {
      cudaGraph_t graph = nullptr;
      EVOC_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal), "begin batch capture");
      const cudaError_t le = launch_all(ctx->stream);
      const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
      if (le != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return cuda_fail(ctx, le, "batch launches");
      }
      EVOC_TRY(ce, "end batch capture");
      const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      EVOC_TRY(ie, "instantiate batch graph");
      ctx->batch_graphs.push_back(
          {f32, keep_odd, gkey, ctx->batch_tab.p, {grids[0], grids[1], grids[2], grids[3]}, exec});
    }
    EVOC_TRY(cudaGraphLaunch(exec, ctx->stream), "launch batch graph");
  } else {
    EVOC_TRY(launch_all(ctx->stream), "batch launches");
  }
  int32_t st2[2] = {0, 0};  // status, fail_count
  EVOC_TRY(cudaMemcpyAsync(st2, &d_hdr->status, sizeof(st2), cudaMemcpyDeviceToHost, ctx->stream),
           "read batch status");
  EVOC_TRY(cudaStreamSynchronize(ctx->stream), "batch");
  int status = st2[0];
  ctx->cert_checked = certify ? L.total_rows : 0;
  if (status == 0 && certify && st2[1] > 0) {
    // Rows that failed the certificate: each request's rescans, as a single call makes them.
    const int64_t nf = std::min<int64_t>(st2[1], L.total_rows);
    std::vector<int32_t> pairs(size_t(nf) * 2);
    EVOC_TRY(cudaMemcpy(pairs.data(), W + L.off_fail, pairs.size() * 4, cudaMemcpyDeviceToHost), "read failed rows");
    std::vector<std::vector<int32_t>> by_job(static_cast<size_t>(n_jobs));
    for (int64_t f = 0; f < nf; f++) by_job[size_t(pairs[size_t(2 * f)])].push_back(pairs[size_t(2 * f + 1)]);
    const CertLayout CL = cert_layout(L.max_n, L.max_n);
    EVOC_TRY(ctx->cert.ensure(CL.total), "alloc certificate");
    uint8_t* cb = ctx->cert.as<uint8_t>();
    int64_t second = 0, exact = 0;
    for (int i = 0; i < n_jobs; i++) {
      std::vector<int32_t>& rows_i = by_job[size_t(i)];
      if (rows_i.empty()) continue;
      std::sort(rows_i.begin(), rows_i.end());
      const BatchJobPlan& J = L.jobs[size_t(i)];
      const evoc::BatchRowJob& R = rj[i];
      int32_t* fail1 = reinterpret_cast<int32_t*>(cb + CL.fail1);
      EVOC_TRY(cudaMemcpyAsync(fail1, rows_i.data(), rows_i.size() * 4, cudaMemcpyHostToDevice, ctx->stream),
               "upload failed rows");
      evoc::CertArgs ca{R.bound, R.rnorm, R.hnorm, R.maxes, int(J.ldb / 2), nullptr, nullptr, 0};
      RescanJob rsj{R.x, int(J.ld), int(J.dim), R.xb, J.ldb / 2, J.rows, J.n, 0, J.n, J.keff, R.half_type, J.C,
                    R.out_idx, R.out_raw, R.out_dist, &d_hdr->status, ca};
      int64_t s2 = 0, ex = 0;
      const int rc = certify_rescan(ctx, rsj, fail1, int64_t(rows_i.size()), reinterpret_cast<int32_t*>(cb + CL.fail2),
                                    reinterpret_cast<float*>(cb + CL.bound2),
                                    reinterpret_cast<int32_t*>(cb + CL.counts), &s2, &ex);
      if (rc) return rc;
      second += s2;
      exact += ex;
    }
    ctx->cert_second = second;
    ctx->cert_exact = exact;
    EVOC_TRY(cudaMemcpyAsync(&status, &d_hdr->status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream),
             "read batch status");
    EVOC_TRY(cudaStreamSynchronize(ctx->stream), "batch rescans");
  }
  total.end();
  if (status == evoc::kStatusBadOrder || status == evoc::kStatusBadCandidate)
    return fail(ctx, EVOC_ERR_CUDA, "device self-check failed in a batch (code " + std::to_string(status) + ")");
  if (status != 0)
    return fail(ctx, EVOC_ERR_TIMEOUT, "a kernel pipeline wait timed out in a batch (stage " +
                                           std::to_string(status) + ")");
  return EVOC_OK;
}

// ---------------------------------------------------------------------------
// Autotuner of the scan's kernel variants
// ---------------------------------------------------------------------------
std::mutex g_tune_file_mu;  // appends to a cache file from several contexts

int tune_load_impl(evoc_gpu_ctx* ctx, const char* path) {
  std::ifstream f(path);
  if (!f) return -1;
  std::string line;
  int loaded = 0;
  while (std::getline(f, line)) {
    int ver = 0, mode = 0, keep = 0, l2 = 0, v = 0;
    long long rb = 0;
    double ms = 0.0;
    if (std::sscanf(line.c_str(), "evoc-tune %d mode=%d keep=%d row_bytes=%lld log2n=%d variant=%d ms=%lf", &ver,
                    &mode, &keep, &rb, &l2, &v, &ms) == 7 &&
        ver == 1 && v >= 0 && v < evoc::kScanVariants) {
      ctx->tune[std::make_tuple(mode, keep, int64_t(rb), l2)] = v;
      loaded++;
    }
  }
  return loaded;
}

int autotune_impl(evoc_gpu_ctx* ctx, int32_t dtype, int32_t form_in, int64_t n, int64_t dim, int32_t k,
                  const char* cache_path, char* report, int32_t report_len) {
  if (!ctx) return EVOC_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  ctx->err.clear();
  if (k <= 0) return fail(ctx, EVOC_ERR_K, "n_neighbors must be positive");
  if (n <= 1 || dim <= 0) return fail(ctx, EVOC_ERR_ARG, "n > 1 and dim > 0 required");
  evoc_gpu_opts opts;
  evoc_gpu_default_opts(&opts);
  const int form = resolve_form(dtype, form_in);
  const int keff = int(std::max<int64_t>(1, std::min<int64_t>(k, n - 1)));
  int mode, keep, final_mode, out_dtype;
  int64_t row_bytes;
  if (dtype == EVOC_DTYPE_F32 && form == EVOC_FORM_BF16_RERANK) {
    mode = evoc::kScanHalf;
    keep = int(bf16_candidates(opts, n, keff));
    row_bytes = round_up(dim, 64) * 2;
    final_mode = 0;
    out_dtype = 0;
  } else if (dtype == EVOC_DTYPE_I8 && form == EVOC_FORM_EXACT_INT) {
    mode = evoc::kScanInt8;
    keep = keff;
    row_bytes = round_up(dim, 128);
    final_mode = 1;
    out_dtype = EVOC_DTYPE_I8;
  } else if (dtype == EVOC_DTYPE_U8 && form == EVOC_FORM_EXACT_INT) {
    mode = evoc::kScanJaccard;
    keep = keff;
    row_bytes = expanded_row_bytes(dim);
    final_mode = 1;
    out_dtype = EVOC_DTYPE_U8;
  } else {
    return fail(ctx, EVOC_ERR_UNSUPPORTED, "only the tensor-core forms (BF16+rerank, exact int8 / binary) are tuned");
  }
  EVOC_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
  // Synthetic rows of the request's shape: a sample that ranks the variants
  // by their cost per (query, key) pair.  65,536 rows, or 262,144 for
  // requests of a million rows and more: the share of the epilogue's heap
  // inserts falls as n grows, so a small sample over-rewards epilogue warps
  // at the expense of pipeline stages.
  const int64_t nt = std::min<int64_t>(n, n >= 1000000 ? 262144 : 65536);
  const int64_t rows = evoc::padded_rows(nt);
  EVOC_TRY(ctx->xb.ensure(size_t(rows * row_bytes)), "alloc tuning rows");
  const int32_t* pc = nullptr;
  if (mode == evoc::kScanJaccard) {
    const int64_t ldp = round_up(dim, 64);
    EVOC_TRY(ctx->x.ensure(size_t(rows * ldp)), "alloc tuning bits");
    EVOC_TRY(evoc::launch_fill_random(2, ctx->x.p, rows, ldp, nt, dim, 0x7157u, ctx->sms, ctx->stream), "fill");
    EVOC_TRY(ctx->popc.ensure(size_t(nt) * 4), "alloc popcounts");
    EVOC_TRY(evoc::launch_popcount_rows(ctx->x.p, nt, int(ldp / 4), ctx->popc.as<int32_t>(), ctx->sms, ctx->stream),
             "popcounts");
    EVOC_TRY(evoc::launch_expand_bits(ctx->x.p, nt, ldp, dim, ctx->xb.p, rows, row_bytes, ctx->sms, ctx->stream),
             "expand bits");
    pc = ctx->popc.as<int32_t>();
  } else {
    const int64_t bytes = mode == evoc::kScanHalf ? dim * 2 : dim;
    EVOC_TRY(evoc::launch_fill_random(mode == evoc::kScanHalf ? 0 : 1, ctx->xb.p, rows, row_bytes, nt, bytes, 0x7157u,
                                      ctx->sms, ctx->stream),
             "fill");
  }
  const int grid = scan_grid(ctx, nt);
  EVOC_TRY(ctx->cand.ensure(size_t(nt) * size_t(keep) * 4), "alloc tuning outputs");
  EVOC_TRY(ctx->out_dist.ensure(size_t(nt) * size_t(keep) * 4), "alloc tuning outputs");
  EVOC_TRY(ctx->scratch.ensure(size_t(grid) * 256 * size_t(keep) * 8), "alloc scratch");
  EVOC_TRY(ctx->flag.ensure(64), "alloc flag");
  int* status = ctx->flag.as<int>() + 1;
  cudaEvent_t e0, e1;
  EVOC_TRY(cudaEventCreate(&e0), "event");
  EVOC_TRY(cudaEventCreate(&e1), "event");
  std::string rep;
  // The automatic choice stays unless another variant is clearly faster:
  // timings within a few percent are noise at this sample size.
  const int automatic = evoc::tc_scan_automatic_variant(mode, keep);
  std::vector<float> times(evoc::kScanVariants, -1.0f);
  for (int v = 0; v < evoc::kScanVariants; v++) {
    if (!evoc::tc_scan_variant_feasible(v, keep, true)) continue;
    auto run = [&]() {
      return evoc::launch_tc_scan(mode, ctx->xb.p, rows, 0, nt, ctx->xb.p, rows, nt, row_bytes, keep,
                                  ctx->scratch.as<uint64_t>(), grid, 1, final_mode, out_dtype, ctx->cand.as<int32_t>(),
                                  nullptr, final_mode ? ctx->out_dist.as<float>() : nullptr, status, ctx->timeout_ns,
                                  pc, ctx->stream, v);
    };
    cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), ctx->stream);
    if (e == cudaSuccess) e = run();  // warm-up
    if (e == cudaSuccess) e = cudaEventRecord(e0, ctx->stream);
    for (int r = 0; r < 2 && e == cudaSuccess; r++) e = run();
    if (e == cudaSuccess) e = cudaEventRecord(e1, ctx->stream);
    int st = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return cuda_fail(ctx, e, "tuning run");
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= 2.0f;
    char buf[160];
    std::snprintf(buf, sizeof(buf), "%d %.3f ms %s%s\n", v, double(ms), evoc::tc_scan_variant_name(v),
                  st ? " (timed out)" : "");
    rep += buf;
    if (st == 0) times[size_t(v)] = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int best = (automatic >= 0 && times[size_t(automatic)] >= 0.0f) ? automatic : -1;
  for (int v = 0; v < evoc::kScanVariants; v++) {
    if (times[size_t(v)] < 0.0f) continue;
    if (best < 0 || times[size_t(v)] < 0.97f * times[size_t(best)]) best = v;
  }
  if (best < 0) return fail(ctx, EVOC_ERR_TIMEOUT, "no variant completed");
  const float best_ms = times[size_t(best)];
  ctx->tune[std::make_tuple(mode, keep, row_bytes, ilog2(n))] = best;
  char line[200];
  std::snprintf(line, sizeof(line), "evoc-tune 1 mode=%d keep=%d row_bytes=%lld log2n=%d variant=%d ms=%.3f\n", mode,
                keep, static_cast<long long>(row_bytes), ilog2(n), best, double(best_ms));
  rep += std::string("chosen: ") + line;
  if (cache_path && cache_path[0]) {
    std::lock_guard<std::mutex> flock(g_tune_file_mu);
    std::ofstream f(cache_path, std::ios::app);
    if (!f) return fail(ctx, EVOC_ERR_ARG, std::string("cannot append to ") + cache_path);
    f << line;
  }
  if (report && report_len > 0) {
    std::strncpy(report, rep.c_str(), size_t(report_len) - 1);
    report[report_len - 1] = '\0';
  }
  return EVOC_OK;
}

}  // namespace

extern "C" {

int evoc_gpu_version(void) { return 200; }

void evoc_gpu_default_opts(evoc_gpu_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->struct_size = sizeof(evoc_gpu_opts);
  o->form = EVOC_FORM_AUTO;
  o->oversample = 0;
  o->delta = 0.001f;
  o->delta_improv = 0.001f;
  o->scan_type = 0;  // FP16 operands
  o->certify = 1;
}

int evoc_gpu_ctx_create(int device, evoc_gpu_ctx** out) {
  if (!out) return EVOC_ERR_ARG;
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) return EVOC_ERR_CUDA;
  if (device < 0 || device >= count) return EVOC_ERR_ARG;
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return EVOC_ERR_CUDA;
  evoc_gpu_ctx* ctx = new evoc_gpu_ctx();
  ctx->device = device;
  cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
  if (const char* v = std::getenv("EVOC_SYNC_CHECK")) ctx->sync_check = v[0] == '1';
  if (const char* v = std::getenv("EVOC_NO_GRAPHS")) ctx->use_graphs = v[0] != '1';
  if (const char* v = std::getenv("EVOC_SYM_MIN_ROWS")) {
    const long long r = std::atoll(v);
    ctx->sym_min_rows = r < 0 ? 0 : r;
  }
  if (const char* v = std::getenv("EVOC_TUNE_CACHE"))
    if (v[0]) tune_load_impl(ctx, v);
  e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete ctx;
    return EVOC_ERR_CUDA;
  }
  ctx->base_stream = ctx->stream;
  *out = ctx;
  return EVOC_OK;
}

void evoc_gpu_ctx_destroy(evoc_gpu_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  ctx->stream = ctx->base_stream;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  DevBuf* bufs[] = {&ctx->x,        &ctx->scratch, &ctx->norms, &ctx->flag,   &ctx->out_idx,
                    &ctx->out_raw,  &ctx->out_dist, &ctx->xb,   &ctx->cand,   &ctx->labels,
                    &ctx->order,    &ctx->hist,    &ctx->cursor, &ctx->pivots, &ctx->popc,
                    &ctx->g_idx,    &ctx->g_dist,  &ctx->g_sigma, &ctx->g_rho, &ctx->g_indptr,
                    &ctx->g_indices, &ctx->g_data, &ctx->g_work, &ctx->nnd_work, &ctx->cert, &ctx->repair};
  for (DevBuf* b : bufs) b->release();
  for (auto& g : ctx->batch_graphs) cudaGraphExecDestroy(g.exec);
  ctx->batch_ws.release();
  ctx->batch_tab.release();
  if (ctx->batch_host) cudaFreeHost(ctx->batch_host);
  if (ctx->lp_pool) cudaMemPoolDestroy(ctx->lp_pool);
  for (auto& r : ctx->stages) {
    if (r.a) cudaEventDestroy(r.a);
    if (r.b) cudaEventDestroy(r.b);
  }
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* evoc_gpu_last_error(const evoc_gpu_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void* evoc_gpu_ctx_stream(const evoc_gpu_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int evoc_gpu_profile_enable(evoc_gpu_ctx* ctx, int enable) {
  if (!ctx) return EVOC_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  ctx->profiling = enable != 0;
  return EVOC_OK;
}

int evoc_gpu_profile_count(const evoc_gpu_ctx* ctx) { return ctx ? ctx->n_stages : 0; }

int evoc_gpu_profile_stage(const evoc_gpu_ctx* ctx, int i, char* name, int name_len, float* ms) {
  if (!ctx || i < 0 || i >= ctx->n_stages) return EVOC_ERR_ARG;
  const StageRec& r = ctx->stages[size_t(i)];
  if (name && name_len > 0) {
    std::strncpy(name, r.name.c_str(), size_t(name_len) - 1);
    name[name_len - 1] = '\0';
  }
  if (ms) {
    cudaSetDevice(ctx->device);
    if (cudaEventElapsedTime(ms, r.a, r.b) != cudaSuccess) return EVOC_ERR_CUDA;
  }
  return EVOC_OK;
}

int evoc_gpu_last_launch_count(const evoc_gpu_ctx* ctx) { return ctx ? ctx->launches : 0; }

int evoc_gpu_last_nndescent(const evoc_gpu_ctx* ctx, int32_t* iterations, int64_t* distance_evals,
                            int64_t* row_bytes) {
  if (!ctx) return EVOC_ERR_ARG;
  if (iterations) *iterations = ctx->nnd_iterations;
  if (distance_evals) *distance_evals = int64_t(ctx->nnd_evals);
  if (row_bytes) *row_bytes = ctx->nnd_row_bytes;
  return EVOC_OK;
}

int evoc_gpu_set_wait_limit(evoc_gpu_ctx* ctx, uint64_t ns, uint64_t producer_delay_ns) {
  if (!ctx) return EVOC_ERR_ARG;
  if (producer_delay_ns > 100000000ull) return fail(ctx, EVOC_ERR_ARG, "producer delay above 100 ms");
  std::lock_guard<std::mutex> lock(ctx->mu);
  ctx->timeout_ns = ns ? ns : 4000000000ull;
  ctx->delay_ns = producer_delay_ns;
  return EVOC_OK;
}

int evoc_gpu_set_symmetric_scan(evoc_gpu_ctx* ctx, int64_t min_rows) {
  if (!ctx) return EVOC_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  ctx->sym_min_rows = min_rows < 0 ? 0 : min_rows;
  return EVOC_OK;
}

int evoc_gpu_last_symmetric(const evoc_gpu_ctx* ctx, int64_t* sample_rows, int64_t* mailbox_cap,
                            int64_t* max_offers, int64_t* overflowed) {
  if (!ctx) return EVOC_ERR_ARG;
  if (sample_rows) *sample_rows = ctx->sym_sample;
  if (mailbox_cap) *mailbox_cap = ctx->sym_cap;
  if (max_offers) *max_offers = ctx->sym_max_offers;
  if (overflowed) *overflowed = ctx->sym_overflow;
  return EVOC_OK;
}

int evoc_gpu_last_certify(const evoc_gpu_ctx* ctx, int64_t* checked, int64_t* second_pass, int64_t* exact_rescan) {
  if (!ctx) return EVOC_ERR_ARG;
  if (checked) *checked = ctx->cert_checked;
  if (second_pass) *second_pass = ctx->cert_second;
  if (exact_rescan) *exact_rescan = ctx->cert_exact;
  return EVOC_OK;
}

int evoc_gpu_smooth_knn_dist(evoc_gpu_ctx* ctx, const float* dist, int64_t n, int32_t k, float n_neighbors,
                             int32_t buffers_on_device, float* sigma, float* rho) {
  return fuzzy_impl(ctx, nullptr, dist, n, k, n_neighbors, 0, buffers_on_device, sigma, rho, false, nullptr, nullptr,
                    nullptr, 0, nullptr);
}

int evoc_gpu_fuzzy_graph(evoc_gpu_ctx* ctx, const int32_t* idx, const float* dist, int64_t n, int32_t k,
                         float n_neighbors, int32_t symmetrize, int32_t buffers_on_device, float* sigma, float* rho,
                         int64_t* indptr, int32_t* indices, float* data, int64_t cap, int64_t* nnz) {
  return fuzzy_impl(ctx, idx, dist, n, k, n_neighbors, symmetrize, buffers_on_device, sigma, rho, true, indptr,
                    indices, data, cap, nnz);
}

int evoc_gpu_knn_graph(evoc_gpu_ctx* ctx, const evoc_gpu_opts* opts, int32_t dtype, const void* data, int64_t n,
                       int64_t dim, int32_t k, const int64_t* rng_state, int32_t* out_idx, float* out_dist,
                       int32_t* out_k) {
  return knn_impl(ctx, opts, dtype, data, n, dim, k, rng_state, out_idx, out_dist, nullptr, out_k);
}

int evoc_gpu_autotune(evoc_gpu_ctx* ctx, int32_t dtype, int32_t form, int64_t n, int64_t dim, int32_t k,
                      const char* cache_path, char* report, int32_t report_len) {
  return autotune_impl(ctx, dtype, form, n, dim, k, cache_path, report, report_len);
}

int evoc_gpu_tune_load(evoc_gpu_ctx* ctx, const char* cache_path) {
  if (!ctx || !cache_path) return -1;
  std::lock_guard<std::mutex> lock(ctx->mu);
  return tune_load_impl(ctx, cache_path);
}

int evoc_gpu_knn_graph_batch(evoc_gpu_ctx* ctx, const evoc_gpu_opts* opts, int32_t dtype, int32_t n_jobs,
                             const void* const* data, const int64_t* n, const int64_t* dim, int32_t k,
                             int32_t* const* out_idx, float* const* out_dist, float* const* out_raw, int32_t* out_k) {
  return knn_batch_impl(ctx, opts, dtype, n_jobs, data, n, dim, k, out_idx, out_dist, out_raw, out_k);
}

int evoc_gpu_knn_graph_raw(evoc_gpu_ctx* ctx, const evoc_gpu_opts* opts, int32_t dtype, const void* data,
                           int64_t n, int64_t dim, int32_t k, const int64_t* rng_state, int32_t* out_idx,
                           float* out_dist, float* out_raw, int32_t* out_k) {
  return knn_impl(ctx, opts, dtype, data, n, dim, k, rng_state, out_idx, out_dist, out_raw, out_k);
}

}  // extern "C"

namespace evoc {

// Mirrors the ensure() calls of knn_impl and the run_* functions above for a
// whole-graph request with device-resident outputs.  A form that fails its
// own checks (k or candidate limits) allocates no more than listed here.
void knn_buffer_needs(const evoc_gpu_ctx* ctx, const evoc_gpu_opts& opts, int32_t dtype, int64_t n, int64_t dim,
                      int32_t k, CtxSizes* need) {
  *need = CtxSizes{};
  size_t* b = need->b;
  const int64_t keff = std::max<int64_t>(1, std::min<int64_t>(k, n - 1));
  const int form = resolve_form(dtype, opts.form, keff);
  const int64_t rows = padded_rows(n);
  const int64_t qblocks = (n + 127) / 128;
  const int64_t grid = std::min<int64_t>(qblocks, ctx->sms);
  auto locality = [&](int64_t row_bytes) {
    const int64_t n_piv = pivot_count(n);
    b[kBufPivots] = size_t(padded_rows(n_piv) * row_bytes);
    b[kBufLabels] = size_t(n) * 4;
    b[kBufOrder] = size_t(n) * 4;
    b[kBufHist] = size_t(n_piv) * 4;
    b[kBufCursor] = size_t(n_piv) * 4;
  };
  auto nnd = [&]() {
    size_t sizes[kNndParts];
    b[kBufNnd] = nnd_work_sizes(n, int(keff), nnd_max_candidates(opts, int(keff)), sizes);
  };
  b[kBufFlag] = 64;
  if (dtype == EVOC_DTYPE_F32) {
    b[kBufX] = size_t(rows * round_up(dim, 16) * 4);
    b[kBufNorms] = size_t(n) * 4;
    const int64_t ldb = round_up(dim, 64);
    if (form == EVOC_FORM_FP32 ||
        (form == EVOC_FORM_BF16_RERANK && bf16_candidates(opts, n, int(keff)) > 256)) {
      const int64_t g = std::min<int64_t>(qblocks, int64_t(ctx->sms) * 2);
      b[kBufScratch] = size_t(g) * 128 * size_t(topk_capacity(int(keff))) * 8;
      b[kBufXb] = size_t(knn_f32_kt_cols(n)) * size_t(round_up(dim, 16)) * 4;  // the k-major copy
    } else if (form == EVOC_FORM_BF16_RERANK) {
      const int64_t C = bf16_candidates(opts, n, int(keff));
      b[kBufXb] = size_t(rows * ldb * 2);
      b[kBufCand] = size_t(n * C) * 4;
      b[kBufScratch] = size_t(grid) * 256 * size_t(C) * 8;
      if (n >= 65536) locality(ldb * 2);
      if (use_symmetric(ctx, opts.certify != 0, n, 0, n, C)) b[kBufSym] = sym_layout(n, C, ldb).total;
      if (opts.certify) {
        // the certificate and, should rows fail it, their rescans (bounded chunks)
        const int64_t C2 = second_pass_candidates(n, 256);  // the largest second pass
        const int64_t R = std::min<int64_t>(n, kRepairChunk);
        b[kBufCert] = cert_layout(n, n).total;
        b[kBufRepair] = repair_layout(R, round_up(dim, 16), ldb, C2, keff).total;
        const int64_t g3 = std::min<int64_t>((R + 127) / 128, int64_t(ctx->sms) * 2);
        b[kBufScratch] = std::max({b[kBufScratch], scan_scratch_bytes(ctx, R, C2),
                                   size_t(g3) * 128 * size_t(topk_capacity(int(keff))) * 8});
      }
    } else if (form == EVOC_FORM_NNDESCENT) {
      b[kBufXb] = size_t(rows * ldb * 2);
      locality(ldb * 2);
      nnd();
      b[kBufCand] = size_t(n) * size_t(keff) * 4;
    }
  } else if (dtype == EVOC_DTYPE_I8) {
    const int64_t ldb = round_up(dim, 128);
    b[kBufX] = size_t(rows * ldb);
    if (form == EVOC_FORM_EXACT_INT) {
      b[kBufScratch] = size_t(grid) * 256 * size_t(keff) * 8;
    } else if (form == EVOC_FORM_NNDESCENT) {
      locality(ldb);
      nnd();
    }
  } else {
    b[kBufX] = size_t(rows * round_up(dim, 64));
    if (form == EVOC_FORM_EXACT_INT) {
      b[kBufPopc] = size_t(n) * 4;
      b[kBufXb] = size_t(rows * expanded_row_bytes(dim));
      b[kBufScratch] = size_t(grid) * 256 * size_t(keff) * 8;
    } else if (form == EVOC_FORM_POPCOUNT) {
      b[kBufPopc] = size_t(n) * 4;
    } else if (form == EVOC_FORM_NNDESCENT) {
      b[kBufPopc] = size_t(n) * 4;
      nnd();
    }
  }
}

bool batch_buffer_needs(const evoc_gpu_opts& opts, int32_t dtype, int32_t n_jobs, const int64_t* n,
                        const int64_t* dim, int32_t k, CtxSizes* need) {
  *need = CtxSizes{};
  const int form = resolve_form(dtype, opts.form);
  const bool f32 = dtype == EVOC_DTYPE_F32;
  if (!((f32 && form == EVOC_FORM_BF16_RERANK) || (dtype == EVOC_DTYPE_I8 && form == EVOC_FORM_EXACT_INT)))
    return false;
  if (n_jobs <= 0 || n_jobs > kBatchMaxJobs || k <= 0) return false;
  BatchLayout L;
  if (batch_layout(f32, opts, n_jobs, n, dim, k, &L) != EVOC_OK || L.max_keep > kBatchMaxKeep) return false;
  need->b[kBufBatchWs] = L.ws_bytes;
  need->b[kBufBatchTab] = L.tab_bytes;
  if (f32 && opts.certify) {
    // rescans of rows that fail the certificate, request by request
    int64_t max_dim = 1, max_keff = 1;
    for (int i = 0; i < n_jobs; i++) {
      max_dim = std::max(max_dim, dim[i]);
      max_keff = std::max<int64_t>(max_keff, std::min<int64_t>(k, n[i] - 1));
    }
    const int64_t R = std::min<int64_t>(L.max_n, kRepairChunk);
    const int64_t C2 = second_pass_candidates(L.max_n, 256);  // the largest second pass
    need->b[kBufCert] = cert_layout(L.max_n, L.max_n).total;
    need->b[kBufRepair] = repair_layout(R, round_up(max_dim, 16), round_up(max_dim, 64), C2, max_keff).total;
    // the batch's plan holds no context scratch: the rescans' scan and exact pass size it
    const int sms = 148;  // upper bound of the grids on B200 (scan_grid caps at the SM count)
    const int64_t g2 = std::min<int64_t>((R + 127) / 128, sms);
    const int64_t g3 = std::min<int64_t>((R + 127) / 128, int64_t(sms) * 2);
    need->b[kBufScratch] = std::max(size_t(g2) * 256 * size_t(C2) * 8,
                                    size_t(g3) * 128 * size_t(topk_capacity(int(max_keff))) * 8);
  }
  return true;
}

void ctx_buffer_sizes(const evoc_gpu_ctx* ctx, CtxSizes* cur) {
  const DevBuf* bufs[kBufCount] = {&ctx->x,      &ctx->scratch, &ctx->norms,    &ctx->flag,      &ctx->xb,
                                   &ctx->cand,   &ctx->labels,  &ctx->order,    &ctx->hist,      &ctx->cursor,
                                   &ctx->pivots, &ctx->popc,    &ctx->nnd_work, &ctx->batch_ws,  &ctx->batch_tab,
                                   &ctx->cert,   &ctx->repair,  &ctx->sym};
  for (int i = 0; i < kBufCount; i++) cur->b[i] = bufs[i]->bytes;
}

CtxSizes grown_sizes(const CtxSizes& cur, const CtxSizes& need) {
  CtxSizes out = cur;
  for (int i = 0; i < kBufCount; i++)
    if (need.b[i] > cur.b[i]) out.b[i] = need.b[i] + need.b[i] / 8;
  return out;
}

void ctx_release_buffers(evoc_gpu_ctx* ctx) {
  std::lock_guard<std::mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  DevBuf* bufs[kBufCount] = {&ctx->x,      &ctx->scratch, &ctx->norms,    &ctx->flag,      &ctx->xb,
                             &ctx->cand,   &ctx->labels,  &ctx->order,    &ctx->hist,      &ctx->cursor,
                             &ctx->pivots, &ctx->popc,    &ctx->nnd_work, &ctx->batch_ws,  &ctx->batch_tab,
                             &ctx->cert,   &ctx->repair,  &ctx->sym};
  for (DevBuf* b : bufs) b->release();
  for (auto& g : ctx->batch_graphs) cudaGraphExecDestroy(g.exec);  // they name the freed tables
  ctx->batch_graphs.clear();
}

}  // namespace evoc
