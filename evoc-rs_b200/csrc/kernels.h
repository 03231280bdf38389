// Internal launcher declarations (not part of the C ABI).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace evoc {

// prep.cu
cudaError_t launch_prepare_float(float* X, int64_t n, int ld, int d, float* norms, int* not_unit, int sms,
                                 cudaStream_t stream);

// exact_f32.cu: plain FP32 exact search with fused top-k.
//   Queries q_begin .. q_end-1 of X against the n rows of X, query q written to output row
//   q - q_begin.  With Q and q_list (query rows gathered from X): query i is row i of Q, row
//   q_row0 + q_list[i] of X for the self rule, and is written to output row q_list[i].
size_t knn_f32_simt_smem();
// Columns of the k-major copy launch_knn_f32_kt writes for n rows.
int64_t knn_f32_kt_cols(int64_t n);
// Exact FP32 kNN from a k-major copy: writes XT (ld x knn_f32_kt_cols(n)
// floats) from the n x ld rows X, then searches queries q_begin .. q_end-1
// (q_begin % 4 == 0) against all n rows.
cudaError_t launch_knn_f32_kt(const float* X, int64_t n, int ld, float* XT, int k, int cap, uint64_t* scratch,
                              int grid, int32_t* out_idx, float* out_raw, float* out_dist, int64_t q_begin,
                              int64_t q_end, int sms, cudaStream_t stream);
cudaError_t launch_knn_f32_simt(const float* X, int64_t n, int ld, int k, int cap, uint64_t* scratch, int grid,
                                int32_t* out_idx, float* out_raw, float* out_dist, int64_t q_begin, int64_t q_end,
                                cudaStream_t stream, const float* Q = nullptr, const int32_t* q_list = nullptr,
                                int64_t q_row0 = 0, int n_splits = 1, uint64_t* partial = nullptr);
// With n_splits > 1, launch_knn_f32_simt writes each split's sorted top-k keys
// of the (q_end - q_begin) rows to `partial` (n_splits x rows x k); this
// takes each row's k best of them into the outputs (row q_list[r], or r).
cudaError_t launch_merge_key_splits(const uint64_t* partial, int64_t rows, int k, int n_splits,
                                    const int32_t* q_list, int32_t* out_idx, float* out_raw, float* out_dist,
                                    int sms, cudaStream_t stream);
// Bound on n_splits x rows x ... : the host keeps n_splits * rows <= this.
constexpr int64_t kSplitRowsMax = 2 * 148 * 128;

// Candidate-buffer capacity used by every fused top-k epilogue for k kept keys.
// Rows allocated for an n-row device matrix: the tensor-core scan's TMA boxes
// are 256 rows high, so every staged matrix is padded to a multiple of 256.
inline int64_t padded_rows(int64_t n) { return ((n < 1 ? 1 : n) + 255) / 256 * 256; }

inline int topk_capacity(int k) {
  int cap = 2 * k;
  if (cap < k + 64) cap = k + 64;
  return (cap + 7) & ~7;
}

}  // namespace evoc

namespace evoc {

// 16-bit operand type of the f32 tensor-core scan (evoc_gpu_opts.scan_type).
enum HalfType { kHalfF16 = 0, kHalfBf16 = 1 };

// prep.cu: f32 rows (ld) -> zero-padded 16-bit rows (ldb elements) for rows
// 0 .. n_rows-1 (rows n .. n_rows-1 zero).  FP16 flushes values below 2^-14
// to zero.  With rnorm/hnorm (n each) and maxes (2 words): each row's
// |x - half(x)| and |half(x)| rounded up, and their maxima as f32 bit patterns.
cudaError_t launch_to_half(const float* X, int64_t n_rows, int64_t n, int ld, int d, void* Y, int ldb, int half_type,
                           float* rnorm, float* hnorm, unsigned int* maxes, int sms, cudaStream_t stream);
// prep.cu: dst row i = src row row0 + list[i] (i < count), zero rows up to rows_out.
cudaError_t launch_gather_rows_list(const void* src, int64_t row_bytes, int64_t row0, const int32_t* list,
                                    int64_t count, int64_t rows_out, void* dst, int sms, cudaStream_t stream);

// tc_scan.cu: tcgen05 exact scan (FP16 or BF16 -> F32, or S8 -> S32) with fused top-k.
//   Q: query rows q_row0 .. q_row0+n_q-1 of a q_rows-row matrix; K: the first n_k of k_rows rows;
//   `row_bytes` per row (multiple of 128, 16-byte aligned bases); q_rows and k_rows are multiples
//   of 256 and rows past the data are zero.  Query i is written to output row i.
//   final_mode 1: out rows of `keep` sorted (idx, raw, transformed dist); 0: candidates (idx, raw).
//   mode 0: 16-bit float rows (half_type), cosine; 1: int8 rows, -(dot); 2: 0/1 int8 rows (expanded
//   bits), Jaccard from the intersection counts and the row popcounts `pc` (self_mode, Q == K).
//   q_self (optional): key index of query i for the self rule is q_self_base + q_self[i] (default
//   q_row0 + i), for query rows gathered from elsewhere.  out_bound (optional): per query, the raw
//   value of the keep-th kept key.
size_t tc_scan_smem_bytes();
enum ScanMode { kScanHalf = 0, kScanInt8 = 1, kScanJaccard = 2 };
cudaError_t launch_tc_scan(int mode, const void* Q, int64_t q_rows, int64_t q_row0, int64_t n_q, const void* K,
                           int64_t k_rows, int64_t n_k, int64_t row_bytes, int keep, uint64_t* scratch, int grid,
                           int self_mode, int final_mode, int dtype, int32_t* out_idx, float* out_raw, float* out_dist,
                           int* status, uint64_t timeout_ns, const int32_t* pc, cudaStream_t stream,
                           int variant = -1, int half_type = kHalfF16, const int32_t* q_self = nullptr,
                           float* out_bound = nullptr, int64_t q_self_base = 0, uint64_t delay_ns = 0);
// Symmetric scan of all n rows against themselves (16-bit operands, self
// rule, candidates out).  X holds the rows in a permuted order: scanned row i
// is data-set row perm[i].  Query block b multiplies only the key tiles from
// its own rows on, and scores of key rows past the block that reach thr[key]
// go to that row's mailbox (count[row] offers, the first cap kept in
// mail[row * cap ..], rows of the data set).  thr and perm hold n_ktiles *
// 256 entries (thr +inf past n), umin the smallest threshold of each 32, all
// in scanned order; out_idx / out_raw rows are data-set rows.  sym.cu
// computes the thresholds and merges the mailboxes.
bool tc_scan_sym_feasible(int keep);
cudaError_t launch_tc_scan_sym(const void* X, int64_t rows, int64_t n, int64_t row_bytes, int keep, int grid,
                               int32_t* out_idx, float* out_raw, int* status, uint64_t timeout_ns,
                               cudaStream_t stream, int half_type, const float* thr, const float* umin,
                               const int32_t* perm, int32_t* count, uint64_t* mail, int cap,
                               uint64_t delay_ns = 0);
// sym.cu.  Row j of dst = row j * stride of src for j < m, zero rows up to m_pad.
cudaError_t launch_gather_strided_rows(const void* src, int64_t row_bytes, int64_t stride, int64_t m, int64_t m_pad,
                                       void* dst, int sms, cudaStream_t stream);
// Mailbox thresholds of the scanned rows from the sample pre-scan's (C+1)-th
// raw values T (scanned order; hnorm of data-set row perm[i]); clears count.
cudaError_t launch_sym_thresholds(int64_t n, int64_t n_pad, const float* T, const float* hnorm,
                                  const int32_t* perm, const unsigned int* maxes, int half_len, float* thr,
                                  float* umin, int32_t* count, int sms, cudaStream_t stream);
// Folds each row's mailbox into its C own-side candidates (cand, own_raw), in
// place; bound[r] = C-th kept raw value (-f32::MAX after an overflow).
// stats[0] += overflowed rows, stats[1] = max(stats[1], most offers to a row).
cudaError_t launch_sym_merge(int64_t n, int C, int32_t* cand, const float* own_raw, const int32_t* count,
                             const uint64_t* mail, int cap, float* bound, int32_t* stats, int sms,
                             cudaStream_t stream);
// Kernel variants of the scan (0..14; -1 = automatic, tc_scan_automatic_variant:
// int8 with small keep 10, else the first that fits shared memory in the order
// 0..3, 14, else 4 with global heaps; 5, the CTA-pair variants 6..9, 12, 13
// and the four-group variant 11 are chosen only by the autotuner).
constexpr int kScanVariants = 15;
bool tc_scan_variant_feasible(int variant, int keep, bool has_scratch);
// Whether a launch with this variant (-1: automatic) and keep keeps its heaps in global scratch.
bool tc_scan_uses_global_heaps(int variant, int keep);
// The variant an automatic (-1) launch of this mode and keep takes.
int tc_scan_automatic_variant(int mode, int keep);
const char* tc_scan_variant_name(int variant);
// prep.cu: synthetic rows for the autotuner (mode 0: FP16 values in [-1, 1];
// 1: int8; 2: packed bits, about 1 in 8 set), zero past n rows / `bytes` bytes.
cudaError_t launch_fill_random(int mode, void* rows, int64_t n_rows_mem, int64_t row_bytes, int64_t n,
                               int64_t bytes, uint64_t seed, int sms, cudaStream_t stream);

// rerank.cu
// Certificate of the 16-bit scan's candidate sets (see rerank.cu): per query row the scan's
// keep-th kept raw value (`bound`, indexed like the candidates), the rows' residual and operand
// norms with their maxima, the operand row length; rows whose k nearest cannot be proven to lie
// among the candidates are appended (output row index) to fail_list.
struct CertArgs {
  const float* bound;
  const float* rnorm;
  const float* hnorm;
  const unsigned int* maxes;
  int half_len;      // elements per 16-bit operand row (the contraction length)
  int32_t* fail_list;
  int32_t* fail_count;
  int64_t fail_cap;
};
// rerank.cu.  n_q work items; order (optional): item w reranks output row order[w] (of n_out
// output rows; default n_q); with by_item the candidates (and the certificate's bound) of item w
// are row w of `cand`, else row order[w].
cudaError_t launch_rerank_f32(const float* X, int ld, int d, int64_t n_q, int64_t n_keys, int64_t q_row0,
                              const int32_t* cand, int C, int k, const int32_t* order, int32_t* out_idx, float* out_raw,
                              float* out_dist, int* status, int sms, cudaStream_t stream,
                              const CertArgs* cert = nullptr, bool by_item = false, int64_t n_out = -1);
cudaError_t launch_gather_pivots(const void* src, int64_t row_bytes, int64_t n, int64_t n_piv, void* dst, int sms,
                                 cudaStream_t stream);
// Counting sort of rows by label.  sorted_cells: rows inside each cell ordered
// by index (deterministic; the NN-descent initialisation reads cells by
// position); otherwise rows inside a cell keep the scatter's order, which is
// enough where the order only schedules work (the rerank).
cudaError_t launch_order_by_label(const int32_t* label, int64_t n, int nb, int32_t* hist, int32_t* cursor,
                                  int32_t* order, bool sorted_cells, int sms, cudaStream_t stream);

// prep.cu: rows of `row_bytes` (packed) -> rows of `ld_bytes` (>= row_bytes),
// columns past row_bytes and rows n..rows-1 zero-filled; SM copy, so it does
// not queue behind host<->device traffic on the copy engines.
cudaError_t launch_copy_rows(const void* src, int64_t n, int64_t row_bytes, void* dst, int64_t rows, int64_t ld_bytes,
                             int sms, cudaStream_t stream);

}  // namespace evoc

namespace evoc {
// brute.cu: the reference's brute_force_knn for i8 (dtype 1) / u8 (dtype 2) rows of row_bytes
// (multiple of 16, zero padded), rows q_begin .. q_end-1, each output row in the reference's heap
// order.  The k-slot heap and the query row sit in shared memory (at most 200 KB per row).
size_t brute_force_smem_per_warp(int64_t row_bytes, int k);
cudaError_t launch_brute_force_heap(int dtype, const void* X, int64_t n, int64_t row_bytes, int k, int64_t q_begin,
                                    int64_t q_end, int32_t* out_idx, float* out_raw, float* out_dist, int sms,
                                    cudaStream_t stream);
}  // namespace evoc

namespace evoc {
// jaccard.cu: exact popcount Jaccard over packed bits with fused top-k.
//   X: rows of ldw 32-bit words (ldw a multiple of 16), pc: n int32 row popcounts (written here).
size_t knn_jaccard_smem(int k);
cudaError_t launch_knn_jaccard(const void* X, int64_t n, int ldw, int k, int32_t* pc, int grid, int32_t* out_idx,
                               float* out_raw, float* out_dist, int64_t q_begin, int64_t q_end, int sms,
                               cudaStream_t stream);
}  // namespace evoc

namespace evoc {
// graph.cu: smooth_knn_dist, membership strengths and the fuzzy union on the device.
struct FuzzyWork {
  int* flags;         // [0]: some row has rho == 0 (its sigma floor needs the global mean)
  float* mean;        // mean of all distances, in ndarray's f32 order (only when flags[0])
  int32_t* a_cols;    // n x k: row i's nonzero memberships, sorted by column
  float* a_vals;
  int32_t* a_cnt;     // n
  int32_t* indeg;     // n: entries per column of A
  int64_t* colptr;    // n + 1: CSR pointer of A^T
  int32_t* fill;      // n
  int32_t* at_rows;   // n x k capacity: A^T row indices per column bucket
  float* at_vals;
  int32_t* row_cnt;   // n: entries per row of the result
  int32_t* big;       // n: column buckets too large for a warp's sort
  int32_t* n_big;     // 1: their count
};
cudaError_t launch_smooth_and_membership(const int32_t* idx, const float* dist, int64_t n, int k, float n_neighbors,
                                         const FuzzyWork& w, float* sigma, float* rho, int sms, cudaStream_t stream);
cudaError_t launch_fuzzy_union_count(int64_t n, int k, int symmetrize, const FuzzyWork& w, int64_t* indptr, int sms,
                                     cudaStream_t stream);
cudaError_t launch_fuzzy_union_write(int64_t n, int k, int symmetrize, const FuzzyWork& w, const int64_t* indptr,
                                     int32_t* indices, float* data, int sms, cudaStream_t stream);
}  // namespace evoc

namespace evoc {
// graph.cu: out[0] = 0, out[i+1] = cnt[0] + ... + cnt[i].
cudaError_t launch_scan_counts(const int32_t* cnt, int64_t n, int64_t* out, cudaStream_t stream);
// jaccard.cu: per-row popcounts of rows of ldw 32-bit words.
cudaError_t launch_popcount_rows(const void* X, int64_t n, int ldw, int32_t* pc, int sms, cudaStream_t stream);
// jaccard.cu: packed bit rows (ld_in bytes apart, nbytes used) -> 0/1 int8 rows of ld_out bytes
// (ld_out >= 8 * nbytes, multiple of 16) for `rows` rows; rows past n and columns past 8*nbytes are 0.
cudaError_t launch_expand_bits(const void* X, int64_t n, int64_t ld_in, int64_t nbytes, void* Y, int64_t rows,
                               int64_t ld_out, int sms, cudaStream_t stream);

// nndescent.cu: GPU NN-descent.
struct NndArgs {
  const uint8_t* X;       // rows of row_bytes (FP16 rows of f32 data, int8, or packed bits)
  int64_t row_bytes;      // multiple of 16
  const int32_t* pc;      // row popcounts (binary rows), else null
  int64_t n;
  int k;                  // <= 64
  int mc;                 // max_candidates, <= 64
  int dtype;              // 0 f32 (joined on FP16 rows), 1 i8, 2 u8
  int sms;
  const int32_t* order;   // visit order (rows grouped by pivot cell) or null
  const int32_t* label;   // pivot cell of each row or null
  const int32_t* cell_end;
  const int32_t* cell_cnt;
  uint64_t seed;
  uint64_t* keys[2];      // n x k sorted (raw, index) keys, double buffered
  uint8_t* isnew[2];      // n x k flags
  int32_t* rcnt;          // n
  int64_t* rptr;          // n + 1
  int32_t* rfill;         // n
  int32_t* rrows;         // n x k
  int32_t* cand;          // n x 2 mc: tagged candidate ids (bit 31 = new), -1 past the end
  unsigned long long* changes;
  double* sum;            // [0]: the new graph's sum of finite raw dissimilarities; [1 ..]: kNndSumParts partials
  unsigned long long* evals;  // distances the joins computed (accumulates over iterations)
};
constexpr int kNndSumParts = 1024;
cudaError_t launch_nnd_init(const NndArgs& a, cudaStream_t stream);
cudaError_t launch_nnd_iteration(const NndArgs& a, int cur, int iter, cudaStream_t stream);
cudaError_t launch_nnd_emit(const NndArgs& a, int cur, int32_t* out_idx, float* out_raw, float* out_dist,
                            cudaStream_t stream);
}  // namespace evoc
