// Label-propagation initialisation and reproducible node embedding: kernel
// launchers (label_prop.cu) used by the C-ABI orchestration (lp_host.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace evoc {
namespace lp {

constexpr int kVoteSlots = 256;   // ordered-table slots per warp in shared memory
constexpr int kRowWarps = 8;      // warps per CTA in the warp-per-row kernels
constexpr int kMaxComponents = 32;

// A graph as CSR on the device: rows may list their columns in any order.
struct Csr {
  const int64_t* indptr;
  const int32_t* indices;
  const float* data;
  int64_t n;
  int64_t nnz;
};

// *bad = 1 unless indptr[0] == 0, indptr is non-decreasing, indptr[n] == nnz
// and every column is in [0, n).
cudaError_t launch_validate_csr(const Csr& g, int32_t* bad, cudaStream_t s);

// Largest row length -> *out (device int64).
cudaError_t launch_max_degree(const int64_t* indptr, int64_t n, int64_t* out, cudaStream_t s);

// Sets labels[idx[i]] = i for i in order (seeds from host draws): one thread, in order.
cudaError_t launch_seed_labels(int32_t* labels, const int64_t* idx, int64_t count, cudaStream_t s);

// One label_prop_iteration sweep.  Rows whose table outgrows shared memory go
// to overflow[] (count in *n_overflow) and are finished by the second launch
// with tables in `scratch` (warps x max_deg slots).
// dix: key_bound ints per overflow warp (labels -1 .. key_bound - 2), all -1, or null.
cudaError_t launch_lp_iteration(const Csr& g, const int32_t* lab_in, int32_t* lab_out, int32_t* overflow,
                                int32_t* n_overflow, int32_t* scratch_key, double* scratch_sum, int64_t max_deg,
                                int32_t* dix, int64_t key_bound, int sms, cudaStream_t s);

// label_outliers (see label_prop.cu): all unlabelled rows walked at once,
// copied labels resolved by pointer jumping.  Buffers: flag, rows, oidx,
// lab[2], nxt[2], big: n ints each; walk: 2 n ints; stacks:
// outlier_stack_entries(sms) ints; big_stack: 64 * max_deg + 1 ints; count,
// max_label, n_big, pending, status: one int each; tmp: lp_outliers_tmp_bytes(n).
struct OutlierScratch {
  int32_t *flag, *rows, *oidx, *lab[2], *nxt[2], *big, *walk, *stacks, *big_stack;
  int32_t *count, *max_label, *n_big, *pending, *status;
  void* tmp;
  size_t tmp_bytes;
};
cudaError_t run_lp_outliers(const Csr& g, int32_t* labels, const int64_t* rs, const OutlierScratch& w, int64_t max_deg,
                            int sms, cudaStream_t s);
size_t lp_outliers_tmp_bytes(int64_t n);
size_t outlier_stack_entries(int sms);

// remap_labels: dense ranks of the labels present (all labels are >= 0 here).
// flags/map hold `bound` ints; *n_parts receives the number of labels.
cudaError_t launch_lp_remap(int32_t* labels, int64_t n, int32_t bound, int32_t* flags, int32_t* map,
                            int32_t* n_parts, int32_t* status, void* tmp, size_t tmp_bytes, cudaStream_t s);
size_t lp_remap_tmp_bytes(int32_t bound);

// Part sizes, member lists (rows grouped by part, ascending within a part),
// and the normalised reduction values x_p = 1/sqrt(c_p) and data-reducer
// weights w_p = x_p / (x_p summed c_p times).
cudaError_t launch_part_members(const int32_t* part, int64_t n, int32_t n_parts, int32_t* count, int64_t* start,
                                int32_t* members, float* xnorm, float* wred, void* tmp, size_t tmp_bytes,
                                int32_t* keys_tmp, int32_t* vals_tmp, cudaStream_t s);
size_t part_members_tmp_bytes(int64_t n, int32_t n_parts);

// reduced_data[p, :] = sum over members (ascending) of f32(f64(w_p) * f64(x[m, :])).
cudaError_t launch_reduce_data(const float* x, int64_t d, const int32_t* members, const int64_t* start,
                               const int32_t* count, const float* wred, int32_t n_parts, float* out, int sms,
                               cudaStream_t s);

// Sort scratch shared by the SMMP reduction and hadamard_symmetric of a graph
// with at most `cap` entries and `rows` rows (reused level by level).
struct ReduceScratch {
  uint64_t* k0;      // cap
  uint64_t* k1;      // cap
  uint32_t* v0;      // cap each
  uint32_t* v1;
  uint32_t* v2;
  uint32_t* v3;
  int32_t* head;     // cap + 1
  int32_t* pos;      // cap + 1
  int64_t* rcount;   // rows + 2
  void* tmp;         // CUB temporary storage
  size_t tmp_bytes;
  int32_t* counter;  // 4 ints
};
size_t reduce_sort_tmp_bytes(int64_t nnz);

// temp = N^T G and reduced = temp R in SciPy SMMP order (see label_prop.cu).
// Writes the reduced CSR (n_parts rows) into r_indptr / r_indices / r_data
// (capacity g.nnz) and its nnz into *r_nnz (device int64).
cudaError_t launch_reduce_graph(const Csr& g, const int32_t* part, const float* xnorm, int32_t n_parts,
                                const ReduceScratch& w, int64_t* r_indptr, int32_t* r_indices, float* r_data,
                                int64_t* r_nnz, cudaStream_t s);

// G o G^T on G's pattern with rows sorted (hadamard_symmetric), written as CSR
// with the same row pointer layout minus dropped entries: s_indptr (n + 1).
cudaError_t launch_hadamard_sym(const Csr& g, const ReduceScratch& w, int64_t* s_indptr, int32_t* s_indices,
                                float* s_data, int64_t* s_nnz, cudaStream_t s);

// result[r, :] = ((expander row r . layout) + layout[part[r], :]) / 2 in the
// reference's rounding; rows whose part table overflows shared memory are
// finished with `scratch` tables.
// dix: key_bound (= number of parts) ints per overflow warp, all -1, or null.
cudaError_t launch_expand(const Csr& sym, const int32_t* part, const float* xnorm, const float* layout, int ncomp,
                          float* result, int32_t* overflow, int32_t* n_overflow, int32_t* scratch_key,
                          float* scratch_sum, int64_t max_deg, int32_t* dix, int64_t key_bound, int sms,
                          cudaStream_t s);

// out[r, c] = f32(f64(scaling) * (f64(result[r, c]) - mean_c)), mean_c the f64
// mean of column c summed in row order.
cudaError_t launch_center_scale(const float* result, int64_t n, int ncomp, float scaling, float* out,
                                double* mean, cudaStream_t s);

// PCA base init of n < 64 rows (f64 Jacobi on the Gram matrix) followed by the
// small-graph normalisation; out is n x ncomp.
// mean_ws holds d floats and vws d doubles of scratch.
cudaError_t launch_pca_init(const float* x, int64_t n, int64_t d, int ncomp, float* out, float* mean_ws,
                            double* vws, int32_t* status, cudaStream_t s);

// Spectral (mode 0) or MDS (mode 1) base init of n <= 64 rows, then the
// small-graph normalisation; out is n x ncomp.
cudaError_t launch_spectral_mds_init(const float* x, int64_t n, int64_t d, int ncomp, int mode, float* out,
                                     cudaStream_t s);

// Rows of r (n x ncomp) divided by their f32 L2 norm (random_unit_init).
cudaError_t launch_unit_rows(float* r, int64_t n, int ncomp, cudaStream_t s);

// The jitter (jitter = 1) or node-embedding (0) upscaler on result (n x ncomp):
// noise holds the f32 draws, part the row's part, layout the reduced layout.
cudaError_t launch_upscale(float* result, const int32_t* part, const float* layout, const float* noise, int64_t n,
                           int ncomp, int jitter, cudaStream_t s);

// node_embedding: per-edge schedules (neg_scale 1.5 for the reproducible epochs, else 1).
cudaError_t launch_ne_schedule(const float* w, int64_t m, int32_t n_epochs, float negative_sample_rate,
                               float neg_scale, float* eps, float* epns, float* eonn, float* eons, float* max_w,
                               cudaStream_t s);
// Row of every edge (head[e], nnz entries).
cudaError_t launch_edge_head(const int64_t* indptr, int64_t n, uint32_t* head, cudaStream_t s);
// One non-reproducible epoch: every edge at once, updates by atomic adds.
cudaError_t launch_ne_hogwild(const Csr& g, const uint32_t* head, float* emb, const float* eps, const float* epns,
                              float* eonn, float* eons, uint32_t rng_state, int ncomp, float alpha, uint8_t epoch,
                              float noise, int sms, cudaStream_t s);
// One block of one epoch: nodes order[bs, be), rows of more than heavy_deg
// edges by one CTA each (heavy_rows holds be - bs ids); then the apply launch.
cudaError_t launch_ne_block(const Csr& g, float* emb, float* upd, const uint32_t* order, int64_t bs, int64_t be,
                            const float* eps, const float* epns, float* eonn, float* eons, uint32_t rng_state,
                            int ncomp, float alpha, uint8_t epoch, float noise, float gamma, float decay,
                            int apply_decay, int64_t heavy_deg, uint32_t* heavy_rows, int32_t* heavy_count, int sms,
                            cudaStream_t s);
cudaError_t launch_ne_apply(float* emb, const float* upd, const uint32_t* order, int64_t bs, int64_t be, int64_t nv,
                            int ncomp, cudaStream_t s);

}  // namespace lp
}  // namespace evoc
