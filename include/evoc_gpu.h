/*
 * evoc_gpu.h -- C ABI of the B200 kNN-graph engine for evoc.
 *
 * Plain pointers and sizes only.  Every entry point returns an evoc_status;
 * evoc_gpu_last_error() gives the message of the last failure on a context.
 * Entry points are synchronous: they return after the results are written.
 * A context owns one CUDA stream and its scratch memory; calls on one context
 * are serialised by the context, calls on different contexts may overlap.
 *
 * Each declaration cites the evoc-rs interface it replaces (paths relative to
 * the evoc-rs source tree).
 */
#ifndef EVOC_GPU_H
#define EVOC_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  1 and 2 are KnnError::{EmptyData, InvalidNeighbors}
 * (src/knn.rs:32-41); the rest are conditions the CPU path never meets. */
typedef enum {
  EVOC_OK = 0,
  EVOC_ERR_EMPTY = 1,       /* n == 0                                   */
  EVOC_ERR_K = 2,           /* k == 0                                   */
  EVOC_ERR_ARG = 3,         /* null pointer, bad dtype/dim, bad option  */
  EVOC_ERR_OOM = 4,         /* device allocation or admission budget    */
  EVOC_ERR_TIMEOUT = 5,     /* a bounded wait ran out                   */
  EVOC_ERR_CUDA = 6,        /* CUDA runtime error                       */
  EVOC_ERR_UNSUPPORTED = 7, /* form not available for this dtype/shape  */
  EVOC_ERR_CANCELLED = 8,   /* serving: job was cancelled               */
  EVOC_ERR_PENDING = 9      /* serving: job has not finished            */
} evoc_status;

/* EmbeddingData variants (src/knn.rs:16-20).  BINARY is the name the
 * reference's README uses for the UInt8 (packed bits, Jaccard) variant. */
typedef enum {
  EVOC_DTYPE_F32 = 0,
  EVOC_DTYPE_I8 = 1,
  EVOC_DTYPE_U8 = 2,
  EVOC_DTYPE_BINARY = 2
} evoc_dtype;

/* How the neighbours are found. */
typedef enum {
  EVOC_FORM_AUTO = 0,        /* f32 -> BF16_RERANK; i8/u8 -> EXACT_INT            */
  EVOC_FORM_FP32 = 1,        /* f32 exact search, FP32 SIMT dot products          */
  EVOC_FORM_BF16_RERANK = 2, /* f32: tcgen05 16-bit scan (FP16 operands by        */
                             /* default, BF16 with scan_type) keeps oversample*k  */
                             /* candidates per row, reranked in FP32 (FP64 at the */
                             /* k-th boundary); every row certified, rows that    */
                             /* fail rescanned (see `certify`)                    */
  EVOC_FORM_HALF_RERANK = 2, /* the same form under its operand-neutral name      */
  EVOC_FORM_EXACT_INT = 3,   /* i8: tcgen05 int8 dots; u8: tcgen05 int8 on bits  */
                             /* expanded to 0/1 bytes (exact intersection counts) */
  EVOC_FORM_NNDESCENT = 4,   /* GPU NN-descent (approximate, all dtypes)          */
  EVOC_FORM_POPCOUNT = 5     /* u8: SIMT AND + popcount over the packed words     */
} evoc_form;

/* Options.  evoc_gpu_default_opts() fills the defaults; fields that mirror
 * KnnGraphOptions (src/knn.rs:44-76) keep its meaning. */
typedef struct {
  uint32_t struct_size;      /* sizeof(evoc_gpu_opts)                          */
  int32_t form;              /* evoc_form                                      */
  int32_t oversample;        /* 16-bit form: candidates per row =             */
                             /* oversample*k; <= 0 (the default) -> ceil(2.5k) */
                             /* (a wider margin between the k-th and the last  */
                             /* kept candidate: fewer rows fail the           */
                             /* certificate)                                   */
  int32_t buffers_on_device; /* 1: data and outputs are device pointers on the */
                             /* context's device; 0: host pointers             */
  int32_t deterministic;     /* KnnGraphOptions.deterministic                  */
  int32_t n_iters;           /* NN-descent; <= 0 -> max(5, round(log2 n))      */
  int32_t max_candidates;    /* NN-descent; <= 0 -> min(60, floor(1.5 k))      */
  float delta;               /* NN-descent; KnnGraphOptions.delta (0.001)      */
  float delta_improv;        /* NN-descent; KnnGraphOptions.delta_improv       */
  int64_t row_begin;         /* exact forms: compute query rows [row_begin,     */
  int64_t row_end;           /* row_end) against all n rows; 0,0 = all rows.    */
                             /* Outputs then hold (row_end-row_begin) rows.     */
  int32_t strict_precision;  /* RlxBackend::knn_graph's strict_precision        */
                             /* (src/rlx_backend/mod.rs:133-144): 1 = the call  */
                             /* must give the Strict backend's bits or fail.    */
                             /* Only the brute-force branch below can; every    */
                             /* other request returns EVOC_ERR_UNSUPPORTED.     */
  int32_t scan_type;         /* BF16_RERANK operands: 0 FP16 (default), 1 BF16  */
  int64_t brute_force_max_n; /* KnnGraphOptions.brute_force_max_n: i8/u8 data  */
                             /* with n <= it take the reference's brute_force_  */
                             /* knn (src/knn.rs:189-281,418-421): self excluded, */
                             /* each row in the reference's max-heap order      */
  int32_t certify;           /* BF16_RERANK: 1 (default) prove for every row    */
                             /* that the candidates hold its k nearest (within  */
                             /* the 1e-6 tie tolerance) and rescan rows that    */
                             /* cannot be proven -- with 256 candidates, then   */
                             /* exactly in FP32; 0 = skip the certificate       */
  int32_t reserved[3];
} evoc_gpu_opts;

typedef struct evoc_gpu_ctx evoc_gpu_ctx;

/* ABI version: major*10000 + minor*100 + patch. */
int evoc_gpu_version(void);

void evoc_gpu_default_opts(evoc_gpu_opts* opts);

/* Context on one CUDA device (one stream + scratch).  No counterpart in
 * evoc-rs, whose backends are stateless trait objects
 * (src/rlx_backend/mod.rs:204-216); the Rust shim keeps one per backend. */
int evoc_gpu_ctx_create(int device, evoc_gpu_ctx** out);
void evoc_gpu_ctx_destroy(evoc_gpu_ctx* ctx);
const char* evoc_gpu_last_error(const evoc_gpu_ctx* ctx);

/*
 * kNN graph.  Replaces knn_graph / knn_graph_impl (src/knn.rs:345-454) behind
 * RlxBackend::knn_graph (src/rlx_backend/mod.rs:135-144).
 *   data       n x dim row-major: f32, i8, or u8 (dim = bytes per row)
 *   k          n_neighbors; clamped to max(1, min(k, n-1)) as the reference does
 *   rng_state  tau seed from NumpyRandomState::randint3_for_tau
 *              (src/numpy_rng.rs:204-212); read by the NN-descent form only,
 *              may be NULL otherwise
 *   out_idx    n x k_eff int32, row-major, each row sorted ascending
 *   out_dist   n x k_eff f32 transformed distances (src/knn.rs:156-187)
 *   out_k      receives k_eff (may be NULL)
 * f32 rows are renormalised first when any row's norm is off by > 1e-5
 * (prepare_float, src/knn.rs:95-113).
 */
int evoc_gpu_knn_graph(evoc_gpu_ctx* ctx, const evoc_gpu_opts* opts, int32_t dtype, const void* data, int64_t n,
                       int64_t dim, int32_t k, const int64_t* rng_state, int32_t* out_idx, float* out_dist,
                       int32_t* out_k);

/*
 * Many independent kNN graphs in one pass: the BF16+rerank form for f32
 * requests, the exact int8 form for i8.  No counterpart in evoc-rs (each
 * fit_predict builds one graph, src/clustering.rs:650-716); it is the serving
 * loop's path for small requests and open to any caller with many small sets.
 * One persistent tensor-core launch takes the query blocks of every request
 * from a device work-list, so requests too small to fill the GPU share it;
 * the kernels read all per-request data from device tables, and the sequence
 * is captured once per context in a CUDA graph and replayed (EVOC_NO_GRAPHS=1
 * launches it directly).  Results are identical to evoc_gpu_knn_graph's on
 * each request.
 *   opts       buffers_on_device must be 1 (all pointers are device pointers);
 *              form AUTO, BF16_RERANK (f32) or EXACT_INT (i8)
 *   dtype      EVOC_DTYPE_F32 or EVOC_DTYPE_I8, the same for every request
 *   n_jobs     1..4096 requests; request i has n[i] rows of dim[i] at data[i]
 *   k          n_neighbors for every request (k_eff_i = max(1, min(k, n_i - 1)));
 *              the kept candidates (2k for f32, k for i8) must be <= 80
 *   out_idx[i], out_dist[i], out_raw[i]   n_i x k_eff_i each (out_dist and
 *              out_raw arrays, or their entries, may be NULL)
 *   out_k      n_jobs entries receiving k_eff_i (may be NULL)
 * The call returns after every graph is written; one failure fails the batch.
 */
int evoc_gpu_knn_graph_batch(evoc_gpu_ctx* ctx, const evoc_gpu_opts* opts, int32_t dtype, int32_t n_jobs,
                             const void* const* data, const int64_t* n, const int64_t* dim, int32_t k,
                             int32_t* const* out_idx, float* const* out_dist, float* const* out_raw, int32_t* out_k);

/*
 * Autotuner.  Times the tensor-core scan's kernel variants (pipeline depth,
 * epilogue warp groups, heaps in shared or global memory) for requests of
 * this shape on synthetic rows (a sample of up to 65,536 rows), keeps the
 * fastest for this context -- later calls with the same dtype, form, k, dim
 * and floor(log2 n) use it -- and, when cache_path is not NULL, appends it to
 * that file.  A context created while EVOC_TUNE_CACHE names such a file loads
 * it.  Only the tensor-core forms are tuned (f32 BF16_RERANK, i8 and u8
 * EXACT_INT); every variant gives the same results.  report (may be NULL)
 * receives one line per variant and the chosen entry.  No counterpart in
 * evoc-rs (its CPU kernels have no tile parameters).
 */
int evoc_gpu_autotune(evoc_gpu_ctx* ctx, int32_t dtype, int32_t form, int64_t n, int64_t dim, int32_t k,
                      const char* cache_path, char* report, int32_t report_len);
/* Loads a tuning cache file into the context; returns the entries loaded,
 * or -1 when the file cannot be read. */
int evoc_gpu_tune_load(evoc_gpu_ctx* ctx, const char* cache_path);

/* As evoc_gpu_knn_graph, and also writes the raw pre-transform
 * dissimilarities the reference's heaps hold (src/knn.rs:456-520 checks
 * them) into out_raw (n x k_eff, may be NULL). */
int evoc_gpu_knn_graph_raw(evoc_gpu_ctx* ctx, const evoc_gpu_opts* opts, int32_t dtype, const void* data,
                           int64_t n, int64_t dim, int32_t k, const int64_t* rng_state, int32_t* out_idx,
                           float* out_dist, float* out_raw, int32_t* out_k);

/*
 * sigma and rho of every row.  Replaces smooth_knn_dist
 * (src/graph_construction.rs:16-80): rho = first positive distance; sigma by
 * f64 bisection (64 steps, tolerance 1e-5) on log2(n_neighbors), floored at
 * 1e-3 x the row mean (rho > 0) or 1e-3 x the mean of all distances.
 *   dist   n x k transformed distances, rows sorted ascending (any k >= 1)
 */
int evoc_gpu_smooth_knn_dist(evoc_gpu_ctx* ctx, const float* dist, int64_t n, int32_t k, float n_neighbors,
                             int32_t buffers_on_device, float* sigma, float* rho);

/*
 * Fuzzy simplicial set as canonical CSR.  Replaces neighbor_graph_matrix /
 * neighbor_graph_matrix_with_coo (src/graph_construction.rs:176-235) with
 * compute_membership_strengths (82-115) and the SciPy-order union
 * A + A^T - A o A^T (src/csr_matmul.rs:62-150); symmetrize = 0 gives A.
 *   idx, dist   n x k output of evoc_gpu_knn_graph (-1 entries skipped)
 *   sigma, rho  n each (may be NULL)
 *   indptr      n + 1 int64; indices int32 / data f32 with room for `cap`
 *               entries (at most 2 n k).  When cap is too small the call
 *               returns EVOC_ERR_ARG and *nnz holds the size needed.
 */
int evoc_gpu_fuzzy_graph(evoc_gpu_ctx* ctx, const int32_t* idx, const float* dist, int64_t n, int32_t k,
                         float n_neighbors, int32_t symmetrize, int32_t buffers_on_device, float* sigma, float* rho,
                         int64_t* indptr, int32_t* indices, float* data, int64_t cap, int64_t* nnz);

/*
 * NumPy RandomState (MT19937) state, the fields of get_state() and of the
 * reference's NumpyRandomState (src/numpy_rng.rs:11-17, from_numpy_state
 * 154-168).  Calls that draw from the caller's RNG advance it in place with
 * the reference's draws, in the reference's order.
 */
typedef struct {
  uint32_t key[624];
  int32_t pos;
  int32_t has_gauss;
  double gauss;
} evoc_numpy_rng;

/*
 * Partition of a graph by label propagation.  Replaces label_prop_loop
 * (src/label_prop.rs:160-185) called on all -1 labels: 3 tau-seed draws,
 * approx_n_parts seeds labels[randint(0, n)] = i, n_iter sweeps of
 * label_prop_iteration (39-91), label_outliers (94-132), remap_labels
 * (135-157).  Bit-identical to the reference.
 *   indptr (n + 1, int64), indices (int32), data (f32): CSR, any column order
 *   labels   n int64 out: part of each row, 0 .. *n_parts - 1
 */
int evoc_gpu_label_prop_loop(evoc_gpu_ctx* ctx, const int64_t* indptr, const int32_t* indices, const float* data,
                             int64_t n, int32_t n_iter, int64_t approx_n_parts, evoc_numpy_rng* rng,
                             int32_t buffers_on_device, int64_t* labels, int64_t* n_parts);

/*
 * Initial node embedding by label propagation.  Replaces label_propagation_init
 * (src/label_prop.rs:464-494) and RlxBackend::label_propagation_init
 * (src/rlx_backend/mod.rs:146-159): recursive init on the reduced graph, PCA
 * base init below 64 vertices, the partition expander.
 *   x        n x dim f32, the caller's rows (reduced level by level; required
 *            when the recursion reaches a graph of fewer than 64 vertices,
 *            else EVOC_ERR_ARG as LabelPropError::PcaRequiresData)
 *   out      n x n_components f32 (n_components 1..32)
 *   random_scale  unused by the partition expander (used by the other
 *            upscalers of evoc_gpu_label_propagation_init_with_options)
 * Partitions, reduced graphs, node orders and the embedding epochs match the
 * reference bit for bit; the PCA base init is f64 eigen-decomposition (the
 * reference uses an f64 thin SVD), equal within its rounding.
 */
int evoc_gpu_label_propagation_init(evoc_gpu_ctx* ctx, const int64_t* indptr, const int32_t* indices,
                                    const float* data, int64_t n, int32_t n_label_prop_iter,
                                    int32_t n_embedding_epochs, int64_t approx_n_parts, int32_t n_components,
                                    float scaling, float random_scale, float noise_level, evoc_numpy_rng* rng,
                                    const float* x, int64_t dim, int32_t buffers_on_device, float* out);

/* Base initialisation of graphs below base_init_threshold vertices (BaseInit,
 * src/label_prop.rs:20-27) and the upscaling of a partition layout (Upscaling,
 * 29-36). */
typedef enum {
  EVOC_BASE_INIT_PCA = 0,       /* pca_init (265-309): needs x */
  EVOC_BASE_INIT_RANDOM = 1,    /* random_unit_init (311-320): normal draws, rows L2-normalised */
  EVOC_BASE_INIT_SPECTRAL = 2,  /* spectral_init (364-423): needs x */
  EVOC_BASE_INIT_MDS = 3        /* mds_init (339-362): needs x */
} evoc_base_init;

typedef enum {
  EVOC_UPSCALE_PARTITION_EXPANDER = 0,  /* src/label_prop.rs:590-605 */
  EVOC_UPSCALE_JITTER_EXPANDER = 1,     /* 606-642: expander averaged with the jittered part layout */
  EVOC_UPSCALE_NODE_EMBEDDING = 2       /* 643-656: part layout plus normal(random_scale) draws */
} evoc_upscaling;

/* The keyword arguments of label_propagation_init_with_options
 * (src/label_prop.rs:497-512).  evoc_lp_options_default gives the values of
 * label_propagation_init: recursive, PCA, 64, partition expander. */
typedef struct {
  int32_t recursive_init;       /* nonzero: the reduced layout starts from the recursive init */
  int32_t base_init;            /* evoc_base_init */
  int64_t base_init_threshold;  /* graphs of fewer vertices take the base init */
  int32_t upscaling;            /* evoc_upscaling */
  int32_t reserved[3];
} evoc_lp_options;

void evoc_lp_options_default(evoc_lp_options* o);

/*
 * label_propagation_init_with_options (src/label_prop.rs:497-674): as
 * evoc_gpu_label_propagation_init, with the options above (NULL: defaults).
 * The options pass down the recursion as in the reference.  RNG draws, in
 * the reference's order per level: label_prop_loop, the recursion, the
 * reduced layout's node_embedding (normal(0.25) initial draws when
 * recursive_init is 0), then the upscaler's n x n_components normals
 * (jitter: normal(random_scale / 4), node embedding: normal(random_scale)).
 * The random base init draws n x n_components normals.  Spectral and MDS
 * eigen-decompose in f64 on the host (the reference: faer's f32 solver), with
 * eigenvalues ascending and each eigenvector's largest-magnitude entry (the
 * first on ties) made positive -- the reference's signs are faer's.
 * Errors: EVOC_ERR_ARG for an unknown base_init / upscaling, a threshold
 * below 0, or a base init that needs x without it.
 */
int evoc_gpu_label_propagation_init_with_options(evoc_gpu_ctx* ctx, const int64_t* indptr, const int32_t* indices,
                                                 const float* data, int64_t n, int32_t n_label_prop_iter,
                                                 int32_t n_embedding_epochs, int64_t approx_n_parts,
                                                 int32_t n_components, float scaling, float random_scale,
                                                 float noise_level, evoc_numpy_rng* rng, const float* x, int64_t dim,
                                                 int32_t buffers_on_device, const evoc_lp_options* options,
                                                 float* out);

/*
 * UMAP-like node embedding.  Replaces node_embedding (src/embed.rs:251-369)
 * and RlxBackend::node_embedding (src/rlx_backend/mod.rs:161-173).
 *   reproducible = 1: block-synchronous epochs (node_embedding_epoch_repr,
 *                  138-248), bit-identical to the reference
 *   reproducible = 0: the non-reproducible epoch (node_embedding_epoch,
 *                  57-135) with every edge of an epoch updating the rows at
 *                  once (lock-free atomic adds, as Python's parallel version);
 *                  same schedules and RNG draws as the reference, embedding
 *                  equal in distribution, not bit for bit
 *   initial_embedding  n x n_components, or NULL for normal(0.25) draws
 */
int evoc_gpu_node_embedding(evoc_gpu_ctx* ctx, const int64_t* indptr, const int32_t* indices, const float* data,
                            int64_t n, int32_t n_components, int32_t n_epochs, const float* initial_embedding,
                            float initial_alpha, float negative_sample_rate, float noise_level, evoc_numpy_rng* rng,
                            int32_t reproducible, int32_t buffers_on_device, float* out);

/*
 * .npy / .npz ingestion.  The reference reads its data sets, graphs and RNG
 * states with ndarray_npy (src/graph_construction.rs:117-154,
 * src/clustering.rs:350-356, src/numpy_rng.rs:170-193).  Here an array is
 * read in place from a read-only mapping of the file: `data` points into the
 * mapping (stored .npz members too), so rows can go straight to
 * evoc_gpu_knn_graph or a server submit (EVOC_SUBMIT_BORROW) without a
 * host-side copy; a deflated .npz member is inflated into a buffer the handle
 * owns.  Little-endian f4/f8/i1/u1/i4/i8/u4/b1 arrays, .npy versions 1-3, ZIP
 * and ZIP64 archives.  Release with evoc_npy_close.
 */
typedef enum {
  EVOC_NPY_F32 = 0,
  EVOC_NPY_F64 = 1,
  EVOC_NPY_I8 = 2,
  EVOC_NPY_U8 = 3,
  EVOC_NPY_I32 = 4,
  EVOC_NPY_I64 = 5,
  EVOC_NPY_U32 = 6,
  EVOC_NPY_BOOL = 7
} evoc_npy_dtype;

typedef struct {
  const void* data;      /* first element                                  */
  int64_t nbytes;        /* bytes of array data                            */
  int64_t shape[8];
  int32_t ndim;
  int32_t dtype;         /* evoc_npy_dtype                                 */
  int32_t fortran_order; /* 1: column-major                                */
  int32_t reserved;
  void* handle;          /* the mapping / buffer; owned by the library     */
} evoc_npy_array;

/* EVOC_ERR_ARG: unreadable file, bad header, missing member;
 * EVOC_ERR_UNSUPPORTED: dtype or format version not listed above. */
int evoc_npy_open(const char* path, evoc_npy_array* out);
int evoc_npz_open(const char* path, const char* name, evoc_npy_array* out); /* name with or without ".npy" */
void evoc_npy_close(evoc_npy_array* a);

/*
 * A graph .npz in the reference's layouts: CSR (indptr, indices, data, shape;
 * load_graph_csr_npz, src/graph_construction.rs:133-154) or COO (rows, cols,
 * data, shape; load_graph_coo_npz, 117-131), returned as CSR.  COO entries
 * are sorted by (row, column) and entries with the same position summed in
 * file order (TriMat::to_csr); CSR is copied as stored.  With indptr == NULL
 * only *n and *nnz are set (a size query); otherwise indptr holds n + 1,
 * indices / data `cap` entries (EVOC_ERR_ARG when cap < *nnz).
 */
int evoc_graph_npz_read(const char* path, int64_t* n, int64_t* nnz, int64_t* indptr, int32_t* indices, float* data,
                        int64_t cap);

/*
 * Minimum spanning tree under mutual-reachability distance, with the core
 * distances.  Replaces build_kdtree (src/kdtree.rs:367-413) and
 * parallel_boruvka with reproducible = false (src/boruvka.rs:437-593), which
 * build_cluster_layers runs on the node embedding (src/clustering.rs:50-80).
 *   data         n x dim f32 points, row-major (dim 1..32)
 *   min_samples  core distance = squared distance to the (min_samples + 1)-th
 *                nearest point, the point itself included; <= 1: zero core
 *                distances (as the reference); at most 31; n must exceed it
 *   out_edges    (n - 1) x 3 f32 rows (from, to, distance), distance the
 *                square root of max(squared distance, core[from], core[to])
 *   out_core     n f32 squared core distances (may be NULL)
 *   n_edges      receives n - 1
 * The total weight and the sorted edge weights equal the reference's; edges
 * (and their order) can differ where several have equal weight, as they do
 * between the reference's non-reproducible runs.
 */
int evoc_gpu_boruvka_mst(evoc_gpu_ctx* ctx, const float* data, int64_t n, int32_t dim, int32_t min_samples,
                         int32_t buffers_on_device, float* out_edges, float* out_core, int64_t* n_edges);

/* FP32 FMA throughput of the context's device (TFLOP/s, 2 FLOPs per FMA),
 * measured with a hand-written kernel over every SM; *ms its duration.  The
 * plain FP32 form's roofline denominator.  No counterpart in evoc-rs. */
int evoc_gpu_peak_ffma(evoc_gpu_ctx* ctx, double* tflops, double* ms);

/* The context's CUDA stream (a cudaStream_t), for callers that record their
 * own CUDA events around calls.  No counterpart in evoc-rs. */
void* evoc_gpu_ctx_stream(const evoc_gpu_ctx* ctx);

/* Device timing of the stages of the last call.  When enabled, every call
 * records CUDA events on the context's stream around each kernel stage.
 * No counterpart in evoc-rs (its bins time stages with Instant,
 * src/bin/bench_huge.rs:71-82). */
int evoc_gpu_profile_enable(evoc_gpu_ctx* ctx, int enable);
int evoc_gpu_profile_count(const evoc_gpu_ctx* ctx);
int evoc_gpu_profile_stage(const evoc_gpu_ctx* ctx, int i, char* name, int name_len, float* ms);

/* Number of kernels the last call launched. */
int evoc_gpu_last_launch_count(const evoc_gpu_ctx* ctx);

/* Limit, in ns, of each wait inside the tensor-core scan's pipeline on this
 * context (its producer, MMA and epilogue roles wait on one another); 0
 * restores the default of 4 s.  A wait that runs out ends the call with
 * EVOC_ERR_TIMEOUT and leaves the context usable: the roles stop together,
 * loads and MMAs already issued are waited for (always with the full 4 s
 * limit) and the tensor memory is freed.  producer_delay_ns (at most 100 ms,
 * normally 0) makes the main scan's producer start that late, so a limit
 * below it is sure to run out: the timeout path's test.  No counterpart in
 * evoc-rs. */
int evoc_gpu_set_wait_limit(evoc_gpu_ctx* ctx, uint64_t ns, uint64_t producer_delay_ns);

/* Symmetric scan of the 16-bit form (opt-in; off by default).  A self-join
 * (all rows as queries, the certificate on) of at least min_rows rows
 * multiplies each pair of rows once: a query block takes only the key tiles
 * from its own rows on, and the scores for later rows reach them through
 * per-row mailboxes, filtered by thresholds from a pre-scan against a strided
 * 1/16 sample of the rows.  Half the tensor-core work of the plain scan and
 * the same candidates, but on B200 at 1M x 768 it measured slower end to end
 * than the plain scan, hence off.  0 or a negative value turns it off.  The
 * environment variable EVOC_SYM_MIN_ROWS sets it when a context is created.
 * No counterpart in evoc-rs (its NN-descent evaluates each pair once per join
 * by its own bookkeeping, src/nndescent/float.rs:552-660). */
int evoc_gpu_set_symmetric_scan(evoc_gpu_ctx* ctx, int64_t min_rows);

/* The last call's symmetric scan: rows of its sample pre-scan (0 when the
 * call did not take it), mailbox capacity per row, the most mailbox keys any
 * row was offered, and rows whose mailbox overflowed (the certificate rescans
 * those).  Any pointer may be NULL. */
int evoc_gpu_last_symmetric(const evoc_gpu_ctx* ctx, int64_t* sample_rows, int64_t* mailbox_cap,
                            int64_t* max_offers, int64_t* overflowed);

/* The last NN-descent call on this context: iterations run, distances its
 * joins computed, and the bytes of each row those distances gathered (the
 * join's algorithmic traffic is distance_evals x row_bytes).  No counterpart
 * in evoc-rs. */
int evoc_gpu_last_nndescent(const evoc_gpu_ctx* ctx, int32_t* iterations, int64_t* distance_evals,
                            int64_t* row_bytes);

/* Certificate counts of the last BF16_RERANK call on this context: query
 * rows checked, rows that failed the first certificate (rescanned with 256
 * candidates), and rows rescanned exactly in FP32 after failing the second.
 * No counterpart in evoc-rs. */
int evoc_gpu_last_certify(const evoc_gpu_ctx* ctx, int64_t* checked, int64_t* second_pass, int64_t* exact_rescan);

/*
 * Exact FP32 kNN that allocates no device memory.  It has no counterpart in
 * evoc-rs.  It is for callers that may not let a library call cudaMalloc:
 * processes that reserve the GPU's memory for their own pool up front, or
 * latency-critical loops that cannot take cudaMalloc's implicit device-wide
 * synchronisation.  All pointers are device pointers; the work is enqueued on
 * `stream` (a cudaStream_t, 0 for the default stream) and the call returns
 * without waiting for it.
 *   rows       n rows of `ld` floats, 16-byte aligned, ld a multiple of 16
 *              (at most INT32_MAX), columns past the data zero, each row
 *              already L2-normalised (this entry point has no working copy
 *              to renormalise into); rows holding NaN or infinities give
 *              undefined neighbours (the call does not scan for them)
 *   k          clamped to max(1, min(k, n-1)); at most 64 after the clamp,
 *              larger values return EVOC_ERR_UNSUPPORTED
 *   out_idx / out_dist   n x k_eff, as evoc_gpu_knn_graph with EVOC_FORM_FP32
 *   errbuf     receives a message on failure (may be NULL)
 * The search's scratch is one fixed 16 MiB array per GPU, held from the
 * library's load until the process exits.  The first call on a device looks
 * up that array's device address (cudaGetSymbolAddress), so make that first
 * call before any stream capture.  All calls on a device share the array:
 * calls whose kernels overlap on the GPU (different streams with no ordering)
 * race and corrupt each other's results.
 */
int evoc_gpu_knn_f32_noalloc(const float* rows, int64_t n, int64_t ld, int32_t k, int32_t* out_idx, float* out_dist,
                             void* stream, int32_t* out_k, char* errbuf, int32_t errlen);

/*
 * Serving: a kNN-graph server with continuous batching.  No counterpart in
 * evoc-rs, whose Evoc::fit_predict builds one data set's graph at a time
 * (src/clustering.rs:650-716); the Rust request loop calls these.
 *
 * Requests of any n, dim and dtype are queued by evoc_gpu_server_submit and
 * run by `max_inflight` lanes, each with its own context (stream and
 * scratch), so several requests are on the device at once.  A lane admits the
 * oldest pending request that fits the budget: n*dim*size(dtype) for the rows
 * + n*k_eff*8 for the graph + what the lane's buffers must grow by for that
 * shape (lane buffers are kept between requests and counted once; an idle lane
 * frees them when they alone keep the oldest request out).  A request passed
 * over 16 times by later ones is admitted next.  Under backlog -- at least 4
 * compatible small requests pending (f32 with the BF16+rerank form or i8 with
 * the exact form, at most 16,384 rows; same dtype, k and form) -- they are
 * admitted together (up to batch_max requests and 4e12 scan operations) and
 * built by one evoc_gpu_knn_graph_batch call; otherwise each runs alone.  The rows go back to the
 * budget once the graph is built; the graph stays resident in HBM until it is
 * fetched without keep_resident or released.  Every job id must end in
 * evoc_gpu_server_result (without keep_resident) or evoc_gpu_server_release.
 */
typedef struct evoc_gpu_server evoc_gpu_server;

typedef struct {
  uint32_t struct_size;  /* sizeof(evoc_gpu_server_opts)                    */
  int32_t device;        /* CUDA device                                     */
  int64_t budget_bytes;  /* HBM admission budget; default 150e9             */
  int32_t max_inflight;  /* lanes (requests on the device at once), 1..64;  */
                         /* default 4                                       */
  int32_t profile;       /* 1: time every request's stages with CUDA events */
                         /* and keep per-stage totals (server_stage)        */
  int32_t batch_max;     /* most small requests in one batch; 0 or 1: no    */
                         /* batching; default 64                            */
  int32_t small_lanes;   /* lanes that admit only requests under 65,536     */
                         /* rows (of max_inflight); default 0              */
  int32_t admission;     /* 0: oldest request first (first fit);           */
                         /* 1: smallest scan (n^2 d) first; both let a     */
                         /* request passed over 16 times go next           */
  int32_t reserved[1];
} evoc_gpu_server_opts;

typedef struct {
  int64_t submitted, completed, failed, cancelled, rejected;
  int64_t pending, running;
  int64_t bytes_in_use;    /* counted against the budget now               */
  int64_t peak_bytes;      /* high-water mark of bytes_in_use              */
  int64_t budget_bytes;
  int64_t workspace_bytes; /* lane contexts' buffers, counted in bytes_in_use */
  int64_t workspace_misses;/* requests whose buffers outgrew the plan       */
  int64_t lanes;
  int64_t batches;         /* multi-request calls (small requests together)  */
  int64_t batched;         /* requests those calls carried                   */
} evoc_gpu_server_counters;

typedef struct {
  int64_t submit_ns, admit_ns, done_ns; /* evoc_gpu_server_now_ns clock; 0 = not yet */
  int64_t n, dim;
  int32_t dtype, k_eff, lane, status;   /* status as evoc_gpu_server_poll returns */
  char error[160];
} evoc_gpu_job_info;

/* submit flag: the server reads the caller's host rows in place instead of
 * copying them at submit; the buffer must stay valid and unchanged until the
 * job has finished. */
#define EVOC_SUBMIT_BORROW 1

void evoc_gpu_server_default_opts(evoc_gpu_server_opts* opts);
int evoc_gpu_server_create(const evoc_gpu_server_opts* opts, evoc_gpu_server** out);
/* Cancels pending jobs, waits for running ones and frees everything. */
void evoc_gpu_server_destroy(evoc_gpu_server* server);
/* Monotonic clock of the job times (CLOCK_MONOTONIC on Linux), in ns. */
int64_t evoc_gpu_server_now_ns(void);

/* Queues one request; arguments as evoc_gpu_knn_graph.  opts may be NULL
 * (defaults); opts->buffers_on_device = 1 means `data` is a device pointer
 * that stays valid until the job has finished (outputs always stay on the
 * device until fetched); row_begin/row_end must be 0.  EVOC_ERR_OOM when the
 * request cannot fit the budget even alone.  *job_id > 0 on success. */
int evoc_gpu_server_submit(evoc_gpu_server* server, const evoc_gpu_opts* opts, int32_t dtype, const void* data,
                           int64_t n, int64_t dim, int32_t k, const int64_t* rng_state, int32_t flags,
                           int64_t* job_id);
/* Bytes a request is admitted against: *resident = rows (unless on the
 * device) + graph; *workspace = lane buffers it needs on a lane that holds
 * none.  A request fits an otherwise empty server when their sum is at most
 * the budget. */
int evoc_gpu_server_request_bytes(evoc_gpu_server* server, const evoc_gpu_opts* opts, int32_t dtype, int64_t n,
                                  int64_t dim, int32_t k, int64_t* resident, int64_t* workspace);
/* EVOC_ERR_PENDING while queued or running, else the job's final status. */
int evoc_gpu_server_poll(evoc_gpu_server* server, int64_t job_id);
/* Waits until the job has finished (timeout_ms < 0: no limit); returns its
 * status or EVOC_ERR_TIMEOUT. */
int evoc_gpu_server_wait(evoc_gpu_server* server, int64_t job_id, int64_t timeout_ms);
/* Waits for the next job to finish that no wait_any or result call has
 * reported yet, in completion order; returns its status, *job_id its id. */
int evoc_gpu_server_wait_any(evoc_gpu_server* server, int64_t timeout_ms, int64_t* job_id);
/* Waits for the job and copies its graph (n x k_eff, as evoc_gpu_knn_graph)
 * into host buffers (either may be NULL).  Unless keep_resident, the job is
 * then released (also when it failed or was cancelled). */
int evoc_gpu_server_result(evoc_gpu_server* server, int64_t job_id, int32_t* out_idx, float* out_dist,
                           int32_t* out_k, int32_t keep_resident);
/* Device pointers of a finished job's graph, valid until it is released. */
int evoc_gpu_server_result_device(evoc_gpu_server* server, int64_t job_id, const int32_t** d_idx,
                                  const float** d_dist, int32_t* out_k);
/* Frees the job (cancelling it first if it has not finished). */
int evoc_gpu_server_release(evoc_gpu_server* server, int64_t job_id);
/* A pending job is dropped; a running job's graph is discarded when its lane
 * finishes.  Its status becomes EVOC_ERR_CANCELLED. */
int evoc_gpu_server_cancel(evoc_gpu_server* server, int64_t job_id);
int evoc_gpu_server_job_info(evoc_gpu_server* server, int64_t job_id, evoc_gpu_job_info* info);
int evoc_gpu_server_stats(evoc_gpu_server* server, evoc_gpu_server_counters* stats);
/* With opts.profile: the number of distinct stages seen, and stage i's name,
 * summed device time (CUDA events on the lanes' streams) and request count.
 * lane_busy_ms sums, over lanes, the host time a lane spent on requests. */
int evoc_gpu_server_stage_count(evoc_gpu_server* server);
int evoc_gpu_server_stage(evoc_gpu_server* server, int i, char* name, int32_t name_len, double* total_ms,
                          int64_t* count);
double evoc_gpu_server_lane_busy_ms(evoc_gpu_server* server);

#ifdef __cplusplus
}
#endif

#endif /* EVOC_GPU_H */
