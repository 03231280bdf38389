// Batches of small requests in one pass (internal; not part of the C ABI).
//
// A batch lives in device tables: a header with the counts and one status
// word, one BatchRowJob per request for the row kernels (copy and pad,
// prepare_float, 16-bit conversion, FP32 rerank), one ScanJob per request for
// the tensor-core scan (its two tensor maps and scan parameters) and a
// work-list of (request, 128-row query block) items.  Every kernel reads its
// counts and pointers from these tables, so its launch parameters do not
// depend on the batch and the whole sequence can be captured once in a CUDA
// graph and replayed for every batch.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace evoc {

struct BatchHeader {
  int32_t n_jobs;        // requests in the batch
  int32_t n_items;       // scan work items
  int32_t status;        // 0 ok; the scan / rerank status codes of any request
  int32_t fail_count;    // f32 requests: rows that failed the certificate
  int64_t total_rows;    // sum of n over the requests (rerank rows)
  int64_t total_blocks;  // sum of ceil(n / 128) (row-norm blocks)
  int32_t* fail_list;    // (request, row) pairs of those rows
  int64_t fail_cap;      // pairs the list holds
};

struct BatchRowJob {
  int64_t n, dim;          // rows, features (f32) or bytes (i8)
  int64_t rows;            // padded rows (multiple of 256)
  int64_t row_bytes;       // packed input bytes per row
  int64_t ld;              // f32 stride in floats (f32 requests)
  int64_t ldb;             // 16-bit / int8 stride in bytes
  int64_t row_base;        // first global row of this request (prefix of n)
  int64_t blk_base;        // first global 128-row block (prefix of ceil(n/128))
  const uint8_t* src;      // packed input rows on the device
  float* x;                // f32 padded rows (f32 requests)
  uint8_t* xb;             // 16-bit or int8 padded rows
  float* norms;            // f32 row norms (f32 requests)
  int32_t* flag;           // prepare_float: some row's norm is off by > 1e-5
  int32_t* cand;           // n x C scan candidates (f32 requests)
  int32_t C, keff;         // candidates kept per row, neighbours returned
  int32_t* out_idx;
  float* out_dist;
  float* out_raw;          // may be null
  // f32 requests: 16-bit operand type and the certificate (rerank.cu): row
  // residual / operand norms, their maxima, the scan's C-th kept value per row
  int32_t half_type, certify;
  float* rnorm;
  float* hnorm;
  unsigned int* maxes;
  float* bound;
};

struct alignas(64) ScanJob {
  CUtensorMap ma, mb;      // query rows (box 128) and key rows (box 256)
  int64_t n_q, n_k, q_row0;
  int32_t n_kchunks, keep, self_mode, final_mode, dtype, pad_;
  int32_t* out_idx;
  float* out_raw;
  float* out_dist;
  const int32_t* pc;
  float* out_bound;        // optional: raw value of each query's keep-th kept key
};

struct ScanItem {
  int32_t job, qb;
};

// tc_scan.cu.  Encodes a request's tensor maps and parameters (self mode:
// every row is a query and a key).  mode 0: 16-bit float rows (half_type);
// 1: int8 rows.
bool encode_scan_job(ScanJob* sj, int mode, const void* rows, int64_t rows_mem, int64_t n, int64_t row_bytes,
                     int keep, int final_mode, int dtype, int32_t* out_idx, float* out_raw, float* out_dist,
                     float* out_bound, int half_type);
// Sets the kernels' shared-memory limit (call before a stream capture).
cudaError_t prepare_tc_scan_batch(int mode, int max_keep);
cudaError_t launch_tc_scan_batch(int mode, BatchHeader* hdr, const ScanJob* jobs, const ScanItem* items,
                                 int max_keep, int grid, uint64_t timeout_ns, cudaStream_t stream, int half_type);

// prep.cu.  f32 requests: copy + pad into x, prepare_float, 16-bit rows into
// xb (with the certificate's norms).  i8 requests: copy + pad into xb.
// Grids are sized by the caller for the batch (grid-stride loops cover any
// count), so a small batch occupies a few SMs and runs beside other work.
cudaError_t launch_batch_rows(bool f32, const BatchHeader* hdr, const BatchRowJob* jobs, int grid_rows,
                              int grid_norms, cudaStream_t stream);
// rerank.cu.  f32 requests: FP32 rerank of the scan candidates into the
// outputs; rows that fail the certificate go to the header's list.
cudaError_t launch_batch_rerank(BatchHeader* hdr, const BatchRowJob* jobs, int grid, cudaStream_t stream);

}  // namespace evoc
