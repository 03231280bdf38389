// Device-memory plan of a context (internal; used by the serving loop's
// admission control).  Not part of the C ABI.
#pragma once
#include <cstddef>
#include <cstdint>

#include "../../include/evoc_gpu.h"

namespace evoc {

// The context buffers a kNN request with device-resident outputs may grow.
enum CtxBuf {
  kBufX,
  kBufScratch,
  kBufNorms,
  kBufFlag,
  kBufXb,
  kBufCand,
  kBufLabels,
  kBufOrder,
  kBufHist,
  kBufCursor,
  kBufPivots,
  kBufPopc,
  kBufNnd,
  kBufBatchWs,   // batches: per-request work arena
  kBufBatchTab,  // batches: device tables
  kBufCert,      // 16-bit form: certificate norms, bounds, failed-row lists
  kBufRepair,    // 16-bit form: rescan arena for rows that failed the certificate
  kBufSym,       // 16-bit form: symmetric scan arena (mailboxes, thresholds, sample rows)
  kBufCount
};

struct CtxSizes {
  size_t b[kBufCount] = {};
  size_t total() const {
    size_t t = 0;
    for (size_t v : b) t += v;
    return t;
  }
};

// Bytes each buffer must hold for evoc_gpu_knn_graph(ctx, opts, dtype, ., n,
// dim, k, ...) with buffers_on_device = 1 and all rows as queries: the sizes
// the form runners pass to DevBuf::ensure.
void knn_buffer_needs(const evoc_gpu_ctx* ctx, const evoc_gpu_opts& opts, int32_t dtype, int64_t n, int64_t dim,
                      int32_t k, CtxSizes* need);

// The buffers evoc_gpu_knn_graph_batch needs for these requests (all other
// entries zero).  Returns false when the batch path does not take them
// (dtype/form, k too large).
bool batch_buffer_needs(const evoc_gpu_opts& opts, int32_t dtype, int32_t n_jobs, const int64_t* n,
                        const int64_t* dim, int32_t k, CtxSizes* need);

// Allocated size of each of the context's buffers.  Call only from the thread
// that makes the context's calls.
void ctx_buffer_sizes(const evoc_gpu_ctx* ctx, CtxSizes* cur);

// The sizes after DevBuf::ensure grows `cur` to cover `need` (a buffer that
// grows is reallocated at need + need/8).
CtxSizes grown_sizes(const CtxSizes& cur, const CtxSizes& need);

// Frees every buffer of the context (they regrow on the next call).
void ctx_release_buffers(evoc_gpu_ctx* ctx);

}  // namespace evoc
