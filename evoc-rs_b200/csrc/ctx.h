// Private to the library: the context every C-ABI translation unit shares
// (device, stream, reusable device buffers, stage timers, last error).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/evoc_gpu.h"

namespace evoc {

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t want) {
    if (want <= bytes) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t grow = want + want / 8;
    cudaError_t e = cudaMalloc(&p, grow);
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    bytes = grow;
    return cudaSuccess;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

struct StageRec {
  std::string name;
  cudaEvent_t a = nullptr, b = nullptr;
};

}  // namespace evoc

struct evoc_gpu_ctx {
  int device = 0;
  int sms = 148;
  cudaStream_t stream = nullptr;       // the stream calls run on (a serving lane may swap in another)
  cudaStream_t base_stream = nullptr;  // the context's own stream (destroyed with it)
  bool scan_per_block = false;         // main scans launch one CTA per query block (serving, big requests)
  std::mutex mu;
  std::string err;
  evoc::DevBuf x, scratch, norms, flag, out_idx, out_raw, out_dist;
  evoc::DevBuf xb, cand, labels, order, hist, cursor, pivots, popc;
  evoc::DevBuf g_idx, g_dist, g_sigma, g_rho, g_indptr, g_indices, g_data, g_work;
  evoc::DevBuf nnd_work;
  // 16-bit form certificate: per-row residual / operand norms, their maxima,
  // the scan's C-th kept value per query row, the lists of rows that failed;
  // and the rescan arena for those rows (bounded chunks).
  evoc::DevBuf cert, repair;
  int64_t cert_checked = 0, cert_second = 0, cert_exact = 0;  // last call's counts
  // Symmetric 16-bit scan (sym.cu, opt-in): self-joins of at least
  // sym_min_rows rows (0: never, the default); the arena; the last call's
  // sample rows (0: not taken), mailbox capacity, most mirror keys a row was
  // offered, overflowed rows.
  evoc::DevBuf sym;
  int64_t sym_min_rows = 0;
  int64_t sym_sample = 0, sym_cap = 0, sym_max_offers = 0, sym_overflow = 0;
  evoc::DevBuf batch_ws, batch_tab;  // batches: per-request work arena, device tables
  void* batch_host = nullptr;  // pinned staging of the tables
  size_t batch_host_bytes = 0;
  struct BatchGraph {
    bool f32;
    int keep_odd;
    int key;  // certificate on/off and the 16-bit operand type
    void* tab;
    int grids[4];  // rows, norms, scan, rerank
    cudaGraphExec_t exec;
  };
  std::vector<BatchGraph> batch_graphs;  // captured batch pipelines, replayed per batch
  bool use_graphs = true;                // EVOC_NO_GRAPHS=1 launches the kernels directly
  // Autotuned scan variants: (scan mode, keep, row bytes, floor(log2 n)) -> variant.
  std::map<std::tuple<int, int, int64_t, int>, int> tune;
  uint64_t timeout_ns = 4000000000ull;  // longest a pipeline wait inside a kernel may take
  uint64_t delay_ns = 0;  // tests of the timeout path: the scan's producer starts this late
  bool sync_check = false;  // EVOC_SYNC_CHECK=1: wait for and check every kernel stage (fault diagnosis)
  bool profiling = false;
  std::vector<evoc::StageRec> stages;  // event pool; the first n_stages belong to the last call
  int n_stages = 0;
  int launches = 0;
  int nnd_iterations = 0;
  unsigned long long nnd_evals = 0;  // distances the last NN-descent call's joins computed
  int64_t nnd_row_bytes = 0;         // bytes of each row those distances gathered
  // Stream-ordered pool of the label-propagation / embedding calls; it keeps
  // freed blocks (release threshold = max) so repeated calls do not remap.
  cudaMemPool_t lp_pool = nullptr;
};

namespace evoc {

inline int fail(evoc_gpu_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

inline int cuda_fail(evoc_gpu_ctx* ctx, cudaError_t e, const char* where) {
  std::string m = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return fail(ctx, e == cudaErrorMemoryAllocation ? EVOC_ERR_OOM : EVOC_ERR_CUDA, m);
}

#define EVOC_TRY(expr, where)                                \
  do {                                                       \
    cudaError_t _e = (expr);                                 \
    if (_e != cudaSuccess) return cuda_fail(ctx, _e, where); \
    if (ctx->sync_check) {                                   \
      _e = cudaStreamSynchronize(ctx->stream);               \
      if (_e != cudaSuccess) return cuda_fail(ctx, _e, where); \
    }                                                        \
  } while (0)

// Records CUDA events around one stage on the context's stream when profiling.
struct Stage {
  evoc_gpu_ctx* ctx;
  int idx = -1;
  Stage(evoc_gpu_ctx* c, const char* name) : ctx(c) {
    if (!ctx->profiling) return;
    if (ctx->n_stages == int(ctx->stages.size())) {
      StageRec r;
      if (cudaEventCreate(&r.a) != cudaSuccess || cudaEventCreate(&r.b) != cudaSuccess) return;
      ctx->stages.push_back(r);
    }
    idx = ctx->n_stages++;
    ctx->stages[size_t(idx)].name = name;
    cudaEventRecord(ctx->stages[size_t(idx)].a, ctx->stream);
  }
  void end() {
    if (idx >= 0) cudaEventRecord(ctx->stages[size_t(idx)].b, ctx->stream);
    idx = -1;
  }
  ~Stage() { end(); }
};


}  // namespace evoc
