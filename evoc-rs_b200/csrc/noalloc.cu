// Exact FP32 kNN entry point that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc: a serving process that
// reserves all of the GPU's memory for its own pool up front and hands
// libraries only the buffers it owns, or a latency-critical loop that cannot
// take the implicit device-wide synchronisation cudaMalloc/cudaFree may
// cause.  evoc_gpu_knn_f32_noalloc serves them: the caller passes the input
// rows and the output buffers (all on the device), and the only scratch the
// search needs -- the per-row candidate buffers of the fused top-k -- lives
// in a fixed array compiled into this library (kScratchWords below).
//
// That array exists once per GPU that loads the library and stays allocated
// until the process exits.  Every call on a GPU uses the same array, so two
// calls whose kernels overlap on the GPU (different streams, no ordering
// between them) corrupt each other's results; calls on one stream are
// ordered and safe.  No part of the array needs to start at zero: each
// launch writes every candidate slot before it reads it.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/evoc_gpu.h"
#include "common.cuh"
#include "kernels.h"

namespace {

// 16 MiB of candidate keys: 2^21 64-bit words.
constexpr int64_t kScratchWords = int64_t(1) << 21;
constexpr int kMaxK = 64;  // topk_capacity(64) = 128 words per row
constexpr int kMaxDevices = 64;

static __device__ __align__(256) uint64_t g_noalloc_scratch[kScratchWords];

std::mutex g_setup_mu;
uint64_t* g_scratch_ptr[kMaxDevices] = {};  // device address of g_noalloc_scratch, per device
int g_sms[kMaxDevices] = {};

void set_err(char* buf, int32_t len, const char* msg) {
  if (buf && len > 0) {
    std::strncpy(buf, msg, size_t(len) - 1);
    buf[len - 1] = '\0';
  }
}

}  // namespace

extern "C" int evoc_gpu_knn_f32_noalloc(const float* rows, int64_t n, int64_t ld, int32_t k, int32_t* out_idx,
                                        float* out_dist, void* stream, int32_t* out_k, char* errbuf, int32_t errlen) {
  if (k <= 0) {
    set_err(errbuf, errlen, "n_neighbors must be positive");
    return EVOC_ERR_K;
  }
  if (n <= 0) {
    set_err(errbuf, errlen, "empty embedding matrix");
    return EVOC_ERR_EMPTY;
  }
  if (!rows || !out_idx) {
    set_err(errbuf, errlen, "null rows or out_idx");
    return EVOC_ERR_ARG;
  }
  if (ld <= 0 || ld % 16 != 0 || (reinterpret_cast<uintptr_t>(rows) & 15) != 0) {
    set_err(errbuf, errlen, "rows must be 16-byte aligned with a row stride (ld) that is a positive multiple of 16");
    return EVOC_ERR_ARG;
  }
  if (n >= (int64_t(1) << 31) - 1) {
    set_err(errbuf, errlen, "n exceeds the int32 index range");
    return EVOC_ERR_ARG;
  }
  // The kernel takes the stride as an int and indexes rows as int64 row * ld.
  if (ld > INT32_MAX || n > INT64_MAX / ld) {
    set_err(errbuf, errlen, "row stride (ld) exceeds the int32 range, or n * ld exceeds the int64 range");
    return EVOC_ERR_ARG;
  }
  int64_t kk = k < n - 1 ? k : n - 1;
  if (kk < 1) kk = 1;
  if (kk > kMaxK) {
    char msg[160];
    std::snprintf(msg, sizeof msg, "k = %lld exceeds the fixed scratch of this entry point (at most %d neighbours)",
                  static_cast<long long>(kk), kMaxK);
    set_err(errbuf, errlen, msg);
    return EVOC_ERR_UNSUPPORTED;
  }
  const int keff = int(kk);
  if (out_k) *out_k = keff;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_err(errbuf, errlen, "no usable current CUDA device");
    return EVOC_ERR_CUDA;
  }
  uint64_t* scratch = nullptr;
  int sms = 0;
  {
    // First call on a device: look up the device address of the fixed array
    // (the array's name is only a host-side stand-in) with that device current.
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        set_err(errbuf, errlen, cudaGetErrorString(e));
        return EVOC_ERR_CUDA;
      }
      int count = 0;
      cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
      g_scratch_ptr[dev] = static_cast<uint64_t*>(p);
      g_sms[dev] = count > 0 ? count : 1;
    }
    scratch = g_scratch_ptr[dev];
    sms = g_sms[dev];
  }

  // Persistent grid sized so every CTA's 128 row buffers fit in the fixed array.
  const int cap = evoc::topk_capacity(keff);
  const int64_t fit = kScratchWords / (int64_t(128) * cap);
  const int64_t qblocks = (n + 127) / 128;
  int64_t grid = qblocks < int64_t(sms) * 2 ? qblocks : int64_t(sms) * 2;
  if (grid > fit) grid = fit;
  cudaError_t e = evoc::launch_knn_f32_simt(rows, n, int(ld), keff, cap, scratch, int(grid), out_idx, nullptr,
                                            out_dist, 0, n, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    set_err(errbuf, errlen, cudaGetErrorString(e));
    return EVOC_ERR_CUDA;
  }
  return EVOC_OK;
}
