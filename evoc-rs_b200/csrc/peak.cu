// FP32 FMA throughput of the device, measured with a hand-written kernel.
//
// The plain FP32 form (exact_f32.cu) is bound by FFMA issue; its roofline
// needs the FFMA rate of this part at the clocks it runs at, which no
// library reports.  Each thread runs 8 independent FMA chains (enough
// independent work per warp to cover the FMA latency at 8 warps per
// scheduler); the grid fills every SM.  FLOPs = 2 per FMA.
#include <cstdint>

#include "../../include/evoc_gpu.h"
#include "ctx.h"

namespace evoc {

namespace {
constexpr int kChains = 8;
constexpr int kUnroll = 16;

__global__ void __launch_bounds__(256) ffma_kernel(float* __restrict__ out, int iters, float b, float c) {
  float a[kChains];
#pragma unroll
  for (int j = 0; j < kChains; j++) a[j] = float(threadIdx.x + j) * 1e-3f;
#pragma unroll 1
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < kUnroll; u++)
#pragma unroll
      for (int j = 0; j < kChains; j++) a[j] = fmaf(a[j], b, c);
  }
  float s = 0.0f;
#pragma unroll
  for (int j = 0; j < kChains; j++) s += a[j];
  out[int64_t(blockIdx.x) * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}
}  // namespace

}  // namespace evoc

extern "C" int evoc_gpu_peak_ffma(evoc_gpu_ctx* ctx, double* tflops, double* ms) {
  using evoc::cuda_fail;
  using evoc::fail;
  if (!ctx || !tflops) return EVOC_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->mu);
  ctx->err.clear();
  EVOC_TRY(cudaSetDevice(ctx->device), "cudaSetDevice");
  const int blocks = ctx->sms * 8, threads = 256, iters = 4096;
  float* out = nullptr;
  EVOC_TRY(cudaMallocAsync(reinterpret_cast<void**>(&out), size_t(blocks) * threads * 4, ctx->stream), "alloc");
  cudaEvent_t e0, e1;
  EVOC_TRY(cudaEventCreate(&e0), "event");
  EVOC_TRY(cudaEventCreate(&e1), "event");
  // b just below 1 and c small keep the values finite and normal for any iteration count
  evoc::ffma_kernel<<<blocks, threads, 0, ctx->stream>>>(out, iters / 8, 0.999999f, 1e-6f);  // warm-up
  cudaEventRecord(e0, ctx->stream);
  evoc::ffma_kernel<<<blocks, threads, 0, ctx->stream>>>(out, iters, 0.999999f, 1e-6f);
  cudaEventRecord(e1, ctx->stream);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  float t = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(out, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "ffma peak");
  const double flops = 2.0 * double(blocks) * threads * double(iters) * evoc::kUnroll * evoc::kChains;
  *tflops = flops / (double(t) * 1e-3) / 1e12;
  if (ms) *ms = t;
  return EVOC_OK;
}
