// FP64 throughput of the device the context lives on, measured by the library itself.
//
// The stencil kernels of the stage (WENO5 reconstruction, the Rusanov fluxes, the
// shock detector) do more FP64 arithmetic per byte than B200's FP64 pipe can keep up
// with at full HBM bandwidth.  Whether such a kernel is "FP64 bound" is judged against
// these two measured rates, not against a datasheet figure:
//   * fused multiply-adds per second (independent chains, no memory traffic), and
//   * IEEE double divisions per second (a / b, round to nearest, as the kernels do).
#include "imex_internal.h"

namespace imex {
namespace {

constexpr int kChains = 8;     // independent dependency chains per thread (hides the pipe latency)
constexpr int kBlocksPerSm = 8;
constexpr int kThreads = 256;

// a <- a * m + c on kChains chains; m < 1 and c > 0 keep every value normal and bounded
__global__ void __launch_bounds__(kThreads) k_peak_dfma(double* sink, int iters, double c) {
  double a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = 1e-3 * (double)(threadIdx.x + 1 + k);
  const double m = 0.9999999;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = fma(a[k], m, c);
  }
  double t = 0.0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) t += a[k];
  if (t < 0.0) sink[0] = t;  // never true (every chain stays positive); keeps the chains live
}

// a <- c / (a + 1) on kChains chains: converges to a fixed point in (0, c), never 0
__global__ void __launch_bounds__(kThreads) k_peak_ddiv(double* sink, int iters, double c) {
  double a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = 1e-3 * (double)(threadIdx.x + 1 + k);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = c / (a[k] + 1.0);
  }
  double t = 0.0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) t += a[k];
  if (t < 0.0) sink[0] = t;
}

}  // namespace

imex_status run_fp64_selftest(imex_ctx* ctx, double* dfma_per_s, double* ddiv_per_s) {
  const int blocks = ctx->num_sms * kBlocksPerSm;
  double* sink = ctx->red;  // one slot, written only if a chain went negative, which it cannot
  cudaEvent_t a = nullptr, b = nullptr;
  cudaError_t e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  if (e != cudaSuccess) return cuda_check(ctx, e, "fp64 self-test events");
  double rates[2] = {0.0, 0.0};
  const int iters[2] = {1 << 15, 1 << 12};
  for (int kind = 0; kind < 2 && e == cudaSuccess; ++kind) {
    float ms = 0.f;
    for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {  // the first launch warms up
      e = cudaEventRecord(a, ctx->stream);
      if (kind == 0)
        k_peak_dfma<<<blocks, kThreads, 0, ctx->stream>>>(sink, iters[kind], 1e-7);
      else
        k_peak_ddiv<<<blocks, kThreads, 0, ctx->stream>>>(sink, iters[kind], 1.5);
      if (e == cudaSuccess) e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaEventRecord(b, ctx->stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(b);
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    }
    const double ops = (double)blocks * kThreads * kChains * (double)iters[kind];
    rates[kind] = ms > 0.f ? ops / (ms * 1e-3) : 0.0;
  }
  ctx->kernel_launches += 4;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (e != cudaSuccess) return cuda_check(ctx, e, "fp64 self-test");
  if (dfma_per_s) *dfma_per_s = rates[0];
  if (ddiv_per_s) *ddiv_per_s = rates[1];
  return IMEX_OK;
}

}  // namespace imex
