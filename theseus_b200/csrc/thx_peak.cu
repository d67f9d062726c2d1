// thx_peak.cu -- FP64 fused-multiply-add throughput of the current GPU,
// measured with CUDA events: the denominator of the FP64-pipe roofline that
// the benchmark reports for the flux-differencing volume kernel (whose pair
// fluxes are FP64 arithmetic with no tensor-core form).
//
// Every thread runs eight independent FMA chains x <- x * a + b (a < 1, so the
// values stay bounded) for `iters` rounds of eight steps, on a grid of eight
// 256-thread CTAs per SM, which keeps every FP64 pipe of every SM busy.  One
// FMA counts two floating-point operations.
#include "theseus_b200.h"

#include <cuda_runtime.h>

namespace {

constexpr int kChains = 8;
constexpr int kUnroll = 8;
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) fp64_fma_chains(int iters, double a, double b, double *sink) {
  double x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = 1e-3 * (threadIdx.x + c);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
#pragma unroll
      for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c];
  if (s == -1.0) sink[blockIdx.x] = s;  // never true; keeps the chains live
}

}  // namespace

extern "C" int thx_measure_fp64_fma_peak(int iters, int repeats, double *flops_per_s, void *stream) {
  if (iters <= 0 || repeats <= 0 || !flops_per_s) return THX_ERR_INVALID_ARGUMENT;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return THX_ERR_NO_DEVICE; }
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return THX_ERR_CUDA;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = 8 * sms;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return THX_ERR_CUDA;
  if (cudaEventCreate(&e1) != cudaSuccess) { cudaEventDestroy(e0); return THX_ERR_CUDA; }
  int st = THX_OK;
  double best = 0.0;
  for (int r = 0; r <= repeats && st == THX_OK; ++r) {  // r == 0: warm-up
    cudaEventRecord(e0, s);
    fp64_fma_chains<<<blocks, kThreads, 0, s>>>(iters, 0.999999, 1e-7, nullptr);
    cudaEventRecord(e1, s);
    if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
      st = THX_ERR_CUDA;
      break;
    }
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) { st = THX_ERR_CUDA; break; }
    const double flops = 2.0 * kChains * kUnroll * (double)iters * blocks * kThreads;
    if (r > 0 && ms > 0.f && flops / (ms * 1e-3) > best) best = flops / (ms * 1e-3);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *flops_per_s = best;
  return st;
}
