// Measured FP32 issue peak of the current GPU: the denominator of the march kernel's FP32 roofline.
//
// The raymarch is bound by FP32 instruction issue (SIMT FMA/FMUL/FADD and the special-function unit), not by HBM, and
// no vendor figure is measured on the box the benchmark runs on.  This kernel measures one: every thread runs
// kChains independent FMA chains (a <- a * b + c), enough independent work per scheduler to cover the FMA latency,
// over a grid of whole-SM blocks, timed with CUDA events.  FLOP/s = 2 * chains * iterations * threads / time.
#include <cuda_runtime.h>

#include <stdexcept>

#include "internal.hpp"

using namespace phx_capi;

namespace {

constexpr int kChains = 8;
constexpr int kPeakThreads = 512;

__global__ void __launch_bounds__(kPeakThreads) k_fma_chains(float b, float c, int iters, float* sink) {
  float a[kChains];
#pragma unroll
  for (int j = 0; j < kChains; j++) a[j] = (float)(threadIdx.x + j);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 16; u++) {
#pragma unroll
      for (int j = 0; j < kChains; j++) a[j] = fmaf(a[j], b, c);
    }
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < kChains; j++) s += a[j];
  if (s == 12345.678f) sink[0] = s;  // keeps the chains live; practically never stores
}

}  // namespace

extern "C" int phx_measure_fp32_peak(int32_t repeats, double* tflops) {
  return guarded([&]() -> int {
    if (!tflops || repeats < 1) throw std::invalid_argument("bad argument");
    int dev = 0, sms = 0;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute");
    float* sink = nullptr;
    ck(cudaMalloc((void**)&sink, sizeof(float)), "cudaMalloc");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ck(cudaEventCreate(&e0), "event");
    ck(cudaEventCreate(&e1), "event");
    const int blocks = sms * (2048 / kPeakThreads), iters = 4096;
    const double flops = 2.0 * kChains * 16.0 * iters * (double)blocks * kPeakThreads;
    double best = 0.0;
    cudaError_t err = cudaSuccess;
    for (int r = 0; r <= repeats && err == cudaSuccess; r++) {  // the first run warms up
      cudaEventRecord(e0);
      k_fma_chains<<<blocks, kPeakThreads>>>(0.999999f, 1e-7f, iters, sink);
      cudaEventRecord(e1);
      err = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
      if (r > 0 && ms > 0.f) best = std::max(best, flops / (ms * 1e-3) * 1e-12);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    ck(err, "fp32 peak kernel");
    *tflops = best;
    return PHX_OK;
  });
}
