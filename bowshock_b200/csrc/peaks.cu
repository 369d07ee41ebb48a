// The FP64 fused multiply-add rate of the current device, measured: the
// denominator for the FP64 fraction of the flux kernels (their residual is
// FP64 arithmetic, bound by the FP64 pipe rather than by HBM). Every thread
// runs kChains independent FMA chains, so the pipe, not a chain's latency,
// sets the rate; the grid fills every SM with full occupancy. No counterpart
// in the reference.
#include <cuda_runtime.h>

#include <string>

#include "bowshock.h"
#include "common.hpp"

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) fma_chains(int iterations, double b, double c, double* out) {
  double a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; k++) a[k] = 1.0 + 1e-3 * (threadIdx.x + k);
  for (int it = 0; it < iterations; it++) {
#pragma unroll
    for (int k = 0; k < kChains; k++) a[k] = fma(a[k], b, c);
  }
  double s = 0;
#pragma unroll
  for (int k = 0; k < kChains; k++) s += a[k];
  // Stored only where it can never be true, so the chains are not dead code.
  if (s == -1.0) out[blockIdx.x] = s;
}

}  // namespace

extern "C" {

bs_status bs_fp64_fma_rate(int32_t iterations, double* tflops, double* ms) {
  if (tflops == nullptr || ms == nullptr || iterations < 1)
    return bs::fail(BS_INVALID_ARGUMENT, "needs iterations >= 1 and two outputs");
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fma_chains, kThreads, 0);
  double* out = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&out), sizeof(double) * 8);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  const int blocks = sms * per_sm;
  float t = 0;
  if (e == cudaSuccess) {
    fma_chains<<<blocks, kThreads>>>(iterations, 0.9999999, 1e-7, out);  // warm-up
    cudaEventRecord(e0);
    fma_chains<<<blocks, kThreads>>>(iterations, 0.9999999, 1e-7, out);
    cudaEventRecord(e1);
    e = cudaEventSynchronize(e1);
  }
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  if (e0 != nullptr) cudaEventDestroy(e0);
  if (e1 != nullptr) cudaEventDestroy(e1);
  if (out != nullptr) cudaFree(out);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return bs::fail(BS_EXECUTION, std::string("FP64 rate: ") + cudaGetErrorString(e));
  }
  const double flops = 2.0 * kChains * double(iterations) * double(blocks) * kThreads;
  *ms = t;
  *tflops = flops / (double(t) * 1e-3) / 1e12;
  return BS_OK;
}

}  // extern "C"
