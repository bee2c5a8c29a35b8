// Device measurement used by the benchmark's roofline: the FP32 FMA issue
// peak of the current device, measured rather than computed from the data
// sheet (SMs x 128 lanes x 2 FLOP x clock), so that the raster's FP32
// fraction is taken against what this GPU sustains at its present clocks.

#include <algorithm>
#include <cuda_runtime.h>

#include "cuda_check.h"
#include "kernels.h"
#include "pipeline.h"
#include "sort_api.h"

namespace gsr {
namespace {

constexpr int kChains = 8;    // independent FMA chains per thread (hides the FMA latency)
constexpr int kUnroll = 16;   // FMAs per chain per loop iteration

// Every thread runs kChains independent chains x = x * a + b; a and b keep
// the values bounded and the final sum is stored only when it equals an
// impossible value, so the compiler keeps every FMA and the kernel writes
// nothing in practice.
__global__ void __launch_bounds__(256) fma_peak_kernel(float *out, int iters, float a, float b) {
  float x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = (float)(threadIdx.x + c) * 1e-3f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
      for (int c = 0; c < kChains; ++c) x[c] = __fmaf_rn(x[c], a, b);
    }
  }
  float s = 0.0f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c];
  if (s == -1.2345e30f) out[blockIdx.x] = s;
}

}  // namespace

void measure_fp32_peak(double *tflops, double *best_ms) {
  require_device();
  const uint32_t sms = device_sm_count();
  const uint32_t blocks = sms * 8;  // 2048 threads per SM: every scheduler has warps to pick
  const int iters = 2048;
  DeviceBuffer out;
  out.reset(4ull * blocks);
  cudaEvent_t e0, e1;
  GSR_CUDA(cudaEventCreate(&e0));
  GSR_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  for (int rep = 0; rep < 6; ++rep) {  // first launch is a warm-up
    GSR_CUDA(cudaEventRecord(e0));
    fma_peak_kernel<<<blocks, 256>>>(out.as<float>(), iters, 0.9999f, 1e-4f);
    GSR_CUDA(cudaEventRecord(e1));
    GSR_CUDA(cudaEventSynchronize(e1));
    float ms = 0.0f;
    GSR_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (rep > 0) best = std::min(best, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const double flop = 2.0 * kChains * kUnroll * (double)iters * blocks * 256.0;
  if (best_ms) *best_ms = best;
  if (tflops) *tflops = flop / (best * 1e-3) / 1e12;
}

}  // namespace gsr
