// FP32 FMA throughput probe: the denominator of the PairHMM roofline, measured
// on the device the engine runs on (the recurrence is FP32-pipe bound, and the
// pool's measured peaks cover only HBM and tensor-core throughput).
#include <cuda_runtime.h>
#include <cstdint>
#include "../../include/vardepth_pairhmm.h"

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) fma_probe(float* sink, int iters, float seed) {
  float a[kChains];
  const float b = 0.999f + 1e-7f * threadIdx.x, c = 1e-3f * seed;
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = seed + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
#pragma unroll
      for (int k = 0; k < kChains; ++k) a[k] = __fmaf_rn(a[k], b, c);
    }
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  if (s == 1234.5f) sink[blockIdx.x * blockDim.x + threadIdx.x] = s;  // never true; keeps the chains live
}

}  // namespace

extern "C" int vd_measure_fp32_peak(int device, double* tflops) {
  if (!tflops) return VD_EINVAL;
  *tflops = 0.0;
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return VD_ENODEV; }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) { cudaSetDevice(prev); return VD_ECUDA; }
  const int blocks = prop.multiProcessorCount * 8, threads = 256, iters = 4096;
  float* sink = nullptr;
  cudaEvent_t e0, e1;
  int rc = VD_OK;
  if (cudaMalloc(&sink, sizeof(float) * blocks * threads) != cudaSuccess) { cudaSetDevice(prev); return VD_ENOMEM; }
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fma_probe<<<blocks, threads>>>(sink, iters / 8, 1.0f);  // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0);
    fma_probe<<<blocks, threads>>>(sink, iters, 1.0f + rep);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess) { rc = VD_ECUDA; break; }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  if (!rc) {
    const double fmas = (double)blocks * threads * iters * 16.0 * kChains;
    *tflops = 2.0 * fmas / (best * 1e-3) / 1e12;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  cudaSetDevice(prev);
  return rc;
}
