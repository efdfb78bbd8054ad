// FP32 FMA issue-rate probe: the roofline denominator for the RF kernels, which
// are bound by the FP32 pipe (no tensor-core or HBM bound applies).  No
// counterpart in the reference.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/geraf_rf.h"

#define GERAF_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

// 8 independent FMA chains per thread: with >= 4 warps per scheduler this
// keeps every FP32 lane issuing one FMA per clock.
__global__ void __launch_bounds__(256) fma_probe_kernel(float* sink, int iters, float seed) {
  float a0 = seed + threadIdx.x * 1e-6f, a1 = a0 + 1e-3f, a2 = a0 + 2e-3f, a3 = a0 + 3e-3f;
  float a4 = a0 + 4e-3f, a5 = a0 + 5e-3f, a6 = a0 + 6e-3f, a7 = a0 + 7e-3f;
  const float m = 0.999999f, c = 1.0e-7f;
#pragma unroll 16
  for (int i = 0; i < iters; ++i) {
    a0 = fmaf(a0, m, c);
    a1 = fmaf(a1, m, c);
    a2 = fmaf(a2, m, c);
    a3 = fmaf(a3, m, c);
    a4 = fmaf(a4, m, c);
    a5 = fmaf(a5, m, c);
    a6 = fmaf(a6, m, c);
    a7 = fmaf(a7, m, c);
  }
  const float s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
  if (s == 1234.5f) sink[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

}  // namespace

// Enqueues blocks x threads threads of `iters` iterations x 8 FMAs each
// (flops = blocks * threads * iters * 16).  `sink` needs blocks*threads floats.
GERAF_EXPORT int32_t geraf_rf_fma_probe(int32_t blocks, int32_t threads, int32_t iters, float* sink,
                                        void* stream) {
  if (blocks <= 0 || threads <= 0 || threads > 256 || iters <= 0 || sink == nullptr) {
    return GERAF_ERR_INVALID_ARGUMENT;
  }
  fma_probe_kernel<<<blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(sink, iters, 0.5f);
  return cudaGetLastError() == cudaSuccess ? GERAF_OK : GERAF_ERR_CUDA;
}
