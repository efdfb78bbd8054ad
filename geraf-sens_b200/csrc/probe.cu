// FP32 FMA issue-rate probe: the roofline denominator for the RF kernels, which
// are bound by the FP32 pipe (no tensor-core or HBM bound applies).  No
// counterpart in the reference.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/geraf_rf.h"
#include "common.cuh"

#define GERAF_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

// 8 independent chains of packed FP32 FMAs (fma.rn.f32x2, two FMAs per
// instruction) per thread.  The packed form measures slightly higher than
// scalar FMA chains on B200 (it needs half the issue slots for the same FMA
// pipe time), so it is the ceiling the kernels are held to.
__global__ void __launch_bounds__(256) fma_probe_kernel(float* sink, int iters, float seed) {
  float2 a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    a[k] = make_float2(seed + threadIdx.x * 1e-6f + k * 1e-3f, seed + 0.5f + k * 1e-3f);
  }
  const float2 m = make_float2(0.999999f, 0.999999f), c = make_float2(1.0e-7f, 1.0e-7f);
#pragma unroll 16
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = geraf::ffma2(a[k], m, c);
  }
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k].x + a[k].y;
  if (s == 1234.5f) sink[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

}  // namespace

// Enqueues blocks x threads threads of `iters` iterations x 16 FMAs each
// (flops = blocks * threads * iters * 32).  `sink` needs blocks*threads floats.
GERAF_EXPORT int32_t geraf_rf_fma_probe(int32_t blocks, int32_t threads, int32_t iters, float* sink,
                                        void* stream) {
  if (blocks <= 0 || threads <= 0 || threads > 256 || iters <= 0 || sink == nullptr) {
    return GERAF_ERR_INVALID_ARGUMENT;
  }
  fma_probe_kernel<<<blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(sink, iters, 0.5f);
  return cudaGetLastError() == cudaSuccess ? GERAF_OK : GERAF_ERR_CUDA;
}
