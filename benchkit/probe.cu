// Measurement probes for the benchmark and the tests (libgeraf_probe.so, not
// part of libgeraf_rf.so): the FP32 FMA issue rate that is the roofline
// denominator of the RF kernels (they are bound by the FP32 pipe; no
// tensor-core or HBM bound applies), the ceiling of the MIXED forward's Horner
// loop, and the sincosf identity check the PLAIN kernels rely on.  No
// counterpart in the reference.  Return codes are those of geraf_rf.h.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../geraf-sens_b200/csrc/common.cuh"
#include "../include/geraf_rf.h"

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

// The MIXED matched-filter forward's inner loop on its own: 4 packed voxel
// pairs per thread run the Horner recurrence P <- P z + s over `rows` rows of
// 256 samples, broadcast from shared memory in the duplicated (s, s) layout,
// with the per-(voxel, antenna) phase set-up left out (the phasors are fixed
// per thread).  Its rate is the ceiling of that loop's instruction form: every
// packed FMA of the complex step reads two or three register operands that
// the instruction before it did not, while the FMA-rate probe above reuses two
// of its three, so this loop stays below the FMA peak however it is scheduled.
__global__ void __launch_bounds__(128) horner_probe_kernel(float* sink, int rows, float seed) {
  constexpr int kLen = 256;
  constexpr int kPairs = 4;
  __shared__ __align__(16) float2 dup[2][kLen];
  for (int i = threadIdx.x; i < kLen; i += blockDim.x) {
    const float v = 1.0e-3f * static_cast<float>(i % 17) - 8.0e-3f;
    dup[0][i] = make_float2(v, v);
    dup[1][i] = make_float2(-v, -v);
  }
  __syncthreads();
  float2 zr[kPairs], zi[kPairs], nzi[kPairs], acc[kPairs];
#pragma unroll
  for (int q = 0; q < kPairs; ++q) {
    float s0, c0, s1, c1;
    sincospif(seed * static_cast<float>(threadIdx.x + 1) * 1.0e-3f + 0.1f * q, &s0, &c0);
    sincospif(seed * static_cast<float>(threadIdx.x + 2) * 1.0e-3f + 0.13f * q, &s1, &c1);
    zr[q] = make_float2(c0, c1);
    zi[q] = make_float2(-s0, -s1);
    nzi[q] = make_float2(s0, s1);
    acc[q] = make_float2(0.0f, 0.0f);
  }
  for (int r = 0; r < rows; ++r) {
    float2 pr[kPairs], pi[kPairs];
#pragma unroll
    for (int q = 0; q < kPairs; ++q) pr[q] = pi[q] = make_float2(0.0f, 0.0f);
#pragma unroll 2
    for (int n = kLen - 2; n >= 0; n -= 2) {
      const float4 a = *reinterpret_cast<const float4*>(&dup[0][n]);
      const float4 b = *reinterpret_cast<const float4*>(&dup[1][n]);
      const float2 sr[2] = {make_float2(a.z, a.w), make_float2(a.x, a.y)};
      const float2 si[2] = {make_float2(b.z, b.w), make_float2(b.x, b.y)};
#pragma unroll
      for (int h = 0; h < 2; ++h) {
#pragma unroll
        for (int q = 0; q < kPairs; ++q) {
          const float2 t1 = geraf::ffma2(pi[q], nzi[q], sr[h]);
          const float2 t2 = geraf::ffma2(pi[q], zr[q], si[h]);
          const float2 npr = geraf::ffma2(pr[q], zr[q], t1);
          pi[q] = geraf::ffma2(pr[q], zi[q], t2);
          pr[q] = npr;
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kPairs; ++q) {
      acc[q].x += pr[q].x + pi[q].y;
      acc[q].y += pi[q].x + pr[q].y;
    }
  }
  float s = 0.0f;
#pragma unroll
  for (int q = 0; q < kPairs; ++q) s += acc[q].x + acc[q].y;
  if (s == 1234.5f) sink[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the loop live
}

// The same sum evaluated by the second-order (Goertzel) recurrence on the
// complex samples: s_n = x_n + 2 cos(theta) s_{n+1} - s_{n+2} runs on the packed
// (re, im) pair of one voxel with a real coefficient, one sub.rn.f32x2 and one
// fma.rn.f32x2 per voxel-sample (8 voxels per thread, samples (re, im) from
// shared memory, no duplication).  Same flop count per row as the Horner probe.
__global__ void __launch_bounds__(128) goertzel_probe_kernel(float* sink, int rows, float seed) {
  constexpr int kLen = 256;
  constexpr int kVox = 8;
  __shared__ __align__(16) float2 xs[kLen];
  for (int i = threadIdx.x; i < kLen; i += blockDim.x) {
    const float v = 1.0e-3f * static_cast<float>(i % 17) - 8.0e-3f;
    xs[i] = make_float2(v, -v);
  }
  __syncthreads();
  float2 c2[kVox], acc[kVox];
#pragma unroll
  for (int q = 0; q < kVox; ++q) {
    float sn, cs;
    sincospif(seed * static_cast<float>(threadIdx.x + 1) * 1.0e-3f + 0.1f * q, &sn, &cs);
    c2[q] = make_float2(2.0f * cs, 2.0f * cs);
    acc[q] = make_float2(0.0f, 0.0f);
  }
  for (int r = 0; r < rows; ++r) {
    float2 s1[kVox], s2[kVox];
#pragma unroll
    for (int q = 0; q < kVox; ++q) s1[q] = s2[q] = make_float2(0.0f, 0.0f);
#pragma unroll 2
    for (int n = kLen - 2; n >= 0; n -= 2) {
      const float4 a = *reinterpret_cast<const float4*>(&xs[n]);  // (x_n, x_n+1)
      const float2 x[2] = {make_float2(a.z, a.w), make_float2(a.x, a.y)};
#pragma unroll
      for (int h = 0; h < 2; ++h) {
#pragma unroll
        for (int q = 0; q < kVox; ++q) {
          const float2 t = geraf::fsub2(x[h], s2[q]);
          s2[q] = s1[q];
          s1[q] = geraf::ffma2(c2[q], s1[q], t);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kVox; ++q) acc[q] = geraf::fadd2(acc[q], geraf::fsub2(s1[q], s2[q]));
  }
  float s = 0.0f;
#pragma unroll
  for (int q = 0; q < kVox; ++q) s += acc[q].x + acc[q].y;
  if (s == 1234.5f) sink[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the loop live
}

// Counts the FP32 inputs, over all 2^32 bit patterns, for which sincosf differs
// in any bit from separate sinf and cosf calls: the PLAIN kernels rely on there
// being none.
__global__ void sincos_identity_kernel(unsigned long long* mismatches) {
  unsigned long long local = 0;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < (1ull << 32);
       i += stride) {
    const float x = __uint_as_float(static_cast<unsigned int>(i));
    float s1, c1;
    sincosf(x, &s1, &c1);
    const float s0 = sinf(x);
    const float c0 = cosf(x);
    if (__float_as_uint(s0) != __float_as_uint(s1) || __float_as_uint(c0) != __float_as_uint(c1)) ++local;
  }
  if (local != 0) atomicAdd(mismatches, local);
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

// Enqueues blocks x threads (threads <= 128) threads of the Horner loop over
// `rows` rows of 256 samples x 8 voxels (flops = blocks * threads * rows * 16384).
// `sink` needs blocks*threads floats.
GERAF_EXPORT int32_t geraf_rf_horner_probe(int32_t blocks, int32_t threads, int32_t rows,
                                           float* sink, void* stream) {
  if (blocks <= 0 || threads <= 0 || threads > 128 || rows <= 0 || sink == nullptr) {
    return GERAF_ERR_INVALID_ARGUMENT;
  }
  horner_probe_kernel<<<blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(sink, rows, 0.5f);
  return cudaGetLastError() == cudaSuccess ? GERAF_OK : GERAF_ERR_CUDA;
}

// As geraf_rf_horner_probe, for the second-order recurrence form of the same
// sum (flops = blocks * threads * rows * 16384).
GERAF_EXPORT int32_t geraf_rf_goertzel_probe(int32_t blocks, int32_t threads, int32_t rows,
                                             float* sink, void* stream) {
  if (blocks <= 0 || threads <= 0 || threads > 128 || rows <= 0 || sink == nullptr) {
    return GERAF_ERR_INVALID_ARGUMENT;
  }
  goertzel_probe_kernel<<<blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(sink, rows, 0.5f);
  return cudaGetLastError() == cudaSuccess ? GERAF_OK : GERAF_ERR_CUDA;
}

// Adds to *mismatches (device memory, zeroed by the caller) the number of FP32
// inputs for which sincosf and separate sinf / cosf calls differ in any bit.
GERAF_EXPORT int32_t geraf_rf_sincos_identity_check(unsigned long long* mismatches, void* stream) {
  if (mismatches == nullptr) return GERAF_ERR_INVALID_ARGUMENT;
  sincos_identity_kernel<<<148 * 16, 256, 0, static_cast<cudaStream_t>(stream)>>>(mismatches);
  return cudaGetLastError() == cudaSuccess ? GERAF_OK : GERAF_ERR_CUDA;
}
