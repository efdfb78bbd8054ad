// Volume sampling at target points (InterpolateMFAtTargets) for sm_100a.
//
// The reference's data workers sample the matched-filter volume at every
// target ray sample on the host with torch grid_sample
// (geraf/datasets/transforms/loading.py:20-25, 78-100): the volume [Nx, Ny, Nz]
// (x slowest) is read as a [1, 1, Nx, Ny, Nz] tensor and the grid is given as
// (z, y, x), so a point's normalised x selects along Nx, y along Ny and z
// along Nz; trilinear weights, zeros outside the volume, align_corners as
// configured (True in every reference config).  Here one thread per point
// forms the source coordinate, the eight corner weights and the bounds-checked
// gathers; the volume (8 MB at 128^3) stays in L2 across a launch, so the
// kernel's HBM traffic is the points in and the samples out.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace geraf {
namespace {

// grid_sample's unnormalisation of coordinate c in [-1, 1] to a source index,
// ((c + 1) / 2) (size - 1) or ((c + 1) size - 1) / 2, each operation rounded on
// its own (no fused multiply-add) as torch's host code rounds it.
__device__ __forceinline__ float source_index(float c, int size, bool align) {
  const float c1 = __fadd_rn(c, 1.0f);
  return align ? __fmul_rn(__fmul_rn(c1, 0.5f), static_cast<float>(size - 1))
               : __fmul_rn(__fsub_rn(__fmul_rn(c1, static_cast<float>(size)), 1.0f), 0.5f);
}

__global__ void __launch_bounds__(256) volume_sample_kernel(const float* __restrict__ vol, int nx,
                                                             int ny, int nz,
                                                             const float* __restrict__ pts,
                                                             int64_t n, float* __restrict__ out,
                                                             int nearest, int align) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    const float fx = source_index(__ldg(pts + 3 * i + 0), nx, align != 0);
    const float fy = source_index(__ldg(pts + 3 * i + 1), ny, align != 0);
    const float fz = source_index(__ldg(pts + 3 * i + 2), nz, align != 0);
    float acc = 0.0f;
    if (nearest) {
      // round half to even, like grid_sample's nearest mode; the range test runs
      // in float so NaN and huge coordinates never reach an integer conversion
      const float rx = nearbyintf(fx), ry = nearbyintf(fy), rz = nearbyintf(fz);
      if (rx >= 0.0f && rx <= nx - 1 && ry >= 0.0f && ry <= ny - 1 && rz >= 0.0f && rz <= nz - 1) {
        acc = __ldg(vol + (static_cast<int64_t>(rx) * ny + static_cast<int64_t>(ry)) * nz +
                    static_cast<int64_t>(rz));
      }
    } else {
      const float x0 = floorf(fx), y0 = floorf(fy), z0 = floorf(fz);
      // corners lie in [x0, x0 + 1]; anything outside [-1, n] contributes nothing
      if (x0 >= -1.0f && x0 <= nx - 1 && y0 >= -1.0f && y0 <= ny - 1 && z0 >= -1.0f && z0 <= nz - 1) {
        const float wx1 = fx - x0, wy1 = fy - y0, wz1 = fz - z0;
        const float wx0 = (x0 + 1.0f) - fx, wy0 = (y0 + 1.0f) - fy, wz0 = (z0 + 1.0f) - fz;
        const int ix = static_cast<int>(x0), iy = static_cast<int>(y0), iz = static_cast<int>(z0);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const int dx = c >> 2, dy = (c >> 1) & 1, dz = c & 1;
          const int jx = ix + dx, jy = iy + dy, jz = iz + dz;
          if (jx < 0 || jx >= nx || jy < 0 || jy >= ny || jz < 0 || jz >= nz) continue;
          const float w = (dx ? wx1 : wx0) * (dy ? wy1 : wy0) * (dz ? wz1 : wz0);
          acc = fmaf(__ldg(vol + (static_cast<int64_t>(jx) * ny + jy) * nz + jz), w, acc);
        }
      }
    }
    out[i] = acc;
  }
}

}  // namespace

cudaError_t volume_sample(const VolumeSampleArgs& a, cudaStream_t st) {
  if (a.num_points == 0) return cudaSuccess;
  const int64_t blocks = std::min<int64_t>((a.num_points + 255) / 256, static_cast<int64_t>(148) * 32);
  volume_sample_kernel<<<static_cast<unsigned>(blocks), 256, 0, st>>>(
      static_cast<const float*>(a.volume), static_cast<int>(a.nx), static_cast<int>(a.ny),
      static_cast<int>(a.nz), static_cast<const float*>(a.points), a.num_points,
      static_cast<float*>(a.out), a.nearest ? 1 : 0, a.align_corners ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace geraf
