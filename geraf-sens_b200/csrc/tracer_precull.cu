// Point pre-cull of the signal tracer: one conservative test per point over the
// whole antenna set of a call, ahead of the per-(point, antenna) kernels, which
// then visit only the listed points.
//
// Every transmitter t_a of the call lies within R_t of a centre c_t and every
// receiver r_a within R_r of c_r.  For a point p with normal n (as given, not
// necessarily unit), i_c = p - c_t, o_c = c_r - p, H = I - 2 n n^T (so the
// unnormalised reflection of i_a = p - t_a is r_a = H i_a, and |H| <= m =
// 1 + 2|n|^2), the exact values of every pair obey
//   i_a.n   >= i_c.n - R_t |n|,                               |i_a| <= |i_c| + R_t,
//   o_a.r_a <= o_c.(H i_c) + R_r |H i_c| + R_t |H o_c| + m R_r R_t,  |o_a| <= |o_c| + R_r.
// So when
//   i_c.n - R_t |n| > 1e-4 (|i_c| + R_t) |n|                       (back-facing to all)
// or the o.r bound is below -1e-4 (|o_c| + R_r)(|i_c| + R_t) m     (reflected away from all)
// every pair of the point meets i.n > 1e-4 |i||n| or o.r < -1e-4 |o||i| m, the
// margins under which the reference's FP32 geometry culls a pair
// (surely_culled() in tracer_geometry.cuh derives them); the per-pair kernels
// would discard all of the point's pairs.  The test runs in FP64 on the FP32
// values the kernels use; its rounding (~1e-16 relative) is far inside the
// 1e-4 margin.  Non-finite values fail both comparisons, so such points are
// listed and decided by the exact form.  Out-of-bounds points are never listed.
//
// Launches: per-point flags with a count per 1024-point chunk, and the ordered
// scatter of the listed point indices, which for the adjoint also writes the
// zero gradients of every point not listed.  Each flags block bounds the
// aperture itself and each scatter block sums the counts before its chunk,
// up to 2048 antennas and 2048 chunks; beyond those, one-block kernels bound
// the aperture and scan the counts once.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "kernels.h"

namespace geraf {
namespace {

constexpr int kChunk = 1024;        // points per flag chunk (32 words)
constexpr int kChunkThreads = 256;  // 4 points per thread (faster than 1024 x 1)
// Up to these sizes the flags kernel bounds the aperture in every block and the
// scatter kernel sums the preceding chunks' counts itself: two launches, not four.
constexpr int64_t kInlineApertureMax = 2048;  // antennas
constexpr int64_t kInlineScanMax = 2048;      // chunks

struct Aperture {
  double ct[3], rt;  // transmitter centre and radius
  double cr[3], rr;  // receiver centre and radius
};

// The aperture bounds of antennas [0, A), by all 256 threads of a block (fixed
// reduction order, so every block that computes them gets the same bits); *out
// is written by thread 0 and published by the closing barrier.
template <typename T>
__device__ void block_aperture(const T* tx, const T* rx, int64_t A, Aperture* out) {
  __shared__ double red[6][256];
  __shared__ double cen[6];
  const int tid = threadIdx.x;
  double s[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int64_t a = tid; a < A; a += 256) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      s[k] += static_cast<double>(ld_f(tx, a * 3 + k));
      s[3 + k] += static_cast<double>(ld_f(rx, a * 3 + k));
    }
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) red[k][tid] = s[k];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (tid < w) {
#pragma unroll
      for (int k = 0; k < 6; ++k) red[k][tid] += red[k][tid + w];
    }
    __syncthreads();
  }
  if (tid < 6) cen[tid] = A > 0 ? red[tid][0] / static_cast<double>(A) : NAN;
  __syncthreads();
  double mt = 0.0, mr = 0.0;
  for (int64_t a = tid; a < A; a += 256) {
    double dt = 0.0, dr = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double et = static_cast<double>(ld_f(tx, a * 3 + k)) - cen[k];
      const double er = static_cast<double>(ld_f(rx, a * 3 + k)) - cen[3 + k];
      dt = fma(et, et, dt);
      dr = fma(er, er, dr);
    }
    // fmax drops a NaN operand; a non-finite antenna makes its centre (and so
    // every test) non-finite instead
    mt = fmax(mt, sqrt(dt));
    mr = fmax(mr, sqrt(dr));
  }
  __syncthreads();  // red is reused
  red[0][tid] = mt;
  red[1][tid] = mr;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (tid < w) {
      red[0][tid] = fmax(red[0][tid], red[0][tid + w]);
      red[1][tid] = fmax(red[1][tid], red[1][tid + w]);
    }
    __syncthreads();
  }
  if (tid == 0) {
    // widen the radii by far more than the FP64 rounding of the distances
    const double st = fabs(cen[0]) + fabs(cen[1]) + fabs(cen[2]);
    const double sr = fabs(cen[3]) + fabs(cen[4]) + fabs(cen[5]);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      out->ct[k] = cen[k];
      out->cr[k] = cen[3 + k];
    }
    out->rt = red[0][0] + 1e-12 * (red[0][0] + st);
    out->rr = red[1][0] + 1e-12 * (red[1][0] + sr);
  }
  __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(256) aperture_kernel(const T* tx, const T* rx, int64_t A, Aperture* out) {
  block_aperture(tx, rx, A, out);
}

__device__ __forceinline__ double dot3d(const double* a, const double* b) {
  return fma(a[2], b[2], fma(a[1], b[1], a[0] * b[0]));
}

// True when every pair of the point is culled with the margin above.
__device__ __forceinline__ bool culled_for_all(const Aperture& ap, const float* nf, const float* pf) {
  double n[3], ic[3], oc[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    n[k] = nf[k];
    ic[k] = static_cast<double>(pf[k]) - ap.ct[k];
    oc[k] = ap.cr[k] - static_cast<double>(pf[k]);
  }
  const double nn = dot3d(n, n);
  const double nrm = sqrt(nn);
  const double m = 1.0 + 2.0 * nn;
  const double icn = dot3d(ic, n);
  const double ni = sqrt(dot3d(ic, ic));
  const double no = sqrt(dot3d(oc, oc));
  if (icn - ap.rt * nrm > 1e-4 * (ni + ap.rt) * nrm) return true;
  const double ocn = dot3d(oc, n);
  double hi[3], ho[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    hi[k] = ic[k] - 2.0 * icn * n[k];
    ho[k] = oc[k] - 2.0 * ocn * n[k];
  }
  const double bound = dot3d(oc, hi) + ap.rr * sqrt(dot3d(hi, hi)) + ap.rt * sqrt(dot3d(ho, ho)) +
                       m * ap.rr * ap.rt;
  return bound < -1e-4 * (no + ap.rr) * (ni + ap.rt) * m;
}

// Flag word w of chunk c covers points c*1024 + w*32 + lane; counts[c] is the
// number of listed points of the chunk.  With a null `aperture` each block
// bounds the antennas itself.
template <typename T>
__global__ void __launch_bounds__(kChunkThreads) point_flags_kernel(const T* normals, const T* points,
                                                                    const uint8_t* inb, int64_t P,
                                                                    const Aperture* aperture, const T* tx,
                                                                    const T* rx, int64_t A, uint32_t* words,
                                                                    int* counts) {
  __shared__ int warp_count[kChunkThreads / 32];
  __shared__ Aperture ap_s;
  if (aperture == nullptr) block_aperture(tx, rx, A, &ap_s);
  const Aperture ap = aperture != nullptr ? *aperture : ap_s;
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kChunk;
  int c = 0;
#pragma unroll
  for (int k = 0; k < kChunk / kChunkThreads; ++k) {
    const int64_t q = base + k * kChunkThreads + threadIdx.x;
    bool listed = false;
    if (q < P && inb[q]) {
      float n[3], pt[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        n[j] = ld_f(normals, q * 3 + j);
        pt[j] = ld_f(points, q * 3 + j);
      }
      listed = !culled_for_all(ap, n, pt);
    }
    const unsigned b = __ballot_sync(0xffffffffu, listed);
    if (lane == 0) {
      words[static_cast<int64_t>(blockIdx.x) * 32 + k * (kChunkThreads / 32) + warp] = b;
      c += __popc(b);
    }
  }
  if (lane == 0) warp_count[warp] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int total = 0;
    for (int w = 0; w < kChunkThreads / 32; ++w) total += warp_count[w];
    counts[blockIdx.x] = total;
  }
}

// Exclusive scan of the chunk counts in one block; *total = the listed points.
__global__ void __launch_bounds__(1024) chunk_scan_kernel(const int* counts, int64_t chunks, int* offsets,
                                                          int* total) {
  __shared__ int warp_sum[32];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  int carry = 0;
  for (int64_t base = 0; base < chunks; base += blockDim.x) {
    const int64_t i = base + threadIdx.x;
    const int v = i < chunks ? counts[i] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      int w = lane < static_cast<int>(blockDim.x >> 5) ? warp_sum[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      warp_sum[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    if (i < chunks) offsets[i] = carry + (warp > 0 ? warp_sum[warp - 1] : 0) + x - v;
    carry += warp_sum[31];
    __syncthreads();  // warp_sum is rewritten by the next piece
  }
  if (threadIdx.x == 0) *total = carry;
}

// Writes the listed point indices of each chunk in ascending order; with
// gradient outputs, every unlisted point gets zero gradients (all antennas'
// grad_sigmas, grad_normals and grad_points).  With a null `offsets` each block
// sums the counts of the chunks before its own, and the last block writes the
// total.
template <typename T>
__global__ void __launch_bounds__(kChunkThreads) point_scatter_kernel(const uint32_t* words, const int* offsets,
                                                                      const int* counts, int64_t chunks,
                                                                      int* total, int64_t P, int* list,
                                                                      int64_t A, T* g_sigmas, T* g_normals,
                                                                      T* g_points) {
  __shared__ uint32_t w_s[32];
  __shared__ int pre_s[32];
  __shared__ int part_s[kChunkThreads / 32];
  __shared__ int off_s;
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t chunk = blockIdx.x;
  if (offsets == nullptr) {
    int x = 0;
    for (int64_t i = threadIdx.x; i < chunk; i += kChunkThreads) x += counts[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) part_s[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
      int t = 0;
      for (int w = 0; w < kChunkThreads / 32; ++w) t += part_s[w];
      off_s = t;
      if (chunk == chunks - 1) *total = t + counts[chunk];
    }
  } else if (threadIdx.x == 0) {
    off_s = offsets[chunk];
  }
  if (warp == 0) {
    const uint32_t w = words[chunk * 32 + lane];
    const int c = __popc(w);
    int x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    w_s[lane] = w;
    pre_s[lane] = x - c;
  }
  __syncthreads();
  const int off = off_s;
  const T zero = from_f<T>(0.0f);
#pragma unroll
  for (int k = 0; k < kChunk / kChunkThreads; ++k) {
    const int wi = k * (kChunkThreads / 32) + warp;
    const int64_t q = chunk * kChunk + wi * 32 + lane;
    if (q >= P) continue;
    const uint32_t w = w_s[wi];
    if ((w >> lane) & 1u) {
      list[off + pre_s[wi] + __popc(w & ((1u << lane) - 1u))] = static_cast<int>(q);
    } else if (g_normals != nullptr) {
#pragma unroll
      for (int j = 0; j < 3; ++j) g_normals[q * 3 + j] = zero;
      if (g_points != nullptr) {
#pragma unroll
        for (int j = 0; j < 3; ++j) g_points[q * 3 + j] = zero;
      }
      for (int64_t a = 0; a < A; ++a) g_sigmas[a * P + q] = zero;
    }
  }
}

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

struct ListLayout {
  size_t aperture, words, counts, offsets, total, list, bytes;
};

ListLayout list_layout(int64_t P) {
  const int64_t chunks = (P + kChunk - 1) / kChunk;
  ListLayout l;
  size_t off = 0;
  l.aperture = off;
  off = align256(off + sizeof(Aperture));
  l.words = off;
  off = align256(off + static_cast<size_t>(chunks) * 32 * sizeof(uint32_t));
  l.counts = off;
  off = align256(off + static_cast<size_t>(chunks) * sizeof(int));
  l.offsets = off;
  off = align256(off + static_cast<size_t>(chunks) * sizeof(int));
  l.total = off;
  off = align256(off + sizeof(int));
  l.list = off;
  off = align256(off + static_cast<size_t>(P) * sizeof(int));
  l.bytes = off;
  return l;
}

template <typename T>
cudaError_t launch_point_list(const TracerArgs& a, void* ws, bool zero_grads, cudaStream_t st) {
  const ListLayout l = list_layout(a.P);
  unsigned char* base = static_cast<unsigned char*>(ws);
  Aperture* ap = reinterpret_cast<Aperture*>(base + l.aperture);
  uint32_t* words = reinterpret_cast<uint32_t*>(base + l.words);
  int* counts = reinterpret_cast<int*>(base + l.counts);
  int* offsets = reinterpret_cast<int*>(base + l.offsets);
  int* total = reinterpret_cast<int*>(base + l.total);
  int* list = reinterpret_cast<int*>(base + l.list);
  const int64_t chunks = (a.P + kChunk - 1) / kChunk;
  const T* tx = static_cast<const T*>(a.tx);
  const T* rx = static_cast<const T*>(a.rx);
  const bool inline_aperture = a.A <= kInlineApertureMax;
  const bool inline_scan = chunks <= kInlineScanMax;
  if (!inline_aperture) aperture_kernel<T><<<1, 256, 0, st>>>(tx, rx, a.A, ap);
  point_flags_kernel<T><<<static_cast<unsigned>(chunks), kChunkThreads, 0, st>>>(
      static_cast<const T*>(a.normals), static_cast<const T*>(a.points), a.inbounds, a.P,
      inline_aperture ? nullptr : ap, tx, rx, a.A, words, counts);
  if (!inline_scan) chunk_scan_kernel<<<1, 1024, 0, st>>>(counts, chunks, offsets, total);
  point_scatter_kernel<T><<<static_cast<unsigned>(chunks), kChunkThreads, 0, st>>>(
      words, inline_scan ? nullptr : offsets, counts, chunks, total, a.P, list, a.A,
      zero_grads ? static_cast<T*>(a.grad_sigmas) : nullptr, zero_grads ? static_cast<T*>(a.grad_normals) : nullptr,
      zero_grads ? static_cast<T*>(a.grad_points) : nullptr);
  return cudaGetLastError();
}

}  // namespace

bool tracer_point_list_applies(const TracerArgs& a) {
  // int32 indices and a grid of one block per 1024-point chunk
  return (a.mode == kMixed || a.mode == kNufft) && a.P > 0 && a.P <= (int64_t{1} << 31) - kChunk;
}

size_t tracer_point_list_bytes(int64_t P) { return list_layout(P).bytes; }

PointList tracer_point_list_view(void* ws, int64_t P) {
  const ListLayout l = list_layout(P);
  unsigned char* base = static_cast<unsigned char*>(ws);
  return PointList{reinterpret_cast<const int*>(base + l.list), reinterpret_cast<const int*>(base + l.total)};
}

cudaError_t tracer_point_list(const TracerArgs& a, void* ws, bool zero_grads, cudaStream_t st) {
  if (a.dtype == kF64) return launch_point_list<double>(a, ws, zero_grads, st);
  return launch_point_list<float>(a, ws, zero_grads, st);
}

}  // namespace geraf
