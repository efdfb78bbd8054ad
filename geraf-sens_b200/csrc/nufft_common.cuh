// Shared pieces of the NUFFT forms (nufft_kernels.cu: matched filter,
// nufft_tracer_kernels.cu: signal tracer): the "exponential of semicircle"
// kernel and its per-tap weight polynomials, the deconvolution factors, the
// per-antenna range-grid FFTs, the per-(point, antenna) NUFFT coordinates, the
// TMA row stager, the bounding-box band bound and the adjoint FFT.  See
// nufft_kernels.cu for the method.
#pragma once

#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "kernels.h"

namespace geraf {
namespace {

constexpr int kGlNodes = 48;  // Gauss-Legendre nodes on [0, W/2] for Phi

struct GlRule {
  double x[kGlNodes];
  double w[kGlNodes];
};

// Gauss-Legendre nodes and weights on [0, b]: Newton iteration on the
// three-term Legendre recurrence from the asymptotic first guesses
// cos(pi (i + 3/4) / (n + 1/2)).
GlRule gauss_legendre(double b) {
  GlRule r;
  const int n = kGlNodes;
  for (int i = 0; i < n; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));
    double dp = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; ++k) {
        const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    // map [-1, 1] -> [0, b]
    r.x[i] = 0.5 * b * (1.0 + z);
    r.w[i] = 0.5 * b * 2.0 / ((1.0 - z * z) * dp * dp);
  }
  return r;
}

// Interpolation weights.  For a point at grid coordinate u = base + W/2 - 1 + f
// (f in [0, 1)), grid point base + k gets phi((f + W/2 - 1 - k) 2 / W).  Each
// tap's weight is a polynomial of degree P in z = 2f - 1: the Chebyshev
// interpolant at P + 1 nodes (FP64 on the host), in monomial form, evaluated by
// Horner in FP32 with the coefficients as kernel parameters.  Degrees are the
// lowest that keep the fit error at or below the FP32 rounding of the weights
// for W >= 8 (~1e-7 absolute) and ten times below the truncation error of the
// kernel for W = 4, 6 (measured: 8.5e-5 at W = 4, 2.7e-6 at W = 6).
constexpr int kMaxTaps = 12;
constexpr int kMaxDegree = 13;
constexpr int kGridPad = 16;  // periodic extension of each grid row (>= kMaxTaps)

__host__ __device__ constexpr int poly_degree(int W) { return W <= 4 ? 5 : (W == 6 ? 6 : W - 1); }

struct EsPoly {
  float c[kMaxTaps][kMaxDegree + 1];  // c[k][i]: coefficient of z^i for tap k
};

double es_kernel(double t, double beta) {
  return std::exp(beta * (std::sqrt(std::max(0.0, 1.0 - t * t)) - 1.0));
}

EsPoly es_poly(int W, double beta) {
  EsPoly e{};
  const int P = poly_degree(W);
  const int n = P + 1;
  for (int k = 0; k < W; ++k) {
    double val[kMaxDegree + 1], z[kMaxDegree + 1];
    for (int j = 0; j < n; ++j) {
      z[j] = std::cos(M_PI * (j + 0.5) / n);
      const double f = 0.5 * (z[j] + 1.0);
      val[j] = es_kernel((f + W / 2 - 1 - k) * 2.0 / W, beta);
    }
    // Chebyshev coefficients a_i, then sum_i a_i T_i(z) expanded to monomials
    double mono[kMaxDegree + 1] = {0.0};
    double t_prev[kMaxDegree + 1] = {0.0}, t_cur[kMaxDegree + 1] = {0.0};
    t_prev[0] = 1.0;  // T_0
    t_cur[1] = 1.0;   // T_1
    for (int i = 0; i < n; ++i) {
      double a = 0.0;
      for (int j = 0; j < n; ++j) a += val[j] * std::cos(i * M_PI * (j + 0.5) / n);
      a *= (i == 0 ? 1.0 : 2.0) / n;
      const double* ti = i == 0 ? t_prev : t_cur;
      for (int q = 0; q <= P; ++q) mono[q] += a * ti[q];
      if (i >= 1) {  // advance: T_{i+1} = 2 z T_i - T_{i-1}
        double t_next[kMaxDegree + 1] = {0.0};
        for (int q = 0; q <= P; ++q) {
          t_next[q] = (q > 0 ? 2.0 * t_cur[q - 1] : 0.0) - t_prev[q];
        }
        for (int q = 0; q <= P; ++q) {
          t_prev[q] = t_cur[q];
          t_cur[q] = t_next[q];
        }
      }
    }
    for (int q = 0; q <= P; ++q) e.c[k][q] = static_cast<float>(mono[q]);
  }
  return e;
}

template <int W>
struct TapWeights {
  float w[W];
};

// phi is even, so tap W-1-k at z is tap k at -z: with tap k's polynomial split
// into even and odd parts E_k(z^2) + z O_k(z^2), the mirror pair is E_k + z O_k
// and E_k - z O_k -- one evaluation for two taps.
template <int W>
__device__ __forceinline__ TapWeights<W> tap_weights(const EsPoly& e, float f) {
  constexpr int P = poly_degree(W);
  constexpr int PE = P & ~1;        // highest even power
  constexpr int PO = (P - 1) | 1;   // highest odd power
  const float z = fmaf(2.0f, f, -1.0f);
  const float z2 = z * z;
  TapWeights<W> r;
#pragma unroll
  for (int k = 0; k < W / 2; ++k) {
    float ev = e.c[k][PE];
#pragma unroll
    for (int i = PE - 2; i >= 0; i -= 2) ev = fmaf(ev, z2, e.c[k][i]);
    float od = e.c[k][PO];
#pragma unroll
    for (int i = PO - 2; i >= 1; i -= 2) od = fmaf(od, z2, e.c[k][i]);
    r.w[k] = fmaf(od, z, ev);
    r.w[W - 1 - k] = fmaf(-od, z, ev);
  }
  return r;
}

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

int grid_points(int64_t S) {
  int M = 16;
  while (M < 2 * S) M *= 2;
  return M;
}

// ---------------------------------------------------------------------------
// 1. Deconvolution factors 1 / Phi((n - h) / M), n in [0, S).
struct DeconvP {
  GlRule gl;
  float* deconv;
  int S, h, M, W;
  double beta;
};

__global__ void nufft_deconv_kernel(const DeconvP p) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= p.S) return;
  const double xi = static_cast<double>(n - p.h) / p.M;
  const double inv_half = 2.0 / p.W;
  double acc = 0.0;
  for (int q = 0; q < kGlNodes; ++q) {
    const double t = p.gl.x[q] * inv_half;
    const double phi = exp(p.beta * (sqrt(fmax(0.0, 1.0 - t * t)) - 1.0));
    acc += p.gl.w[q] * phi * cospi(2.0 * xi * p.gl.x[q]);
  }
  p.deconv[n] = static_cast<float>(1.0 / (2.0 * acc));
}

// ---------------------------------------------------------------------------
// 2. Fine range grid per antenna: deconvolve, zero-pad to M, radix-2 FFT in
// shared memory (decimation in time, e^{-j 2 pi k l / M}).
template <typename T>
struct GridP {
  const T* real;
  const T* imag;
  const float* deconv;
  float2* g;  // [A][M + kGridPad]: the M grid points, then the first kGridPad again
  int64_t A;
  int S, h, M, log2M;
  int index_weight;  // 1: grid of n * s[a, n] instead of s[a, n]
};

__device__ __forceinline__ unsigned bit_reverse(unsigned x, int bits) {
  return __brev(x) >> (32 - bits);
}

// In-place radix-2 FFT of fbuf[M] (input already in bit-reversed order),
// decimation in time, kernel e^{sign j 2 pi k l / M}.  Called by the whole
// block; ends with a barrier.
__device__ __forceinline__ void fft_radix2(float2* fbuf, int M, float sign) {
  for (int half = 1; half < M; half *= 2) {
    for (int b = threadIdx.x; b < M / 2; b += blockDim.x) {
      const int k = b & (half - 1);
      const int i0 = ((b - k) << 1) + k;
      const int i1 = i0 + half;
      float sn, cs;
      sincospif(sign * static_cast<float>(k) / static_cast<float>(half), &sn, &cs);
      const float2 x0 = fbuf[i0];
      const float2 x1 = fbuf[i1];
      const float2 tw = make_float2(fmaf(cs, x1.x, -sn * x1.y), fmaf(cs, x1.y, sn * x1.x));
      fbuf[i0] = make_float2(x0.x + tw.x, x0.y + tw.y);
      fbuf[i1] = make_float2(x0.x - tw.x, x0.y - tw.y);
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void __launch_bounds__(512) nufft_grid_kernel(const GridP<T> p) {
  extern __shared__ float2 fbuf[];  // [M]
  const int M = p.M;
  for (int64_t a = blockIdx.x; a < p.A; a += gridDim.x) {
    for (int idx = threadIdx.x; idx < M; idx += blockDim.x) {
      const int m = idx < M / 2 ? idx : idx - M;
      const int n = m + p.h;
      float2 v = make_float2(0.0f, 0.0f);
      if (n >= 0 && n < p.S) {
        const float c = p.index_weight ? p.deconv[n] * static_cast<float>(n) : p.deconv[n];
        v = make_float2(ld_f(p.real, a * p.S + n) * c, ld_f(p.imag, a * p.S + n) * c);
      }
      fbuf[bit_reverse(static_cast<unsigned>(idx), p.log2M)] = v;
    }
    __syncthreads();
    fft_radix2(fbuf, M, -1.0f);
    const int Mp = M + kGridPad;
    for (int l = threadIdx.x; l < Mp; l += blockDim.x) p.g[a * Mp + l] = fbuf[l & (M - 1)];
    __syncthreads();
  }
}

// Per (voxel, antenna) NUFFT coordinates: the frequency d reduced to [-1/2, 1/2]
// as u = d M split into floor and fraction, and the combined phase
// c0 + h d reduced to [-1/2, 1/2] cycles (FP64, as the MIXED form).
struct NufftPoint {
  int base;     // first grid point of the W-point stencil (unwrapped)
  float f;      // fractional grid offset in [0, 1)
  float frac;   // c0 + h d in cycles, reduced
};

template <int W>
__device__ __forceinline__ NufftPoint nufft_point(double tx, double ty, double tz, double rx, double ry,
                                                  double rz, double x, double y, double z, double k0,
                                                  double b0, double k1, double b1, int h, float fM) {
  const double st = fma(tz - z, tz - z, fma(ty - y, ty - y, (tx - x) * (tx - x)));
  const double sr = fma(rz - z, rz - z, fma(ry - y, ry - y, (rx - x) * (rx - x)));
  const double dist = sqrt_f64_fast(st) + sqrt_f64_fast(sr);
  const double dc = fma(dist, k1, b1);
  const float df = static_cast<float>(dc - rint(dc));
  const double c = fma(dist, k0, b0) + static_cast<double>(h) * static_cast<double>(df);
  NufftPoint q;
  q.frac = static_cast<float>(c - rint(c));
  const float u = df * fM;  // exact: M is a power of two
  const float fl = floorf(u);
  q.f = u - fl;
  q.base = static_cast<int>(fl) - W / 2 + 1;
  return q;
}

// ---------------------------------------------------------------------------
// Double-buffered TMA ring of grid rows (one float2 array): thread 0 issues one
// cp.async.bulk per stage; completion on the stage's mbarrier, waits bounded.
struct RowStager {
  float2* buf;    // [2 stages][rows_max * row]
  uint64_t* bar;  // [2]
  int row;        // float2 per row (multiple of 2: 16-byte rows)
  int rows_max;

  __device__ __forceinline__ float2* stage_ptr(int stage) const {
    return buf + static_cast<int64_t>(stage) * rows_max * row;
  }
  __device__ __forceinline__ void issue(int stage, const float2* src, int64_t row0, int rows) {
    if (threadIdx.x == 0) {
      const uint32_t bytes = static_cast<uint32_t>(rows) * row * sizeof(float2);
      mbar_arrive_expect_tx(&bar[stage], bytes);
      bulk_g2s(stage_ptr(stage), src + row0 * row, bytes, &bar[stage]);
    }
  }
  __device__ __forceinline__ bool wait(int stage, uint32_t parity, int* status) {
    const bool ok = mbar_wait_bounded(&bar[stage], parity, status);
    return __syncthreads_and(ok) != 0;
  }
  __device__ __forceinline__ void drain(int stage, uint32_t parity, int* status) {
    if (threadIdx.x == 0) mbar_wait_bounded(&bar[stage], parity, status);
  }
};

cudaError_t launch_deconv(float* deconv, int64_t S, int h, int M, int W, double beta, cudaStream_t st) {
  DeconvP dp;
  dp.gl = gauss_legendre(0.5 * W);
  dp.deconv = deconv;
  dp.S = static_cast<int>(S);
  dp.h = h;
  dp.M = M;
  dp.W = W;
  dp.beta = beta;
  nufft_deconv_kernel<<<static_cast<unsigned>((S + 127) / 128), 128, 0, st>>>(dp);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Band bound and private-window spreading parameters (see nufft_kernels.cu).
constexpr int kWin = 48;
constexpr int kSpreadThreads = 128;
constexpr int kWinLd = kSpreadThreads + 1;  // padded column stride: conflict-free sums
constexpr int kVoxelsPerThread = 4096;      // per block and antenna: bounds FP32 sums
constexpr int kStatusInternal = 6;          // GERAF_ERR_DEVICE_CHECK

template <typename T>
struct BboxP {
  const T* voxel;  // element (v, c) at v * pstride + c * cstride: [3, N] or [N, 3]
  int64_t N, pstride, cstride;
  float* partial;  // [blocks][6]
  float* bbox;     // [6]: lo xyz, hi xyz
};

template <typename T>
__global__ void __launch_bounds__(256) voxel_bbox_partial_kernel(const BboxP<T> p) {
  __shared__ float red[6][256];
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < p.N;
       v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float x = ld_f(p.voxel, v * p.pstride + c * p.cstride);
      lo[c] = fminf(lo[c], x);
      hi[c] = fmaxf(hi[c], x);
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    red[c][threadIdx.x] = lo[c];
    red[3 + c][threadIdx.x] = hi[c];
  }
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        red[c][threadIdx.x] = fminf(red[c][threadIdx.x], red[c][threadIdx.x + w]);
        red[3 + c][threadIdx.x] = fmaxf(red[3 + c][threadIdx.x], red[3 + c][threadIdx.x + w]);
      }
    }
    __syncthreads();
  }
  if (threadIdx.x < 6) p.partial[blockIdx.x * 6 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void voxel_bbox_final_kernel(const float* partial, int blocks, float* bbox) {
  const int c = threadIdx.x;
  if (c >= 6) return;
  float r = c < 3 ? INFINITY : -INFINITY;
  for (int b = 0; b < blocks; ++b) r = c < 3 ? fminf(r, partial[b * 6 + c]) : fmaxf(r, partial[b * 6 + c]);
  bbox[c] = r;
}

// Range of path lengths |t - x| + |r - x| over x in the box [lo, hi].
__device__ __forceinline__ void path_range(const double* t, const double* r, const float* box, double& dlo,
                                           double& dhi) {
  double nt = 0.0, nr = 0.0, ft = 0.0, fr = 0.0;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double lo = box[c], hi = box[3 + c];
    const double et = fmax(fmax(lo - t[c], 0.0), t[c] - hi);
    const double er = fmax(fmax(lo - r[c], 0.0), r[c] - hi);
    nt += et * et;
    nr += er * er;
    const double gt = fmax(fabs(t[c] - lo), fabs(t[c] - hi));
    const double gr = fmax(fabs(r[c] - lo), fabs(r[c] - hi));
    ft += gt * gt;
    fr += gr * gr;
  }
  dlo = sqrt(nt) + sqrt(nr);
  dhi = sqrt(ft) + sqrt(fr);
}

template <typename T>
struct AdjFftP {
  const float2* grid;  // [vsplits][A][M]
  const float* deconv;
  T* out_r;  // [A][S]
  T* out_i;
  int64_t A;
  int S, h, M, log2M, vsplits;
  float scale;  // 1/A (matched-filter adjoint) or 1/P (tracer forward)
};

template <typename T>
__global__ void __launch_bounds__(512) nufft_adjoint_fft_kernel(const AdjFftP<T> p) {
  extern __shared__ float2 fbuf[];  // [M]
  const int M = p.M;
  for (int64_t a = blockIdx.x; a < p.A; a += gridDim.x) {
    for (int l = threadIdx.x; l < M; l += blockDim.x) {
      float2 acc = make_float2(0.0f, 0.0f);
      for (int vs = 0; vs < p.vsplits; ++vs) {
        const float2 v = p.grid[(static_cast<int64_t>(vs) * p.A + a) * M + l];
        acc.x += v.x;
        acc.y += v.y;
      }
      fbuf[bit_reverse(static_cast<unsigned>(l), p.log2M)] = acc;
    }
    __syncthreads();
    fft_radix2(fbuf, M, 1.0f);
    for (int n = threadIdx.x; n < p.S; n += blockDim.x) {
      const int idx = (n - p.h) & (M - 1);
      const float c = p.deconv[n] * p.scale;
      const float2 v = fbuf[idx];
      p.out_r[a * p.S + n] = from_f<T>(v.x * c);
      p.out_i[a * p.S + n] = from_f<T>(v.y * c);
    }
    __syncthreads();
  }
}

constexpr int kBboxBlocks = 256;


}  // namespace
}  // namespace geraf
