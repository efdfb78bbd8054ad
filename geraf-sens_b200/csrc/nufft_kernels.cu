// Fast approximate matched filter (MODE_NUFFT): the per-antenna sample sum of
// the MIXED form evaluated through an oversampled range FFT and a short
// interpolation kernel instead of S Horner steps.
//
// With the MIXED phase model (common.cuh, path_cycles) the forward is
//   y_v = (1/A) sum_a e^{-j 2 pi c0(v,a)} P_a(d(v,a)),   P_a(d) = sum_n s[a,n] e^{-j 2 pi n d},
// where c0 is the carrier phase in cycles and d the per-sample phase step in
// cycles.  P_a is a trigonometric polynomial of degree S, so it is evaluated
// at the N non-uniform frequencies d(v, a) by a type-2 non-uniform FFT
// (Dutt & Rokhlin 1993; kernel and parameters of Barnett, Magland & af Klinteberg,
// "A parallel non-uniform fast Fourier transform library based on an
// 'exponential of semicircle' kernel", SIAM J. Sci. Comput. 41(5), 2019):
//   1. centre the modes, m = n - h with h = S / 2:  P_a(d) = e^{-j 2 pi h d} Q_a(d);
//   2. deconvolve, c^_m = s[a, m + h] / Phi(m / M), with Phi the Fourier
//      transform of the kernel phi(u) = exp(beta (sqrt(1 - (2u/W)^2) - 1)),
//      |u| < W/2, beta = 2.30 W (FP64 Gauss-Legendre quadrature);
//   3. an M-point FFT per antenna (M = the power of two >= 2S) gives the
//      fine range grid g[a, l] = sum_m c^_m e^{-j 2 pi m l / M};
//   4. per (voxel, antenna): Q(d) = sum over the W grid points l nearest to
//      u = d M of g[a, l] phi(u - l), then y += e^{-j 2 pi (c0 + h d)} Q(d),
//      compensated across antennas.
// The truncation error falls like 10^{-(W-1)} (W = 8: ~1e-7 relative), below
// the FP32 rounding of the grid and the weights (~1e-6).  The phase model,
// the FP64 reduction and the geometry are those of the MIXED form; only the
// sample sum changes.  Work per (voxel, antenna) is O(W) instead of O(S).
//
// The reference has no such path: its range-bin kernels
// (MatchedFilter_cuda_kernel.cu:117-169) gather one precomputed bin with no
// interpolation.  This is an addition of this library.
#include <algorithm>
#include <cmath>
#include <vector>

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

struct NufftShape {
  int M = 0;      // fine grid points per antenna (power of two)
  int Mp = 0;     // grid row length in shared / global memory: M + kGridPad
  int log2M = 0;
  int h = 0;      // mode centre, S / 2
  int W = 0;      // kernel width in grid points
  double beta = 0.0;
  int threads = 128, vpt = 4, rows = 8, splits = 1;
  int64_t ant_per_split = 0;
  size_t deconv_off = 0, grid_off = 0, partial_off = 0, total = 0;
  size_t smem = 0, pos_off = 0, buf_off = 0;
};

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

int grid_points(int64_t S) {
  int M = 16;
  while (M < 2 * S) M *= 2;
  return M;
}

// Shared memory of the gather kernel: 2 mbarriers | positions [2][rows][6]
// double | grid ring [2 stages][rows][M + pad] float2.
size_t gather_buf_off(int rows) { return align256(128 + 2 * static_cast<size_t>(rows) * 6 * sizeof(double)); }
size_t gather_smem(int rows, int M) {
  return gather_buf_off(rows) + 2 * static_cast<size_t>(rows) * (M + kGridPad) * sizeof(float2);
}

NufftShape nufft_shape(const MfArgs& a, const Tuning& t) {
  NufftShape s;
  s.M = grid_points(a.S);
  s.Mp = s.M + kGridPad;
  s.log2M = 0;
  while ((1 << s.log2M) < s.M) ++s.log2M;
  s.h = static_cast<int>(a.S / 2);
  s.W = t.taps;
  s.beta = 2.30 * s.W;
  s.threads = t.threads;
  s.vpt = t.items;
  s.rows = t.stage_rows;
  s.splits = t.splits;
  const int64_t rows_total = (a.A + s.rows - 1) / s.rows;
  const int64_t rows_per_split = (rows_total + s.splits - 1) / s.splits;
  s.ant_per_split = std::max<int64_t>(1, rows_per_split) * s.rows;
  // workspace: deconvolution factors [S] | grid [A][M + pad] float2 | partials [splits][N]
  s.deconv_off = 0;
  s.grid_off = align256(static_cast<size_t>(std::max<int64_t>(a.S, 1)) * sizeof(float));
  s.partial_off = s.grid_off + align256(static_cast<size_t>(a.A) * s.Mp * sizeof(float2));
  s.total = s.partial_off +
            (s.splits > 1 ? align256(static_cast<size_t>(s.splits) * a.N * sizeof(float2)) : 0);
  s.pos_off = 128;
  s.buf_off = gather_buf_off(s.rows);
  s.smem = gather_smem(s.rows, s.M);
  return s;
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
        const float c = p.deconv[n];
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

// ---------------------------------------------------------------------------
// 4. Gather: VPT voxels per thread, antenna rows of the fine grid staged by
// TMA into a double-buffered ring (as the MIXED forward stages IF samples).
// Each row carries a periodic extension, so a stencil starting at any grid
// point reads W consecutive entries without wrapping.
template <typename T>
struct GatherP {
  EsPoly poly;
  const float2* g;  // [A][M + kGridPad]
  const T* tx;
  const T* rx;
  const T* voxel;
  T* out_r;
  T* out_i;
  float2* partial;
  int* status;
  int64_t A, N, ant_per_split;
  int M, h, rows, splits;
  double k0, b0, k1, b1;
  size_t pos_off, buf_off;
};

template <typename T, int VPT, int W>
__global__ void __launch_bounds__(256) nufft_gather_kernel(const GatherP<T> p) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  double* pos = reinterpret_cast<double*>(smem + p.pos_off);
  const int Mp = p.M + kGridPad;
  RowStager stg{reinterpret_cast<float2*>(smem + p.buf_off), bar, Mp, p.rows};

  const int split = blockIdx.x % p.splits;
  const int64_t vtile = blockIdx.x / p.splits;
  const int64_t a_begin = static_cast<int64_t>(split) * p.ant_per_split;
  const int64_t a_end = min(p.A, a_begin + p.ant_per_split);
  const int ntiles = a_end > a_begin ? ceil_div(a_end - a_begin, p.rows) : 0;
  const int mask = p.M - 1;
  const float fM = static_cast<float>(p.M);

  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();

  double vx[VPT], vy[VPT], vz[VPT];
  int64_t vid[VPT];
#pragma unroll
  for (int j = 0; j < VPT; ++j) {
    vid[j] = vtile * blockDim.x * VPT + threadIdx.x + static_cast<int64_t>(j) * blockDim.x;
    const bool ok = vid[j] < p.N;
    vx[j] = ok ? static_cast<double>(ld_f(p.voxel, vid[j])) : 0.0;
    vy[j] = ok ? static_cast<double>(ld_f(p.voxel, p.N + vid[j])) : 0.0;
    vz[j] = ok ? static_cast<double>(ld_f(p.voxel, 2 * p.N + vid[j])) : 0.0;
  }
  float yr[VPT], yi[VPT], cr[VPT], ci[VPT];
#pragma unroll
  for (int j = 0; j < VPT; ++j) yr[j] = yi[j] = cr[j] = ci[j] = 0.0f;

  auto issue = [&](int tile, int stage) {
    const int64_t a0 = a_begin + static_cast<int64_t>(tile) * p.rows;
    const int rws = static_cast<int>(min(static_cast<int64_t>(p.rows), a_end - a0));
    stg.issue(stage, p.g, a0, rws);
    stage_positions<T, double>(pos, stage, p.rows, p.tx, p.rx, a0, rws);
  };
  if (ntiles > 0) issue(0, 0);
  if (ntiles > 1) issue(1, 1);

  for (int t = 0; t < ntiles; ++t) {
    const int s = t & 1;
    if (!stg.wait(s, (t >> 1) & 1, p.status)) {
      if (t + 1 < ntiles) stg.drain(s ^ 1, ((t + 1) >> 1) & 1, p.status);
      return;
    }
    const int64_t a0 = a_begin + static_cast<int64_t>(t) * p.rows;
    const int rws = static_cast<int>(min(static_cast<int64_t>(p.rows), a_end - a0));
    for (int r = 0; r < rws; ++r) {
      const double* ps = pos + (s * p.rows + r) * 6;
      const double tx = ps[0], ty = ps[1], tz = ps[2], rx = ps[3], ry = ps[4], rz = ps[5];
      const float2* row = stg.stage_ptr(s) + r * Mp;
#pragma unroll
      for (int j = 0; j < VPT; ++j) {
        const NufftPoint q = nufft_point<W>(tx, ty, tz, rx, ry, rz, vx[j], vy[j], vz[j], p.k0, p.b0,
                                            p.k1, p.b1, p.h, fM);
        const TapWeights<W> wt = tap_weights<W>(p.poly, q.f);
        const float2* gp = row + (q.base & mask);
        float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int k = 0; k < W; ++k) acc = ffma2(make_float2(wt.w[k], wt.w[k]), gp[k], acc);
        const float2 e = cis_cycles(q.frac);  // e^{+j 2 pi frac}; the forward uses its conjugate
        const float tr = fmaf(e.x, acc.x, e.y * acc.y);
        const float ti = fmaf(e.x, acc.y, -e.y * acc.x);
        kahan_add(yr[j], cr[j], tr);
        kahan_add(yi[j], ci[j], ti);
      }
    }
    __syncthreads();
    if (t + 2 < ntiles) issue(t + 2, s);
  }

#pragma unroll
  for (int j = 0; j < VPT; ++j) {
    if (vid[j] >= p.N) continue;
    if (p.splits == 1) {
      p.out_r[vid[j]] = from_f<T>(yr[j] / static_cast<float>(p.A));
      p.out_i[vid[j]] = from_f<T>(yi[j] / static_cast<float>(p.A));
    } else {
      p.partial[split * p.N + vid[j]] = make_float2(yr[j], yi[j]);
    }
  }
}

template <typename T, int VPT>
const void* gather_ptr(int W) {
  switch (W) {
    case 4: return reinterpret_cast<const void*>(&nufft_gather_kernel<T, VPT, 4>);
    case 6: return reinterpret_cast<const void*>(&nufft_gather_kernel<T, VPT, 6>);
    case 10: return reinterpret_cast<const void*>(&nufft_gather_kernel<T, VPT, 10>);
    case 12: return reinterpret_cast<const void*>(&nufft_gather_kernel<T, VPT, 12>);
    default: return reinterpret_cast<const void*>(&nufft_gather_kernel<T, VPT, 8>);
  }
}

template <typename T>
const void* gather_kernel_ptr(int vpt, int W) {
  if (vpt == 1) return gather_ptr<T, 1>(W);
  if (vpt == 2) return gather_ptr<T, 2>(W);
  return gather_ptr<T, 4>(W);
}

cudaError_t launch_deconv(float* deconv, int64_t S, const NufftShape& s, cudaStream_t st) {
  DeconvP dp;
  dp.gl = gauss_legendre(0.5 * s.W);
  dp.deconv = deconv;
  dp.S = static_cast<int>(S);
  dp.h = s.h;
  dp.M = s.M;
  dp.W = s.W;
  dp.beta = s.beta;
  nufft_deconv_kernel<<<static_cast<unsigned>((S + 127) / 128), 128, 0, st>>>(dp);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Adjoint (type-1 NUFFT), the exact transpose of the forward above:
//   H[a, n] = (1/A) sum_v G_v e^{+j 2 pi (c0 + n d)},  G = grad_real + j grad_imag,
// which gives grad_real = Re H, grad_imag = Im H (the reference's adjoint,
// MatchedFilter_cuda_kernel.cu:171-220, for the MIXED phase model).
//   1. spread: f[a, l] = sum_v G_v e^{+j 2 pi (c0 + h d)} phi(u - l) on the fine grid;
//   2. per antenna an M-point FFT with kernel e^{+j 2 pi m l / M}, then
//      H[a, m + h] = F(m) / Phi(m / M) / A.
// Spreading.  Per antenna, all voxels fall in a narrow band of grid points
// (their path lengths lie between the nearest and farthest point of the voxel
// set's bounding box).  When that band, with the stencil and one point of
// margin each side, fits kWin grid points, every thread accumulates its voxels
// into a private column of a [kWin x threads] shared window with plain
// read-modify-writes, and the columns are summed in a fixed order at the end:
// no atomics, bit-reproducible results.  Otherwise (bands wider than kWin, or
// a band that crosses the +-1/2-cycle wrap) the block accumulates into one
// shared row with FP32 atomics, whose summation order varies from run to run.
constexpr int kWin = 48;
constexpr int kSpreadThreads = 128;
constexpr int kWinLd = kSpreadThreads + 1;  // padded column stride: conflict-free sums
constexpr int kVoxelsPerThread = 4096;      // per block and antenna: bounds FP32 sums
constexpr int kStatusInternal = 6;          // GERAF_ERR_DEVICE_CHECK

template <typename T>
struct BboxP {
  const T* voxel;  // [3, N]
  int64_t N;
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
      const float x = ld_f(p.voxel, c * p.N + v);
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
struct SpreadP {
  EsPoly poly;
  const T* tx;
  const T* rx;
  const T* voxel;
  const T* gr;
  const T* gi;
  const float* bbox;  // [6]
  float2* grid;       // [vsplits][A][M]
  int* status;
  int64_t A, N, vox_per_split;
  int M, h, vsplits;
  double k0, b0, k1, b1;
};

template <typename T, int W>
__global__ void __launch_bounds__(kSpreadThreads) nufft_spread_kernel(const SpreadP<T> p) {
  extern __shared__ __align__(128) unsigned char smem[];
  float* buf = reinterpret_cast<float*>(smem);  // window [2][kWin][kWinLd] or row [2][M]
  __shared__ double pos[6];
  __shared__ int s_mode, s_w0;
  __shared__ float sums[2 * kWin];
  const int vs = blockIdx.x % p.vsplits;
  const int64_t a = blockIdx.x / p.vsplits;
  const int mask = p.M - 1;
  const float fM = static_cast<float>(p.M);
  if (threadIdx.x < 6) {
    const T* src = threadIdx.x < 3 ? p.tx : p.rx;
    pos[threadIdx.x] = static_cast<double>(ld_f(src, a * 3 + (threadIdx.x % 3)));
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double dlo, dhi;
    path_range(pos, pos + 3, p.bbox, dlo, dhi);
    double c_lo = fma(dlo, p.k1, p.b1), c_hi = fma(dhi, p.k1, p.b1);
    if (c_lo > c_hi) {
      const double tmp = c_lo;
      c_lo = c_hi;
      c_hi = tmp;
    }
    const double r0 = rint(c_lo);
    int mode = 0;  // 0: shared row with atomics, 1: private windows
    int w0 = 0;
    if (rint(c_hi) == r0 && c_lo - r0 > -0.5 + 1e-6 && c_hi - r0 < 0.5 - 1e-6) {
      const int b_lo = static_cast<int>(floor((c_lo - r0) * p.M)) - W / 2;      // one point of margin
      const int b_hi = static_cast<int>(floor((c_hi - r0) * p.M)) - W / 2 + 2;  // one point of margin
      if (b_hi + W - b_lo <= kWin) {
        mode = 1;
        w0 = b_lo;
      }
    }
    s_mode = mode;
    s_w0 = w0;
  }
  __syncthreads();
  const int mode = s_mode;
  const int w0 = s_w0;
  const int cells = mode ? 2 * kWin * kWinLd : 2 * p.M;
  for (int i = threadIdx.x; i < cells; i += blockDim.x) buf[i] = 0.0f;
  __syncthreads();

  const int64_t v_begin = static_cast<int64_t>(vs) * p.vox_per_split;
  const int64_t v_end = min(p.N, v_begin + p.vox_per_split);
  float* col_re = buf + threadIdx.x;             // window column of this thread
  float* col_im = buf + kWin * kWinLd + threadIdx.x;
  for (int64_t v = v_begin + threadIdx.x; v < v_end; v += blockDim.x) {
    const double x = static_cast<double>(ld_f(p.voxel, v));
    const double y = static_cast<double>(ld_f(p.voxel, p.N + v));
    const double z = static_cast<double>(ld_f(p.voxel, 2 * p.N + v));
    const float g_r = ld_f(p.gr, v);
    const float g_i = ld_f(p.gi, v);
    const NufftPoint q = nufft_point<W>(pos[0], pos[1], pos[2], pos[3], pos[4], pos[5], x, y, z, p.k0,
                                        p.b0, p.k1, p.b1, p.h, fM);
    const float2 e = cis_cycles(q.frac);
    const float wr = fmaf(g_r, e.x, -g_i * e.y);
    const float wi = fmaf(g_r, e.y, g_i * e.x);
    const TapWeights<W> wt = tap_weights<W>(p.poly, q.f);
    if (mode) {
      const int o = q.base - w0;
      if (static_cast<unsigned>(o) > static_cast<unsigned>(kWin - W)) {
        // outside the band bound from the bounding box: cannot happen for finite inputs
        if (p.status != nullptr) atomicExch(p.status, kStatusInternal);
        continue;
      }
#pragma unroll
      for (int k = 0; k < W; ++k) {
        col_re[(o + k) * kWinLd] += wt.w[k] * wr;
        col_im[(o + k) * kWinLd] += wt.w[k] * wi;
      }
    } else {
#pragma unroll
      for (int k = 0; k < W; ++k) {
        const int l = (q.base + k) & mask;
        atomicAdd(buf + l, wt.w[k] * wr);
        atomicAdd(buf + p.M + l, wt.w[k] * wi);
      }
    }
  }
  __syncthreads();
  float2* out = p.grid + (static_cast<int64_t>(vs) * p.A + a) * p.M;
  if (mode) {
    if (threadIdx.x < 2 * kWin) {
      const float* rowp = buf + threadIdx.x * kWinLd;
      float acc = 0.0f;
      for (int t = 0; t < kSpreadThreads; ++t) acc += rowp[t];
      sums[threadIdx.x] = acc;
    }
    __syncthreads();
    for (int l = threadIdx.x; l < p.M; l += blockDim.x) {
      // window points j and j + M are the same grid point when M < kWin
      float2 v = make_float2(0.0f, 0.0f);
      for (int j = (l - w0) & mask; j < kWin; j += p.M) {
        v.x += sums[j];
        v.y += sums[kWin + j];
      }
      out[l] = v;
    }
  } else {
    for (int l = threadIdx.x; l < p.M; l += blockDim.x) out[l] = make_float2(buf[l], buf[p.M + l]);
  }
}

template <typename T>
struct AdjFftP {
  const float2* grid;  // [vsplits][A][M]
  const float* deconv;
  T* out_r;  // [A][S]
  T* out_i;
  int64_t A;
  int S, h, M, log2M, vsplits;
  float inv_A;
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
      const float c = p.deconv[n] * p.inv_A;
      const float2 v = fbuf[idx];
      p.out_r[a * p.S + n] = from_f<T>(v.x * c);
      p.out_i[a * p.S + n] = from_f<T>(v.y * c);
    }
    __syncthreads();
  }
}

template <typename T>
const void* spread_kernel_ptr(int W) {
  switch (W) {
    case 4: return reinterpret_cast<const void*>(&nufft_spread_kernel<T, 4>);
    case 6: return reinterpret_cast<const void*>(&nufft_spread_kernel<T, 6>);
    case 10: return reinterpret_cast<const void*>(&nufft_spread_kernel<T, 10>);
    case 12: return reinterpret_cast<const void*>(&nufft_spread_kernel<T, 12>);
    default: return reinterpret_cast<const void*>(&nufft_spread_kernel<T, 8>);
  }
}

// Dynamic shared memory of the spread kernel: the private windows or the
// fallback row, whichever is larger.
size_t spread_smem(int M) {
  return std::max(2 * static_cast<size_t>(kWin) * kWinLd, 2 * static_cast<size_t>(M)) * sizeof(float);
}
constexpr int kBboxBlocks = 256;

struct AdjShape {
  NufftShape base;
  int vsplits = 1;
  int64_t vox_per_split = 0;
  size_t deconv_off = 0, bbox_off = 0, grid_off = 0, total = 0;
};

AdjShape adj_shape(const MfArgs& a, const Tuning& t) {
  AdjShape s;
  s.base = nufft_shape(a, t);
  s.vsplits = t.splits;
  s.vox_per_split = std::max<int64_t>(1, (a.N + s.vsplits - 1) / s.vsplits);
  // workspace: deconvolution [S] | bbox partials [kBboxBlocks][6] + bbox [6] | grids [vsplits][A][M]
  s.deconv_off = 0;
  s.bbox_off = align256(static_cast<size_t>(std::max<int64_t>(a.S, 1)) * sizeof(float));
  s.grid_off = s.bbox_off + align256((kBboxBlocks + 1) * 6 * sizeof(float));
  s.total = s.grid_off + align256(static_cast<size_t>(s.vsplits) * a.A * s.base.M * sizeof(float2));
  return s;
}

template <typename T>
cudaError_t launch_nufft_backward(const MfArgs& a, const Tuning& t, void* ws, cudaStream_t st) {
  const AdjShape s = adj_shape(a, t);
  const NufftShape& b = s.base;
  unsigned char* base = static_cast<unsigned char*>(ws);
  float* deconv = reinterpret_cast<float*>(base + s.deconv_off);
  float2* grid = reinterpret_cast<float2*>(base + s.grid_off);
  const DeviceInfo dev = current_device_info();
  cudaError_t err = launch_deconv(deconv, a.S, b, st);
  if (err != cudaSuccess) return err;

  float* bbox_partial = reinterpret_cast<float*>(base + s.bbox_off);
  float* bbox = bbox_partial + kBboxBlocks * 6;
  if (a.N > 0) {
    BboxP<T> bp;
    bp.voxel = static_cast<const T*>(a.voxel);
    bp.N = a.N;
    bp.partial = bbox_partial;
    bp.bbox = bbox;
    const int nb = static_cast<int>(std::min<int64_t>(kBboxBlocks, (a.N + 255) / 256));
    voxel_bbox_partial_kernel<T><<<nb, 256, 0, st>>>(bp);
    voxel_bbox_final_kernel<<<1, 32, 0, st>>>(bbox_partial, nb, bbox);
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
  }

  SpreadP<T> sp;
  sp.poly = es_poly(b.W, b.beta);
  sp.tx = static_cast<const T*>(a.tx);
  sp.rx = static_cast<const T*>(a.rx);
  sp.voxel = static_cast<const T*>(a.voxel);
  sp.gr = static_cast<const T*>(a.grad_real_out);
  sp.gi = static_cast<const T*>(a.grad_imag_out);
  sp.bbox = bbox;
  sp.grid = grid;
  sp.status = device_status_ptr();
  sp.A = a.A;
  sp.N = a.N;
  sp.vox_per_split = s.vox_per_split;
  sp.M = b.M;
  sp.h = b.h;
  sp.vsplits = s.vsplits;
  const PhaseConsts pc = phase_consts(kMfStartFrequency, a.As, a.fs);
  sp.k0 = pc.k0;
  sp.b0 = pc.b0;
  sp.k1 = pc.k1;
  sp.b1 = pc.b1;
  const size_t ssmem = spread_smem(b.M);
  const void* fn = spread_kernel_ptr<T>(b.W);
  err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(ssmem));
  if (err != cudaSuccess) return err;
  const int64_t blocks = a.A * s.vsplits;
  if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
  void* args[] = {&sp};
  err = cudaLaunchKernel(fn, dim3(static_cast<unsigned>(blocks)), dim3(kSpreadThreads), args, ssmem, st);
  if (err != cudaSuccess) return err;

  AdjFftP<T> fp;
  fp.grid = grid;
  fp.deconv = deconv;
  fp.out_r = static_cast<T*>(a.out_real);
  fp.out_i = static_cast<T*>(a.out_imag);
  fp.A = a.A;
  fp.S = static_cast<int>(a.S);
  fp.h = b.h;
  fp.M = b.M;
  fp.log2M = b.log2M;
  fp.vsplits = s.vsplits;
  fp.inv_A = 1.0f / static_cast<float>(a.A);
  const size_t fsmem = static_cast<size_t>(b.M) * sizeof(float2);
  err = cudaFuncSetAttribute(&nufft_adjoint_fft_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(fsmem));
  if (err != cudaSuccess) return err;
  const int fthreads = std::min(512, std::max(32, b.M / 2));
  const int64_t fblocks = std::min<int64_t>(a.A, static_cast<int64_t>(dev.sm_count) * 16);
  nufft_adjoint_fft_kernel<T><<<static_cast<unsigned>(fblocks), fthreads, fsmem, st>>>(fp);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_nufft_forward(const MfArgs& a, const NufftShape& s, void* ws, cudaStream_t st) {
  unsigned char* base = static_cast<unsigned char*>(ws);
  float* deconv = reinterpret_cast<float*>(base + s.deconv_off);
  float2* grid = reinterpret_cast<float2*>(base + s.grid_off);
  const DeviceInfo dev = current_device_info();

  if (a.S > 0) {
    cudaError_t err = launch_deconv(deconv, a.S, s, st);
    if (err != cudaSuccess) return err;

    GridP<T> gp;
    gp.real = static_cast<const T*>(a.real);
    gp.imag = static_cast<const T*>(a.imag);
    gp.deconv = deconv;
    gp.g = grid;
    gp.A = a.A;
    gp.S = static_cast<int>(a.S);
    gp.h = s.h;
    gp.M = s.M;
    gp.log2M = s.log2M;
    const size_t fsmem = static_cast<size_t>(s.M) * sizeof(float2);
    err = cudaFuncSetAttribute(&nufft_grid_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(fsmem));
    if (err != cudaSuccess) return err;
    const int fthreads = std::min(512, std::max(32, s.M / 2));
    const int64_t fblocks = std::min<int64_t>(a.A, static_cast<int64_t>(dev.sm_count) * 16);
    if (fblocks > 0) {
      nufft_grid_kernel<T><<<static_cast<unsigned>(fblocks), fthreads, fsmem, st>>>(gp);
      err = cudaGetLastError();
      if (err != cudaSuccess) return err;
    }
  } else if (a.A > 0) {
    // No samples: every grid point is zero.
    cudaError_t err = cudaMemsetAsync(grid, 0, static_cast<size_t>(a.A) * s.Mp * sizeof(float2), st);
    if (err != cudaSuccess) return err;
  }

  GatherP<T> p;
  p.poly = es_poly(s.W, s.beta);
  p.g = grid;
  p.tx = static_cast<const T*>(a.tx);
  p.rx = static_cast<const T*>(a.rx);
  p.voxel = static_cast<const T*>(a.voxel);
  p.out_r = static_cast<T*>(a.out_real);
  p.out_i = static_cast<T*>(a.out_imag);
  p.partial = reinterpret_cast<float2*>(base + s.partial_off);
  p.status = device_status_ptr();
  p.A = a.A;
  p.N = a.N;
  p.ant_per_split = s.ant_per_split;
  p.M = s.M;
  p.h = s.h;
  p.rows = s.rows;
  p.splits = s.splits;
  const PhaseConsts pc = phase_consts(kMfStartFrequency, a.As, a.fs);
  p.k0 = pc.k0;
  p.b0 = pc.b0;
  p.k1 = pc.k1;
  p.b1 = pc.b1;
  p.pos_off = s.pos_off;
  p.buf_off = s.buf_off;

  const void* fn = gather_kernel_ptr<T>(s.vpt, s.W);
  cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(s.smem));
  if (err != cudaSuccess) return err;
  const int64_t vtiles = (a.N + static_cast<int64_t>(s.threads) * s.vpt - 1) /
                         (static_cast<int64_t>(s.threads) * s.vpt);
  const int64_t blocks = vtiles * s.splits;
  if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
  void* args[] = {&p};
  err = cudaLaunchKernel(fn, dim3(static_cast<unsigned>(blocks)), dim3(s.threads), args, s.smem, st);
  if (err != cudaSuccess) return err;
  if (s.splits > 1) {
    err = launch_finalize_partials(a.dtype, p.partial, s.splits, a.N, static_cast<float>(a.A),
                                   a.out_real, a.out_imag, st);
  }
  return err;
}

}  // namespace

// ---------------------------------------------------------------------------
Tuning mf_nufft_forward_resolve(const MfArgs& a, const Tuning& req) {
  Tuning t = req;
  if (t.threads != 64 && t.threads != 128 && t.threads != 256) t.threads = 128;
  if (t.items != 1 && t.items != 2 && t.items != 4) t.items = 4;
  if (t.taps != 4 && t.taps != 6 && t.taps != 8 && t.taps != 10 && t.taps != 12) t.taps = 8;
  if (t.stage_rows <= 0) t.stage_rows = 4;
  t.stage_rows = std::min(t.stage_rows, 64);
  const int M = grid_points(a.S);
  const DeviceInfo dev = current_device_info();
  // keep the double-buffered grid ring within the opt-in shared memory
  while (t.stage_rows > 1 && gather_smem(t.stage_rows, M) > static_cast<size_t>(dev.max_smem_optin)) {
    t.stage_rows /= 2;
  }
  const int64_t rows_total = std::max<int64_t>(1, (a.A + t.stage_rows - 1) / t.stage_rows);
  if (t.splits <= 0) {
    const int64_t vtiles = (a.N + static_cast<int64_t>(t.threads) * t.items - 1) /
                           (static_cast<int64_t>(t.threads) * t.items);
    const int per_sm = std::max(1, 1024 / t.threads);
    t.splits = pick_splits(vtiles, per_sm, dev.sm_count, rows_total);
  }
  t.splits = static_cast<int>(std::min<int64_t>(std::max(t.splits, 1), rows_total));
  return t;
}

bool mf_nufft_supported(int64_t S) { return S <= kNufftMaxSamples; }

Tuning mf_nufft_backward_resolve(const MfArgs& a, const Tuning& req) {
  Tuning t = req;
  // one block of kSpreadThreads per (antenna, voxel split)
  t.threads = kSpreadThreads;
  if (t.taps != 4 && t.taps != 6 && t.taps != 8 && t.taps != 10 && t.taps != 12) t.taps = 8;
  t.items = 1;
  t.stage_rows = 1;
  // voxel splits: at most kVoxelsPerThread voxels per thread and block, and
  // enough (antenna, split) blocks to fill the GPU
  const int64_t min_vs = std::max<int64_t>(
      1, (a.N + int64_t{kSpreadThreads} * kVoxelsPerThread - 1) / (int64_t{kSpreadThreads} * kVoxelsPerThread));
  const int64_t max_vs = std::max<int64_t>(min_vs, a.N / (4 * kSpreadThreads));
  if (t.splits <= 0) {
    const DeviceInfo dev = current_device_info();
    t.splits = std::max<int>(static_cast<int>(min_vs), pick_splits(std::max<int64_t>(1, a.A), 4, dev.sm_count, max_vs));
  }
  t.splits = static_cast<int>(std::min<int64_t>(std::max(t.splits, 1), std::max<int64_t>(1, a.N)));
  return t;
}

size_t mf_nufft_backward_workspace(const MfArgs& a, const Tuning& t) {
  if (a.A == 0 || a.S == 0) return 0;
  return adj_shape(a, t).total;
}

cudaError_t mf_nufft_backward(const MfArgs& a, const Tuning& t, void* ws, cudaStream_t st) {
  if (a.A == 0 || a.S == 0) return cudaSuccess;
  switch (a.dtype) {
    case kF64: return launch_nufft_backward<double>(a, t, ws, st);
    case kF16: return launch_nufft_backward<__half>(a, t, ws, st);
    default: return launch_nufft_backward<float>(a, t, ws, st);
  }
}

size_t mf_nufft_forward_workspace(const MfArgs& a, const Tuning& t) {
  if (a.N == 0) return 0;
  return nufft_shape(a, t).total;
}

cudaError_t mf_nufft_forward(const MfArgs& a, const Tuning& t, void* ws, cudaStream_t st) {
  if (a.N == 0) return cudaSuccess;
  const NufftShape s = nufft_shape(a, t);
  switch (a.dtype) {
    case kF64: return launch_nufft_forward<double>(a, s, ws, st);
    case kF16: return launch_nufft_forward<__half>(a, s, ws, st);
    default: return launch_nufft_forward<float>(a, s, ws, st);
  }
}

}  // namespace geraf
