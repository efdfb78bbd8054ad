// Fast approximate signal tracer (MODE_NUFFT): the per-antenna sample sums of
// the MIXED tracer evaluated through the same oversampled range grids and
// "exponential of semicircle" interpolation as the NUFFT matched filter
// (nufft_kernels.cu has the method), O(W) instead of O(S) work per
// (point, antenna) pair.
//
// With the MIXED phase model the tracer forward is, per antenna a,
//   x[a, n] = (1/P) sum_p amp(p, a) e^{+j 2 pi (c0 + n d)},
//   amp = sigma[a, p] rho / D^2 (0 for culled or out-of-bounds points)
// (SignalTracer_cuda_kernel.cu:351-450) -- a type-1 NUFFT with the points'
// amplitudes as sources, the exact shape of the matched filter's NUFFT adjoint:
// spread onto the fine grid (private windows bounded from the points' bounding
// box), then the adjoint FFT scaled by 1/P.
//
// The adjoint (SignalTracer_cuda_kernel.cu:452-587, plus the position gradient)
// needs, per live (point, antenna) pair, Q = sum_n conj(g_n) zeta^n and
// Q1 = sum_n n conj(g_n) zeta^n with zeta = e^{+j 2 pi d}: the conjugates of
// type-2 NUFFTs of the residual rows g and n g.  Two fine grids per antenna are
// built (the matched filter's grid kernel, once plain and once with the
// coefficients weighted by n), and one gather with shared weights evaluates
// both; the gradient formulas are those of the MIXED adjoint.
//
// No counterpart in the reference.
#include <algorithm>

#include "nufft_common.cuh"
#include "tracer_geometry.cuh"

namespace geraf {
namespace {

using namespace tracer;

// ---------------------------------------------------------------------------
// Forward: spread.  Block = (antenna, point split), as the matched filter's
// adjoint spread, with the tracer's amplitude and culling per pair.
template <typename T>
struct TrSpreadP {
  EsPoly poly;
  const T* normals;
  const T* sigmas;
  const T* points;
  const T* tx;
  const T* rx;
  const uint8_t* inb;
  const float* bbox;  // [6]
  float2* grid;       // [vsplits][A][M]
  int* status;
  // the points left by the per-point pre-cull and their number (device);
  // null: every in-bounds point is visited
  const int* plist;
  const int* plist_count;
  int64_t A, P, pts_per_split;
  int M, h, vsplits;
  double k0, b0, k1, b1;
};

struct SpreadPoint {
  float nx, ny, nz, px, py, pz, sig;
  bool inb;
};

// Loads the point at position k: listed point list[k], or point k.
template <typename T>
__device__ __forceinline__ SpreadPoint load_spread_point(const TrSpreadP<T>& p, int64_t a, int64_t k,
                                                         int64_t p_end) {
  SpreadPoint s{0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f, false};
  if (k >= p_end) return s;
  const int64_t q = p.plist != nullptr ? static_cast<int64_t>(p.plist[k]) : k;
  s.inb = p.plist != nullptr || p.inb[q];  // listed points are in bounds
  if (s.inb) {
    s.nx = ld_f(p.normals, q * 3 + 0);
    s.ny = ld_f(p.normals, q * 3 + 1);
    s.nz = ld_f(p.normals, q * 3 + 2);
    s.px = ld_f(p.points, q * 3 + 0);
    s.py = ld_f(p.points, q * 3 + 1);
    s.pz = ld_f(p.points, q * 3 + 2);
    s.sig = ld_f(p.sigmas, a * p.P + q);
  }
  return s;
}

template <typename T, int W>
__global__ void __launch_bounds__(kSpreadThreads) nufft_tracer_spread_kernel(const TrSpreadP<T> p) {
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

  const float txp[3] = {static_cast<float>(pos[0]), static_cast<float>(pos[1]), static_cast<float>(pos[2])};
  const float rxp[3] = {static_cast<float>(pos[3]), static_cast<float>(pos[4]), static_cast<float>(pos[5])};
  const int64_t npts = p.plist != nullptr ? static_cast<int64_t>(*p.plist_count) : p.P;
  const int64_t per_split = p.plist != nullptr ? (npts + p.vsplits - 1) / p.vsplits : p.pts_per_split;
  const int64_t p_begin = static_cast<int64_t>(vs) * per_split;
  const int64_t p_end = min(npts, p_begin + per_split);
  float* col_re = buf + threadIdx.x;
  float* col_im = buf + kWin * kWinLd + threadIdx.x;
  // The next point's inputs are loaded while the current one is spread (the
  // shared windows leave room for few warps to hide the load latency).
  SpreadPoint next = load_spread_point(p, a, p_begin + threadIdx.x, p_end);
  for (int64_t q = p_begin + threadIdx.x; q < p_end; q += blockDim.x) {
    const SpreadPoint cur = next;
    next = load_spread_point(p, a, q + blockDim.x, p_end);
    if (!cur.inb) continue;
    const float nrm[3] = {cur.nx, cur.ny, cur.nz};
    const float pt[3] = {cur.px, cur.py, cur.pz};
    const float sig = cur.sig;
    if (surely_culled(txp, rxp, nrm, pt)) continue;
    SpecGeom geo;
    specular_geometry(txp, rxp, nrm, pt, geo);
    if (culled(geo)) continue;
    const float amp = sig * geo.align / sq(path_distance(txp, rxp, pt));
    const NufftPoint np = nufft_point<W>(pos[0], pos[1], pos[2], pos[3], pos[4], pos[5],
                                         static_cast<double>(pt[0]), static_cast<double>(pt[1]),
                                         static_cast<double>(pt[2]), p.k0, p.b0, p.k1, p.b1, p.h, fM);
    const float2 e = cis_cycles(np.frac);
    const float wr = amp * e.x;
    const float wi = amp * e.y;
    const TapWeights<W> wt = tap_weights<W>(p.poly, np.f);
    if (mode) {
      const int o = np.base - w0;
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
        const int l = (np.base + k) & mask;
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

// ---------------------------------------------------------------------------
// Adjoint: gather.  A block owns blockDim points and streams the antennas'
// two grids (g and n g) through a double-buffered TMA ring.
struct GridPairStager {
  float2* buf;    // [2 stages][2 grids][rows_max * row]
  uint64_t* bar;  // [2]
  int row;        // float2 per row (even: 16-byte rows)
  int rows_max;

  __device__ __forceinline__ float2* stage_ptr(int stage, int which) const {
    return buf + (static_cast<int64_t>(stage) * 2 + which) * rows_max * row;
  }
  __device__ __forceinline__ void issue(int stage, const float2* g1, const float2* g2, int64_t row0, int rows) {
    if (threadIdx.x == 0) {
      const uint32_t bytes = static_cast<uint32_t>(rows) * row * sizeof(float2);
      mbar_arrive_expect_tx(&bar[stage], 2 * bytes);
      bulk_g2s(stage_ptr(stage, 0), g1 + row0 * row, bytes, &bar[stage]);
      bulk_g2s(stage_ptr(stage, 1), g2 + row0 * row, bytes, &bar[stage]);
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

template <typename T>
struct TrGatherP {
  EsPoly poly;
  const float2* g1;  // [A][M + kGridPad]: grid of g
  const float2* g2;  // [A][M + kGridPad]: grid of n g
  const T* normals;
  const T* sigmas;
  const T* points;
  const T* tx;
  const T* rx;
  const uint8_t* inb;
  T* g_normals;
  T* g_sigmas;
  T* g_points;
  float* partial;  // [splits][P][6] when splits > 1
  int* status;
  const int* plist;  // as in TrSpreadP
  const int* plist_count;
  int64_t A, P, per_split;
  int M, h, rows, splits;
  double k0, b0, k1, b1;
  float w0, w1s;
  size_t pos_off, buf_off;
};

template <typename T, int W, bool WITH_POINTS>
__global__ void __launch_bounds__(128) nufft_tracer_gather_kernel(const TrGatherP<T> p) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  double* pos = reinterpret_cast<double*>(smem + p.pos_off);
  const int Mp = p.M + kGridPad;
  GridPairStager stg{reinterpret_cast<float2*>(smem + p.buf_off), bar, Mp, p.rows};

  const int split = blockIdx.x % p.splits;
  const int64_t ptile = blockIdx.x / p.splits;
  // thread t owns point position k (listed point list[k], or point k); the grid
  // covers all P points and blocks past the listed ones have nothing to do
  const int64_t npts = p.plist != nullptr ? static_cast<int64_t>(*p.plist_count) : p.P;
  const int64_t p_base = ptile * blockDim.x;
  if (p_base >= npts) return;
  const int64_t k_own = p_base + threadIdx.x;
  const bool inside = k_own < npts;
  const int64_t pi = !inside ? 0 : p.plist != nullptr ? static_cast<int64_t>(p.plist[k_own]) : k_own;
  const int64_t a_begin = static_cast<int64_t>(split) * p.per_split;
  const int64_t a_end = min(p.A, a_begin + p.per_split);
  const int ntiles = a_end > a_begin ? ceil_div(a_end - a_begin, p.rows) : 0;
  const bool active = inside && (p.plist != nullptr || p.inb[pi]);
  const int mask = p.M - 1;
  const float fM = static_cast<float>(p.M);

  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();

  float nrm[3] = {0.0f, 0.0f, 1.0f}, pt[3] = {0.0f, 0.0f, 0.0f};
  if (active) {
    nrm[0] = ld_f(p.normals, pi * 3 + 0);
    nrm[1] = ld_f(p.normals, pi * 3 + 1);
    nrm[2] = ld_f(p.normals, pi * 3 + 2);
    pt[0] = ld_f(p.points, pi * 3 + 0);
    pt[1] = ld_f(p.points, pi * 3 + 1);
    pt[2] = ld_f(p.points, pi * 3 + 2);
  }
  float gnorm[3] = {0.0f, 0.0f, 0.0f};
  float gpt[3] = {0.0f, 0.0f, 0.0f};

  auto issue = [&](int tile, int stage) {
    const int64_t a0 = a_begin + static_cast<int64_t>(tile) * p.rows;
    const int rws = static_cast<int>(min(static_cast<int64_t>(p.rows), a_end - a0));
    stg.issue(stage, p.g1, p.g2, a0, rws);
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
    for (int r = 0; r < rws && inside; ++r) {
      const int64_t a = a0 + r;
      const double* ps = pos + (s * p.rows + r) * 6;
      const float txp[3] = {static_cast<float>(ps[0]), static_cast<float>(ps[1]), static_cast<float>(ps[2])};
      const float rxp[3] = {static_cast<float>(ps[3]), static_cast<float>(ps[4]), static_cast<float>(ps[5])};
      SpecGeom geo;
      bool live = false;
      if (active && !surely_culled(txp, rxp, nrm, pt)) {
        specular_geometry(txp, rxp, nrm, pt, geo);
        live = !culled(geo);
      }
      if (!live) {
        p.g_sigmas[a * p.P + pi] = from_f<T>(0.0f);
        continue;
      }
      const NufftPoint np = nufft_point<W>(ps[0], ps[1], ps[2], ps[3], ps[4], ps[5],
                                           static_cast<double>(pt[0]), static_cast<double>(pt[1]),
                                           static_cast<double>(pt[2]), p.k0, p.b0, p.k1, p.b1, p.h, fM);
      const TapWeights<W> wt = tap_weights<W>(p.poly, np.f);
      const float2* q1p = stg.stage_ptr(s, 0) + r * Mp + (np.base & mask);
      const float2* q2p = stg.stage_ptr(s, 1) + r * Mp + (np.base & mask);
      float2 qc = make_float2(0.0f, 0.0f), q1c = make_float2(0.0f, 0.0f);
#pragma unroll
      for (int k = 0; k < W; ++k) {
        const float2 w2 = make_float2(wt.w[k], wt.w[k]);
        qc = ffma2(w2, q1p[k], qc);
        if (WITH_POINTS) q1c = ffma2(w2, q2p[k], q1c);
      }
      // e = e^{j 2 pi (c0 + h d)};  exp(j phi0) Q = e conj(Qc),
      // exp(j phi0) (w0 Q + w1s Q1) = e conj(w0 Qc + w1s Q1c)
      const float2 e = cis_cycles(np.frac);
      const float sum_re = fmaf(e.x, qc.x, e.y * qc.y);  // Re(e conj(qc))
      const float propagation_distance = path_distance(txp, rxp, pt);
      const float propagation_attenuation = 1.0f / sq(propagation_distance);
      const float sigma_value = ld_f(p.sigmas, a * p.P + pi);
      p.g_sigmas[a * p.P + pi] =
          from_f<T>(propagation_attenuation * geo.align * sum_re / static_cast<float>(p.P));
      float gsa[3];
      align_normal_gradient(geo, nrm, gsa);
      const float normal_scale = sigma_value * propagation_attenuation;
#pragma unroll
      for (int k = 0; k < 3; ++k) gnorm[k] += normal_scale * gsa[k] * sum_re;
      if (WITH_POINTS) {
        const float fr = fmaf(p.w0, qc.x, p.w1s * q1c.x);
        const float fi = fmaf(p.w0, qc.y, p.w1s * q1c.y);
        const float f_im = fmaf(e.y, fr, -e.x * fi);  // Im(e conj(fr + j fi))
        const float amp = sigma_value * geo.align * propagation_attenuation;
        const float d_tau = -amp * f_im;
        const float dist_t = sqrtf(sq(txp[0] - pt[0]) + sq(txp[1] - pt[1]) + sq(txp[2] - pt[2]));
        const float dist_r = sqrtf(sq(rxp[0] - pt[0]) + sq(rxp[1] - pt[1]) + sq(rxp[2] - pt[2]));
        float drho[3];
        align_point_gradient(geo, nrm, dist_t, dist_r, drho);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const float dD = geo.inc[k] - geo.ret[k];
          const float damp_dp = normal_scale * drho[k] - 2.0f * amp / propagation_distance * dD;
          gpt[k] += sum_re * damp_dp + d_tau * dD / kSpeedOfLight;
        }
      }
    }
    __syncthreads();
    if (t + 2 < ntiles) issue(t + 2, s);
  }
  if (!inside) return;
  if (p.splits == 1) {
    const float inv = static_cast<float>(p.P);
#pragma unroll
    for (int k = 0; k < 3; ++k) p.g_normals[pi * 3 + k] = from_f<T>(gnorm[k] / inv);
    if (WITH_POINTS) {
#pragma unroll
      for (int k = 0; k < 3; ++k) p.g_points[pi * 3 + k] = from_f<T>(gpt[k] / inv);
    }
  } else {
    float* dst = p.partial + (split * p.P + pi) * 6;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      dst[k] = gnorm[k];
      dst[3 + k] = WITH_POINTS ? gpt[k] : 0.0f;
    }
  }
}

template <typename T, bool WP>
const void* gather_ptr(int W) {
  switch (W) {
    case 4: return reinterpret_cast<const void*>(&nufft_tracer_gather_kernel<T, 4, WP>);
    case 6: return reinterpret_cast<const void*>(&nufft_tracer_gather_kernel<T, 6, WP>);
    case 10: return reinterpret_cast<const void*>(&nufft_tracer_gather_kernel<T, 10, WP>);
    case 12: return reinterpret_cast<const void*>(&nufft_tracer_gather_kernel<T, 12, WP>);
    default: return reinterpret_cast<const void*>(&nufft_tracer_gather_kernel<T, 8, WP>);
  }
}

template <typename T>
const void* spread_ptr(int W) {
  switch (W) {
    case 4: return reinterpret_cast<const void*>(&nufft_tracer_spread_kernel<T, 4>);
    case 6: return reinterpret_cast<const void*>(&nufft_tracer_spread_kernel<T, 6>);
    case 10: return reinterpret_cast<const void*>(&nufft_tracer_spread_kernel<T, 10>);
    case 12: return reinterpret_cast<const void*>(&nufft_tracer_spread_kernel<T, 12>);
    default: return reinterpret_cast<const void*>(&nufft_tracer_spread_kernel<T, 8>);
  }
}

struct TrNufftShape {
  int M = 16, Mp = 32, log2M = 4, h = 0, W = 8;
  double beta = 0.0;
  // forward
  int vsplits = 1;
  int64_t pts_per_split = 0;
  // adjoint
  int rows = 4, splits = 1;
  int64_t ant_per_split = 0;
  size_t deconv_off = 0, bbox_off = 0, grid_off = 0, grid2_off = 0, partial_off = 0, list_off = 0, total = 0;
  size_t pos_off = 128, buf_off = 0, smem = 0;
};

size_t gather_smem_tr(int rows, int Mp, size_t* buf_off) {
  const size_t b = align256(128 + 2 * static_cast<size_t>(rows) * 6 * sizeof(double));
  if (buf_off != nullptr) *buf_off = b;
  return b + 4 * static_cast<size_t>(rows) * Mp * sizeof(float2);
}

TrNufftShape tr_shape(const TracerArgs& a, const Tuning& t, bool backward) {
  TrNufftShape s;
  s.M = grid_points(a.S);
  s.Mp = s.M + kGridPad;
  s.log2M = 0;
  while ((1 << s.log2M) < s.M) ++s.log2M;
  s.h = static_cast<int>(a.S / 2);
  s.W = t.taps;
  s.beta = 2.30 * s.W;
  s.deconv_off = 0;
  const size_t after_deconv = align256(static_cast<size_t>(std::max<int64_t>(a.S, 1)) * sizeof(float));
  if (!backward) {
    s.vsplits = t.splits;
    s.pts_per_split = std::max<int64_t>(1, (a.P + s.vsplits - 1) / s.vsplits);
    s.bbox_off = after_deconv;
    s.grid_off = s.bbox_off + align256((kBboxBlocks + 1) * 6 * sizeof(float));
    s.total = s.grid_off + align256(static_cast<size_t>(s.vsplits) * a.A * s.M * sizeof(float2));
  } else {
    s.rows = t.stage_rows;
    s.splits = t.splits;
    const int64_t rows_total = std::max<int64_t>(1, (a.A + s.rows - 1) / s.rows);
    s.ant_per_split = ((rows_total + s.splits - 1) / s.splits) * s.rows;
    s.grid_off = after_deconv;
    s.grid2_off = s.grid_off + align256(static_cast<size_t>(a.A) * s.Mp * sizeof(float2));
    s.partial_off = s.grid2_off + align256(static_cast<size_t>(a.A) * s.Mp * sizeof(float2));
    s.total = s.partial_off + (s.splits > 1 ? align256(static_cast<size_t>(s.splits) * a.P * 6 * sizeof(float)) : 0);
    s.smem = gather_smem_tr(s.rows, s.Mp, &s.buf_off);
  }
  s.list_off = s.total;
  if (tracer_point_list_applies(a)) s.total = s.list_off + tracer_point_list_bytes(a.P);
  return s;
}

template <typename T>
cudaError_t launch_tracer_nufft_forward(const TracerArgs& a, const Tuning& t, void* ws, cudaStream_t st) {
  const TrNufftShape s = tr_shape(a, t, false);
  unsigned char* base = static_cast<unsigned char*>(ws);
  float* deconv = reinterpret_cast<float*>(base + s.deconv_off);
  float* bbox_partial = reinterpret_cast<float*>(base + s.bbox_off);
  float* bbox = bbox_partial + kBboxBlocks * 6;
  float2* grid = reinterpret_cast<float2*>(base + s.grid_off);
  const DeviceInfo dev = current_device_info();
  cudaError_t err = launch_deconv(deconv, a.S, s.h, s.M, s.W, s.beta, st);
  if (err != cudaSuccess) return err;
  if (a.P > 0) {
    BboxP<T> bp;
    bp.voxel = static_cast<const T*>(a.points);
    bp.N = a.P;
    bp.pstride = 3;
    bp.cstride = 1;
    bp.partial = bbox_partial;
    bp.bbox = bbox;
    const int nb = static_cast<int>(std::min<int64_t>(kBboxBlocks, (a.P + 255) / 256));
    voxel_bbox_partial_kernel<T><<<nb, 256, 0, st>>>(bp);
    voxel_bbox_final_kernel<<<1, 32, 0, st>>>(bbox_partial, nb, bbox);
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
  }
  TrSpreadP<T> sp;
  sp.poly = es_poly(s.W, s.beta);
  sp.normals = static_cast<const T*>(a.normals);
  sp.sigmas = static_cast<const T*>(a.sigmas);
  sp.points = static_cast<const T*>(a.points);
  sp.tx = static_cast<const T*>(a.tx);
  sp.rx = static_cast<const T*>(a.rx);
  sp.inb = a.inbounds;
  sp.bbox = bbox;
  sp.grid = grid;
  sp.status = device_status_ptr();
  sp.plist = nullptr;
  sp.plist_count = nullptr;
  if (tracer_point_list_applies(a)) {
    err = tracer_point_list(a, base + s.list_off, false, st);
    if (err != cudaSuccess) return err;
    const PointList pl = tracer_point_list_view(base + s.list_off, a.P);
    sp.plist = pl.list;
    sp.plist_count = pl.count;
  }
  sp.A = a.A;
  sp.P = a.P;
  sp.pts_per_split = s.pts_per_split;
  sp.M = s.M;
  sp.h = s.h;
  sp.vsplits = s.vsplits;
  const PhaseConsts pc = phase_consts(a.f0, a.As, a.fs);
  sp.k0 = pc.k0;
  sp.b0 = pc.b0;
  sp.k1 = pc.k1;
  sp.b1 = pc.b1;
  const size_t ssmem = std::max(2 * static_cast<size_t>(kWin) * kWinLd, 2 * static_cast<size_t>(s.M)) * sizeof(float);
  const void* fn = spread_ptr<T>(s.W);
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
  fp.h = s.h;
  fp.M = s.M;
  fp.log2M = s.log2M;
  fp.vsplits = s.vsplits;
  fp.scale = 1.0f / static_cast<float>(a.P);
  const size_t fsmem = static_cast<size_t>(s.M) * sizeof(float2);
  err = cudaFuncSetAttribute(&nufft_adjoint_fft_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(fsmem));
  if (err != cudaSuccess) return err;
  const int fthreads = std::min(512, std::max(32, s.M / 2));
  const int64_t fblocks = std::min<int64_t>(a.A, static_cast<int64_t>(dev.sm_count) * 16);
  nufft_adjoint_fft_kernel<T><<<static_cast<unsigned>(fblocks), fthreads, fsmem, st>>>(fp);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_tracer_nufft_backward(const TracerArgs& a, const Tuning& t, void* ws, cudaStream_t st) {
  const TrNufftShape s = tr_shape(a, t, true);
  unsigned char* base = static_cast<unsigned char*>(ws);
  float* deconv = reinterpret_cast<float*>(base + s.deconv_off);
  float2* g1 = reinterpret_cast<float2*>(base + s.grid_off);
  float2* g2 = reinterpret_cast<float2*>(base + s.grid2_off);
  const DeviceInfo dev = current_device_info();
  const bool with_points = a.grad_points != nullptr;
  cudaError_t err = cudaSuccess;
  if (a.A > 0 && a.S == 0) {
    // no samples: both grids are zero
    err = cudaMemsetAsync(base + s.grid_off, 0, s.partial_off - s.grid_off, st);
    if (err != cudaSuccess) return err;
  } else if (a.A > 0) {
    err = launch_deconv(deconv, a.S, s.h, s.M, s.W, s.beta, st);
    if (err != cudaSuccess) return err;
    GridP<T> gp;
    gp.real = static_cast<const T*>(a.grad_real_out);
    gp.imag = static_cast<const T*>(a.grad_imag_out);
    gp.deconv = deconv;
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
    for (int wgt = 0; wgt < (with_points ? 2 : 1); ++wgt) {
      gp.g = wgt ? g2 : g1;
      gp.index_weight = wgt;
      nufft_grid_kernel<T><<<static_cast<unsigned>(fblocks), fthreads, fsmem, st>>>(gp);
      err = cudaGetLastError();
      if (err != cudaSuccess) return err;
    }
  }
  TrGatherP<T> p;
  p.poly = es_poly(s.W, s.beta);
  p.g1 = g1;
  p.g2 = with_points ? g2 : g1;  // without position gradients the second grid is never read
  p.normals = static_cast<const T*>(a.normals);
  p.sigmas = static_cast<const T*>(a.sigmas);
  p.points = static_cast<const T*>(a.points);
  p.tx = static_cast<const T*>(a.tx);
  p.rx = static_cast<const T*>(a.rx);
  p.inb = a.inbounds;
  p.g_normals = static_cast<T*>(a.grad_normals);
  p.g_sigmas = static_cast<T*>(a.grad_sigmas);
  p.g_points = static_cast<T*>(a.grad_points);
  p.partial = reinterpret_cast<float*>(base + s.partial_off);
  p.status = device_status_ptr();
  p.plist = nullptr;
  p.plist_count = nullptr;
  if (tracer_point_list_applies(a)) {
    // lists the points and zeroes the gradients of every point it leaves out
    err = tracer_point_list(a, base + s.list_off, true, st);
    if (err != cudaSuccess) return err;
    const PointList pl = tracer_point_list_view(base + s.list_off, a.P);
    p.plist = pl.list;
    p.plist_count = pl.count;
  }
  p.A = a.A;
  p.P = a.P;
  p.per_split = s.ant_per_split;
  p.M = s.M;
  p.h = s.h;
  p.rows = s.rows;
  p.splits = s.splits;
  const PhaseConsts pc = phase_consts(a.f0, a.As, a.fs);
  p.k0 = pc.k0;
  p.b0 = pc.b0;
  p.k1 = pc.k1;
  p.b1 = pc.b1;
  // w0 and w1/fs in rad per unit delay, as exact FP64 products of the FP32 constants
  p.w0 = static_cast<float>(2.0 * static_cast<double>(kPiF) * a.f0);
  p.w1s = static_cast<float>(2.0 * static_cast<double>(kPiF) * a.As / a.fs);
  p.pos_off = s.pos_off;
  p.buf_off = s.buf_off;
  const void* fn = with_points ? gather_ptr<T, true>(s.W) : gather_ptr<T, false>(s.W);
  err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(s.smem));
  if (err != cudaSuccess) return err;
  const int64_t ptiles = (a.P + t.threads - 1) / t.threads;
  const int64_t blocks = ptiles * s.splits;
  if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
  void* args[] = {&p};
  err = cudaLaunchKernel(fn, dim3(static_cast<unsigned>(blocks)), dim3(t.threads), args, s.smem, st);
  if (err != cudaSuccess) return err;
  if (s.splits > 1) {
    err = launch_tracer_bwd_finalize(a.dtype, p.partial, s.splits, a.P, a.grad_normals,
                                     with_points ? a.grad_points : nullptr, st, p.plist, p.plist_count);
  }
  return err;
}

}  // namespace

// ---------------------------------------------------------------------------
Tuning tracer_nufft_forward_resolve(const TracerArgs& a, const Tuning& req) {
  Tuning t = req;
  t.threads = kSpreadThreads;
  if (t.taps != 4 && t.taps != 6 && t.taps != 8 && t.taps != 10 && t.taps != 12) t.taps = 8;
  t.items = 1;
  t.stage_rows = 1;
  // point splits: at most kVoxelsPerThread points per thread and block, and
  // enough (antenna, split) blocks to fill the GPU
  const int64_t min_vs = std::max<int64_t>(
      1, (a.P + int64_t{kSpreadThreads} * kVoxelsPerThread - 1) / (int64_t{kSpreadThreads} * kVoxelsPerThread));
  const int64_t max_vs = std::max<int64_t>(min_vs, a.P / (4 * kSpreadThreads));
  if (t.splits <= 0) {
    const DeviceInfo dev = current_device_info();
    t.splits = std::max<int>(static_cast<int>(min_vs), pick_splits(std::max<int64_t>(1, a.A), 4, dev.sm_count, max_vs));
  }
  t.splits = static_cast<int>(std::min<int64_t>(std::max(t.splits, 1), std::max<int64_t>(1, a.P)));
  return t;
}

size_t tracer_nufft_forward_workspace(const TracerArgs& a, const Tuning& t) {
  if (a.A == 0 || a.S == 0) return 0;
  return tr_shape(a, t, false).total;
}

cudaError_t tracer_nufft_forward(const TracerArgs& a, const Tuning& t, void* ws, cudaStream_t st) {
  if (a.A == 0 || a.S == 0) return cudaSuccess;
  if (a.dtype == kF64) return launch_tracer_nufft_forward<double>(a, t, ws, st);
  return launch_tracer_nufft_forward<float>(a, t, ws, st);
}

Tuning tracer_nufft_backward_resolve(const TracerArgs& a, const Tuning& req) {
  Tuning t = req;
  if (t.threads != 64 && t.threads != 128) t.threads = 128;
  if (t.taps != 4 && t.taps != 6 && t.taps != 8 && t.taps != 10 && t.taps != 12) t.taps = 8;
  t.items = 1;
  // two antennas per grid stage: half the shared memory of four, so twice the
  // blocks fit each SM (measured: 128 antennas x 262144 points x 256 samples,
  // 0.43 ms against 0.64 ms; 64 x 524288 x 128, 0.37 ms against 0.39 ms)
  if (t.stage_rows <= 0) t.stage_rows = 2;
  t.stage_rows = std::min(t.stage_rows, 64);
  const int Mp = grid_points(a.S) + kGridPad;
  const DeviceInfo dev = current_device_info();
  while (t.stage_rows > 1 && gather_smem_tr(t.stage_rows, Mp, nullptr) > static_cast<size_t>(dev.max_smem_optin)) {
    t.stage_rows /= 2;
  }
  const int64_t rows_total = std::max<int64_t>(1, (a.A + t.stage_rows - 1) / t.stage_rows);
  if (t.splits <= 0) {
    int64_t ptiles = std::max<int64_t>(1, (a.P + t.threads - 1) / t.threads);
    // only the blocks of points the pre-cull lists have work; a quarter is assumed
    if (tracer_point_list_applies(a)) ptiles = std::max<int64_t>(1, ptiles / 4);
    const int per_sm = std::max(1, 1024 / t.threads);
    t.splits = pick_splits(ptiles, per_sm, dev.sm_count, rows_total);
  }
  t.splits = static_cast<int>(std::min<int64_t>(std::max(t.splits, 1), rows_total));
  return t;
}

size_t tracer_nufft_backward_workspace(const TracerArgs& a, const Tuning& t) {
  if (a.P == 0) return 0;
  return tr_shape(a, t, true).total;
}

cudaError_t tracer_nufft_backward(const TracerArgs& a, const Tuning& t, void* ws, cudaStream_t st) {
  if (a.P == 0) return cudaSuccess;
  if (a.dtype == kF64) return launch_tracer_nufft_backward<double>(a, t, ws, st);
  return launch_tracer_nufft_backward<float>(a, t, ws, st);
}

}  // namespace geraf
