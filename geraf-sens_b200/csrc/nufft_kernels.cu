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

#include "nufft_common.cuh"

namespace geraf {
namespace {

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

struct SpreadVoxel {
  float x, y, z, gr, gi;
};

template <typename T>
__device__ __forceinline__ SpreadVoxel load_spread_voxel(const SpreadP<T>& p, int64_t v, int64_t v_end) {
  SpreadVoxel s{0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  if (v < v_end) {
    s.x = ld_f(p.voxel, v);
    s.y = ld_f(p.voxel, p.N + v);
    s.z = ld_f(p.voxel, 2 * p.N + v);
    s.gr = ld_f(p.gr, v);
    s.gi = ld_f(p.gi, v);
  }
  return s;
}

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
  // The next voxel's inputs are loaded while the current one is spread (the
  // shared windows leave room for few warps to hide the load latency).
  SpreadVoxel next = load_spread_voxel(p, v_begin + threadIdx.x, v_end);
  for (int64_t v = v_begin + threadIdx.x; v < v_end; v += blockDim.x) {
    const SpreadVoxel cur = next;
    next = load_spread_voxel(p, v + blockDim.x, v_end);
    const double x = static_cast<double>(cur.x);
    const double y = static_cast<double>(cur.y);
    const double z = static_cast<double>(cur.z);
    const float g_r = cur.gr;
    const float g_i = cur.gi;
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
  cudaError_t err = launch_deconv(deconv, a.S, b.h, b.M, b.W, b.beta, st);
  if (err != cudaSuccess) return err;

  float* bbox_partial = reinterpret_cast<float*>(base + s.bbox_off);
  float* bbox = bbox_partial + kBboxBlocks * 6;
  if (a.N > 0) {
    BboxP<T> bp;
    bp.voxel = static_cast<const T*>(a.voxel);
    bp.N = a.N;
    bp.pstride = 1;
    bp.cstride = a.N;
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
  fp.scale = 1.0f / static_cast<float>(a.A);
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
    cudaError_t err = launch_deconv(deconv, a.S, s.h, s.M, s.W, s.beta, st);
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
    gp.index_weight = 0;
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
