// Matched-filter backprojection (RFMatchedFilter) kernels for sm_100a.
//
// Forward  y[v]   = (1/A) sum_a sum_n s[a,n] exp(-j phi(a,v,n))       (voxel-major)
// Adjoint  g[a,n] = (1/A) sum_v G[v]   exp(+j phi(a,v,n))             (sample-major)
// with phi(a,v,n) = 2 pi f0 tau(a,v) + 2 pi As (n/fs) tau(a,v), f0 = 773.704,
// tau = (|tx_a - v| + |rx_a - v| + 0.15) / 2.9979
// (reference: geraf/ops/RFMatchedFilter/csrc/matched_filter/MatchedFilter_cuda_kernel.cu:28-115,171-220).
//
// PLAIN kernels evaluate the reference's FP32 expressions per (v, a, n) with
// accurate cosf/sinf and keep the reference's per-output summation order, so
// their outputs track the reference to the last few ulps; their speed comes
// from TMA-staged sample tiles, a per-sample constant table and per-(v,a)
// geometry hoisting.
//
// MIXED kernels use that phi is linear in n: with z = exp(-j 2 pi dcyc) the
// forward inner sum is exp(-j phi0) * P_a(z), P_a(z) = sum_n s[a,n] z^n,
// evaluated by a second-order (Goertzel) recurrence on packed complex samples
// in 128- or 64-sample blocks; the adjoint generates
// G[v] exp(j phi0) zeta^n by a three-term recurrence per real component,
// re-seeded from exact phasors every K samples.  phi0 is reduced modulo one
// cycle in FP64 (path_cycles), so only two phasors per (v, a) are evaluated.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace geraf {
namespace {

// ---------------------------------------------------------------------------
// Shared-memory layout of the voxel-major forward kernels.
struct FwdSmem {
  size_t pos_off, kn_off, buf_off, dup_off, total;
};

// MIXED (`dup`): after the TMA ring, a float2 buffer holding the staged samples
// interleaved as (re, im) pairs, so that one 16-byte shared load yields two
// samples' packed operands.
template <typename T, typename PosT>
FwdSmem fwd_smem_layout(int rows, int ld, bool with_kn, bool dup) {
  FwdSmem s;
  s.pos_off = 128;  // two mbarriers, padded
  size_t off = s.pos_off + 2 * static_cast<size_t>(rows) * 6 * sizeof(PosT);
  off = (off + 127) & ~static_cast<size_t>(127);
  s.kn_off = off;
  if (with_kn) off += static_cast<size_t>(ld) * sizeof(float);
  off = (off + 127) & ~static_cast<size_t>(127);
  s.buf_off = off;
  off += 4 * static_cast<size_t>(rows) * ld * sizeof(T);
  off = (off + 127) & ~static_cast<size_t>(127);
  s.dup_off = off;
  if (dup) off += static_cast<size_t>(rows) * ld * sizeof(float2);
  s.total = (off + 127) & ~static_cast<size_t>(127);
  return s;
}

template <typename T>
struct MfFwdP {
  const T* real;
  const T* imag;
  const T* tx;
  const T* rx;
  T* out_r;
  T* out_i;
  const T* voxel;
  float2* partial;  // [splits][N] when splits > 1
  int* status;
  int64_t A, S, N;
  float fs, As;
  double k0, b0, k1, b1;
  int rows, ld, splits, bulk;
  int64_t ant_per_split;
  size_t pos_off, kn_off, buf_off, dup_off;
};

__device__ __forceinline__ float sq(float x) { return x * x; }

// ---------------------------------------------------------------------------
// MIXED forward: VPT voxels per thread, antennas streamed through a
// double-buffered TMA ring of `rows` antennas x S samples.  After each stage
// lands, the block interleaves it into (re, im) pairs in shared memory.  Per
// (voxel, antenna) the sample sum P(z) = sum_n x_n z^n, z = exp(-j theta), is
// evaluated by the second-order (Goertzel / Clenshaw) recurrence on the
// packed complex samples, from the highest sample down:
//   b_n = x_n + 2 cos(theta) b_{n+1} - b_{n+2}    (one sub.f32x2 + one fma.f32x2)
// so that sum_{n in block} x_n z^(n - lo) = b_lo - exp(j theta) b_{lo+1}, since
// z^m = U_m(cos theta) - exp(j theta) U_{m-1}(cos theta) (Chebyshev polynomials of
// the second kind).  The recurrence restarts every 128 samples (64 where
// |sin theta| < 0.1), which bounds its error growth, and the block sums are
// combined by Horner in z^128 (z^64).  Per
// voxel-sample this is 2 issue slots and 4 FP32 lane-operations, like the
// packed complex Horner step it replaces, but the sample operand is shared by
// all the thread's voxels and the coefficient is real: the loop alone runs
// ~15% faster on B200 (geraf_rf_goertzel_probe against geraf_rf_horner_probe).
template <typename T, int VPT>
__global__ void __launch_bounds__(256) mf_fwd_mixed_kernel(const MfFwdP<T> p) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  double* pos = reinterpret_cast<double*>(smem + p.pos_off);
  float2* dup = reinterpret_cast<float2*>(smem + p.dup_off);  // [rows][ld] interleaved (re, im)
  PairStager<T> stg{reinterpret_cast<T*>(smem + p.buf_off), bar, p.ld, p.rows, p.bulk != 0};

  // Split-major block order: the blocks resident at one time work on the same
  // antenna split, so the IF rows they stream (A/splits of them) stay in L2.
  const int64_t vtiles = gridDim.x / p.splits;
  const int split = static_cast<int>(blockIdx.x / vtiles);
  const int64_t vtile = blockIdx.x - static_cast<int64_t>(split) * vtiles;
  const int64_t a_begin = static_cast<int64_t>(split) * p.ant_per_split;
  const int64_t a_end = min(p.A, a_begin + p.ant_per_split);
  const int ntiles = a_end > a_begin ? ceil_div(a_end - a_begin, p.rows) : 0;
  const int S = static_cast<int>(p.S);

  if (p.bulk && threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();

  float vx[VPT], vy[VPT], vz[VPT];
  int64_t vid[VPT];
#pragma unroll
  for (int j = 0; j < VPT; ++j) {
    vid[j] = vtile * blockDim.x * VPT + threadIdx.x + static_cast<int64_t>(j) * blockDim.x;
    const bool ok = vid[j] < p.N;
    vx[j] = ok ? ld_f(p.voxel, vid[j]) : 0.0f;
    vy[j] = ok ? ld_f(p.voxel, p.N + vid[j]) : 0.0f;
    vz[j] = ok ? ld_f(p.voxel, 2 * p.N + vid[j]) : 0.0f;
  }
  float yr[VPT], yi[VPT], cr[VPT], ci[VPT];
#pragma unroll
  for (int j = 0; j < VPT; ++j) yr[j] = yi[j] = cr[j] = ci[j] = 0.0f;

  auto issue = [&](int tile, int stage) {
    const int64_t a0 = a_begin + static_cast<int64_t>(tile) * p.rows;
    const int rws = static_cast<int>(min(static_cast<int64_t>(p.rows), a_end - a0));
    stg.issue(stage, p.real, p.imag, a0, rws, S);
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
    {  // expand the stage into interleaved (re, im) samples; samples past S stay zero
      const T* sre = stg.stage_ptr(s, 0);
      const T* sim = stg.stage_ptr(s, 1);
      for (int i = threadIdx.x; i < rws * p.ld; i += blockDim.x) {
        const int c = i % p.ld;
        const float vr = c < S ? static_cast<float>(sre[i]) : 0.0f;
        const float vi = c < S ? static_cast<float>(sim[i]) : 0.0f;
        dup[i] = make_float2(vr, vi);
      }
    }
    __syncthreads();
    // The recurrence restarts every B = 64 samples, or every 2B for a voxel whose
    // |sin theta| >= 0.1: its rounding errors grow at most ~m eps / |sin theta|
    // over m samples, so 128 samples keep them below ~1e-4 relative even in the
    // worst case at |sin theta| = 0.1 (measured ~5e-7 on the 49152 x 256 x 128^3
    // workload, where theta is 0.2 to 0.4 rad), and only near theta = 0 or pi do
    // the shorter blocks matter.  The longer blocks halve the block extractions.
    constexpr int B = 64;
    // z^B and z^2B are raised to at most nb - 1 powers; up to 8 blocks their
    // hardware phasors are accurate enough (phase error <= 8 x 4e-7 rad)
    const int nb = (p.ld + B - 1) / B;
    const bool few_blocks = nb <= kFastPowers;
    for (int r = 0; r < rws; ++r) {
      const double* ps = pos + (s * p.rows + r) * 6;
      const double tx = ps[0], ty = ps[1], tz = ps[2], rx = ps[3], ry = ps[4], rz = ps[5];
      float frac0[VPT], sn[VPT];
      float2 C2[VPT], ZB[VPT], R[VPT];
      unsigned long_blocks = 0;  // bit j: voxel j restarts every 2B samples
#pragma unroll
      for (int j = 0; j < VPT; ++j) {
        const double dx = static_cast<double>(vx[j]), dy = static_cast<double>(vy[j]),
                     dz = static_cast<double>(vz[j]);
        const PhaseCycles pc =
            path_cycles(tx - dx, ty - dy, tz - dz, rx - dx, ry - dy, rz - dz, p.k0, p.b0, p.k1, p.b1);
        const float2 c1 = cis_cycles(pc.dcyc);  // (cos, sin) of theta; z = exp(-j theta)
        frac0[j] = pc.frac0;
        C2[j] = make_float2(2.0f * c1.x, 2.0f * c1.x);
        sn[j] = c1.y;
        const bool lng = fabsf(c1.y) >= 0.1f;
        long_blocks |= lng ? (1u << j) : 0u;
        // the multiplier of a block of this voxel's length: z^2B or z^B
        const float kb = pc.dcyc * static_cast<float>(lng ? 2 * B : B);
        const float2 zb = few_blocks ? cis_cycles_fast(kb - rintf(kb)) : cis_cycles(kb - rintf(kb));
        ZB[j] = make_float2(zb.x, -zb.y);
        R[j] = make_float2(0.0f, 0.0f);
      }
      const float2* row = dup + r * p.ld;
      float2 b1[VPT], b2[VPT];
#pragma unroll
      for (int j = 0; j < VPT; ++j) b1[j] = b2[j] = make_float2(0.0f, 0.0f);
      // The recurrence over samples [lo, hi), from the highest down.
      auto recur = [&](int lo, int hi) {
#pragma unroll 2
        for (int n = hi - 2; n >= lo; n -= 2) {
          const float4 a = *reinterpret_cast<const float4*>(row + n);  // (x_n, x_n+1)
          const float2 xh = make_float2(a.z, a.w), xl = make_float2(a.x, a.y);
#pragma unroll
          for (int j = 0; j < VPT; ++j) {
            const float2 t = fsub2(xh, b2[j]);
            b2[j] = b1[j];
            b1[j] = ffma2(C2[j], b1[j], t);
          }
#pragma unroll
          for (int j = 0; j < VPT; ++j) {
            const float2 t = fsub2(xl, b2[j]);
            b2[j] = b1[j];
            b1[j] = ffma2(C2[j], b1[j], t);
          }
        }
      };
      // Voxel j's block ends: its sum b1 - exp(j theta) b2 enters the Horner over
      // blocks, R <- R z^len + block sum, and the recurrence restarts.  (The first
      // block from the top may be shorter; R is still zero then.)
      auto end_block = [&](int j) {
        const float2 e = make_float2(0.5f * C2[j].x, sn[j]);
        const float2 eb = cmul(e, b2[j]);
        const float2 pb = make_float2(b1[j].x - eb.x, b1[j].y - eb.y);
        const float2 rz = cmul(R[j], ZB[j]);
        R[j] = make_float2(rz.x + pb.x, rz.y + pb.y);
        b1[j] = b2[j] = make_float2(0.0f, 0.0f);
      };
      if (!__any_sync(0xffffffffu, (~long_blocks & ((1u << VPT) - 1u)) != 0u)) {
        // every voxel of the warp has 2B-sample blocks (the usual case)
        for (int lo = ((nb - 1) >> 1) * 2 * B; lo >= 0; lo -= 2 * B) {
          recur(lo, min(p.ld, lo + 2 * B));
#pragma unroll
          for (int j = 0; j < VPT; ++j) end_block(j);
        }
      } else {
        // B-sample steps; a voxel with long blocks ends one at every second step
        for (int blk = nb - 1; blk >= 0; --blk) {
          recur(blk * B, min(p.ld, blk * B + B));
          const bool even = (blk & 1) == 0;
#pragma unroll
          for (int j = 0; j < VPT; ++j) {
            if (even || !((long_blocks >> j) & 1u)) end_block(j);
          }
        }
      }
#pragma unroll
      for (int j = 0; j < VPT; ++j) {
        const float2 c0 = cis_cycles_fast(frac0[j]);
        const float2 e0 = make_float2(c0.x, -c0.y);  // exp(-j phi0)
        const float2 term = cmul(e0, R[j]);
        kahan_add(yr[j], cr[j], term.x);
        kahan_add(yi[j], ci[j], term.y);
      }
    }
    __syncthreads();  // stage s (raw samples and positions) and xs are free again
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

// ---------------------------------------------------------------------------
// PLAIN forward: the reference's per-(v, a, n) FP32 arithmetic
// (MatchedFilter_cuda_kernel.cu:28-58, 86-114), one accumulator per voxel in
// the reference's (a, n) order.
template <typename T, int VPT>
__global__ void __launch_bounds__(256) mf_fwd_plain_kernel(const MfFwdP<T> p) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  float* pos = reinterpret_cast<float*>(smem + p.pos_off);
  float* kn = reinterpret_cast<float*>(smem + p.kn_off);
  PairStager<T> stg{reinterpret_cast<T*>(smem + p.buf_off), bar, p.ld, p.rows, p.bulk != 0};

  const int64_t vtiles = gridDim.x / p.splits;  // split-major, as the MIXED forward
  const int split = static_cast<int>(blockIdx.x / vtiles);
  const int64_t vtile = blockIdx.x - static_cast<int64_t>(split) * vtiles;
  const int64_t a_begin = static_cast<int64_t>(split) * p.ant_per_split;
  const int64_t a_end = min(p.A, a_begin + p.ant_per_split);
  const int ntiles = a_end > a_begin ? ceil_div(a_end - a_begin, p.rows) : 0;
  const int S = static_cast<int>(p.S);

  if (p.bulk && threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  // Per-sample factor of the reference's phase, 2*kPi*As*(n/fs), evaluated in
  // the reference's order ((2*pi)*As)*t_n with t_n = float(n)/fs.
  for (int n = threadIdx.x; n < p.ld; n += blockDim.x) {
    const float sample_time = static_cast<float>(n) / p.fs;
    kn[n] = 2.0f * kPiF * p.As * sample_time;
  }
  __syncthreads();

  float vx[VPT], vy[VPT], vz[VPT];
  int64_t vid[VPT];
  float ar[VPT], ai[VPT];
#pragma unroll
  for (int j = 0; j < VPT; ++j) {
    vid[j] = vtile * blockDim.x * VPT + threadIdx.x + static_cast<int64_t>(j) * blockDim.x;
    const bool ok = vid[j] < p.N;
    vx[j] = ok ? ld_f(p.voxel, vid[j]) : 0.0f;
    vy[j] = ok ? ld_f(p.voxel, p.N + vid[j]) : 0.0f;
    vz[j] = ok ? ld_f(p.voxel, 2 * p.N + vid[j]) : 0.0f;
    ar[j] = 0.0f;
    ai[j] = 0.0f;
  }

  auto issue = [&](int tile, int stage) {
    const int64_t a0 = a_begin + static_cast<int64_t>(tile) * p.rows;
    const int rws = static_cast<int>(min(static_cast<int64_t>(p.rows), a_end - a0));
    stg.issue(stage, p.real, p.imag, a0, rws, S);
    stage_positions<T, float>(pos, stage, p.rows, p.tx, p.rx, a0, rws);
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
    const T* sre = stg.stage_ptr(s, 0);
    const T* sim = stg.stage_ptr(s, 1);
    for (int r = 0; r < rws; ++r) {
      const float* ps = pos + (s * p.rows + r) * 6;
      const float tx_x = ps[0], tx_y = ps[1], tx_z = ps[2];
      const float rx_x = ps[3], rx_y = ps[4], rx_z = ps[5];
      const T* rowr = sre + r * p.ld;
      const T* rowi = sim + r * p.ld;
#pragma unroll
      for (int j = 0; j < VPT; ++j) {
        const float tx_distance = sqrtf(sq(tx_x - vx[j]) + sq(tx_y - vy[j]) + sq(tx_z - vz[j]));
        const float rx_distance = sqrtf(sq(rx_x - vx[j]) + sq(rx_y - vy[j]) + sq(rx_z - vz[j]));
        const float distance = tx_distance + rx_distance + kPathBias;
        const float tau = distance / kSpeedOfLight;
        const float base_phase = 2.0f * kPiF * kMfStartFrequency * tau;
        float acc_r = ar[j], acc_i = ai[j];
        for (int n = 0; n < S; ++n) {
          const float phase = base_phase + kn[n] * tau;
          float cos_phase, sin_phase;
          cos_sin(phase, &cos_phase, &sin_phase);
          const float neg_sin_phase = -sin_phase;
          const float sample_real = static_cast<float>(rowr[n]);
          const float sample_imag = static_cast<float>(rowi[n]);
          acc_r += cos_phase * sample_real - neg_sin_phase * sample_imag;
          acc_i += cos_phase * sample_imag + neg_sin_phase * sample_real;
        }
        ar[j] = acc_r;
        ai[j] = acc_i;
      }
    }
    __syncthreads();
    if (t + 2 < ntiles) issue(t + 2, s);
  }

  const int total_ant_size = static_cast<int>(p.A);
#pragma unroll
  for (int j = 0; j < VPT; ++j) {
    if (vid[j] >= p.N) continue;
    if (p.splits == 1) {
      p.out_r[vid[j]] = from_f<T>(ar[j] / total_ant_size);
      p.out_i[vid[j]] = from_f<T>(ai[j] / total_ant_size);
    } else {
      p.partial[split * p.N + vid[j]] = make_float2(ar[j], ai[j]);
    }
  }
}

// Sums `splits` partial rows of `count` complex values in a fixed order (FP64)
// and divides by `divisor`.
template <typename T>
__global__ void finalize_partials_kernel(const float2* __restrict__ partial, int splits,
                                         int64_t count, float divisor, T* out_r, T* out_i) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double sr = 0.0, si = 0.0;
    for (int s = 0; s < splits; ++s) {
      const float2 v = partial[s * count + i];
      sr += v.x;
      si += v.y;
    }
    out_r[i] = from_f<T>(static_cast<float>(sr) / divisor);
    out_i[i] = from_f<T>(static_cast<float>(si) / divisor);
  }
}

// ---------------------------------------------------------------------------
// Adjoint kernels.
template <typename T>
struct MfBwdP {
  const T* gr;  // [N]
  const T* gi;
  const T* tx;
  const T* rx;
  const T* voxel;
  T* out_r;  // [A,S]
  T* out_i;
  float2* partial;  // [splits][A][S]
  int64_t A, S, N;
  float fs, As;
  double k0, b0, k1, b1;
  int splits;
  int64_t vox_per_split;
  int groups;  // sample groups per block
};

// MIXED adjoint.  Block = (antenna, voxel split, sample range).  Phase 1:
// thread t forms w = G[v] exp(j phi0) and the group seeds w zeta^(g K) of
// voxel v0 + t.  Phase 2: thread (group g, lane l) runs each seed of its
// lane's voxels through K samples by the packed three-term recurrence
// (rotate_accumulate: 2 issue slots per voxel-sample), accumulating in
// registers; a two-level FP32 sum (flushed per tile) bounds the error growth
// over long voxel ranges.
template <typename T, int K>
__global__ void __launch_bounds__(256) mf_bwd_mixed_kernel(const MfBwdP<T> p) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int TILE = blockDim.x;
  const int G = p.groups;
  const int L = blockDim.x / G;
  float2* seeds = reinterpret_cast<float2*>(smem);  // [G][TILE]
  float2* zeta = seeds + static_cast<size_t>(G) * TILE;  // [TILE]

  const int64_t a = blockIdx.x / p.splits;
  const int split = blockIdx.x % p.splits;
  const int64_t n_begin = static_cast<int64_t>(blockIdx.y) * G * K;
  const int64_t v_begin = static_cast<int64_t>(split) * p.vox_per_split;
  const int64_t v_end = min(p.N, v_begin + p.vox_per_split);

  const double tx = ld_f(p.tx, a * 3 + 0), ty = ld_f(p.tx, a * 3 + 1), tz = ld_f(p.tx, a * 3 + 2);
  const double rx = ld_f(p.rx, a * 3 + 0), ry = ld_f(p.rx, a * 3 + 1), rz = ld_f(p.rx, a * 3 + 2);

  const int g = threadIdx.x / L;
  const int l = threadIdx.x - g * L;
  float2 acc[K], hi[K];
#pragma unroll
  for (int m = 0; m < K; ++m) acc[m] = hi[m] = make_float2(0.0f, 0.0f);

  for (int64_t v0 = v_begin; v0 < v_end; v0 += TILE) {
    {  // phase 1
      const int64_t v = v0 + threadIdx.x;
      float2 w = make_float2(0.0f, 0.0f), zt = make_float2(1.0f, 0.0f), zk = make_float2(1.0f, 0.0f);
      if (v < v_end) {
        const double vx = ld_f(p.voxel, v), vy = ld_f(p.voxel, p.N + v), vz = ld_f(p.voxel, 2 * p.N + v);
        const PhaseCycles pc =
            path_cycles(tx - vx, ty - vy, tz - vz, rx - vx, ry - vy, rz - vz, p.k0, p.b0, p.k1, p.b1);
        float start = pc.frac0;
        if (n_begin != 0) {
          const double c = static_cast<double>(pc.frac0) + static_cast<double>(n_begin) * pc.dcyc;
          start = static_cast<float>(c - rint(c));
        }
        const float2 e = cis_cycles_fast(start);
        const float2 gv = make_float2(ld_f(p.gr, v), ld_f(p.gi, v));
        w = cmul(gv, e);
        zt = cis_cycles(pc.dcyc);
        const float kc = pc.dcyc * static_cast<float>(K);
        zk = G <= kFastPowers ? cis_cycles_fast(kc - rintf(kc)) : cis_cycles(kc - rintf(kc));
      }
      zeta[threadIdx.x] = zt;
      for (int gg = 0; gg < G; ++gg) {
        seeds[gg * TILE + threadIdx.x] = w;
        w = cmul(w, zk);
      }
    }
    __syncthreads();
    {  // phase 2
      const int count = static_cast<int>(min(static_cast<int64_t>(TILE), v_end - v0));
      rotate_tile<K>(seeds + g * TILE, zeta, l, L, count, acc);
#pragma unroll
      for (int m = 0; m < K; ++m) hi[m] = fadd2(hi[m], acc[m]);
    }
    __syncthreads();
  }

  // Reduce the L lanes of each group through shared memory (fixed order).
  float2* red = reinterpret_cast<float2*>(smem);  // [G][K][L]
#pragma unroll
  for (int m = 0; m < K; ++m) red[(g * K + m) * L + l] = hi[m];
  __syncthreads();
  for (int idx = threadIdx.x; idx < G * K; idx += blockDim.x) {
    const int64_t n = n_begin + idx;
    if (n >= p.S) continue;
    float sr = 0.0f, si = 0.0f;
    for (int ll = 0; ll < L; ++ll) {
      const float2 v = red[idx * L + ll];
      sr += v.x;
      si += v.y;
    }
    if (p.splits == 1) {
      p.out_r[a * p.S + n] = from_f<T>(sr / static_cast<float>(p.A));
      p.out_i[a * p.S + n] = from_f<T>(si / static_cast<float>(p.A));
    } else {
      p.partial[(split * p.A + a) * p.S + n] = make_float2(sr, si);
    }
  }
}

// PLAIN adjoint: thread = (antenna, sample), voxels in the reference's order
// (MatchedFilter_cuda_kernel.cu:186-219).  Per-(a, v) path delays are formed
// once per voxel tile in shared memory.
template <typename T>
__global__ void __launch_bounds__(128) mf_bwd_plain_kernel(const MfBwdP<T> p) {
  constexpr int TILE = 256;
  __shared__ float s_tau[TILE], s_gr[TILE], s_gi[TILE];
  const int64_t a = blockIdx.x;
  const int64_t n = static_cast<int64_t>(blockIdx.y) * blockDim.x + threadIdx.x;
  const bool active = n < p.S;
  const float tx_x = ld_f(p.tx, a * 3 + 0), tx_y = ld_f(p.tx, a * 3 + 1), tx_z = ld_f(p.tx, a * 3 + 2);
  const float rx_x = ld_f(p.rx, a * 3 + 0), rx_y = ld_f(p.rx, a * 3 + 1), rx_z = ld_f(p.rx, a * 3 + 2);
  const float sample_time = static_cast<float>(n) / p.fs;
  const float kn = 2.0f * kPiF * p.As * sample_time;
  float acc_r = 0.0f, acc_i = 0.0f;
  for (int64_t v0 = 0; v0 < p.N; v0 += TILE) {
    const int count = static_cast<int>(min(static_cast<int64_t>(TILE), p.N - v0));
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
      const int64_t v = v0 + i;
      const float vx = ld_f(p.voxel, v), vy = ld_f(p.voxel, p.N + v), vz = ld_f(p.voxel, 2 * p.N + v);
      const float tx_distance = sqrtf(sq(tx_x - vx) + sq(tx_y - vy) + sq(tx_z - vz));
      const float rx_distance = sqrtf(sq(rx_x - vx) + sq(rx_y - vy) + sq(rx_z - vz));
      const float distance = tx_distance + rx_distance + kPathBias;
      s_tau[i] = distance / kSpeedOfLight;
      s_gr[i] = ld_f(p.gr, v);
      s_gi[i] = ld_f(p.gi, v);
    }
    __syncthreads();
    if (active) {
      for (int i = 0; i < count; ++i) {
        const float tau = s_tau[i];
        const float phase = 2.0f * kPiF * kMfStartFrequency * tau + kn * tau;
        float cos_phase, sin_phase;
        cos_sin(phase, &cos_phase, &sin_phase);
        const float neg_sin_phase = -sin_phase;
        const float grad_real_out = s_gr[i];
        const float grad_imag_out = s_gi[i];
        // The reference's expressions with the FMA contraction its build makes
        // (identified against its outputs): the cos product is fused in both.
        acc_r = __fadd_rn(acc_r, __fmaf_rn(cos_phase, grad_real_out, __fmul_rn(neg_sin_phase, grad_imag_out)));
        acc_i = __fadd_rn(acc_i, __fmaf_rn(cos_phase, grad_imag_out, __fmul_rn(sin_phase, grad_real_out)));
      }
    }
    __syncthreads();
  }
  if (active) {
    const int total_ant_size = static_cast<int>(p.A);
    p.out_r[a * p.S + n] = from_f<T>(acc_r / total_ant_size);
    p.out_i[a * p.S + n] = from_f<T>(acc_i / total_ant_size);
  }
}

// ---------------------------------------------------------------------------
// Range-bin (FFT) variants, reference arithmetic (MatchedFilter_cuda_kernel.cu:117-169, 222-279).
template <typename T>
struct MfFftP {
  const T* real;
  const T* imag;
  const T* tx;
  const T* rx;
  const T* voxel;
  const T* gr;
  const T* gi;
  T* out_r;
  T* out_i;
  int64_t A, bins, N;
  float spacing;
  int consistent_bins;
};

// Largest path delay kept by the range-bin kernels: the reference's
// spacing * bins (MatchedFilter_cuda_kernel.cu:143-148), or twice that when the
// bound is made consistent with the bin index floor(d / spacing / 2).
template <typename T>
__device__ __forceinline__ float fft_bound(const MfFftP<T>& p, int num_range_bins) {
  return p.consistent_bins ? 2.0f * (p.spacing * num_range_bins) : p.spacing * num_range_bins;
}

template <typename T>
__global__ void __launch_bounds__(256) mf_fft_fwd_kernel(const MfFftP<T> p) {
  const int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (v >= p.N) return;
  const float vx = ld_f(p.voxel, v), vy = ld_f(p.voxel, p.N + v), vz = ld_f(p.voxel, 2 * p.N + v);
  const int num_range_bins = static_cast<int>(p.bins);
  float acc_r = 0.0f, acc_i = 0.0f;
  for (int64_t a = 0; a < p.A; ++a) {
    const float tx_x = ld_f(p.tx, a * 3 + 0), tx_y = ld_f(p.tx, a * 3 + 1), tx_z = ld_f(p.tx, a * 3 + 2);
    const float rx_x = ld_f(p.rx, a * 3 + 0), rx_y = ld_f(p.rx, a * 3 + 1), rx_z = ld_f(p.rx, a * 3 + 2);
    const float tx_distance = sqrtf(sq(tx_x - vx) + sq(tx_y - vy) + sq(tx_z - vz));
    const float rx_distance = sqrtf(sq(rx_x - vx) + sq(rx_y - vy) + sq(rx_z - vz));
    const float distance = tx_distance + rx_distance + kPathBias;
    if (distance < 0.0f || distance > fft_bound(p, num_range_bins)) continue;
    const int range_bin = static_cast<int>(floorf(distance / p.spacing / 2.0f));
    if (range_bin < 0 || range_bin >= num_range_bins) continue;
    const float tau = distance / kSpeedOfLight;
    const float phase = 2.0f * kPiF * kMfStartFrequency * tau;
    float cos_phase, sin_phase;
    cos_sin(phase, &cos_phase, &sin_phase);
    const float neg_sin_phase = -sin_phase;
    const float sample_real = ld_f(p.real, a * p.bins + range_bin);
    const float sample_imag = ld_f(p.imag, a * p.bins + range_bin);
    acc_r += cos_phase * sample_real - neg_sin_phase * sample_imag;
    acc_i += cos_phase * sample_imag + neg_sin_phase * sample_real;
  }
  const int total_ant_size = static_cast<int>(p.A);
  p.out_r[v] = from_f<T>(acc_r / total_ant_size);
  p.out_i[v] = from_f<T>(acc_i / total_ant_size);
}

// Adjoint: thread = (antenna, bin); per voxel tile the bin and delay of every
// voxel are formed once in shared memory, then each thread gathers the voxels
// of its bin in voxel order (the reference's order).
template <typename T>
__global__ void __launch_bounds__(128) mf_fft_bwd_kernel(const MfFftP<T> p) {
  constexpr int TILE = 256;
  __shared__ int s_bin[TILE];
  __shared__ float s_tau[TILE], s_gr[TILE], s_gi[TILE];
  const int64_t a = blockIdx.x;
  const int64_t b = static_cast<int64_t>(blockIdx.y) * blockDim.x + threadIdx.x;
  const int num_range_bins = static_cast<int>(p.bins);
  const float tx_x = ld_f(p.tx, a * 3 + 0), tx_y = ld_f(p.tx, a * 3 + 1), tx_z = ld_f(p.tx, a * 3 + 2);
  const float rx_x = ld_f(p.rx, a * 3 + 0), rx_y = ld_f(p.rx, a * 3 + 1), rx_z = ld_f(p.rx, a * 3 + 2);
  float acc_r = 0.0f, acc_i = 0.0f;
  for (int64_t v0 = 0; v0 < p.N; v0 += TILE) {
    const int count = static_cast<int>(min(static_cast<int64_t>(TILE), p.N - v0));
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
      const int64_t v = v0 + i;
      const float vx = ld_f(p.voxel, v), vy = ld_f(p.voxel, p.N + v), vz = ld_f(p.voxel, 2 * p.N + v);
      const float tx_distance = sqrtf(sq(tx_x - vx) + sq(tx_y - vy) + sq(tx_z - vz));
      const float rx_distance = sqrtf(sq(rx_x - vx) + sq(rx_y - vy) + sq(rx_z - vz));
      const float distance = tx_distance + rx_distance + kPathBias;
      int bin = -1;
      if (!(distance < 0.0f || distance > fft_bound(p, num_range_bins))) {
        bin = static_cast<int>(floorf(distance / p.spacing / 2.0f));
      }
      s_bin[i] = bin;
      s_tau[i] = distance / kSpeedOfLight;
      s_gr[i] = ld_f(p.gr, v);
      s_gi[i] = ld_f(p.gi, v);
    }
    __syncthreads();
    if (b < p.bins) {
      for (int i = 0; i < count; ++i) {
        if (s_bin[i] != b) continue;
        const float tau = s_tau[i];
        const float phase = 2.0f * kPiF * kMfStartFrequency * tau;
        float cos_phase, sin_phase;
        cos_sin(phase, &cos_phase, &sin_phase);
        const float neg_sin_phase = -sin_phase;
        const float grad_real_out = s_gr[i];
        const float grad_imag_out = s_gi[i];
        // The reference's expressions with the FMA contraction its build makes
        // (identified against its outputs): the cos product is fused in both.
        acc_r = __fadd_rn(acc_r, __fmaf_rn(cos_phase, grad_real_out, __fmul_rn(neg_sin_phase, grad_imag_out)));
        acc_i = __fadd_rn(acc_i, __fmaf_rn(cos_phase, grad_imag_out, __fmul_rn(sin_phase, grad_real_out)));
      }
    }
    __syncthreads();
  }
  if (b < p.bins) {
    const int total_ant_size = static_cast<int>(p.A);
    p.out_r[a * p.bins + b] = from_f<T>(acc_r / total_ant_size);
    p.out_i[a * p.bins + b] = from_f<T>(acc_i / total_ant_size);
  }
}

// ---------------------------------------------------------------------------
// Host-side launch logic.
size_t elem_size(int dtype) { return dtype == kF64 ? 8 : dtype == kF16 ? 2 : 4; }

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Forward shape: threads, voxels per thread, antenna rows per stage, splits.
struct FwdShape {
  int threads, vpt, rows, ld, splits;
  int64_t ant_per_split;
  bool bulk;
  size_t smem;
  FwdSmem layout;
};

template <typename T>
const void* fwd_kernel_ptr(int mode, int vpt) {
  if (mode == kMixed) {
    if (vpt <= 2) return reinterpret_cast<const void*>(&mf_fwd_mixed_kernel<T, 2>);
    if (vpt == 4) return reinterpret_cast<const void*>(&mf_fwd_mixed_kernel<T, 4>);
    return reinterpret_cast<const void*>(&mf_fwd_mixed_kernel<T, 8>);
  }
  if (vpt == 1) return reinterpret_cast<const void*>(&mf_fwd_plain_kernel<T, 1>);
  if (vpt == 2) return reinterpret_cast<const void*>(&mf_fwd_plain_kernel<T, 2>);
  return reinterpret_cast<const void*>(&mf_fwd_plain_kernel<T, 4>);
}

FwdShape fwd_shape(const MfArgs& a, const Tuning& t) {
  FwdShape s;
  s.threads = t.threads;
  s.vpt = t.items;
  s.splits = t.splits;
  const size_t es = elem_size(a.dtype);
  // TMA writes rows back to back, so the shared row stride must equal S.
  s.bulk = (a.S > 0) && (a.S % 4 == 0) && ((a.S * es) % 16 == 0) && aligned16(a.real) &&
           aligned16(a.imag);
  s.ld = static_cast<int>(((std::max<int64_t>(a.S, 1) + 3) / 4) * 4);
  s.rows = t.stage_rows;
  const bool mixed = a.mode == kMixed;
  auto layout = [&](int rows) {
    if (a.dtype == kF64) return mixed ? fwd_smem_layout<double, double>(rows, s.ld, false, true)
                                      : fwd_smem_layout<double, float>(rows, s.ld, true, false);
    if (a.dtype == kF16) return mixed ? fwd_smem_layout<__half, double>(rows, s.ld, false, true)
                                      : fwd_smem_layout<__half, float>(rows, s.ld, true, false);
    return mixed ? fwd_smem_layout<float, double>(rows, s.ld, false, true)
                 : fwd_smem_layout<float, float>(rows, s.ld, true, false);
  };
  const DeviceInfo dev = current_device_info();
  s.layout = layout(s.rows);
  while (s.rows > 1 && s.layout.total > static_cast<size_t>(dev.max_smem_optin)) {
    s.rows /= 2;
    s.layout = layout(s.rows);
  }
  s.smem = s.layout.total;
  const int64_t rows_total = (a.A + s.rows - 1) / s.rows;
  const int64_t rows_per_split = (rows_total + s.splits - 1) / s.splits;
  s.ant_per_split = std::max<int64_t>(1, rows_per_split) * s.rows;
  return s;
}

template <typename T>
cudaError_t launch_fwd(const MfArgs& a, const FwdShape& s, void* ws, cudaStream_t st) {
  MfFwdP<T> p;
  p.real = static_cast<const T*>(a.real);
  p.imag = static_cast<const T*>(a.imag);
  p.tx = static_cast<const T*>(a.tx);
  p.rx = static_cast<const T*>(a.rx);
  p.out_r = static_cast<T*>(a.out_real);
  p.out_i = static_cast<T*>(a.out_imag);
  p.voxel = static_cast<const T*>(a.voxel);
  p.partial = static_cast<float2*>(ws);
  p.status = device_status_ptr();
  p.A = a.A;
  p.S = a.S;
  p.N = a.N;
  p.fs = a.fs;
  p.As = a.As;
  const PhaseConsts pc = phase_consts(kMfStartFrequency, a.As, a.fs);
  p.k0 = pc.k0;
  p.b0 = pc.b0;
  p.k1 = pc.k1;
  p.b1 = pc.b1;
  p.rows = s.rows;
  p.ld = s.ld;
  p.splits = s.splits;
  p.bulk = s.bulk ? 1 : 0;
  p.ant_per_split = s.ant_per_split;
  p.pos_off = s.layout.pos_off;
  p.kn_off = s.layout.kn_off;
  p.buf_off = s.layout.buf_off;
  p.dup_off = s.layout.dup_off;

  const void* fn = fwd_kernel_ptr<T>(a.mode, s.vpt);
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
    const int fin_blocks = static_cast<int>(std::min<int64_t>((a.N + 255) / 256, 148 * 16));
    finalize_partials_kernel<T><<<std::max(fin_blocks, 1), 256, 0, st>>>(
        p.partial, s.splits, a.N, static_cast<float>(a.A), p.out_r, p.out_i);
    err = cudaGetLastError();
  }
  return err;
}

// Sample groups per block (a power of two, at most 64 so the seed table fits
// in shared memory); longer sample axes are split over grid.y ranges.
int bwd_groups(int64_t S, int chunk, int threads) {
  const int64_t g = (S + chunk - 1) / chunk;
  int groups = 1;
  while (groups < g && groups < threads && groups < 64) groups *= 2;
  return groups;
}

template <typename T, int K>
cudaError_t launch_bwd_mixed_k(const MfBwdP<T>& p, dim3 grid, int threads, size_t smem,
                               cudaStream_t st) {
  const void* fn = reinterpret_cast<const void*>(&mf_bwd_mixed_kernel<T, K>);
  cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  void* args[] = {const_cast<MfBwdP<T>*>(&p)};
  return cudaLaunchKernel(fn, grid, dim3(threads), args, smem, st);
}

size_t bwd_mixed_smem(int threads, int groups, int chunk) {
  const size_t seeds = (static_cast<size_t>(groups) + 1) * threads * sizeof(float2);
  const size_t red = static_cast<size_t>(threads) * chunk * sizeof(float2);
  return std::max(seeds, red);
}

template <typename T>
cudaError_t launch_bwd(const MfArgs& a, const Tuning& t, void* ws, cudaStream_t st) {
  MfBwdP<T> p;
  p.gr = static_cast<const T*>(a.grad_real_out);
  p.gi = static_cast<const T*>(a.grad_imag_out);
  p.tx = static_cast<const T*>(a.tx);
  p.rx = static_cast<const T*>(a.rx);
  p.voxel = static_cast<const T*>(a.voxel);
  p.out_r = static_cast<T*>(a.out_real);
  p.out_i = static_cast<T*>(a.out_imag);
  p.partial = static_cast<float2*>(ws);
  p.A = a.A;
  p.S = a.S;
  p.N = a.N;
  p.fs = a.fs;
  p.As = a.As;
  const PhaseConsts pc = phase_consts(kMfStartFrequency, a.As, a.fs);
  p.k0 = pc.k0;
  p.b0 = pc.b0;
  p.k1 = pc.k1;
  p.b1 = pc.b1;
  p.splits = 1;
  p.vox_per_split = a.N;
  p.groups = 1;
  if (a.mode == kPlain) {
    const int threads = 128;
    dim3 grid(static_cast<unsigned>(a.A), static_cast<unsigned>((a.S + threads - 1) / threads));
    mf_bwd_plain_kernel<T><<<grid, threads, 0, st>>>(p);
    return cudaGetLastError();
  }
  const int threads = t.threads;
  const int chunk = t.chunk;
  const int groups = bwd_groups(a.S, chunk, threads);
  p.groups = groups;
  p.splits = t.splits;
  p.vox_per_split = (a.N + t.splits - 1) / t.splits;
  const int64_t ranges = (a.S + static_cast<int64_t>(groups) * chunk - 1) /
                         (static_cast<int64_t>(groups) * chunk);
  dim3 grid(static_cast<unsigned>(a.A * t.splits), static_cast<unsigned>(ranges));
  const size_t smem = bwd_mixed_smem(threads, groups, chunk);
  cudaError_t err;
  if (chunk == 8) err = launch_bwd_mixed_k<T, 8>(p, grid, threads, smem, st);
  else if (chunk == 32) err = launch_bwd_mixed_k<T, 32>(p, grid, threads, smem, st);
  else err = launch_bwd_mixed_k<T, 16>(p, grid, threads, smem, st);
  if (err != cudaSuccess) return err;
  if (t.splits > 1) {
    const int64_t count = a.A * a.S;
    const int fin_blocks = static_cast<int>(std::min<int64_t>((count + 255) / 256, 148 * 16));
    finalize_partials_kernel<T><<<std::max(fin_blocks, 1), 256, 0, st>>>(
        p.partial, t.splits, count, static_cast<float>(a.A), p.out_r, p.out_i);
    err = cudaGetLastError();
  }
  return err;
}

template <typename T>
cudaError_t launch_fft(const MfFftArgs& a, bool backward, cudaStream_t st) {
  MfFftP<T> p;
  p.real = static_cast<const T*>(a.real);
  p.imag = static_cast<const T*>(a.imag);
  p.tx = static_cast<const T*>(a.tx);
  p.rx = static_cast<const T*>(a.rx);
  p.voxel = static_cast<const T*>(a.voxel);
  p.gr = static_cast<const T*>(a.grad_real_out);
  p.gi = static_cast<const T*>(a.grad_imag_out);
  p.out_r = static_cast<T*>(a.out_real);
  p.out_i = static_cast<T*>(a.out_imag);
  p.A = a.A;
  p.bins = a.bins;
  p.N = a.N;
  p.spacing = a.spacing;
  p.consistent_bins = a.consistent_bins ? 1 : 0;
  if (!backward) {
    const int64_t blocks = (a.N + 255) / 256;
    mf_fft_fwd_kernel<T><<<static_cast<unsigned>(blocks), 256, 0, st>>>(p);
  } else {
    dim3 grid(static_cast<unsigned>(a.A), static_cast<unsigned>((a.bins + 127) / 128));
    mf_fft_bwd_kernel<T><<<grid, 128, 0, st>>>(p);
  }
  return cudaGetLastError();
}

}  // namespace

// ---------------------------------------------------------------------------
cudaError_t launch_finalize_partials(int dtype, const float2* partial, int splits, int64_t count,
                                     float divisor, void* out_r, void* out_i, cudaStream_t st) {
  const int blocks = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((count + 255) / 256, 148 * 16)));
  switch (dtype) {
    case kF64:
      finalize_partials_kernel<double><<<blocks, 256, 0, st>>>(
          partial, splits, count, divisor, static_cast<double*>(out_r), static_cast<double*>(out_i));
      break;
    case kF16:
      finalize_partials_kernel<__half><<<blocks, 256, 0, st>>>(
          partial, splits, count, divisor, static_cast<__half*>(out_r), static_cast<__half*>(out_i));
      break;
    default:
      finalize_partials_kernel<float><<<blocks, 256, 0, st>>>(
          partial, splits, count, divisor, static_cast<float*>(out_r), static_cast<float*>(out_i));
  }
  return cudaGetLastError();
}

// Resident blocks per SM of the forward kernel at this shape, from the
// occupancy calculator (registers and dynamic shared memory both count); the
// thread-count bound when no device answers (workspace queries on a host
// without a GPU never launch).
int fwd_blocks_per_sm(const MfArgs& a, const Tuning& t) {
  Tuning one = t;
  one.splits = 1;
  const FwdShape s = fwd_shape(a, one);
  const void* fn = a.dtype == kF64   ? fwd_kernel_ptr<double>(a.mode, s.vpt)
                   : a.dtype == kF16 ? fwd_kernel_ptr<__half>(a.mode, s.vpt)
                                     : fwd_kernel_ptr<float>(a.mode, s.vpt);
  int n = 0;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(s.smem)) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, s.threads, s.smem) != cudaSuccess ||
      n <= 0) {
    cudaGetLastError();
    return std::max(1, 1024 / t.threads);
  }
  return n;
}

Tuning mf_forward_resolve(const MfArgs& a, const Tuning& req) {
  if (a.mode == kNufft) return mf_nufft_forward_resolve(a, req);
  Tuning t = req;
  if (t.threads != 64 && t.threads != 128 && t.threads != 256) t.threads = 128;
  // MIXED keeps 2, 4 or 8 voxels per thread, each with its own recurrence state;
  // four measured fastest on B200 for 49152 x 256 samples x 128^3 voxels
  // (50.0 TFLOP/s at 128 or 256 threads x 4 voxels, against 46.8 at 128 x 8:
  // 124 against 242 registers, so twice the resident blocks).  PLAIN takes 1, 2 or 4.
  if (a.mode == kMixed) {
    if (t.items != 2 && t.items != 4 && t.items != 8) t.items = t.items == 1 ? 2 : 4;
  } else if (t.items != 1 && t.items != 2 && t.items != 4) {
    t.items = 1;
  }
  if (t.stage_rows <= 0) t.stage_rows = 8;
  t.stage_rows = std::min(t.stage_rows, 64);
  const int64_t rows_total = std::max<int64_t>(1, (a.A + t.stage_rows - 1) / t.stage_rows);
  if (t.splits <= 0) {
    const int64_t vtiles = (a.N + static_cast<int64_t>(t.threads) * t.items - 1) /
                           (static_cast<int64_t>(t.threads) * t.items);
    const DeviceInfo dev = current_device_info();
    t.splits = a.mode == kPlain
                   ? 1
                   : pick_splits(vtiles, fwd_blocks_per_sm(a, t), dev.sm_count, rows_total);
    if (a.mode == kMixed) {
      // Enough splits that one split's IF rows (streamed by every block resident
      // at the same time, the blocks being split-major) stay within 32 MiB of L2:
      // 3 splits of 32 MiB for 49152 x 256 samples.  The split count changes the
      // kernel's time by under 0.3% (measured 1 to 6 on B200); the partial sums
      // cost one pass over splits x N x 8 bytes.
      const int64_t if_bytes = 2 * a.A * a.S * static_cast<int64_t>(elem_size(a.dtype));
      const int64_t for_l2 = (if_bytes + (int64_t{32} << 20) - 1) >> 25;
      t.splits = static_cast<int>(std::max<int64_t>(t.splits, std::min<int64_t>(for_l2, 64)));
    }
  }
  t.splits = static_cast<int>(std::min<int64_t>(std::max(t.splits, 1), rows_total));
  if (t.chunk <= 0) t.chunk = 16;
  return t;
}

size_t mf_forward_workspace(const MfArgs& a, const Tuning& t) {
  if (a.mode == kNufft) return mf_nufft_forward_workspace(a, t);
  if (t.splits <= 1 || a.N == 0) return 0;
  return static_cast<size_t>(t.splits) * a.N * sizeof(float2);
}

cudaError_t mf_forward(const MfArgs& a, const Tuning& t, void* ws, cudaStream_t st) {
  if (a.mode == kNufft) return mf_nufft_forward(a, t, ws, st);
  if (a.N == 0) return cudaSuccess;
  const FwdShape s = fwd_shape(a, t);
  switch (a.dtype) {
    case kF64: return launch_fwd<double>(a, s, ws, st);
    case kF16: return launch_fwd<__half>(a, s, ws, st);
    default: return launch_fwd<float>(a, s, ws, st);
  }
}

Tuning mf_backward_resolve(const MfArgs& a, const Tuning& req) {
  if (a.mode == kNufft) return mf_nufft_backward_resolve(a, req);
  Tuning t = req;
  // MIXED: 128 threads; 32-sample chunks for rows of 256 samples or more (measured
  // on B200 for the 49152 x 256 x 128^3 adjoint: 4.48 s, 4% faster than 16-sample
  // chunks; 256 threads and 8-sample chunks are slower), 16 for shorter rows.
  if (t.threads != 64 && t.threads != 128 && t.threads != 256) t.threads = a.mode == kMixed ? 128 : 256;
  if (t.chunk != 8 && t.chunk != 16 && t.chunk != 32) t.chunk = a.mode == kMixed && a.S >= 256 ? 32 : 16;
  if (t.items <= 0) t.items = 1;
  if (t.stage_rows <= 0) t.stage_rows = 8;
  if (a.mode == kPlain) {
    t.splits = 1;
    return t;
  }
  const int groups = bwd_groups(a.S, t.chunk, t.threads);
  const int64_t ranges = (a.S + static_cast<int64_t>(groups) * t.chunk - 1) /
                         (static_cast<int64_t>(groups) * t.chunk);
  const int64_t vtiles = std::max<int64_t>(1, (a.N + t.threads - 1) / t.threads);
  if (t.splits <= 0) {
    const DeviceInfo dev = current_device_info();
    const int per_sm = std::max(1, 512 / t.threads);
    t.splits = pick_splits(std::max<int64_t>(1, a.A * ranges), per_sm, dev.sm_count, vtiles);
  }
  t.splits = static_cast<int>(std::min<int64_t>(std::max(t.splits, 1), vtiles));
  return t;
}

size_t mf_backward_workspace(const MfArgs& a, const Tuning& t) {
  if (a.mode == kNufft) return mf_nufft_backward_workspace(a, t);
  if (a.mode == kPlain || t.splits <= 1) return 0;
  return static_cast<size_t>(t.splits) * a.A * a.S * sizeof(float2);
}

cudaError_t mf_backward(const MfArgs& a, const Tuning& t, void* ws, cudaStream_t st) {
  if (a.mode == kNufft) return mf_nufft_backward(a, t, ws, st);
  if (a.A == 0 || a.S == 0) return cudaSuccess;
  switch (a.dtype) {
    case kF64: return launch_bwd<double>(a, t, ws, st);
    case kF16: return launch_bwd<__half>(a, t, ws, st);
    default: return launch_bwd<float>(a, t, ws, st);
  }
}

cudaError_t mf_fft_forward(const MfFftArgs& a, cudaStream_t st) {
  if (a.N == 0) return cudaSuccess;
  switch (a.dtype) {
    case kF64: return launch_fft<double>(a, false, st);
    case kF16: return launch_fft<__half>(a, false, st);
    default: return launch_fft<float>(a, false, st);
  }
}

cudaError_t mf_fft_backward(const MfFftArgs& a, cudaStream_t st) {
  if (a.A == 0 || a.bins == 0) return cudaSuccess;
  switch (a.dtype) {
    case kF64: return launch_fft<double>(a, true, st);
    case kF16: return launch_fft<__half>(a, true, st);
    default: return launch_fft<float>(a, true, st);
  }
}

}  // namespace geraf
