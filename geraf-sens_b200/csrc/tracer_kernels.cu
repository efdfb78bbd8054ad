// Lensless specular signal tracer (RFSignalTracer) and along-ray resampler
// kernels for sm_100a.
//
// Forward  x[a,n] = (1/P) sum_p amp(a,p) exp(+j (w0 + w1 t_n) tau(a,p))          (sample-major)
// Adjoint  dL/dsigma[a,p], dL/dnormal[p], dL/dpoint[p]                             (point-major)
// amp = sigma[a,p] rho / D^2, rho = <normalize(rx-p), normalize(i - 2(i.n)n)>,
// i = normalize(p - tx), culled when rho < 1e-6 or i.n > 0, D = |tx-p| + |rx-p|,
// tau = (D + 0.15)/2.9979, w0 = 2 pi f0, w1 = 2 pi As
// (reference: geraf/ops/RFSignalTracer/csrc/signal_tracer/SignalTracer_cuda_kernel.cu:19-197, 351-587).
//
// The reference recomputes the specular geometry for every (point, antenna,
// sample) triple.  Here the geometry is formed once per (point, antenna) --
// in the reference's FP32 operation order, so amplitudes and culling decisions
// are bit-identical -- and the sample loop works on (amplitude, delay) only.
// PLAIN forms then evaluate the reference's per-sample phase with accurate
// cosf/sinf in its summation order; MIXED forms reduce the carrier phase in
// FP64 and generate the per-sample phasors with a three-term recurrence
// (forward) or a Horner recurrence (adjoint), which also yields the position gradient the
// reference does not provide.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "tracer_geometry.cuh"

namespace geraf {
namespace {

using namespace tracer;

// ---------------------------------------------------------------------------
template <typename T>
struct TrP {
  const T* normals;
  const T* sigmas;
  const T* points;
  const T* tx;
  const T* rx;
  const uint8_t* inb;
  T* out_r;
  T* out_i;
  const T* gr;
  const T* gi;
  T* g_normals;
  T* g_sigmas;
  T* g_points;
  float* partial;  // forward: [splits][A][S][2]; adjoint: [splits][P][6]
  int* status;
  int64_t A, S, P;
  float fs, f0, As;
  double k0, b0, k1, b1;
  int splits;
  int64_t per_split;  // points (forward) or antennas (adjoint) per split
  int groups;         // forward: sample groups per block
  int rows, ld, bulk;  // adjoint: antenna stage
  size_t pos_off, buf_off;
  size_t cnt_off, list_off, contrib_off;  // MIXED adjoint: per-tile work lists
  // MIXED: the points left by the per-point pre-cull (tracer_precull.cu), in
  // ascending order, and their number (device); null: every point is visited
  const int* plist;
  const int* plist_count;
};

template <typename T>
__device__ __forceinline__ void load3(const T* base, int64_t i, float* out) {
  out[0] = ld_f(base, i * 3 + 0);
  out[1] = ld_f(base, i * 3 + 1);
  out[2] = ld_f(base, i * 3 + 2);
}

// PLAIN forward: block = (sample block, antenna).  Per point tile, the
// (amplitude, delay) of each point is formed once in shared memory; each
// thread then accumulates its sample over the tile in point order, with the
// reference's phase expression and accurate cosf/sinf
// (SignalTracer_cuda_kernel.cu:375-449).
template <typename T>
__global__ void __launch_bounds__(128) tracer_fwd_plain_kernel(const TrP<T> p) {
  constexpr int TILE = 256;
  __shared__ float s_amp[TILE], s_tau[TILE];
  __shared__ int s_valid[TILE];
  const int64_t a = blockIdx.x;
  const int64_t n = static_cast<int64_t>(blockIdx.y) * blockDim.x + threadIdx.x;
  const bool active = n < p.S;
  float txp[3], rxp[3];
  load3(p.tx, a, txp);
  load3(p.rx, a, rxp);
  const float sample_time = static_cast<float>(n) / p.fs;
  const float w = phase_rate(p.f0, p.As, sample_time);
  float acc_r = 0.0f, acc_i = 0.0f;
  for (int64_t p0 = 0; p0 < p.P; p0 += TILE) {
    const int count = static_cast<int>(min(static_cast<int64_t>(TILE), p.P - p0));
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
      const int64_t pi = p0 + i;
      int valid = 0;
      float amp = 0.0f, tau = 0.0f;
      if (p.inb[pi]) {
        float nrm[3], pt[3];
        load3(p.normals, pi, nrm);
        load3(p.points, pi, pt);
        SpecGeom g;
        specular_geometry(txp, rxp, nrm, pt, g);
        if (!culled(g)) {
          float propagation_distance = path_distance(txp, rxp, pt);
          amp = ld_f(p.sigmas, a * p.P + pi) * g.align / sq(propagation_distance);
          propagation_distance += kPathBias;
          tau = propagation_distance / kSpeedOfLight;
          valid = 1;
        }
      }
      s_valid[i] = valid;
      s_amp[i] = amp;
      s_tau[i] = tau;
    }
    __syncthreads();
    if (active) {
      for (int i = 0; i < count; ++i) {
        if (!s_valid[i]) continue;
        const float phase = __fmul_rn(w, s_tau[i]);
        float c, sn;
        cos_sin(phase, &c, &sn);
        acc_r += s_amp[i] * c;
        acc_i += s_amp[i] * sn;
      }
    }
    __syncthreads();
  }
  if (active) {
    const int total_point_size = static_cast<int>(p.P);
    p.out_r[a * p.S + n] = from_f<T>(acc_r / total_point_size);
    p.out_i[a * p.S + n] = from_f<T>(acc_i / total_point_size);
  }
}

// MIXED forward.  Block = (antenna x point split, sample range).  Phase 1:
// thread t forms the geometry of point p0 + t, culled and out-of-bounds
// points are compacted away, and each surviving point stores its group seeds
// amp exp(j phi(n_g)) and its per-sample rotator zeta.  Phase 2: thread
// (group g, lane l) runs the seeds of its lane's points through K samples
// (rotate_accumulate: packed three-term recurrence).
template <typename T, int K>
__global__ void __launch_bounds__(256) tracer_fwd_mixed_kernel(const TrP<T> p) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int TILE = blockDim.x;
  const int G = p.groups;
  const int L = blockDim.x / G;
  float2* seeds = reinterpret_cast<float2*>(smem);        // [G][TILE]
  float2* zeta = seeds + static_cast<size_t>(G) * TILE;   // [TILE]
  int* warp_base = reinterpret_cast<int*>(zeta + TILE);   // [32]

  const int64_t a = blockIdx.x / p.splits;
  const int split = blockIdx.x % p.splits;
  const int64_t n_begin = static_cast<int64_t>(blockIdx.y) * G * K;
  // the point positions k visited: listed points list[k], or every point k
  const int64_t npts = p.plist != nullptr ? static_cast<int64_t>(*p.plist_count) : p.P;
  const int64_t per_split = p.plist != nullptr ? (npts + p.splits - 1) / p.splits : p.per_split;
  const int64_t pt_begin = static_cast<int64_t>(split) * per_split;
  const int64_t pt_end = min(npts, pt_begin + per_split);

  float txp[3], rxp[3];
  load3(p.tx, a, txp);
  load3(p.rx, a, rxp);
  const double tx = txp[0], ty = txp[1], tz = txp[2], rx = rxp[0], ry = rxp[1], rz = rxp[2];

  const int g = threadIdx.x / L;
  const int l = threadIdx.x - g * L;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  float2 acc[K], hi[K];
#pragma unroll
  for (int m = 0; m < K; ++m) acc[m] = hi[m] = make_float2(0.0f, 0.0f);

  // The point data of tile k + 1 are loaded while tile k's samples are summed.
  float nrm[3] = {0.0f, 0.0f, 1.0f}, pt[3] = {0.0f, 0.0f, 0.0f}, sig = 0.0f;
  bool inb = false;
  auto load_point = [&](int64_t k) {
    inb = false;
    if (k < pt_end) {
      const int64_t q = p.plist != nullptr ? static_cast<int64_t>(p.plist[k]) : k;
      inb = p.plist != nullptr || p.inb[q];  // listed points are in bounds
      if (inb) {
        load3(p.normals, q, nrm);
        load3(p.points, q, pt);
        sig = ld_f(p.sigmas, a * p.P + q);
      }
    }
  };
  load_point(pt_begin + threadIdx.x);
  for (int64_t p0 = pt_begin; p0 < pt_end; p0 += TILE) {
    bool valid = false;
    float2 w = make_float2(0.0f, 0.0f), zt = make_float2(1.0f, 0.0f), zk = make_float2(1.0f, 0.0f);
    if (inb && !surely_culled(txp, rxp, nrm, pt)) {
      SpecGeom geo;
      specular_geometry(txp, rxp, nrm, pt, geo);
      if (!culled(geo)) {
        const float propagation_distance = path_distance(txp, rxp, pt);
        const float amp = sig * geo.align / sq(propagation_distance);
        const double px = pt[0], py = pt[1], pz = pt[2];
        const PhaseCycles pc =
            path_cycles(tx - px, ty - py, tz - pz, rx - px, ry - py, rz - pz, p.k0, p.b0, p.k1, p.b1);
        float start = pc.frac0;
        if (n_begin != 0) {
          const double c = static_cast<double>(pc.frac0) + static_cast<double>(n_begin) * pc.dcyc;
          start = static_cast<float>(c - rint(c));
        }
        const float2 e = cis_cycles_fast(start);
        w = make_float2(amp * e.x, amp * e.y);
        zt = cis_cycles(pc.dcyc);
        const float kc = pc.dcyc * static_cast<float>(K);
        zk = G <= kFastPowers ? cis_cycles_fast(kc - rintf(kc)) : cis_cycles(kc - rintf(kc));
        valid = true;
      }
    }
    // Compact the surviving points of the tile.
    const unsigned ballot = __ballot_sync(0xffffffffu, valid);
    if (lane == 0) warp_base[warp] = __popc(ballot);
    __syncthreads();
    if (threadIdx.x == 0) {
      int run = 0;
      for (int wi = 0; wi < nwarps; ++wi) {
        const int c = warp_base[wi];
        warp_base[wi] = run;
        run += c;
      }
      warp_base[nwarps] = run;
    }
    __syncthreads();
    const int count = warp_base[nwarps];
    if (valid) {
      const int slot = warp_base[warp] + __popc(ballot & ((1u << lane) - 1u));
      zeta[slot] = zt;
      for (int gg = 0; gg < G; ++gg) {
        seeds[gg * TILE + slot] = w;
        w = cmul(w, zk);
      }
    }
    load_point(p0 + TILE + threadIdx.x);  // in flight during the sums below
    __syncthreads();
    rotate_tile<K>(seeds + g * TILE, zeta, l, L, count, acc);
#pragma unroll
    for (int m = 0; m < K; ++m) hi[m] = fadd2(hi[m], acc[m]);
    __syncthreads();
  }

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
      p.out_r[a * p.S + n] = from_f<T>(sr / static_cast<float>(p.P));
      p.out_i[a * p.S + n] = from_f<T>(si / static_cast<float>(p.P));
    } else {
      float* dst = p.partial + ((split * p.A + a) * p.S + n) * 2;
      dst[0] = sr;
      dst[1] = si;
    }
  }
}

template <typename T>
__global__ void tracer_fwd_finalize_kernel(const float* __restrict__ partial, int splits,
                                           int64_t count, float divisor, T* out_r, T* out_i) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double sr = 0.0, si = 0.0;
    for (int s = 0; s < splits; ++s) {
      sr += partial[(s * count + i) * 2 + 0];
      si += partial[(s * count + i) * 2 + 1];
    }
    out_r[i] = from_f<T>(static_cast<float>(sr) / divisor);
    out_i[i] = from_f<T>(static_cast<float>(si) / divisor);
  }
}

// ---------------------------------------------------------------------------
// Adjoint (point-major).  Block = point tile x antenna split; the residual
// rows g[a, :] stream through a double-buffered TMA ring.
struct AdjSmem {
  size_t pos_off, buf_off, total;
};

template <typename T>
AdjSmem adj_smem_layout(int rows, int ld) {
  AdjSmem s;
  s.pos_off = 128;
  size_t off = s.pos_off + 2 * static_cast<size_t>(rows) * 6 * sizeof(float);
  off = (off + 127) & ~static_cast<size_t>(127);
  s.buf_off = off;
  off += 4 * static_cast<size_t>(rows) * ld * sizeof(T);
  s.total = (off + 127) & ~static_cast<size_t>(127);
  return s;
}

// MIXED adjoint: the staged ring as above, then per-tile work lists -- live
// (point, antenna) counts [rows], their point slots [rows][threads] and the
// per-point gradient contributions [rows][nc][threads].
struct AdjMixedSmem {
  size_t pos_off, buf_off, cnt_off, list_off, contrib_off, total;
};

template <typename T>
AdjMixedSmem adj_mixed_smem_layout(int rows, int ld, int threads, int nc) {
  const AdjSmem base = adj_smem_layout<T>(rows, ld);
  AdjMixedSmem s;
  s.pos_off = base.pos_off;
  s.buf_off = base.buf_off;
  size_t off = base.total;
  s.cnt_off = off;
  off += (static_cast<size_t>(rows) * sizeof(int) + 127) & ~static_cast<size_t>(127);
  s.list_off = off;
  off += (static_cast<size_t>(rows) * threads * sizeof(int) + 127) & ~static_cast<size_t>(127);
  s.contrib_off = off;
  off += static_cast<size_t>(rows) * nc * threads * sizeof(float);
  s.total = (off + 127) & ~static_cast<size_t>(127);
  return s;
}

template <typename T>
__device__ __forceinline__ void stage_positions_f(float* pos, int stage, int rows_max, const T* tx,
                                                  const T* rx, int64_t a0, int rws) {
  for (int i = threadIdx.x; i < rws * 6; i += blockDim.x) {
    const int r = i / 6;
    const int c = i - r * 6;
    const T* src = c < 3 ? tx : rx;
    pos[(stage * rows_max + r) * 6 + c] = ld_f(src, (a0 + r) * 3 + (c % 3));
  }
}

// Writes one point's accumulated normal / position gradients (or partials).
template <typename T>
__device__ __forceinline__ void store_point_grads(const TrP<T>& p, int split, int64_t pi,
                                                  const float* gn, const float* gp, bool with_points) {
  if (p.splits == 1) {
    const int total_point_size = static_cast<int>(p.P);
#pragma unroll
    for (int k = 0; k < 3; ++k) p.g_normals[pi * 3 + k] = from_f<T>(gn[k] / total_point_size);
    if (with_points) {
#pragma unroll
      for (int k = 0; k < 3; ++k) p.g_points[pi * 3 + k] = from_f<T>(gp[k] / total_point_size);
    }
  } else {
    float* dst = p.partial + (split * p.P + pi) * 6;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      dst[k] = gn[k];
      dst[3 + k] = with_points ? gp[k] : 0.0f;
    }
  }
}

// PLAIN adjoint: thread = point, antennas and samples in the reference's order
// (SignalTracer_cuda_kernel.cu:491-586).  With grad_points requested, the delay
// derivative sum_n w_n (g_i cos - g_r sin) is accumulated alongside.
template <typename T, bool WITH_POINTS>
__global__ void __launch_bounds__(128) tracer_bwd_plain_kernel(const TrP<T> p) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  float* pos = reinterpret_cast<float*>(smem + p.pos_off);
  PairStager<T> stg{reinterpret_cast<T*>(smem + p.buf_off), bar, p.ld, p.rows, p.bulk != 0};

  const int split = blockIdx.x % p.splits;
  const int64_t ptile = blockIdx.x / p.splits;
  const int64_t pi = ptile * blockDim.x + threadIdx.x;
  const int64_t a_begin = static_cast<int64_t>(split) * p.per_split;
  const int64_t a_end = min(p.A, a_begin + p.per_split);
  const int ntiles = a_end > a_begin ? ceil_div(a_end - a_begin, p.rows) : 0;
  const int S = static_cast<int>(p.S);
  const bool inside = pi < p.P;
  const bool active = inside && p.inb[pi];

  if (p.bulk && threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();

  float nrm[3] = {0.0f, 0.0f, 0.0f}, pt[3] = {0.0f, 0.0f, 0.0f};
  if (active) {
    load3(p.normals, pi, nrm);
    load3(p.points, pi, pt);
  }
  float accum_grad_normal[3] = {0.0f, 0.0f, 0.0f};
  float accum_grad_point[3] = {0.0f, 0.0f, 0.0f};

  auto issue = [&](int tile, int stage) {
    const int64_t a0 = a_begin + static_cast<int64_t>(tile) * p.rows;
    const int rws = static_cast<int>(min(static_cast<int64_t>(p.rows), a_end - a0));
    stg.issue(stage, p.gr, p.gi, a0, rws, S);
    stage_positions_f<T>(pos, stage, p.rows, p.tx, p.rx, a0, rws);
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
      if (!active) {
        p.g_sigmas[a * p.P + pi] = from_f<T>(0.0f);
        continue;
      }
      const float* ps = pos + (s * p.rows + r) * 6;
      const float txp[3] = {ps[0], ps[1], ps[2]};
      const float rxp[3] = {ps[3], ps[4], ps[5]};
      SpecGeom g;
      specular_geometry(txp, rxp, nrm, pt, g);
      if (culled(g)) {
        p.g_sigmas[a * p.P + pi] = from_f<T>(0.0f);
        continue;
      }
      float gsa[3];
      align_normal_gradient(g, nrm, gsa);
      float propagation_distance = path_distance(txp, rxp, pt);
      const float propagation_attenuation = 1.0f / sq(propagation_distance);
      const float sigma_value = ld_f(p.sigmas, a * p.P + pi);
      const float dist_path = propagation_distance;
      propagation_distance += kPathBias;
      const float tau = propagation_distance / kSpeedOfLight;
      const T* rowr = stg.stage_ptr(s, 0) + r * p.ld;
      const T* rowi = stg.stage_ptr(s, 1) + r * p.ld;
      float accum_grad_sigma = 0.0f;
      float accum_raw = 0.0f;
      float accum_tau = 0.0f;
      for (int n = 0; n < S; ++n) {
        const float sample_time = static_cast<float>(n) / p.fs;
        const float omega = adjoint_phase_rate<T>(p.f0, p.As, sample_time);
        const float phase = __fmul_rn(omega, tau);
        float phase_real, phase_imag;
        cos_sin(phase, &phase_real, &phase_imag);
        const float gro = static_cast<float>(rowr[n]);
        const float gio = static_cast<float>(rowi[n]);
        const float grad_real = gro * phase_real;
        const float grad_imag = gio * phase_imag;
        const float normal_scale = sigma_value * propagation_attenuation;
        accum_grad_normal[0] += normal_scale * gsa[0] * (grad_real + grad_imag);
        accum_grad_normal[1] += normal_scale * gsa[1] * (grad_real + grad_imag);
        accum_grad_normal[2] += normal_scale * gsa[2] * (grad_real + grad_imag);
        accum_grad_sigma += propagation_attenuation * g.align * (grad_real + grad_imag);
        if (WITH_POINTS) {
          accum_raw += grad_real + grad_imag;
          accum_tau += omega * (gio * phase_real - gro * phase_imag);
        }
      }
      p.g_sigmas[a * p.P + pi] = from_f<T>(accum_grad_sigma / static_cast<int>(p.P));
      if (WITH_POINTS) {
        // dL/dp = dL/damp * damp/dp + dL/dtau * dtau/dp (before the 1/P factor)
        const float amp = sigma_value * g.align * propagation_attenuation;
        const float d_amp = accum_raw;
        const float dist_t = sqrtf(sq(txp[0] - pt[0]) + sq(txp[1] - pt[1]) + sq(txp[2] - pt[2]));
        const float dist_r = sqrtf(sq(rxp[0] - pt[0]) + sq(rxp[1] - pt[1]) + sq(rxp[2] - pt[2]));
        float drho[3];
        align_point_gradient(g, nrm, dist_t, dist_r, drho);
        const float d_tau = amp * accum_tau;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const float dD = g.inc[k] - g.ret[k];
          const float damp_dp =
              sigma_value * propagation_attenuation * drho[k] - 2.0f * amp / dist_path * dD;
          accum_grad_point[k] += d_amp * damp_dp + d_tau * dD / kSpeedOfLight;
        }
      }
    }
    __syncthreads();
    if (t + 2 < ntiles) issue(t + 2, s);
  }
  if (inside) store_point_grads(p, split, pi, accum_grad_normal, accum_grad_point, WITH_POINTS);
}

// MIXED adjoint: a block owns blockDim points (one per thread) and streams
// antenna rows of the residual through a TMA ring.  Per (point, antenna) the
// residual polynomial Q(zeta) = sum_n conj(g[a,n]) zeta^n is evaluated by
// Horner in zeta^2 on the even and odd samples in the two lanes of packed
// f32x2 operations (2 instructions per sample) and, for position gradients,
// Q1 = sum_n n conj(g) zeta^n alongside (2 more).
//
// Culled pairs (back-facing or grazing, rho < 1e-6) skip all of that, so per
// stage the block first lists the (point, antenna) pairs that the early test
// cannot cull and then deals them out evenly over all threads, which form each
// pair's exact geometry once: no lane idles beside a lane that works.
// Each pair's normal / position contributions land in shared memory, and the
// point's owner thread adds them up in antenna order -- the same sums, in the
// same order, as one thread walking its point's antennas.  Six blocks are kept
// resident per SM (80 registers): 1-6% faster than the five that 93
// registers allowed, measured on 64 antennas x 524288 points x 128 samples and
// 128 antennas x 262144 points x 256 samples.
template <typename T, bool WITH_POINTS>
__global__ void __launch_bounds__(128, 6) tracer_bwd_mixed_kernel(const TrP<T> p) {
  constexpr int NC = WITH_POINTS ? 6 : 3;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  float* pos = reinterpret_cast<float*>(smem + p.pos_off);
  int* cnt = reinterpret_cast<int*>(smem + p.cnt_off);           // [rows]
  int* list = reinterpret_cast<int*>(smem + p.list_off);         // [rows][TILE]
  float* contrib = reinterpret_cast<float*>(smem + p.contrib_off);  // [rows][NC][TILE]
  PairStager<T> stg{reinterpret_cast<T*>(smem + p.buf_off), bar, p.ld, p.rows, p.bulk != 0};

  const int TILE = blockDim.x;
  const int split = blockIdx.x % p.splits;
  const int64_t ptile = blockIdx.x / p.splits;
  // Thread t owns point position k = ptile * TILE + t: listed point list[k],
  // or point k when every point is visited.  The grid covers all P points;
  // blocks past the listed ones have nothing to do.
  const int64_t npts = p.plist != nullptr ? static_cast<int64_t>(*p.plist_count) : p.P;
  const int64_t p_base = ptile * TILE;
  if (p_base >= npts) return;
  const int64_t k_own = p_base + threadIdx.x;
  const bool inside = k_own < npts;
  const int64_t pi = !inside ? 0 : p.plist != nullptr ? static_cast<int64_t>(p.plist[k_own]) : k_own;
  const int64_t a_begin = static_cast<int64_t>(split) * p.per_split;
  const int64_t a_end = min(p.A, a_begin + p.per_split);
  const int ntiles = a_end > a_begin ? ceil_div(a_end - a_begin, p.rows) : 0;
  const bool active = inside && (p.plist != nullptr || p.inb[pi]);

  if (p.bulk && threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();

  float own_nrm[3] = {0.0f, 0.0f, 1.0f}, own_pt[3] = {0.0f, 0.0f, 0.0f};
  if (active) {
    load3(p.normals, pi, own_nrm);
    load3(p.points, pi, own_pt);
  }
  // w0 and w1/fs in rad per unit delay, as exact FP64 products of the FP32 constants.
  const float w0 = static_cast<float>(2.0 * static_cast<double>(kPiF) * p.f0);
  const float w1s = static_cast<float>(2.0 * static_cast<double>(kPiF) * p.As / p.fs);
  float gnorm[3] = {0.0f, 0.0f, 0.0f};
  float gpt[3] = {0.0f, 0.0f, 0.0f};

  auto issue = [&](int tile, int stage) {
    const int64_t a0 = a_begin + static_cast<int64_t>(tile) * p.rows;
    const int rws = static_cast<int>(min(static_cast<int64_t>(p.rows), a_end - a0));
    stg.issue(stage, p.gr, p.gi, a0, rws, static_cast<int>(p.S));
    stage_positions_f<T>(pos, stage, p.rows, p.tx, p.rx, a0, rws);
  };
  if (ntiles > 0) issue(0, 0);
  if (ntiles > 1) issue(1, 1);

  for (int t = 0; t < ntiles; ++t) {
    const int s = t & 1;
    for (int r = threadIdx.x; r < p.rows; r += TILE) cnt[r] = 0;
    if (!stg.wait(s, (t >> 1) & 1, p.status)) {  // (its barrier also publishes cnt)
      if (t + 1 < ntiles) stg.drain(s ^ 1, ((t + 1) >> 1) & 1, p.status);
      return;
    }
    const int64_t a0 = a_begin + static_cast<int64_t>(t) * p.rows;
    const int rws = static_cast<int>(min(static_cast<int64_t>(p.rows), a_end - a0));

    // 1. list the stage's candidate pairs, those the early test cannot cull (the
    //    exact geometry, formed once in step 2, decides them); the other pairs get
    //    zero gradients here
    for (int r = 0; r < rws; ++r) {
      if (!inside) break;
      const float* ps = pos + (s * p.rows + r) * 6;
      const float txp[3] = {ps[0], ps[1], ps[2]};
      const float rxp[3] = {ps[3], ps[4], ps[5]};
      const bool live = active && !surely_culled(txp, rxp, own_nrm, own_pt);
      if (live) {
        list[r * TILE + atomicAdd(&cnt[r], 1)] = threadIdx.x;
      } else {
        p.g_sigmas[(a0 + r) * p.P + pi] = from_f<T>(0.0f);
#pragma unroll
        for (int k = 0; k < NC; ++k) contrib[(r * NC + k) * TILE + threadIdx.x] = 0.0f;
      }
    }
    __syncthreads();

    // 2. every thread takes candidate pairs k = tid, tid + TILE, ... in (row, list) order
    int total = 0;
    for (int r = 0; r < rws; ++r) total += cnt[r];
    int r_cur = 0, r_start = 0;
    for (int k = threadIdx.x; k < total; k += TILE) {
      while (k >= r_start + cnt[r_cur]) {
        r_start += cnt[r_cur];
        ++r_cur;
      }
      const int r = r_cur;
      const int slot = list[r * TILE + (k - r_start)];
      const int64_t pj = p.plist != nullptr ? static_cast<int64_t>(p.plist[p_base + slot]) : p_base + slot;
      const int64_t a = a0 + r;
      float nrm[3], pt[3];
      load3(p.normals, pj, nrm);
      load3(p.points, pj, pt);
      const float* ps = pos + (s * p.rows + r) * 6;
      const float txp[3] = {ps[0], ps[1], ps[2]};
      const float rxp[3] = {ps[3], ps[4], ps[5]};
      SpecGeom geo;
      specular_geometry(txp, rxp, nrm, pt, geo);
      if (culled(geo)) {
        p.g_sigmas[a * p.P + pj] = from_f<T>(0.0f);
#pragma unroll
        for (int c = 0; c < NC; ++c) contrib[(r * NC + c) * TILE + slot] = 0.0f;
        continue;
      }
      const double px = pt[0], py = pt[1], pz = pt[2];
      const PhaseCycles pc = path_cycles(ps[0] - px, ps[1] - py, ps[2] - pz, ps[3] - px,
                                         ps[4] - py, ps[5] - pz, p.k0, p.b0, p.k1, p.b1);
      const float2 zt = cis_cycles(pc.dcyc);
      const T* rowr = stg.stage_ptr(s, 0) + r * p.ld;
      const T* rowi = stg.stage_ptr(s, 1) + r * p.ld;
      float2 qv, q1;  // Q and Q1 = zeta Q'(zeta): packed even/odd Horner in zeta^2
      residual_sums<WITH_POINTS>(rowr, rowi, p.ld, zt, qv, q1);
      const float qr = qv.x, qi = qv.y;
      const float2 e0 = cis_cycles_fast(pc.frac0);
      const float2 eq = cmul(e0, make_float2(qr, qi));
      // sum_n (g_r cos + g_i sin) = Re(exp(j phi0) Q)
      const float sum_re = eq.x;
      const float propagation_distance = path_distance(txp, rxp, pt);
      const float propagation_attenuation = 1.0f / sq(propagation_distance);
      const float sigma_value = ld_f(p.sigmas, a * p.P + pj);
      p.g_sigmas[a * p.P + pj] =
          from_f<T>(propagation_attenuation * geo.align * sum_re / static_cast<float>(p.P));
      float gsa[3];
      align_normal_gradient(geo, nrm, gsa);
      const float normal_scale = sigma_value * propagation_attenuation;
#pragma unroll
      for (int c = 0; c < 3; ++c) contrib[(r * NC + c) * TILE + slot] = normal_scale * gsa[c] * sum_re;
      if (WITH_POINTS) {
        // sum_n w_n (g_i cos - g_r sin) = -Im(exp(j phi0) (w0 Q + w1s Q1))
        const float2 f = cmul(e0, make_float2(w0 * qr + w1s * q1.x, w0 * qi + w1s * q1.y));
        const float amp = sigma_value * geo.align * propagation_attenuation;
        const float d_tau = -amp * f.y;
        const float dist_t = sqrtf(sq(txp[0] - pt[0]) + sq(txp[1] - pt[1]) + sq(txp[2] - pt[2]));
        const float dist_r = sqrtf(sq(rxp[0] - pt[0]) + sq(rxp[1] - pt[1]) + sq(rxp[2] - pt[2]));
        float drho[3];
        align_point_gradient(geo, nrm, dist_t, dist_r, drho);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float dD = geo.inc[c] - geo.ret[c];
          const float damp_dp =
              normal_scale * drho[c] - 2.0f * amp / propagation_distance * dD;
          contrib[(r * NC + 3 + c) * TILE + slot] = sum_re * damp_dp + d_tau * dD / kSpeedOfLight;
        }
      }
    }
    __syncthreads();

    // 3. each owner adds its point's contributions in antenna order
    if (inside) {
      for (int r = 0; r < rws; ++r) {
#pragma unroll
        for (int c = 0; c < 3; ++c) gnorm[c] += contrib[(r * NC + c) * TILE + threadIdx.x];
        if (WITH_POINTS) {
#pragma unroll
          for (int c = 0; c < 3; ++c) gpt[c] += contrib[(r * NC + 3 + c) * TILE + threadIdx.x];
        }
      }
    }
    __syncthreads();
    if (t + 2 < ntiles) issue(t + 2, s);
  }
  if (inside) store_point_grads(p, split, pi, gnorm, gpt, WITH_POINTS);
}

// With a point list, only the listed points' partials are summed (the others'
// gradients were zeroed by the pre-cull).
template <typename T>
__global__ void tracer_bwd_finalize_kernel(const float* __restrict__ partial, int splits, int64_t P,
                                           T* g_normals, T* g_points, const int* plist,
                                           const int* plist_count) {
  const int64_t count = plist != nullptr ? static_cast<int64_t>(*plist_count) : P;
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < count;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = plist != nullptr ? static_cast<int64_t>(plist[k]) : k;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int s = 0; s < splits; ++s) {
      const float* src = partial + (s * P + i) * 6;
      for (int k = 0; k < 6; ++k) acc[k] += src[k];
    }
    const float inv = static_cast<float>(P);
    for (int k = 0; k < 3; ++k) g_normals[i * 3 + k] = from_f<T>(static_cast<float>(acc[k]) / inv);
    if (g_points != nullptr) {
      for (int k = 0; k < 3; ++k) g_points[i * 3 + k] = from_f<T>(static_cast<float>(acc[3 + k]) / inv);
    }
  }
}

// ---------------------------------------------------------------------------
// Along-ray linear resampler (SignalTracer_cuda_kernel.cu:199-349).  One warp
// per ray: the bracketing index and weights of every target depth are found
// once per ray (binary search over the ray's coarse depths) and reused for all
// A sigma rows; arithmetic is in the element type, as in the reference.
template <typename T>
struct BiP {
  const T* normals;
  const T* sigmas;
  const T* z;
  const T* tz;
  T* out_n;
  T* out_s;
  uint8_t* out_inb;
  int64_t A, R, S, T_;
};

template <typename T>
__device__ __forceinline__ int bracket_lower(const T* z, int S, T target) {
  int lower_index = 0;
  int upper_index = S - 1;
  while (lower_index < upper_index - 1) {
    const int mid_index = (lower_index + upper_index) / 2;
    if (z[mid_index] <= target) lower_index = mid_index;
    else upper_index = mid_index;
  }
  return lower_index;
}

template <typename T>
__device__ __forceinline__ T tmax(T a, T b) { return a > b ? a : b; }

// acc + w * g with the product rounded before the sum (never fused), as an
// atomicAdd of a precomputed product does in the reference.
__device__ __forceinline__ float add_product(float acc, float w, float g) {
  return __fadd_rn(acc, __fmul_rn(w, g));
}
__device__ __forceinline__ double add_product(double acc, double w, double g) {
  return __dadd_rn(acc, __dmul_rn(w, g));
}

template <typename T>
__global__ void __launch_bounds__(256) bilinear_fwd_kernel(const BiP<T> p) {
  const int64_t ray = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (ray >= p.R) return;
  const int S = static_cast<int>(p.S);
  const T* z = p.z + ray * p.S;
  const T* nrm = p.normals + ray * p.S * 3;
  for (int64_t t = lane; t < p.T_; t += 32) {
    const T target = p.tz[ray * p.T_ + t];
    const int lo = bracket_lower(z, S, target);
    const T z0 = z[lo];
    const T z1 = z[lo + 1];
    const bool oob = (target < z0) || (target > z1);
    p.out_inb[ray * p.T_ + t] = oob ? 0 : 1;
    T* on = p.out_n + (ray * p.T_ + t) * 3;
    if (oob) {
      on[0] = T(0.0f);
      on[1] = T(0.0f);
      on[2] = T(0.0f);
      for (int64_t a = 0; a < p.A; ++a) p.out_s[(a * p.R + ray) * p.T_ + t] = T(0.0f);
      continue;
    }
    const T weight_upper = (target - z0) / tmax(z1 - z0, static_cast<T>(1.0e-6f));
    const T weight_lower = static_cast<T>(1) - weight_upper;
    for (int axis = 0; axis < 3; ++axis) {
      const T normal_lower = nrm[lo * 3 + axis];
      const T normal_upper = nrm[(lo + 1) * 3 + axis];
      on[axis] = weight_lower * normal_lower + weight_upper * normal_upper;
    }
    for (int64_t a = 0; a < p.A; ++a) {
      const T* sg = p.sigmas + (a * p.R + ray) * p.S;
      p.out_s[(a * p.R + ray) * p.T_ + t] = weight_lower * sg[lo] + weight_upper * sg[lo + 1];
    }
  }
}

// Adjoint, gather form: lane j of the ray's warp owns coarse sample j and adds
// the contributions of the targets bracketing it in target order -- the same
// per-element order as the reference's single-writer atomicAdd sequence --
// onto the existing gradient value.
template <typename T>
__global__ void __launch_bounds__(256) bilinear_bwd_kernel(const BiP<T> p) {
  const int64_t ray = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (ray >= p.R) return;
  const int S = static_cast<int>(p.S);
  const T* z = p.z + ray * p.S;
  // p.normals = grad_output_normals [R,T,3], p.sigmas = grad_output_sigmas [A,R,T]
  for (int j = lane; j < S; j += 32) {
    T gn[3] = {p.out_n[(ray * p.S + j) * 3 + 0], p.out_n[(ray * p.S + j) * 3 + 1],
               p.out_n[(ray * p.S + j) * 3 + 2]};
    for (int64_t t = 0; t < p.T_; ++t) {
      const T target = p.tz[ray * p.T_ + t];
      const int lo = bracket_lower(z, S, target);
      if (lo != j && lo + 1 != j) continue;
      const T z0 = z[lo];
      const T z1 = z[lo + 1];
      if (target < z0 || target > z1) continue;
      const T weight_upper = (target - z0) / tmax(z1 - z0, static_cast<T>(1.0e-6f));
      const T weight_lower = static_cast<T>(1) - weight_upper;
      const T* gno = p.normals + (ray * p.T_ + t) * 3;
      for (int axis = 0; axis < 3; ++axis) {
        if (lo == j) gn[axis] = add_product(gn[axis], weight_lower, gno[axis]);
        if (lo + 1 == j) gn[axis] = add_product(gn[axis], weight_upper, gno[axis]);
      }
    }
    for (int axis = 0; axis < 3; ++axis) p.out_n[(ray * p.S + j) * 3 + axis] = gn[axis];
  }
  for (int64_t a = 0; a < p.A; ++a) {
    const T* gso = p.sigmas + (a * p.R + ray) * p.T_;
    T* gs = p.out_s + (a * p.R + ray) * p.S;
    for (int j = lane; j < S; j += 32) {
      T acc = gs[j];
      for (int64_t t = 0; t < p.T_; ++t) {
        const T target = p.tz[ray * p.T_ + t];
        const int lo = bracket_lower(z, S, target);
        if (lo != j && lo + 1 != j) continue;
        const T z0 = z[lo];
        const T z1 = z[lo + 1];
        if (target < z0 || target > z1) continue;
        const T weight_upper = (target - z0) / tmax(z1 - z0, static_cast<T>(1.0e-6f));
        const T weight_lower = static_cast<T>(1) - weight_upper;
        if (lo == j) acc = add_product(acc, weight_lower, gso[t]);
        if (lo + 1 == j) acc = add_product(acc, weight_upper, gso[t]);
      }
      gs[j] = acc;
    }
  }
}

// ---------------------------------------------------------------------------
bool aligned16(const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; }

template <typename T>
TrP<T> make_params(const TracerArgs& a) {
  TrP<T> p;
  p.normals = static_cast<const T*>(a.normals);
  p.sigmas = static_cast<const T*>(a.sigmas);
  p.points = static_cast<const T*>(a.points);
  p.tx = static_cast<const T*>(a.tx);
  p.rx = static_cast<const T*>(a.rx);
  p.inb = a.inbounds;
  p.out_r = static_cast<T*>(a.out_real);
  p.out_i = static_cast<T*>(a.out_imag);
  p.gr = static_cast<const T*>(a.grad_real_out);
  p.gi = static_cast<const T*>(a.grad_imag_out);
  p.g_normals = static_cast<T*>(a.grad_normals);
  p.g_sigmas = static_cast<T*>(a.grad_sigmas);
  p.g_points = static_cast<T*>(a.grad_points);
  p.partial = nullptr;
  p.status = device_status_ptr();
  p.A = a.A;
  p.S = a.S;
  p.P = a.P;
  p.fs = a.fs;
  p.f0 = a.f0;
  p.As = a.As;
  const PhaseConsts pc = phase_consts(a.f0, a.As, a.fs);
  p.k0 = pc.k0;
  p.b0 = pc.b0;
  p.k1 = pc.k1;
  p.b1 = pc.b1;
  p.splits = 1;
  p.per_split = 0;
  p.groups = 1;
  p.rows = 1;
  p.ld = 4;
  p.bulk = 0;
  p.pos_off = p.buf_off = 0;
  p.plist = nullptr;
  p.plist_count = nullptr;
  return p;
}

// Sample groups per block (power of two, at most 64: shared-memory bound).
int fwd_groups(int64_t S, int chunk, int threads) {
  const int64_t g = (S + chunk - 1) / chunk;
  int groups = 1;
  while (groups < g && groups < threads && groups < 64) groups *= 2;
  return groups;
}

template <typename T, int K>
cudaError_t launch_tr_fwd_mixed_k(const TrP<T>& p, dim3 grid, int threads, size_t smem,
                                  cudaStream_t st) {
  const void* fn = reinterpret_cast<const void*>(&tracer_fwd_mixed_kernel<T, K>);
  cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  void* args[] = {const_cast<TrP<T>*>(&p)};
  return cudaLaunchKernel(fn, grid, dim3(threads), args, smem, st);
}

size_t fwd_mixed_smem(int threads, int groups, int chunk) {
  const size_t seeds = (static_cast<size_t>(groups) + 1) * threads * sizeof(float2) + 33 * sizeof(int);
  const size_t red = static_cast<size_t>(threads) * chunk * sizeof(float2);
  return std::max(seeds, red);
}

// Workspace of the MIXED forward and adjoint: the split partials, then (when the
// pre-cull applies) the point list region.
size_t list_region_offset(size_t partial_bytes) { return (partial_bytes + 255) & ~static_cast<size_t>(255); }

template <typename T>
cudaError_t launch_tracer_fwd(const TracerArgs& a, const Tuning& t, void* ws, cudaStream_t st) {
  TrP<T> p = make_params<T>(a);
  p.partial = static_cast<float*>(ws);
  if (a.mode == kPlain) {
    const int threads = 128;
    dim3 grid(static_cast<unsigned>(a.A), static_cast<unsigned>((a.S + threads - 1) / threads));
    tracer_fwd_plain_kernel<T><<<grid, threads, 0, st>>>(p);
    return cudaGetLastError();
  }
  const int threads = t.threads;
  const int chunk = t.chunk;
  const int groups = fwd_groups(a.S, chunk, threads);
  p.groups = groups;
  p.splits = t.splits;
  p.per_split = (a.P + t.splits - 1) / t.splits;
  const int64_t ranges = (a.S + static_cast<int64_t>(groups) * chunk - 1) /
                         (static_cast<int64_t>(groups) * chunk);
  dim3 grid(static_cast<unsigned>(a.A * t.splits), static_cast<unsigned>(ranges));
  const size_t smem = fwd_mixed_smem(threads, groups, chunk);
  cudaError_t err;
  if (tracer_point_list_applies(a)) {
    const size_t partial_bytes = t.splits > 1 ? static_cast<size_t>(t.splits) * a.A * a.S * 2 * sizeof(float) : 0;
    void* lws = static_cast<unsigned char*>(ws) + list_region_offset(partial_bytes);
    err = tracer_point_list(a, lws, false, st);
    if (err != cudaSuccess) return err;
    const PointList pl = tracer_point_list_view(lws, a.P);
    p.plist = pl.list;
    p.plist_count = pl.count;
  }
  if (chunk == 8) err = launch_tr_fwd_mixed_k<T, 8>(p, grid, threads, smem, st);
  else if (chunk == 32) err = launch_tr_fwd_mixed_k<T, 32>(p, grid, threads, smem, st);
  else err = launch_tr_fwd_mixed_k<T, 16>(p, grid, threads, smem, st);
  if (err != cudaSuccess) return err;
  if (t.splits > 1) {
    const int64_t count = a.A * a.S;
    const int fin_blocks = static_cast<int>(std::min<int64_t>((count + 255) / 256, 148 * 16));
    tracer_fwd_finalize_kernel<T><<<std::max(fin_blocks, 1), 256, 0, st>>>(
        p.partial, t.splits, count, static_cast<float>(a.P), p.out_r, p.out_i);
    err = cudaGetLastError();
  }
  return err;
}

template <typename T>
cudaError_t launch_tracer_bwd(const TracerArgs& a, const Tuning& t, void* ws, cudaStream_t st) {
  TrP<T> p = make_params<T>(a);
  p.partial = static_cast<float*>(ws);
  const int threads = t.threads;
  p.splits = t.splits;
  const int64_t rows_total = std::max<int64_t>(1, (a.A + t.stage_rows - 1) / t.stage_rows);
  p.per_split = ((rows_total + t.splits - 1) / t.splits) * t.stage_rows;
  p.ld = static_cast<int>(((std::max<int64_t>(a.S, 1) + 3) / 4) * 4);
  const size_t es = a.dtype == kF64 ? 8 : 4;
  p.bulk = (a.S > 0 && a.S % 4 == 0 && (a.S * es) % 16 == 0 && aligned16(a.grad_real_out) &&
            aligned16(a.grad_imag_out))
               ? 1
               : 0;
  int rows = t.stage_rows;
  const bool with_points = a.grad_points != nullptr;
  const int nc = with_points ? 6 : 3;
  auto layout = [&](int rw) {
    if (a.mode == kPlain) {
      const AdjSmem b = adj_smem_layout<T>(rw, p.ld);
      return AdjMixedSmem{b.pos_off, b.buf_off, 0, 0, 0, b.total};
    }
    return adj_mixed_smem_layout<T>(rw, p.ld, threads, nc);
  };
  AdjMixedSmem lay = layout(rows);
  const DeviceInfo dev = current_device_info();
  while (rows > 1 && lay.total > static_cast<size_t>(dev.max_smem_optin)) {
    rows /= 2;
    lay = layout(rows);
  }
  if (rows != t.stage_rows) {
    p.per_split = ((std::max<int64_t>(1, (a.A + rows - 1) / rows) + t.splits - 1) / t.splits) * rows;
  }
  p.rows = rows;
  p.pos_off = lay.pos_off;
  p.buf_off = lay.buf_off;
  p.cnt_off = lay.cnt_off;
  p.list_off = lay.list_off;
  p.contrib_off = lay.contrib_off;
  const void* fn;
  if (a.mode == kPlain) {
    fn = with_points ? reinterpret_cast<const void*>(&tracer_bwd_plain_kernel<T, true>)
                     : reinterpret_cast<const void*>(&tracer_bwd_plain_kernel<T, false>);
  } else {
    fn = with_points ? reinterpret_cast<const void*>(&tracer_bwd_mixed_kernel<T, true>)
                     : reinterpret_cast<const void*>(&tracer_bwd_mixed_kernel<T, false>);
  }
  cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(lay.total));
  if (err != cudaSuccess) return err;
  const int64_t ptiles = (a.P + threads - 1) / threads;
  const int64_t blocks = ptiles * t.splits;
  if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
  if (a.mode == kMixed && tracer_point_list_applies(a)) {
    // lists the points and zeroes the gradients of every point it leaves out
    const size_t partial_bytes = t.splits > 1 ? static_cast<size_t>(t.splits) * a.P * 6 * sizeof(float) : 0;
    void* lws = static_cast<unsigned char*>(ws) + list_region_offset(partial_bytes);
    err = tracer_point_list(a, lws, true, st);
    if (err != cudaSuccess) return err;
    const PointList pl = tracer_point_list_view(lws, a.P);
    p.plist = pl.list;
    p.plist_count = pl.count;
  }
  void* args[] = {&p};
  err = cudaLaunchKernel(fn, dim3(static_cast<unsigned>(blocks)), dim3(threads), args, lay.total, st);
  if (err != cudaSuccess) return err;
  if (t.splits > 1) {
    const int fin_blocks = static_cast<int>(std::min<int64_t>((a.P + 255) / 256, 148 * 16));
    tracer_bwd_finalize_kernel<T><<<std::max(fin_blocks, 1), 256, 0, st>>>(
        p.partial, t.splits, a.P, p.g_normals, with_points ? p.g_points : nullptr, p.plist, p.plist_count);
    err = cudaGetLastError();
  }
  return err;
}

template <typename T>
BiP<T> make_bi(const BilinearArgs& a) {
  BiP<T> p;
  p.normals = static_cast<const T*>(a.normals);
  p.sigmas = static_cast<const T*>(a.sigmas);
  p.z = static_cast<const T*>(a.z_vals);
  p.tz = static_cast<const T*>(a.tz_vals);
  p.out_n = static_cast<T*>(a.out_normals);
  p.out_s = static_cast<T*>(a.out_sigmas);
  p.out_inb = a.out_inbounds;
  p.A = a.A;
  p.R = a.R;
  p.S = a.S;
  p.T_ = a.T;
  return p;
}

}  // namespace

// ---------------------------------------------------------------------------
cudaError_t launch_tracer_bwd_finalize(int dtype, const float* partial, int splits, int64_t P, void* g_normals,
                                       void* g_points, cudaStream_t st, const int* plist,
                                       const int* plist_count) {
  const int blocks = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((P + 255) / 256, 148 * 16)));
  if (dtype == kF64) {
    tracer_bwd_finalize_kernel<double><<<blocks, 256, 0, st>>>(partial, splits, P, static_cast<double*>(g_normals),
                                                               static_cast<double*>(g_points), plist, plist_count);
  } else {
    tracer_bwd_finalize_kernel<float><<<blocks, 256, 0, st>>>(partial, splits, P, static_cast<float*>(g_normals),
                                                              static_cast<float*>(g_points), plist, plist_count);
  }
  return cudaGetLastError();
}

// Resident blocks per SM of the MIXED forward at this shape, from the occupancy
// calculator; the thread-count bound when no device answers.
int tr_fwd_blocks_per_sm(const TracerArgs& a, const Tuning& t, int groups) {
  const bool f64 = a.dtype == kF64;
  const void* fn = t.chunk == 8    ? (f64 ? reinterpret_cast<const void*>(&tracer_fwd_mixed_kernel<double, 8>)
                                          : reinterpret_cast<const void*>(&tracer_fwd_mixed_kernel<float, 8>))
                   : t.chunk == 32 ? (f64 ? reinterpret_cast<const void*>(&tracer_fwd_mixed_kernel<double, 32>)
                                          : reinterpret_cast<const void*>(&tracer_fwd_mixed_kernel<float, 32>))
                                   : (f64 ? reinterpret_cast<const void*>(&tracer_fwd_mixed_kernel<double, 16>)
                                          : reinterpret_cast<const void*>(&tracer_fwd_mixed_kernel<float, 16>));
  const size_t smem = fwd_mixed_smem(t.threads, groups, t.chunk);
  int n = 0;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
          cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, t.threads, smem) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return std::max(1, 512 / t.threads);
  }
  return n;
}

Tuning tracer_forward_resolve(const TracerArgs& a, const Tuning& req) {
  if (a.mode == kNufft) return tracer_nufft_forward_resolve(a, req);
  Tuning t = req;
  // MIXED: 64-thread blocks of 16-sample chunks (measured on B200 for 64 antennas x
  // 524288 points x 128 samples with the point pre-cull: 12% faster than 8-sample
  // chunks, which led before it; 256-thread blocks are slower).  Small blocks stall
  // fewer warps at the per-tile compaction barriers.
  if (t.threads != 64 && t.threads != 128 && t.threads != 256) t.threads = a.mode == kMixed ? 64 : 256;
  if (t.chunk != 8 && t.chunk != 16 && t.chunk != 32) t.chunk = 16;
  if (t.items <= 0) t.items = 1;
  if (t.stage_rows <= 0) t.stage_rows = 8;
  if (a.mode == kPlain) {
    t.splits = 1;
    return t;
  }
  const int groups = fwd_groups(a.S, t.chunk, t.threads);
  const int64_t ranges = (a.S + static_cast<int64_t>(groups) * t.chunk - 1) /
                         (static_cast<int64_t>(groups) * t.chunk);
  const int64_t ptiles = std::max<int64_t>(1, (a.P + t.threads - 1) / t.threads);
  if (t.splits <= 0) {
    const DeviceInfo dev = current_device_info();
    t.splits = pick_splits(std::max<int64_t>(1, a.A * ranges), tr_fwd_blocks_per_sm(a, t, groups),
                           dev.sm_count, ptiles);
  }
  t.splits = static_cast<int>(std::min<int64_t>(std::max(t.splits, 1), ptiles));
  return t;
}

size_t tracer_forward_workspace(const TracerArgs& a, const Tuning& t) {
  if (a.mode == kNufft) return tracer_nufft_forward_workspace(a, t);
  if (a.mode == kPlain) return 0;
  const size_t partial_bytes = t.splits > 1 ? static_cast<size_t>(t.splits) * a.A * a.S * 2 * sizeof(float) : 0;
  if (!tracer_point_list_applies(a)) return partial_bytes;
  return list_region_offset(partial_bytes) + tracer_point_list_bytes(a.P);
}

cudaError_t tracer_forward(const TracerArgs& a, const Tuning& t, void* ws, cudaStream_t st) {
  if (a.mode == kNufft) return tracer_nufft_forward(a, t, ws, st);
  if (a.A == 0 || a.S == 0) return cudaSuccess;
  if (a.dtype == kF64) return launch_tracer_fwd<double>(a, t, ws, st);
  return launch_tracer_fwd<float>(a, t, ws, st);
}

Tuning tracer_backward_resolve(const TracerArgs& a, const Tuning& req) {
  if (a.mode == kNufft) return tracer_nufft_backward_resolve(a, req);
  Tuning t = req;
  if (t.threads != 64 && t.threads != 128) t.threads = 128;
  if (t.items <= 0) t.items = 1;
  // MIXED: 4-antenna stages keep 6 blocks resident per SM (8 fit 4, by shared
  // memory); 5% faster on 64 antennas x 524288 points x 128 samples
  if (t.stage_rows <= 0) t.stage_rows = a.mode == kMixed ? 4 : 8;
  t.stage_rows = std::min(t.stage_rows, 64);
  if (t.chunk <= 0) t.chunk = 16;
  const int64_t rows_total = std::max<int64_t>(1, (a.A + t.stage_rows - 1) / t.stage_rows);
  if (t.splits <= 0) {
    int64_t ptiles = std::max<int64_t>(1, (a.P + t.threads - 1) / t.threads);
    // With the point pre-cull only the blocks of listed points have work; the
    // default assumes a quarter of the points are listed (14% on 64 antennas
    // looking at a 4096-ray SDF scene).
    if (a.mode == kMixed && tracer_point_list_applies(a)) ptiles = std::max<int64_t>(1, ptiles / 4);
    const DeviceInfo dev = current_device_info();
    const int per_sm = std::max(1, 1024 / t.threads);
    t.splits = a.mode == kPlain ? 1 : pick_splits(ptiles, per_sm, dev.sm_count, rows_total);
  }
  t.splits = static_cast<int>(std::min<int64_t>(std::max(t.splits, 1), rows_total));
  return t;
}

size_t tracer_backward_workspace(const TracerArgs& a, const Tuning& t) {
  if (a.mode == kNufft) return tracer_nufft_backward_workspace(a, t);
  const size_t partial_bytes = t.splits > 1 && a.P > 0 ? static_cast<size_t>(t.splits) * a.P * 6 * sizeof(float) : 0;
  if (!tracer_point_list_applies(a)) return partial_bytes;
  return list_region_offset(partial_bytes) + tracer_point_list_bytes(a.P);
}

cudaError_t tracer_backward(const TracerArgs& a, const Tuning& t, void* ws, cudaStream_t st) {
  if (a.mode == kNufft) return tracer_nufft_backward(a, t, ws, st);
  if (a.P == 0) return cudaSuccess;
  if (a.dtype == kF64) return launch_tracer_bwd<double>(a, t, ws, st);
  return launch_tracer_bwd<float>(a, t, ws, st);
}

cudaError_t bilinear_forward(const BilinearArgs& a, cudaStream_t st) {
  if (a.R == 0 || a.T == 0) return cudaSuccess;
  const int64_t blocks = (a.R * 32 + 255) / 256;
  if (a.dtype == kF64) bilinear_fwd_kernel<double><<<static_cast<unsigned>(blocks), 256, 0, st>>>(make_bi<double>(a));
  else bilinear_fwd_kernel<float><<<static_cast<unsigned>(blocks), 256, 0, st>>>(make_bi<float>(a));
  return cudaGetLastError();
}

cudaError_t bilinear_backward(const BilinearArgs& a, cudaStream_t st) {
  if (a.R == 0 || a.S == 0) return cudaSuccess;
  const int64_t blocks = (a.R * 32 + 255) / 256;
  if (a.dtype == kF64) bilinear_bwd_kernel<double><<<static_cast<unsigned>(blocks), 256, 0, st>>>(make_bi<double>(a));
  else bilinear_bwd_kernel<float><<<static_cast<unsigned>(blocks), 256, 0, st>>>(make_bi<float>(a));
  return cudaGetLastError();
}

}  // namespace geraf
