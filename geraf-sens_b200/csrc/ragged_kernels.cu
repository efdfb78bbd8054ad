// Batched signal tracer over all antennas of a step, each antenna with its own
// uneven set of points (rays x samples surviving the filter-based culling),
// in the MIXED arithmetic form.
//
// Layout: points / normals [P, 3], sigmas [P] and inbounds [P] hold the points
// of antenna 0, then antenna 1, ... ; point_offsets [A + 1] (int64, CSR) gives
// antenna a the points [offsets[a], offsets[a+1]).  Per antenna the result is
// exactly the reference's tracer over that antenna's points:
//   x[a, n] = (1 / P_a) sum_{p of a} sigma[p] rho / D^2 exp(+j (w0 + w1 t_n) tau)
// (SignalTracer_cuda_kernel.cu:351-450 with total_point_size = P_a).
//
// Forward: one persistent launch.  A one-block prep pass validates the
// offsets and lays out work items (antenna, chunk of `chunk` points); resident
// blocks then take items from an atomic counter until none are left, so
// antennas with 512 rays and antennas with 8192 rays load-balance; a finish
// pass sums each antenna's item partials in item order (deterministic).
// Adjoint: a point belongs to one antenna, so its gradients need no reduction
// across antennas; blocks screen tiles of points and deal the live ones out
// over their threads.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "tracer_geometry.cuh"

namespace geraf {
namespace {

using namespace tracer;

constexpr int kStatusBadOffsets = 1;  // GERAF_ERR_INVALID_ARGUMENT

template <typename T>
struct RgP {
  const T* normals;
  const T* sigmas;
  const T* points;
  const int64_t* offsets;
  const T* tx;
  const T* rx;
  const uint8_t* inb;  // may be null: all points in bounds
  T* out_r;
  T* out_i;
  const T* gr;
  const T* gi;
  T* g_normals;
  T* g_sigmas;
  T* g_points;
  float2* partial;        // [max_items][S]
  int64_t* item_offsets;  // [A + 1]
  unsigned long long* counter;
  int* status;
  int64_t A, S, P, max_items;
  int chunk, groups;
  float fs, f0, As;
  double k0, b0, k1, b1;
};

template <typename T>
__device__ __forceinline__ void ld3(const T* base, int64_t i, float* out) {
  out[0] = ld_f(base, i * 3 + 0);
  out[1] = ld_f(base, i * 3 + 1);
  out[2] = ld_f(base, i * 3 + 2);
}

// Validates the CSR offsets and writes item_offsets (prefix sums of
// ceil(P_a / chunk)); resets the work counter.  Malformed offsets give zero
// items and raise the status word, so nothing downstream reads a point.
template <typename T>
__global__ void __launch_bounds__(1024) ragged_prep_kernel(const RgP<T> p) {
  __shared__ int bad;
  __shared__ long long carry;
  if (threadIdx.x == 0) {
    bad = (p.offsets[0] != 0 || p.offsets[p.A] != p.P) ? 1 : 0;
    carry = 0;
    *p.counter = 0ull;
  }
  __syncthreads();
  for (int64_t a = threadIdx.x; a < p.A; a += blockDim.x) {
    if (p.offsets[a + 1] < p.offsets[a]) bad = 1;
  }
  __syncthreads();
  if (bad) {
    for (int64_t a = threadIdx.x; a <= p.A; a += blockDim.x) p.item_offsets[a] = 0;
    if (threadIdx.x == 0 && p.status != nullptr) atomicExch(p.status, kStatusBadOffsets);
    return;
  }
  // Block-wide exclusive scan of item counts, blockDim antennas at a time.
  __shared__ long long warp_sums[32];
  for (int64_t base = 0; base < p.A; base += blockDim.x) {
    const int64_t a = base + threadIdx.x;
    long long cnt = 0;
    if (a < p.A) cnt = (p.offsets[a + 1] - p.offsets[a] + p.chunk - 1) / p.chunk;
    long long incl = cnt;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = 1; d < 32; d <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += y;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const int nw = blockDim.x >> 5;
      long long v = lane < nw ? warp_sums[lane] : 0;
      for (int d = 1; d < 32; d <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += y;
      }
      if (lane < nw) warp_sums[lane] = v;
    }
    __syncthreads();
    const long long before = (warp > 0 ? warp_sums[warp - 1] : 0) + carry;
    if (a < p.A) p.item_offsets[a] = before + incl - cnt;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = before + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) p.item_offsets[p.A] = carry;
}

// Antenna owning work item `item`: the last a with item_offsets[a] <= item.
__device__ __forceinline__ int64_t item_antenna(const int64_t* item_offsets, int64_t A, int64_t item) {
  int64_t lo = 0, hi = A;  // invariant: item_offsets[lo] <= item < item_offsets[hi]
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (item_offsets[mid] <= item) lo = mid;
    else hi = mid;
  }
  return lo;
}

template <typename T, int K>
__global__ void __launch_bounds__(256) ragged_fwd_kernel(const RgP<T> p) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int TILE = blockDim.x;
  const int G = p.groups;
  const int L = blockDim.x / G;
  float2* seeds = reinterpret_cast<float2*>(smem);       // [G][TILE]
  float2* zeta = seeds + static_cast<size_t>(G) * TILE;  // [TILE]
  int* warp_base = reinterpret_cast<int*>(zeta + TILE);  // [33]
  __shared__ long long s_item;

  const int g = threadIdx.x / L;
  const int l = threadIdx.x - g * L;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const int64_t total = p.item_offsets[p.A];

  for (;;) {
    if (threadIdx.x == 0) s_item = static_cast<long long>(atomicAdd(p.counter, 1ull));
    __syncthreads();
    const int64_t item = s_item;
    __syncthreads();
    if (item >= total) break;
    const int64_t a = item_antenna(p.item_offsets, p.A, item);
    const int64_t c = item - p.item_offsets[a];
    const int64_t pt_begin = p.offsets[a] + c * p.chunk;
    const int64_t pt_end = min(p.offsets[a + 1], pt_begin + p.chunk);
    float txp[3], rxp[3];
    ld3(p.tx, a, txp);
    ld3(p.rx, a, rxp);
    const double tx = txp[0], ty = txp[1], tz = txp[2], rx = rxp[0], ry = rxp[1], rz = rxp[2];

    float2 acc[K], hi[K];
#pragma unroll
    for (int m = 0; m < K; ++m) acc[m] = hi[m] = make_float2(0.0f, 0.0f);

    // The point data of tile k + 1 are loaded while tile k's samples are summed.
    float nrm[3] = {0.0f, 0.0f, 1.0f}, pt[3] = {0.0f, 0.0f, 0.0f}, sig = 0.0f;
    bool inb = false;
    auto load_point = [&](int64_t q) {
      inb = q < pt_end && (p.inb == nullptr || p.inb[q]);
      if (inb) {
        ld3(p.normals, q, nrm);
        ld3(p.points, q, pt);
        sig = ld_f(p.sigmas, q);
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
          const PhaseCycles pc = path_cycles(tx - px, ty - py, tz - pz, rx - px, ry - py, rz - pz,
                                             p.k0, p.b0, p.k1, p.b1);
          const float2 e = cis_cycles(pc.frac0);
          w = make_float2(amp * e.x, amp * e.y);
          zt = cis_cycles(pc.dcyc);
          const float kc = pc.dcyc * static_cast<float>(K);
          zk = cis_cycles(kc - rintf(kc));
          valid = true;
        }
      }
      const unsigned ballot = __ballot_sync(0xffffffffu, valid);
      if (lane == 0) warp_base[warp] = __popc(ballot);
      __syncthreads();
      if (threadIdx.x == 0) {
        int run = 0;
        for (int wi = 0; wi < nwarps; ++wi) {
          const int cnt = warp_base[wi];
          warp_base[wi] = run;
          run += cnt;
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
    // Reduce the lanes of each sample group and store this item's partial row.
    float2* red = reinterpret_cast<float2*>(smem);  // [G][K][L]
#pragma unroll
    for (int m = 0; m < K; ++m) red[(g * K + m) * L + l] = hi[m];
    __syncthreads();
    for (int idx = threadIdx.x; idx < G * K; idx += blockDim.x) {
      if (idx >= p.S) continue;
      float sr = 0.0f, si = 0.0f;
      for (int ll = 0; ll < L; ++ll) {
        const float2 v = red[idx * L + ll];
        sr += v.x;
        si += v.y;
      }
      p.partial[item * p.S + idx] = make_float2(sr, si);
    }
    __syncthreads();
  }
}

// x[a, n] = (sum of antenna a's item partials, in item order) / P_a.
template <typename T>
__global__ void ragged_finish_kernel(const RgP<T> p) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < p.A * p.S;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t a = i / p.S;
    const int64_t n = i - a * p.S;
    double sr = 0.0, si = 0.0;
    for (int64_t it = p.item_offsets[a]; it < p.item_offsets[a + 1]; ++it) {
      const float2 v = p.partial[it * p.S + n];
      sr += v.x;
      si += v.y;
    }
    const float pa = static_cast<float>(p.offsets[a + 1] - p.offsets[a]);
    p.out_r[i] = from_f<T>(static_cast<float>(sr) / pa);
    p.out_i[i] = from_f<T>(static_cast<float>(si) / pa);
  }
}

// Antenna owning point pi: the last a with offsets[a] <= pi.  *owned is false
// when the offsets do not cover pi (malformed input).
__device__ __forceinline__ int64_t point_antenna(const int64_t* offsets, int64_t A, int64_t pi,
                                                 bool* owned) {
  int64_t lo = 0, hi = A;
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (offsets[mid] <= pi) lo = mid;
    else hi = mid;
  }
  *owned = A > 0 && offsets[lo] <= pi && pi < offsets[lo + 1];
  return lo;
}

// Gradients of one in-bounds point pi of antenna a that the early test cannot
// cull (zeros when its exact geometry culls it).  The residual row comes from
// shared memory (rr, ri: ld floats each) or, when rr is null, from global
// memory.
template <typename T, bool WITH_POINTS>
__device__ __forceinline__ void ragged_point_grads(const RgP<T>& p, int64_t pi, int64_t a, const float* rr,
                                                   const float* ri, int ld) {
  float nrm[3], pt[3], txp[3], rxp[3];
  ld3(p.normals, pi, nrm);
  ld3(p.points, pi, pt);
  ld3(p.tx, a, txp);
  ld3(p.rx, a, rxp);
  SpecGeom geo;
  specular_geometry(txp, rxp, nrm, pt, geo);
  if (culled(geo)) {  // a candidate the exact geometry culls
    p.g_sigmas[pi] = from_f<T>(0.0f);
#pragma unroll
    for (int q = 0; q < 3; ++q) p.g_normals[pi * 3 + q] = from_f<T>(0.0f);
    if (WITH_POINTS) {
#pragma unroll
      for (int q = 0; q < 3; ++q) p.g_points[pi * 3 + q] = from_f<T>(0.0f);
    }
    return;
  }
  const double px = pt[0], py = pt[1], pz = pt[2];
  const PhaseCycles pc = path_cycles(txp[0] - px, txp[1] - py, txp[2] - pz, rxp[0] - px, rxp[1] - py,
                                     rxp[2] - pz, p.k0, p.b0, p.k1, p.b1);
  const float2 zt = cis_cycles(pc.dcyc);
  float qr = 0.0f, qi = 0.0f, dr = 0.0f, di = 0.0f;
  float2 q1 = make_float2(0.0f, 0.0f);
  auto step = [&](float cr, float ci) {
    if (WITH_POINTS) {
      const float ndr = fmaf(dr, zt.x, fmaf(-di, zt.y, qr));
      const float ndi = fmaf(dr, zt.y, fmaf(di, zt.x, qi));
      dr = ndr;
      di = ndi;
    }
    const float nqr = fmaf(qr, zt.x, fmaf(-qi, zt.y, cr));
    const float nqi = fmaf(qr, zt.y, fmaf(qi, zt.x, -ci));
    qr = nqr;
    qi = nqi;
  };
  if (rr != nullptr) {
    // staged row: packed even/odd Horner in zeta^2
    float2 qv;
    residual_sums<WITH_POINTS>(rr, ri, ld, zt, qv, q1);
    qr = qv.x;
    qi = qv.y;
  } else {
    // row read from global memory: scalar Horner, Q1 = zeta Q'(zeta) from its derivative chain
    for (int64_t n = p.S - 1; n >= 0; --n) step(ld_f(p.gr, a * p.S + n), ld_f(p.gi, a * p.S + n));
    q1 = cmul(zt, make_float2(dr, di));
  }
  const float inv_pa = 1.0f / static_cast<float>(p.offsets[a + 1] - p.offsets[a]);
  const float2 e0 = cis_cycles(pc.frac0);
  const float sum_re = cmul(e0, make_float2(qr, qi)).x;
  const float propagation_distance = path_distance(txp, rxp, pt);
  const float atten = 1.0f / sq(propagation_distance);
  const float sigma_value = ld_f(p.sigmas, pi);
  p.g_sigmas[pi] = from_f<T>(atten * geo.align * sum_re * inv_pa);
  float gsa[3];
  align_normal_gradient(geo, nrm, gsa);
  const float normal_scale = sigma_value * atten;
#pragma unroll
  for (int k = 0; k < 3; ++k) p.g_normals[pi * 3 + k] = from_f<T>(normal_scale * gsa[k] * sum_re * inv_pa);
  if (WITH_POINTS) {
    const float w0 = static_cast<float>(2.0 * static_cast<double>(kPiF) * p.f0);
    const float w1s = static_cast<float>(2.0 * static_cast<double>(kPiF) * p.As / p.fs);
    const float2 f = cmul(e0, make_float2(w0 * qr + w1s * q1.x, w0 * qi + w1s * q1.y));
    const float amp = sigma_value * geo.align * atten;
    const float d_tau = -amp * f.y;
    const float dist_t = sqrtf(sq(txp[0] - pt[0]) + sq(txp[1] - pt[1]) + sq(txp[2] - pt[2]));
    const float dist_r = sqrtf(sq(rxp[0] - pt[0]) + sq(rxp[1] - pt[1]) + sq(rxp[2] - pt[2]));
    float drho[3];
    align_point_gradient(geo, nrm, dist_t, dist_r, drho);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float dD = geo.inc[k] - geo.ret[k];
      const float damp_dp = normal_scale * drho[k] - 2.0f * amp / propagation_distance * dD;
      p.g_points[pi * 3 + k] = from_f<T>((sum_re * damp_dp + d_tau * dD / kSpeedOfLight) * inv_pa);
    }
  }
}

// Adjoint.  A block screens kBwdTile consecutive points, kBwdCand per thread:
// it finds each point's antenna, applies the early cull test, and writes zero
// gradients for culled, out-of-bounds and unowned points; the other points are
// listed in shared memory and then dealt out over the block, so every lane forms
// a listed point's exact geometry and, unless that culls it, runs its full
// sample recurrence (packed even/odd Horner, residual_sums).  (About 60% of a typical
// step's points are live; with one point per thread 40% of the lanes would sit
// out the recurrence.)  A point's gradients depend on that point only, so the
// results do not depend on the list order.  Residual rows of the antennas the
// tile spans are staged in shared memory when there are few of them (points
// are grouped by antenna, so a tile usually lies within one antenna).
constexpr int kBwdThreads = 128;
constexpr int kBwdCand = 8;
constexpr int kBwdTile = kBwdThreads * kBwdCand;

template <typename T, bool WITH_POINTS>
__global__ void __launch_bounds__(kBwdThreads) ragged_bwd_kernel(const RgP<T> p, int ld, int max_rows) {
  extern __shared__ __align__(16) float srow[];  // [max_rows][2][ld]
  __shared__ int s_live[kBwdTile];
  __shared__ int s_nlive;
  __shared__ long long s_a0, s_a1;
  __shared__ int s_single;
  const int64_t base = blockIdx.x * static_cast<int64_t>(kBwdTile);
  const int lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    bool owned0, owned1;
    s_nlive = 0;
    s_a0 = point_antenna(p.offsets, p.A, base, &owned0);
    s_a1 = point_antenna(p.offsets, p.A, min(p.P, base + kBwdTile) - 1, &owned1);
    // Both ends owned by one antenna: with offsets[a] <= first <= pi <= last <
    // offsets[a + 1], that antenna owns every point between, no search needed.
    s_single = owned0 && owned1 && s_a0 == s_a1;
  }
  __syncthreads();
  const bool single = s_single != 0;
  const int64_t a_single = s_a0;
  for (int k = 0; k < kBwdCand; ++k) {
    const int c = threadIdx.x + k * kBwdThreads;
    const int64_t pi = base + c;
    bool live = false;
    if (pi < p.P) {
      bool owned = true;
      const int64_t a = single ? a_single : point_antenna(p.offsets, p.A, pi, &owned);
      if (!owned && p.status != nullptr) atomicExch(p.status, kStatusBadOffsets);
      if (owned && (p.inb == nullptr || p.inb[pi])) {
        float nrm[3], pt[3], txp[3], rxp[3];
        ld3(p.normals, pi, nrm);
        ld3(p.points, pi, pt);
        ld3(p.tx, a, txp);
        ld3(p.rx, a, rxp);
        // a candidate: the exact geometry, formed once when its gradients are, decides it
        live = !surely_culled(txp, rxp, nrm, pt);
      }
      if (!live) {
        p.g_sigmas[pi] = from_f<T>(0.0f);
#pragma unroll
        for (int q = 0; q < 3; ++q) p.g_normals[pi * 3 + q] = from_f<T>(0.0f);
        if (WITH_POINTS) {
#pragma unroll
          for (int q = 0; q < 3; ++q) p.g_points[pi * 3 + q] = from_f<T>(0.0f);
        }
      }
    }
    const unsigned ballot = __ballot_sync(0xffffffffu, live);
    if (ballot != 0u) {
      int wbase = 0;
      if (lane == 0) wbase = atomicAdd(&s_nlive, __popc(ballot));
      wbase = __shfl_sync(0xffffffffu, wbase, 0);
      if (live) s_live[wbase + __popc(ballot & ((1u << lane) - 1u))] = c;
    }
  }
  const int64_t a0 = s_a0;
  const int64_t a1 = max(s_a0, s_a1);
  const bool staged = p.A > 0 && (a1 - a0 + 1) <= max_rows;
  if (staged) {
    const int rows = static_cast<int>(a1 - a0 + 1);
    for (int i = threadIdx.x; i < rows * ld; i += kBwdThreads) {
      const int r = i / ld, c = i - r * ld;
      float vr = 0.0f, vi = 0.0f;
      if (c < p.S) {
        vr = ld_f(p.gr, (a0 + r) * p.S + c);
        vi = ld_f(p.gi, (a0 + r) * p.S + c);
      }
      srow[(r * 2 + 0) * ld + c] = vr;
      srow[(r * 2 + 1) * ld + c] = vi;
    }
  }
  __syncthreads();
  const int nlive = s_nlive;
  for (int i = threadIdx.x; i < nlive; i += kBwdThreads) {
    const int64_t pi = base + s_live[i];
    bool owned;
    const int64_t a = single ? a_single : point_antenna(p.offsets, p.A, pi, &owned);
    // A row outside the staged span (possible only with non-monotonic offsets) is read from global memory.
    const bool row_staged = staged && a >= a0 && a <= a1;
    const float* rr = row_staged ? srow + ((a - a0) * 2 + 0) * ld : nullptr;
    const float* ri = row_staged ? srow + ((a - a0) * 2 + 1) * ld : nullptr;
    ragged_point_grads<T, WITH_POINTS>(p, pi, a, rr, ri, ld);
  }
}

// ---------------------------------------------------------------------------
struct RaggedLayout {
  int64_t max_items;
  size_t partial_off, items_off, counter_off, total;
  int chunk;
};

// Points per work item: items_per_thread x threads when tuned, else at least
// 2048 and more for large steps (fewer partial rows); a multiple of 256.
int ragged_chunk(int64_t P, const Tuning& t) {
  int64_t c = t.items > 0 ? static_cast<int64_t>(t.items) * t.threads
                          : std::max<int64_t>(2048, std::min<int64_t>(16384, P / (148 * 8 + 1)));
  c = std::max<int64_t>(256, std::min<int64_t>(c, 1 << 20));
  return static_cast<int>((c + 255) / 256 * 256);
}

RaggedLayout ragged_layout(int64_t A, int64_t S, int64_t P, const Tuning& t) {
  RaggedLayout l;
  l.chunk = ragged_chunk(P, t);
  l.max_items = P / l.chunk + A + 1;
  l.partial_off = 0;
  size_t off = static_cast<size_t>(l.max_items) * std::max<int64_t>(S, 1) * sizeof(float2);
  off = (off + 255) & ~static_cast<size_t>(255);
  l.items_off = off;
  off += static_cast<size_t>(A + 1) * sizeof(int64_t);
  off = (off + 255) & ~static_cast<size_t>(255);
  l.counter_off = off;
  off += 256;
  l.total = off;
  return l;
}

// Sample groups of a forward block: a power of two, G * K >= S (at most 64 and
// at most the block's threads, so every group has a lane).
int ragged_groups(int64_t S, int K, int threads) {
  int groups = 1;
  while (groups * K < S && groups < 64 && groups * 2 <= threads) groups *= 2;
  return groups;
}

template <typename T>
RgP<T> make_rg(const RaggedArgs& a, const Tuning& t, void* ws) {
  RgP<T> p{};
  p.normals = static_cast<const T*>(a.normals);
  p.sigmas = static_cast<const T*>(a.sigmas);
  p.points = static_cast<const T*>(a.points);
  p.offsets = a.offsets;
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
  if (ws != nullptr) {
    const RaggedLayout l = ragged_layout(a.A, a.S, a.P, t);
    unsigned char* base = static_cast<unsigned char*>(ws);
    p.partial = reinterpret_cast<float2*>(base + l.partial_off);
    p.item_offsets = reinterpret_cast<int64_t*>(base + l.items_off);
    p.counter = reinterpret_cast<unsigned long long*>(base + l.counter_off);
    p.max_items = l.max_items;
    p.chunk = l.chunk;
  }
  p.groups = ragged_groups(a.S, t.chunk, t.threads);
  return p;
}

template <typename T, int K>
cudaError_t launch_ragged_fwd_k(RgP<T>& p, int threads, cudaStream_t st) {
  const void* fn = reinterpret_cast<const void*>(&ragged_fwd_kernel<T, K>);
  const size_t smem = std::max((static_cast<size_t>(p.groups) + 1) * threads * sizeof(float2) + 33 * sizeof(int),
                               static_cast<size_t>(threads) * K * sizeof(float2));
  cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  int per_sm = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
  if (err != cudaSuccess) return err;
  const DeviceInfo dev = current_device_info();
  const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>(static_cast<int64_t>(per_sm) * dev.sm_count,
                                                                p.max_items));
  void* args[] = {&p};
  return cudaLaunchKernel(fn, dim3(static_cast<unsigned>(blocks)), dim3(threads), args, smem, st);
}

template <typename T>
cudaError_t launch_ragged_fwd(const RaggedArgs& a, const Tuning& t, void* ws, cudaStream_t st) {
  RgP<T> p = make_rg<T>(a, t, ws);
  ragged_prep_kernel<T><<<1, 1024, 0, st>>>(p);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  if (t.chunk == 8) err = launch_ragged_fwd_k<T, 8>(p, t.threads, st);
  else if (t.chunk == 32) err = launch_ragged_fwd_k<T, 32>(p, t.threads, st);
  else err = launch_ragged_fwd_k<T, 16>(p, t.threads, st);
  if (err != cudaSuccess) return err;
  const int fin = static_cast<int>(std::min<int64_t>((a.A * a.S + 255) / 256, 148 * 16));
  ragged_finish_kernel<T><<<std::max(fin, 1), 256, 0, st>>>(p);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_ragged_bwd(const RaggedArgs& a, const Tuning& t, cudaStream_t st) {
  RgP<T> p = make_rg<T>(a, t, nullptr);
  const int ld = static_cast<int>(((std::max<int64_t>(a.S, 1) + 3) / 4) * 4);
  const int max_rows = t.stage_rows;
  const size_t smem = static_cast<size_t>(max_rows) * 2 * ld * sizeof(float);
  const bool with_points = a.grad_points != nullptr;
  const void* fn = with_points ? reinterpret_cast<const void*>(&ragged_bwd_kernel<T, true>)
                               : reinterpret_cast<const void*>(&ragged_bwd_kernel<T, false>);
  cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  const int64_t blocks = (a.P + kBwdTile - 1) / kBwdTile;
  if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
  void* args[] = {&p, const_cast<int*>(&ld), const_cast<int*>(&max_rows)};
  return cudaLaunchKernel(fn, dim3(static_cast<unsigned>(blocks)), dim3(kBwdThreads), args, smem, st);
}

}  // namespace

Tuning tracer_ragged_forward_resolve(const RaggedArgs& a, const Tuning& req) {
  Tuning t = req;
  // 128 threads x 16-sample chunks: 33.1 ms per ragged step against 33.7 ms at 256 threads
  if (t.threads != 64 && t.threads != 128 && t.threads != 256) t.threads = 128;
  if (t.chunk != 8 && t.chunk != 16 && t.chunk != 32) t.chunk = 16;
  // a block's sample groups must cover all S samples (S <= 1024 is checked at the boundary)
  while (t.chunk < 32 && static_cast<int64_t>(ragged_groups(a.S, t.chunk, t.threads)) * t.chunk < a.S) {
    t.chunk *= 2;
  }
  if (t.items < 0) t.items = 0;
  t.items = std::min(t.items, 4096);
  return t;
}

Tuning tracer_ragged_backward_resolve(const RaggedArgs& a, const Tuning& req) {
  Tuning t = req;
  const int64_t ld = ((std::max<int64_t>(a.S, 1) + 3) / 4) * 4;
  // staged rows within 48 KB of shared memory
  const int cap = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(8, (48 * 1024) / (8 * ld))));
  if (t.stage_rows <= 0) t.stage_rows = 4;
  t.stage_rows = std::max(1, std::min(t.stage_rows, cap));
  return t;
}

size_t tracer_ragged_workspace(int64_t A, int64_t S, int64_t P, const Tuning& t) {
  return ragged_layout(A, S, P, t).total;
}

cudaError_t tracer_forward_ragged(const RaggedArgs& a, const Tuning& t, void* ws, cudaStream_t st) {
  if (a.A == 0 || a.S == 0) return cudaSuccess;
  if (a.dtype == kF64) return launch_ragged_fwd<double>(a, t, ws, st);
  return launch_ragged_fwd<float>(a, t, ws, st);
}

cudaError_t tracer_backward_ragged(const RaggedArgs& a, const Tuning& t, cudaStream_t st) {
  if (a.P == 0) return cudaSuccess;
  if (a.dtype == kF64) return launch_ragged_bwd<double>(a, t, st);
  return launch_ragged_bwd<float>(a, t, st);
}

}  // namespace geraf
