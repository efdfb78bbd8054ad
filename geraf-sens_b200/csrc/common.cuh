// Shared device helpers of libgeraf_rf: reference constants, element-type
// conversion, 1-D TMA (cp.async.bulk) staging with bounded mbarrier waits,
// the device status word, and the FP64 carrier-phase reduction used by the
// MIXED arithmetic form.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace geraf {

// ---------------------------------------------------------------------------
// Constants of the reference kernels, as FP32 literals
// (geraf/ops/RFMatchedFilter/csrc/matched_filter/MatchedFilter_cuda_kernel.cu:13-17,
//  geraf/ops/RFSignalTracer/csrc/signal_tracer/SignalTracer_cuda_kernel.cu:13-17).
// Positions are in metres, tau = D / 2.9979 in units of 1e-8 s, frequencies in
// units of 1e8 Hz.  The matched filter ignores the radar's fc_start and always
// uses 773.704 (77.3704 GHz); the tracer takes its start frequency as an argument.
constexpr float kSpeedOfLight = 2.9979f;
constexpr float kMfStartFrequency = 773.704f;
constexpr float kPathBias = 0.15f;
constexpr float kNormEps = 1.0e-7f;
constexpr float kPiF = 3.14159265358979323846f;

// A bounded wait that gives up stores GERAF_ERR_DEVICE_TIMEOUT (5) into the
// library's device status word (passed to every kernel that waits) and its
// kernel returns early instead of hanging.
constexpr int kStatusTimeout = 5;

// ---------------------------------------------------------------------------
// Element types.  All arithmetic of the PLAIN form is FP32, like the reference
// (`LoadAsFloat`); loads widen and stores narrow with round-to-nearest.
template <typename T>
__device__ __forceinline__ float ld_f(const T* p, int64_t i) {
  return static_cast<float>(p[i]);
}
template <>
__device__ __forceinline__ float ld_f<__half>(const __half* p, int64_t i) {
  return __half2float(p[i]);
}
template <typename T>
__device__ __forceinline__ T from_f(float v) {
  return static_cast<T>(v);
}
template <>
__device__ __forceinline__ __half from_f<__half>(float v) {
  return __float2half_rn(v);
}

// Four consecutive elements from a 4-element-aligned shared-memory address.
__device__ __forceinline__ float4 lds4(const float* p) {
  return *reinterpret_cast<const float4*>(p);
}
__device__ __forceinline__ float4 lds4(const double* p) {
  const double2 a = *reinterpret_cast<const double2*>(p);
  const double2 b = *reinterpret_cast<const double2*>(p + 2);
  return make_float4(static_cast<float>(a.x), static_cast<float>(a.y),
                     static_cast<float>(b.x), static_cast<float>(b.y));
}
__device__ __forceinline__ float4 lds4(const __half* p) {
  const uint2 raw = *reinterpret_cast<const uint2*>(p);
  const __half2 lo = *reinterpret_cast<const __half2*>(&raw.x);
  const __half2 hi = *reinterpret_cast<const __half2*>(&raw.y);
  const float2 a = __half22float2(lo);
  const float2 b = __half22float2(hi);
  return make_float4(a.x, a.y, b.x, b.y);
}

// ---------------------------------------------------------------------------
// 1-D TMA staging: cp.async.bulk global -> shared, completion on an mbarrier.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

// Makes initialised barriers visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Source and destination 16-byte aligned, bytes a multiple of 16 (checked on the host).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Wall-time limit of every bounded wait of the operators (2 s).
constexpr uint64_t kWaitLimitNs = 2000000000ull;

// Waits for phase `parity` of `bar` for at most `limit_ns` of wall time (and at
// most 2^26 polls).  Returns false (and raises *status) when it gives up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* status,
                                                  uint64_t limit_ns = kWaitLimitNs) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  for (uint32_t it = 0; it < (1u << 26); ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255u) == 255u && global_timer_ns() - t0 > limit_ns) break;
  }
  if (status != nullptr) atomicExch(status, kStatusTimeout);
  return false;
}

// Stages `rows` consecutive rows of two [R, S] arrays (e.g. the real and
// imaginary IF samples of a block of antennas) into a double-buffered
// shared-memory ring.  Bulk (TMA) mode: thread 0 issues one cp.async.bulk per
// array per stage and the consumers wait on the stage's mbarrier.  Fallback
// mode (unaligned rows): all threads copy, rows padded to `ld` elements with
// zeros, published by the barrier in wait().
template <typename T>
struct PairStager {
  T* buf;          // [2 stages][2 arrays][rows_max * ld]
  uint64_t* bar;   // [2]
  int ld;          // shared row stride in elements (multiple of 4)
  int rows_max;
  bool bulk;
  uint64_t wait_ns = kWaitLimitNs;  // limit of each bounded wait

  __device__ __forceinline__ T* stage_ptr(int stage, int which) const {
    return buf + (static_cast<int64_t>(stage) * 2 + which) * rows_max * ld;
  }

  // Called by all threads.  In bulk mode only thread 0 does anything.
  __device__ __forceinline__ void issue(int stage, const T* a, const T* b, int64_t row0,
                                        int rows, int S) {
    if (bulk) {
      if (threadIdx.x == 0) {
        const uint32_t bytes = static_cast<uint32_t>(rows) * S * sizeof(T);
        mbar_arrive_expect_tx(&bar[stage], 2 * bytes);
        bulk_g2s(stage_ptr(stage, 0), a + row0 * S, bytes, &bar[stage]);
        bulk_g2s(stage_ptr(stage, 1), b + row0 * S, bytes, &bar[stage]);
      }
    } else {
      T* da = stage_ptr(stage, 0);
      T* db = stage_ptr(stage, 1);
      const int total = rows * ld;
      for (int i = threadIdx.x; i < total; i += blockDim.x) {
        const int r = i / ld;
        const int c = i - r * ld;
        T va = T(0.0f), vb = T(0.0f);
        if (c < S) {
          va = a[(row0 + r) * S + c];
          vb = b[(row0 + r) * S + c];
        }
        da[i] = va;
        db[i] = vb;
      }
    }
  }

  // Called by all threads; returns false on a device-side timeout (uniform
  // across the block, so the caller can return without stranding a barrier).
  __device__ __forceinline__ bool wait(int stage, uint32_t parity, int* status) {
    bool ok = true;
    if (bulk) ok = mbar_wait_bounded(&bar[stage], parity, status, wait_ns);
    return __syncthreads_and(ok) != 0;
  }

  // After a timeout: thread 0 waits (bounded) for a copy still in flight
  // into `stage`, so the block never exits with TMA writes pending.
  __device__ __forceinline__ void drain(int stage, uint32_t parity, int* status) {
    if (bulk && threadIdx.x == 0) mbar_wait_bounded(&bar[stage], parity, status, wait_ns);
  }
};

// ---------------------------------------------------------------------------
// MIXED form carrier phase.  With float inputs promoted to FP64, the path
// length D = |tx - x| + |rx - x| is formed with two Newton-corrected square
// roots (relative error ~1e-13) and the phase is reduced in cycles:
//   cycles0 = (D + 0.15) * k0,  k0 = (pi_f / pi) * f0 / c   (so 2 pi cycles0 = 2 pi_f f0 tau)
//   dcyc    = (D + 0.15) * k1,  k1 = (pi_f / pi) * As / (fs c)
// where pi_f is the FP32 value of pi used by the reference's 2*kPi factor.
// frac0 = cycles0 - rint(cycles0) in [-1/2, 1/2] keeps ~1e-9 cycle accuracy
// where the FP32 reference loses ~2e-5 cycles at 5e3 rad.
__device__ __forceinline__ double sqrt_f64_fast(double s) {
  const float r = rsqrtf(static_cast<float>(s));  // MUFU, ~2^-22 relative
  const double d0 = s * static_cast<double>(r);
  const double res = fma(-d0, d0, s);
  return fma(0.5 * static_cast<double>(r), res, d0);  // one Newton step: ~2^-44
}

struct PhaseCycles {
  float frac0;  // carrier phase in cycles, reduced to [-1/2, 1/2]
  float dcyc;   // per-sample phase step in cycles
};

__device__ __forceinline__ PhaseCycles path_cycles(double dtx, double dty, double dtz, double drx,
                                                   double dry, double drz, double k0, double b0,
                                                   double k1, double b1) {
  const double st = fma(dtz, dtz, fma(dty, dty, dtx * dtx));
  const double sr = fma(drz, drz, fma(dry, dry, drx * drx));
  const double d = sqrt_f64_fast(st) + sqrt_f64_fast(sr);
  const double c0 = fma(d, k0, b0);
  PhaseCycles out;
  out.frac0 = static_cast<float>(c0 - rint(c0));
  out.dcyc = static_cast<float>(fma(d, k1, b1));
  return out;
}

// e^{j 2 pi x} for x in cycles (|x| <= ~1), accurate to ~1 ulp.
__device__ __forceinline__ float2 cis_cycles(float x) {
  float s, c;
  sincospif(2.0f * x, &s, &c);
  return make_float2(c, s);
}

// e^{j 2 pi x} for |x| <= 1/2 from the hardware sine and cosine (__sincosf,
// absolute error ~4e-7 on [-pi, pi]): for the phasor that multiplies a term
// once (its carrier or start phase), and for a rotator raised to at most
// kFastPowers powers (per sample block, per sample group), whose phase error
// then stays below ~3e-6 rad, far inside the MIXED form's bound.  The
// per-sample rotators, and block or group rotators of longer rows, keep
// cis_cycles: their error grows with the steps they take.
constexpr int kFastPowers = 8;
__device__ __forceinline__ float2 cis_cycles_fast(float x) {
  float s, c;
  __sincosf(6.28318530717958647692f * x, &s, &c);
  return make_float2(c, s);
}

// cosf(x) and sinf(x) from one sincosf call.  sincosf returns the same bits as
// the two separate calls for every FP32 input -- geraf_rf_sincos_identity_check
// compares all 2^32 inputs on the device -- so the PLAIN kernels keep the
// reference's results while the argument reduction is done once.
__device__ __forceinline__ void cos_sin(float x, float* c, float* s) { sincosf(x, s, c); }

// Packed FP32 fused multiply-add on two lanes (fma.rn.f32x2, sm_100+): one
// instruction for two independent FMAs, halving the issue slots of FMA-bound
// loops.  Results are those of two fmaf calls.
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
      "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}

// Packed FP32 add and subtract on two lanes (add/sub.rn.f32x2, sm_100+).
__device__ __forceinline__ float2 fadd2(float2 a, float2 b) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 fsub2(float2 a, float2 b) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// acc[m] += s0 * z^m for m = 0 .. K-1, |z| = 1.
//
// Each real component of u_m = s0 z^m is A cos(m theta + c), so it obeys the
// three-term (Chebyshev / Goertzel) recurrence u_{m+1} = 2 cos(theta) u_m - u_{m-1}:
// one FMA per component per sample instead of the 4-operation complex product
// of a rotator.  The (re, im) pair of one term runs in one packed register:
// one fma.rn.f32x2 for the recurrence and one add/sub.rn.f32x2 for the
// accumulation, 2 issue slots per (term, sample).  So that no negation is
// issued, the recurrence carries x_m = sigma_m u_m with the sign pattern
// sigma = (+, +, -, -, +, +, ...):  x_{m+1} = (+-2 cos theta) x_m + x_{m-1}
// (coefficient +2cos for odd m+1, -2cos for even), and x_m is added for
// m mod 4 in {0, 1}, subtracted for {2, 3}.  RN rounding is sign-symmetric,
// so the sums are bit-identical to the scalar recurrence.  Rounding errors of
// the recurrence grow at most ~m^2 eps (theta near 0 or pi) and ~m eps /
// |sin theta| otherwise, which is why callers re-seed from exact phasors
// every K samples.
// ASSIGN: acc is set to this term's samples instead of added to (the first term
// of a tile), which spares zeroing the accumulators between tiles.
template <int K, bool ASSIGN = false>
__device__ __forceinline__ void rotate_accumulate(float2 s0, float2 z, float2 (&acc)[K]) {
  static_assert(K >= 2, "the recurrence needs two seeds");
  const float2 c2 = make_float2(2.0f * z.x, 2.0f * z.x);
  const float2 nc2 = make_float2(-2.0f * z.x, -2.0f * z.x);
  const float2 zero = make_float2(0.0f, 0.0f);
  float2 xm1 = s0;
  float2 x = cmul(s0, z);
  acc[0] = ASSIGN ? xm1 : fadd2(acc[0], xm1);
  acc[1] = ASSIGN ? x : fadd2(acc[1], x);
#pragma unroll
  for (int m = 2; m < K; ++m) {
    const float2 xn = ffma2((m & 1) ? c2 : nc2, x, xm1);
    xm1 = x;
    x = xn;
    if (ASSIGN) acc[m] = (m & 2) ? fsub2(zero, x) : x;
    else acc[m] = (m & 2) ? fsub2(acc[m], x) : fadd2(acc[m], x);
  }
}

// One tile of a sample-major kernel for lane l of L: acc = the sum over the
// tile's terms vl = l, l + L, ... < count of rotate_accumulate, each term from
// its seed and rotator (the first term assigns, so acc needs no zeroing).
template <int K>
__device__ __forceinline__ void rotate_tile(const float2* seeds, const float2* zeta, int l, int L, int count,
                                            float2 (&acc)[K]) {
  int vl = l;
  if (vl < count) {
    rotate_accumulate<K, true>(seeds[vl], zeta[vl], acc);
    vl += L;
  } else {
#pragma unroll
    for (int m = 0; m < K; ++m) acc[m] = make_float2(0.0f, 0.0f);
  }
  for (; vl < count; vl += L) rotate_accumulate<K>(seeds[vl], zeta[vl], acc);
}

// Residual sums of the tracer adjoints for one (point, antenna) pair, from a
// residual row g (real and imaginary parts, ld samples, ld a multiple of 4,
// samples past S zero) in shared memory:
//   Q  = sum_n conj(g_n) zeta^n,   Q1 = zeta Q'(zeta) = sum_n n conj(g_n) zeta^n.
// Horner in w = zeta^2 on the even and odd samples at once, one chain per lane
// of packed f32x2 operands.  The lanes carry the conjugates
// E = sum_m g_2m conj(w)^m, O = sum_m g_2m+1 conj(w)^m (so no operand needs a
// negation) and their derivatives E', O' in conj(w):
//   conj(Q)  = E + conj(zeta) O,
//   conj(Q1) = 2 conj(w) E' + conj(zeta) (2 conj(w) O' + O).
// Per two samples: 4 fma.rn.f32x2 for (E, O), 4 more for (E', O') when Q1 is
// wanted.
template <bool WITH_Q1, typename R>
__device__ __forceinline__ void residual_sums(const R* rowr, const R* rowi, int ld, float2 zt, float2& q,
                                              float2& q1) {
  const float2 wz = cmul(zt, zt);
  const float2 wr2 = make_float2(wz.x, wz.x), wi2 = make_float2(wz.y, wz.y);
  const float2 nwi2 = make_float2(-wz.y, -wz.y);
  float2 pr = make_float2(0.0f, 0.0f), pim = make_float2(0.0f, 0.0f);  // (E, O) real, imaginary
  float2 dr2 = make_float2(0.0f, 0.0f), di2 = make_float2(0.0f, 0.0f);  // (E', O')
#pragma unroll 2
  for (int n = ld - 4; n >= 0; n -= 4) {
    const float4 a4 = lds4(rowr + n);
    const float4 b4 = lds4(rowi + n);
    const float2 gre[2] = {make_float2(a4.z, a4.w), make_float2(a4.x, a4.y)};
    const float2 gim[2] = {make_float2(b4.z, b4.w), make_float2(b4.x, b4.y)};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (WITH_Q1) {  // D <- D conj(w) + P (P before its update)
        const float2 ndr = ffma2(dr2, wr2, ffma2(di2, wi2, pr));
        const float2 ndi = ffma2(di2, wr2, ffma2(dr2, nwi2, pim));
        dr2 = ndr;
        di2 = ndi;
      }
      // P <- P conj(w) + g
      const float2 npr = ffma2(pr, wr2, ffma2(pim, wi2, gre[h]));
      const float2 npi = ffma2(pim, wr2, ffma2(pr, nwi2, gim[h]));
      pr = npr;
      pim = npi;
    }
  }
  const float2 zc = make_float2(zt.x, -zt.y);
  const float2 qc = cmul(zc, make_float2(pr.y, pim.y));
  q = make_float2(pr.x + qc.x, -(pim.x + qc.y));
  if (WITH_Q1) {
    const float2 wc = make_float2(wz.x, -wz.y);
    const float2 de = cmul(wc, make_float2(dr2.x, di2.x));
    const float2 dodd = cmul(wc, make_float2(dr2.y, di2.y));
    const float2 t1 = cmul(zc, make_float2(2.0f * dodd.x + pr.y, 2.0f * dodd.y + pim.y));
    q1 = make_float2(2.0f * de.x + t1.x, -(2.0f * de.y + t1.y));
  } else {
    q1 = make_float2(0.0f, 0.0f);
  }
}

// Stages the tx and rx positions of `rws` antennas from a0 into slot `stage`
// of a [2][rows_max][6] shared table, as PosT (float or double).
template <typename T, typename PosT>
__device__ __forceinline__ void stage_positions(PosT* pos, int stage, int rows_max, const T* tx,
                                                const T* rx, int64_t a0, int rws) {
  for (int i = threadIdx.x; i < rws * 6; i += blockDim.x) {
    const int r = i / 6;
    const int c = i - r * 6;
    const T* src = c < 3 ? tx : rx;
    pos[(stage * rows_max + r) * 6 + c] = static_cast<PosT>(ld_f(src, (a0 + r) * 3 + (c % 3)));
  }
}

// Kahan-compensated accumulation of one component.
__device__ __forceinline__ void kahan_add(float& sum, float& comp, float x) {
  const float y = x - comp;
  const float t = sum + y;
  comp = (t - sum) - y;
  sum = t;
}

__host__ __device__ constexpr int ceil_div(int64_t a, int64_t b) {
  return static_cast<int>((a + b - 1) / b);
}

}  // namespace geraf
