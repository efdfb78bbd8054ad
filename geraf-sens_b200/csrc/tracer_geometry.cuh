// Specular geometry of the lensless signal tracer, shared by the tracer
// kernels (reference: geraf/ops/RFSignalTracer/csrc/signal_tracer/SignalTracer_cuda_kernel.cu:19-197).
// Everything is evaluated in the reference's FP32 operation order, so
// amplitudes and culling decisions match the reference bit for bit.
#pragma once

#include "common.cuh"

namespace geraf {
namespace tracer {

__device__ __forceinline__ float sq(float x) { return x * x; }

__device__ __forceinline__ float dot3(const float* a, const float* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// normalize with the reference's epsilon: v / (|v| + 1e-7)
__device__ __forceinline__ void normalize3(const float* in, float* out) {
  const float norm = sqrtf(dot3(in, in));
  const float inv_norm = 1.0f / (norm + kNormEps);
  out[0] = in[0] * inv_norm;
  out[1] = in[1] * inv_norm;
  out[2] = in[2] * inv_norm;
}

// Specular geometry of one (point, antenna) pair in the reference's FP32
// operation order (SignalTracer_cuda_kernel.cu:172-197).
struct SpecGeom {
  float inc[3];       // normalize(p - tx)
  float refl_raw[3];  // inc - 2 (inc.n) n
  float refl[3];      // normalize(refl_raw)
  float ret[3];       // normalize(rx - p)
  float align;        // rho
  float idn;          // inc . n
};

__device__ __forceinline__ void specular_geometry(const float* tx, const float* rx, const float* nrm,
                                                  const float* pt, SpecGeom& g) {
  float inc_raw[3], ret_raw[3];
#pragma unroll
  for (int axis = 0; axis < 3; ++axis) {
    inc_raw[axis] = pt[axis] - tx[axis];
    ret_raw[axis] = rx[axis] - pt[axis];
  }
  normalize3(inc_raw, g.inc);
  g.idn = dot3(g.inc, nrm);
  const float incident_dot_normal = dot3(g.inc, nrm);
#pragma unroll
  for (int axis = 0; axis < 3; ++axis) {
    g.refl_raw[axis] = g.inc[axis] - 2.0f * incident_dot_normal * nrm[axis];
  }
  normalize3(g.refl_raw, g.refl);
  normalize3(ret_raw, g.ret);
  g.align = dot3(g.ret, g.refl);
}

__device__ __forceinline__ bool culled(const SpecGeom& g) {
  return g.align < 1.0e-6f || g.idn > 0.0f;
}

// A conservative early test for culled(): true only for pairs that the
// reference-order geometry culls with a wide margin, from unnormalised vectors
// and no division or square root (about 30 FP32 operations against ~150 for
// specular_geometry).  With i = p - tx, o = rx - p and r = i - 2 (i.n) n (the
// reflection of the unnormalised incident ray, a positive multiple of the
// reference's refl_raw):
//   inc.n > 0   has the sign of i.n,
//   rho < 1e-6  holds when o.r < 0, since rho = o.r / (positive norms).
// The test fires only when i.n > 1e-4 |i| |n|, or o.r < -1e-4 |o| M with
// M = |i| (1 + 2 |n|^2) the size of the terms r is formed from (compared as
// squares).  The reference's FP32 evaluation errs by ~1e-6 |n| in inc.n and by
// ~1e-6 M / |r| in rho (the error of normalising r, which the margin keeps away
// from cancellation: |r| >= |o.r| / |o| > 1e-4 M), so every pair the test culls
// is culled by culled(specular_geometry(...)) as well, and a pair it lets
// through is decided by the exact form.  Non-finite inputs fail every
// comparison and go to the exact form too.
__device__ __forceinline__ bool surely_culled(const float* tx, const float* rx, const float* nrm,
                                              const float* pt) {
  float i[3], o[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    i[k] = pt[k] - tx[k];
    o[k] = rx[k] - pt[k];
  }
  const float in = dot3(i, nrm);
  const float ii = dot3(i, i), nn = dot3(nrm, nrm);
  if (in > 0.0f && in * in > 1.0e-8f * (ii * nn)) return true;  // back-facing
  float r[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) r[k] = i[k] - 2.0f * in * nrm[k];
  const float orr = dot3(o, r);
  const float m = 1.0f + 2.0f * nn;
  return orr < 0.0f && orr * orr > 1.0e-8f * (dot3(o, o) * ii * (m * m));  // reflected away
}

// |tx - p| + |rx - p| in the reference's order (ComputePathDistance).
__device__ __forceinline__ float path_distance(const float* tx, const float* rx, const float* pt) {
  return sqrtf(sq(tx[0] - pt[0]) + sq(tx[1] - pt[1]) + sq(tx[2] - pt[2])) +
         sqrtf(sq(rx[0] - pt[0]) + sq(rx[1] - pt[1]) + sq(rx[2] - pt[2]));
}

// d rho / d n through the reflection and its normalisation, in the reference's
// order (SignalTracer_cuda_kernel.cu:91-170, 531-542).
__device__ __forceinline__ void align_normal_gradient(const SpecGeom& g, const float* nrm,
                                                      float* gsa) {
  const float incident_dot_normal = dot3(g.inc, nrm);
  float jac[9];
#pragma unroll
  for (int row = 0; row < 3; ++row) {
#pragma unroll
    for (int col = 0; col < 3; ++col) {
      const float shared_term = -2.0f * nrm[row] * g.inc[col];
      jac[row * 3 + col] = row == col ? shared_term - 2.0f * incident_dot_normal : shared_term;
    }
  }
  const float value_norm = sqrtf(dot3(g.refl_raw, g.refl_raw));
  const float x = g.refl[0], y = g.refl[1], z = g.refl[2];
  const float inv_norm = 1.0f / (value_norm + kNormEps);
  float nj[9];
  nj[0] = ((1.0f - x * x) * jac[0] + (-x * y) * jac[3] + (-x * z) * jac[6]) * inv_norm;
  nj[1] = ((1.0f - x * x) * jac[1] + (-x * y) * jac[4] + (-x * z) * jac[7]) * inv_norm;
  nj[2] = ((1.0f - x * x) * jac[2] + (-x * y) * jac[5] + (-x * z) * jac[8]) * inv_norm;
  nj[3] = ((-y * x) * jac[0] + (1.0f - y * y) * jac[3] + (-y * z) * jac[6]) * inv_norm;
  nj[4] = ((-y * x) * jac[1] + (1.0f - y * y) * jac[4] + (-y * z) * jac[7]) * inv_norm;
  nj[5] = ((-y * x) * jac[2] + (1.0f - y * y) * jac[5] + (-y * z) * jac[8]) * inv_norm;
  nj[6] = ((-z * x) * jac[0] + (-z * y) * jac[3] + (1.0f - z * z) * jac[6]) * inv_norm;
  nj[7] = ((-z * x) * jac[1] + (-z * y) * jac[4] + (1.0f - z * z) * jac[7]) * inv_norm;
  nj[8] = ((-z * x) * jac[2] + (-z * y) * jac[5] + (1.0f - z * z) * jac[8]) * inv_norm;
#pragma unroll
  for (int axis = 0; axis < 3; ++axis) {
    float value = 0.0f;
#pragma unroll
    for (int component = 0; component < 3; ++component) {
      value += nj[component * 3 + axis] * g.ret[component];
    }
    gsa[axis] = value;
  }
}

// d rho / d p (no reference counterpart): rho = <o, r/|r|>, r = H i, H = I - 2 n n^T,
// i = (p - tx)/|p - tx|, o = (rx - p)/|rx - p|.
__device__ __forceinline__ void align_point_gradient(const SpecGeom& g, const float* nrm, float dist_t,
                                                     float dist_r, float* out) {
  const float rnorm = sqrtf(dot3(g.refl_raw, g.refl_raw));
  const float ro = dot3(g.refl, g.ret);
  float u[3], v[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) u[k] = (g.ret[k] - g.refl[k] * ro) / rnorm;
  const float nu = dot3(nrm, u);
#pragma unroll
  for (int k = 0; k < 3; ++k) v[k] = u[k] - 2.0f * nu * nrm[k];
  const float iv = dot3(g.inc, v);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float w = (v[k] - g.inc[k] * iv) / dist_t;
    const float q = -(g.refl[k] - g.ret[k] * ro) / dist_r;
    out[k] = w + q;
  }
}

// Per-sample phase rate of the reference, w_n = 2*kPi*f0 + (2*kPi*As) * t_n
// (SignalTracer_cuda_kernel.cu:375-377, 440).  The reference's compiled code
// fuses the 2*kPi*f0 product into the sum and rounds the slope term first;
// that rounding is pinned here with explicit intrinsics (it was identified
// from the reference's outputs: it is the only choice that reproduces them).
__device__ __forceinline__ float phase_rate(float f0, float As, float sample_time) {
  const float phase_slope = 2.0f * kPiF * As;
  return __fmaf_rn(2.0f * kPiF, f0, __fmul_rn(phase_slope, sample_time));
}

// The same rate as the reference's adjoint forms it (SignalTracer_cuda_kernel.cu:552-554):
// there the FP32 instantiation fuses the slope product instead,
// fma(2*kPi*As, t_n, 2*kPi*f0), while the FP64 instantiation rounds as the
// forward does.  Both were identified from the reference's outputs.
template <typename T>
__device__ __forceinline__ float adjoint_phase_rate(float f0, float As, float sample_time) {
  return phase_rate(f0, As, sample_time);
}
template <>
__device__ __forceinline__ float adjoint_phase_rate<float>(float f0, float As, float sample_time) {
  const float phase_base = 2.0f * kPiF * f0;
  const float phase_slope = 2.0f * kPiF * As;
  return __fmaf_rn(phase_slope, sample_time, phase_base);
}

}  // namespace tracer
}  // namespace geraf
