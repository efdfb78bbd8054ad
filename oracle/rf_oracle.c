/*
 * rf_oracle.c -- CPU restatement of GeRaF's RF operator kernels.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, by __graft_entry__.smoke() as the
 * checker and by bench.py's CPU-baseline leg.  Never part of the product path.
 *
 * Two forms of every kernel of the reference (paths relative to GeRaF-SENS):
 *   *_f64  exact-arithmetic model: the reference's expressions evaluated in
 *          double precision with the reference's FP32 constants (2.9979f,
 *          773.704f, 0.15f, 1e-7f, and pi as the float kPi) promoted exactly;
 *          cos/sin from libm.  This is the accuracy target ("vs FP64").
 *   *_f32  the reference's FP32 arithmetic in its expression and summation
 *          order (compiled with -ffp-contract=off, so no fused multiply-adds);
 *          the timed CPU baseline.
 * Inputs are FP32 arrays in the reference's layouts; voxels are [3, N].
 *
 * Parity is pinned by golden vectors produced by the reference's own CUDA
 * kernels (tests/golden/make_golden.py) -- the reference ships no tests.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define K_C 2.9979f
#define K_F0MF 773.704f
#define K_BIAS 0.15f
#define K_EPS 1.0e-7f
#define K_PI 3.14159265358979323846f

static inline float sqf(float x) { return x * x; }
static inline double sqd(double x) { return x * x; }

/* ======================= matched filter =================================
 * MatchedFilter_cuda_kernel.cu:28-58 (distance, phase), :65-115 (forward),
 * :171-220 (adjoint), :117-169 / :222-279 (range-bin variants). */

static inline float mf_distance_f32(const float* tx, const float* rx, int64_t a, float vx, float vy,
                                    float vz) {
  const float txd = sqrtf(sqf(tx[a * 3 + 0] - vx) + sqf(tx[a * 3 + 1] - vy) + sqf(tx[a * 3 + 2] - vz));
  const float rxd = sqrtf(sqf(rx[a * 3 + 0] - vx) + sqf(rx[a * 3 + 1] - vy) + sqf(rx[a * 3 + 2] - vz));
  return txd + rxd + K_BIAS;
}

static inline double mf_distance_f64(const float* tx, const float* rx, int64_t a, double vx,
                                     double vy, double vz) {
  const double txd = sqrt(sqd(tx[a * 3 + 0] - vx) + sqd(tx[a * 3 + 1] - vy) + sqd(tx[a * 3 + 2] - vz));
  const double rxd = sqrt(sqd(rx[a * 3 + 0] - vx) + sqd(rx[a * 3 + 1] - vy) + sqd(rx[a * 3 + 2] - vz));
  return txd + rxd + (double)K_BIAS;
}

void oracle_mf_forward_f64(const float* re, const float* im, const float* tx, const float* rx,
                           const float* vox, int64_t A, int64_t S, int64_t N, float fs, float As,
                           double* out_re, double* out_im) {
  const double w0 = 2.0 * (double)K_PI * (double)K_F0MF;
  const double w1 = 2.0 * (double)K_PI * (double)As;
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t v = 0; v < N; ++v) {
    const double vx = vox[v], vy = vox[N + v], vz = vox[2 * N + v];
    double ar = 0.0, ai = 0.0;
    for (int64_t a = 0; a < A; ++a) {
      const double tau = mf_distance_f64(tx, rx, a, vx, vy, vz) / (double)K_C;
      for (int64_t n = 0; n < S; ++n) {
        const double phase = (w0 + w1 * ((double)n / (double)fs)) * tau;
        const double c = cos(phase), s = sin(phase);
        const double sr = re[a * S + n], si = im[a * S + n];
        ar += c * sr + s * si;
        ai += c * si - s * sr;
      }
    }
    out_re[v] = ar / (double)A;
    out_im[v] = ai / (double)A;
  }
}

void oracle_mf_forward_f32(const float* re, const float* im, const float* tx, const float* rx,
                           const float* vox, int64_t A, int64_t S, int64_t N, float fs, float As,
                           float* out_re, float* out_im) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t v = 0; v < N; ++v) {
    const float vx = vox[v], vy = vox[N + v], vz = vox[2 * N + v];
    float ar = 0.0f, ai = 0.0f;
    for (int64_t a = 0; a < A; ++a) {
      const float distance = mf_distance_f32(tx, rx, a, vx, vy, vz);
      const float tau = distance / K_C;
      const float base_phase = 2.0f * K_PI * K_F0MF * tau;
      for (int64_t n = 0; n < S; ++n) {
        const float sample_time = (float)n / fs;
        const float phase = base_phase + 2.0f * K_PI * As * sample_time * tau;
        const float c = cosf(phase), ns = -sinf(phase);
        const float sr = re[a * S + n], si = im[a * S + n];
        ar += c * sr - ns * si;
        ai += c * si + ns * sr;
      }
    }
    out_re[v] = ar / (float)A;
    out_im[v] = ai / (float)A;
  }
}

void oracle_mf_backward_f64(const float* gr, const float* gi, const float* tx, const float* rx,
                            const float* vox, int64_t A, int64_t S, int64_t N, float fs, float As,
                            double* grad_re, double* grad_im) {
  const double w0 = 2.0 * (double)K_PI * (double)K_F0MF;
  const double w1 = 2.0 * (double)K_PI * (double)As;
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t a = 0; a < A; ++a) {
    for (int64_t n = 0; n < S; ++n) {
      const double wn = w0 + w1 * ((double)n / (double)fs);
      double ar = 0.0, ai = 0.0;
      for (int64_t v = 0; v < N; ++v) {
        const double tau = mf_distance_f64(tx, rx, a, vox[v], vox[N + v], vox[2 * N + v]) / (double)K_C;
        const double phase = wn * tau;
        const double c = cos(phase), s = sin(phase);
        ar += c * gr[v] - s * gi[v];
        ai += s * gr[v] + c * gi[v];
      }
      grad_re[a * S + n] = ar / (double)A;
      grad_im[a * S + n] = ai / (double)A;
    }
  }
}

void oracle_mf_backward_f32(const float* gr, const float* gi, const float* tx, const float* rx,
                            const float* vox, int64_t A, int64_t S, int64_t N, float fs, float As,
                            float* grad_re, float* grad_im) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t a = 0; a < A; ++a) {
    for (int64_t n = 0; n < S; ++n) {
      const float sample_time = (float)n / fs;
      float ar = 0.0f, ai = 0.0f;
      for (int64_t v = 0; v < N; ++v) {
        const float distance = mf_distance_f32(tx, rx, a, vox[v], vox[N + v], vox[2 * N + v]);
        const float tau = distance / K_C;
        const float phase = 2.0f * K_PI * K_F0MF * tau + 2.0f * K_PI * As * sample_time * tau;
        const float c = cosf(phase), ns = -sinf(phase);
        ar += c * gr[v] + ns * gi[v];
        ai += (-ns) * gr[v] + c * gi[v];
      }
      grad_re[a * S + n] = ar / (float)A;
      grad_im[a * S + n] = ai / (float)A;
    }
  }
}

/* The *_f64 model above with the per-sample phasors of one (voxel, antenna)
 * pair generated by an FP64 rotation instead of one libm cos/sin per sample:
 * phase(n) = (w0 + w1 n / fs) tau is linear in n, so
 * e^{j phase(n+1)} = e^{j phase(n)} e^{j w1 tau / fs}.  Every REC_SEED samples
 * the phasor is re-seeded from libm at the *_f64 form's own phase expression,
 * which bounds the rotation's drift to a few 1e-16 relative.  The results agree
 * with *_f64 to ~1e-13 (checked on the CPU) at a fraction of its cost; the
 * parity checks of the full-size workloads (49152 channels x 256 samples) use
 * them.  The forward sums four antenna streams separately and adds them at the
 * end; the adjoint keeps the *_f64 summation order. */
#define REC_SEED 16

void oracle_mf_forward_f64r(const float* re, const float* im, const float* tx, const float* rx,
                            const float* vox, int64_t A, int64_t S, int64_t N, float fs, float As,
                            double* out_re, double* out_im) {
  const double w0 = 2.0 * (double)K_PI * (double)K_F0MF;
  const double w1 = 2.0 * (double)K_PI * (double)As;
  enum { L = 4 }; /* antennas whose rotations run interleaved (independent chains) */
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t v = 0; v < N; ++v) {
    const double vx = vox[v], vy = vox[N + v], vz = vox[2 * N + v];
    double ar[L] = {0.0}, ai[L] = {0.0};
    for (int64_t a0 = 0; a0 < A; a0 += L) {
      const int cnt = A - a0 < L ? (int)(A - a0) : L;
      double tau[L], zc[L], zs[L];
      for (int k = 0; k < L; ++k) {
        tau[k] = k < cnt ? mf_distance_f64(tx, rx, a0 + k, vx, vy, vz) / (double)K_C : 0.0;
        zc[k] = cos(w1 / (double)fs * tau[k]);
        zs[k] = sin(w1 / (double)fs * tau[k]);
      }
      for (int64_t n0 = 0; n0 < S; n0 += REC_SEED) {
        double c[L], s[L];
        for (int k = 0; k < L; ++k) {
          const double phase = (w0 + w1 * ((double)n0 / (double)fs)) * tau[k];
          c[k] = cos(phase);
          s[k] = sin(phase);
        }
        const int64_t n1 = n0 + REC_SEED < S ? n0 + REC_SEED : S;
        for (int64_t n = n0; n < n1; ++n) {
          for (int k = 0; k < L; ++k) {
            const double sr = k < cnt ? re[(a0 + k) * S + n] : 0.0;
            const double si = k < cnt ? im[(a0 + k) * S + n] : 0.0;
            ar[k] += c[k] * sr + s[k] * si;
            ai[k] += c[k] * si - s[k] * sr;
            const double cn = c[k] * zc[k] - s[k] * zs[k];
            s[k] = s[k] * zc[k] + c[k] * zs[k];
            c[k] = cn;
          }
        }
      }
    }
    double sr = 0.0, si = 0.0;
    for (int k = 0; k < L; ++k) {
      sr += ar[k];
      si += ai[k];
    }
    out_re[v] = sr / (double)A;
    out_im[v] = si / (double)A;
  }
}

void oracle_mf_backward_f64r(const float* gr, const float* gi, const float* tx, const float* rx,
                             const float* vox, int64_t A, int64_t S, int64_t N, float fs, float As,
                             double* grad_re, double* grad_im) {
  const double w0 = 2.0 * (double)K_PI * (double)K_F0MF;
  const double w1 = 2.0 * (double)K_PI * (double)As;
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t a = 0; a < A; ++a) {
    double* ar = grad_re + a * S;
    double* ai = grad_im + a * S;
    for (int64_t n = 0; n < S; ++n) ar[n] = ai[n] = 0.0;
    for (int64_t v = 0; v < N; ++v) {
      const double tau = mf_distance_f64(tx, rx, a, vox[v], vox[N + v], vox[2 * N + v]) / (double)K_C;
      const double step = w1 / (double)fs * tau;
      const double zc = cos(step), zs = sin(step);
      const double g_r = gr[v], g_i = gi[v];
      for (int64_t n0 = 0; n0 < S; n0 += REC_SEED) {
        const double phase = (w0 + w1 * ((double)n0 / (double)fs)) * tau;
        double c = cos(phase), s = sin(phase);
        const int64_t n1 = n0 + REC_SEED < S ? n0 + REC_SEED : S;
        for (int64_t n = n0; n < n1; ++n) {
          ar[n] += c * g_r - s * g_i;
          ai[n] += s * g_r + c * g_i;
          const double cn = c * zc - s * zs;
          s = s * zc + c * zs;
          c = cn;
        }
      }
    }
    for (int64_t n = 0; n < S; ++n) {
      ar[n] /= (double)A;
      ai[n] /= (double)A;
    }
  }
}

/* Range-bin variants: FP32 reference order only (the bin index is a
 * floor of an FP32 quotient, so an FP64 form would bin differently). */
/* consistent != 0: keep delays up to 2 * spacing * bins, the bound that matches
 * the bin index (the reference keeps only d <= spacing * bins). */
void oracle_mf_fft_forward_f32(const float* re, const float* im, const float* tx, const float* rx,
                               const float* vox, int64_t A, int64_t B, int64_t N, float spacing,
                               int consistent, float* out_re, float* out_im) {
  const int bins = (int)B;
  const float bound = consistent ? 2.0f * (spacing * bins) : spacing * bins;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t v = 0; v < N; ++v) {
    float ar = 0.0f, ai = 0.0f;
    for (int64_t a = 0; a < A; ++a) {
      const float distance = mf_distance_f32(tx, rx, a, vox[v], vox[N + v], vox[2 * N + v]);
      if (distance < 0.0f || distance > bound) continue;
      const int bin = (int)floorf(distance / spacing / 2.0f);
      if (bin < 0 || bin >= bins) continue;
      const float tau = distance / K_C;
      const float phase = 2.0f * K_PI * K_F0MF * tau;
      const float c = cosf(phase), ns = -sinf(phase);
      const float sr = re[a * B + bin], si = im[a * B + bin];
      ar += c * sr - ns * si;
      ai += c * si + ns * sr;
    }
    out_re[v] = ar / (float)A;
    out_im[v] = ai / (float)A;
  }
}

void oracle_mf_fft_backward_f32(const float* gr, const float* gi, const float* tx, const float* rx,
                                const float* vox, int64_t A, int64_t B, int64_t N, float spacing,
                                int consistent, float* grad_re, float* grad_im) {
  const int bins = (int)B;
  const float bound = consistent ? 2.0f * (spacing * bins) : spacing * bins;
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t a = 0; a < A; ++a) {
    for (int64_t b = 0; b < B; ++b) {
      float ar = 0.0f, ai = 0.0f;
      for (int64_t v = 0; v < N; ++v) {
        const float distance = mf_distance_f32(tx, rx, a, vox[v], vox[N + v], vox[2 * N + v]);
        if (distance < 0.0f || distance > bound) continue;
        const int vb = (int)floorf(distance / spacing / 2.0f);
        if (vb != (int)b) continue;
        const float tau = distance / K_C;
        const float phase = 2.0f * K_PI * K_F0MF * tau;
        const float c = cosf(phase), ns = -sinf(phase);
        ar += c * gr[v] + ns * gi[v];
        ai += (-ns) * gr[v] + c * gi[v];
      }
      grad_re[a * B + b] = ar / (float)A;
      grad_im[a * B + b] = ai / (float)A;
    }
  }
}

/* ======================= signal tracer ==================================
 * SignalTracer_cuda_kernel.cu:19-197 (geometry, Jacobians), :351-450
 * (forward), :452-587 (adjoint onto sigma and normals). */

typedef struct {
  double inc[3], refl_raw[3], refl[3], ret[3];
  double align, idn, dist_t, dist_r;
} geo64;

static inline double dot3d(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

static inline void nrm3d(const double* in, double* out) {
  const double inv = 1.0 / (sqrt(dot3d(in, in)) + (double)K_EPS);
  out[0] = in[0] * inv;
  out[1] = in[1] * inv;
  out[2] = in[2] * inv;
}

static void geometry_f64(const float* tx, const float* rx, const float* nrm, const float* pt, geo64* g) {
  double ir[3], rr[3], n[3];
  for (int k = 0; k < 3; ++k) {
    ir[k] = (double)pt[k] - (double)tx[k];
    rr[k] = (double)rx[k] - (double)pt[k];
    n[k] = nrm[k];
  }
  g->dist_t = sqrt(dot3d(ir, ir));
  g->dist_r = sqrt(dot3d(rr, rr));
  nrm3d(ir, g->inc);
  g->idn = dot3d(g->inc, n);
  for (int k = 0; k < 3; ++k) g->refl_raw[k] = g->inc[k] - 2.0 * g->idn * n[k];
  nrm3d(g->refl_raw, g->refl);
  nrm3d(rr, g->ret);
  g->align = dot3d(g->ret, g->refl);
}

void oracle_tracer_forward_f64(const float* normals, const float* sigmas, const float* points,
                               const float* tx, const float* rx, const uint8_t* inb, int64_t A,
                               int64_t S, int64_t P, float fs, float f0, float As, double* out_re,
                               double* out_im) {
  const double w0 = 2.0 * (double)K_PI * (double)f0;
  const double w1 = 2.0 * (double)K_PI * (double)As;
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t a = 0; a < A; ++a) {
    double* ar = out_re + a * S;
    double* ai = out_im + a * S;
    for (int64_t n = 0; n < S; ++n) ar[n] = ai[n] = 0.0;
    for (int64_t p = 0; p < P; ++p) {
      if (!inb[p]) continue;
      geo64 g;
      geometry_f64(tx + a * 3, rx + a * 3, normals + p * 3, points + p * 3, &g);
      if (g.align < 1.0e-6 || g.idn > 0.0) continue;
      const double D = g.dist_t + g.dist_r;
      const double amp = (double)sigmas[a * P + p] * g.align / (D * D);
      const double tau = (D + (double)K_BIAS) / (double)K_C;
      for (int64_t n = 0; n < S; ++n) {
        const double phase = (w0 + w1 * ((double)n / (double)fs)) * tau;
        ar[n] += amp * cos(phase);
        ai[n] += amp * sin(phase);
      }
    }
    for (int64_t n = 0; n < S; ++n) {
      ar[n] /= (double)P;
      ai[n] /= (double)P;
    }
  }
}

/* FP32 reference-order geometry (ComputeSpecularGeometry and helpers). */
static inline float dot3f(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

static inline void nrm3f(const float* in, float* out) {
  const float norm = sqrtf(dot3f(in, in));
  const float inv = 1.0f / (norm + K_EPS);
  out[0] = in[0] * inv;
  out[1] = in[1] * inv;
  out[2] = in[2] * inv;
}

typedef struct {
  float inc[3], refl_raw[3], refl[3], ret[3];
  float align, idn;
} geo32;

static void geometry_f32(const float* tx, const float* rx, const float* n, const float* pt, geo32* g) {
  float ir[3], rr[3];
  for (int k = 0; k < 3; ++k) {
    ir[k] = pt[k] - tx[k];
    rr[k] = rx[k] - pt[k];
  }
  nrm3f(ir, g->inc);
  g->idn = dot3f(g->inc, n);
  for (int k = 0; k < 3; ++k) g->refl_raw[k] = g->inc[k] - 2.0f * g->idn * n[k];
  nrm3f(g->refl_raw, g->refl);
  nrm3f(rr, g->ret);
  g->align = dot3f(g->ret, g->refl);
}

static inline float path_distance_f32(const float* tx, const float* rx, const float* pt) {
  return sqrtf(sqf(tx[0] - pt[0]) + sqf(tx[1] - pt[1]) + sqf(tx[2] - pt[2])) +
         sqrtf(sqf(rx[0] - pt[0]) + sqf(rx[1] - pt[1]) + sqf(rx[2] - pt[2]));
}

void oracle_tracer_forward_f32(const float* normals, const float* sigmas, const float* points,
                               const float* tx, const float* rx, const uint8_t* inb, int64_t A,
                               int64_t S, int64_t P, float fs, float f0, float As, float* out_re,
                               float* out_im) {
  const float phase_base = 2.0f * K_PI * f0;
  const float phase_slope = 2.0f * K_PI * As;
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t a = 0; a < A; ++a) {
    for (int64_t n = 0; n < S; ++n) {
      const float sample_time = (float)n / fs;
      float ar = 0.0f, ai = 0.0f;
      for (int64_t p = 0; p < P; ++p) {
        if (!inb[p]) continue;
        geo32 g;
        geometry_f32(tx + a * 3, rx + a * 3, normals + p * 3, points + p * 3, &g);
        if (g.align < 1.0e-6f || g.idn > 0.0f) continue;
        float d = path_distance_f32(tx + a * 3, rx + a * 3, points + p * 3);
        const float amp = sigmas[a * P + p] * g.align / sqf(d);
        d += K_BIAS;
        const float tau = d / K_C;
        const float phase = (phase_base + phase_slope * sample_time) * tau;
        ar += amp * cosf(phase);
        ai += amp * sinf(phase);
      }
      out_re[a * S + n] = ar / (float)P;
      out_im[a * S + n] = ai / (float)P;
    }
  }
}

/* d rho / d n (reference Jacobian chain, exact arithmetic). */
static void drho_dn_f64(const geo64* g, const double* n, double* out) {
  double J[9], M[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) J[r * 3 + c] = -2.0 * n[r] * g->inc[c] - (r == c ? 2.0 * g->idn : 0.0);
  const double inv = 1.0 / (sqrt(dot3d(g->refl_raw, g->refl_raw)) + (double)K_EPS);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v += ((r == k ? 1.0 : 0.0) - g->refl[r] * g->refl[k]) * J[k * 3 + c];
      M[r * 3 + c] = v * inv;
    }
  for (int ax = 0; ax < 3; ++ax) {
    double v = 0.0;
    for (int k = 0; k < 3; ++k) v += M[k * 3 + ax] * g->ret[k];
    out[ax] = v;
  }
}

/* d rho / d p (no reference counterpart). */
static void drho_dp_f64(const geo64* g, const double* n, double* out) {
  const double rnorm = sqrt(dot3d(g->refl_raw, g->refl_raw));
  const double ro = dot3d(g->refl, g->ret);
  double u[3], v[3];
  for (int k = 0; k < 3; ++k) u[k] = (g->ret[k] - g->refl[k] * ro) / rnorm;
  const double nu = dot3d(n, u);
  for (int k = 0; k < 3; ++k) v[k] = u[k] - 2.0 * nu * n[k];
  const double iv = dot3d(g->inc, v);
  for (int k = 0; k < 3; ++k) out[k] = (v[k] - g->inc[k] * iv) / g->dist_t - (g->refl[k] - g->ret[k] * ro) / g->dist_r;
}

/* Adjoint in exact arithmetic.  grad_points may be NULL.  Out-of-bounds
 * points get zero gradients (the reference leaves them unwritten). */
void oracle_tracer_backward_f64(const float* gr, const float* gi, const float* normals,
                                const float* sigmas, const float* points, const float* tx,
                                const float* rx, const uint8_t* inb, int64_t A, int64_t S, int64_t P,
                                float fs, float f0, float As, double* g_normals, double* g_sigmas,
                                double* g_points) {
  const double w0 = 2.0 * (double)K_PI * (double)f0;
  const double w1 = 2.0 * (double)K_PI * (double)As;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t p = 0; p < P; ++p) {
    double gn[3] = {0, 0, 0}, gp[3] = {0, 0, 0};
    const double n[3] = {normals[p * 3], normals[p * 3 + 1], normals[p * 3 + 2]};
    for (int64_t a = 0; a < A; ++a) {
      g_sigmas[a * P + p] = 0.0;
      if (!inb[p]) continue;
      geo64 g;
      geometry_f64(tx + a * 3, rx + a * 3, normals + p * 3, points + p * 3, &g);
      if (g.align < 1.0e-6 || g.idn > 0.0) continue;
      const double D = g.dist_t + g.dist_r;
      const double atten = 1.0 / (D * D);
      const double sigma = sigmas[a * P + p];
      const double amp = sigma * g.align * atten;
      const double tau = (D + (double)K_BIAS) / (double)K_C;
      double sum_amp = 0.0, sum_tau = 0.0;
      for (int64_t s = 0; s < S; ++s) {
        const double wn = w0 + w1 * ((double)s / (double)fs);
        const double c = cos(wn * tau), sn = sin(wn * tau);
        const double r_ = gr[a * S + s], i_ = gi[a * S + s];
        sum_amp += r_ * c + i_ * sn;
        sum_tau += wn * (i_ * c - r_ * sn);
      }
      g_sigmas[a * P + p] = atten * g.align * sum_amp / (double)P;
      double dn[3];
      drho_dn_f64(&g, n, dn);
      for (int k = 0; k < 3; ++k) gn[k] += sigma * atten * dn[k] * sum_amp;
      if (g_points) {
        double dp[3];
        drho_dp_f64(&g, n, dp);
        for (int k = 0; k < 3; ++k) {
          const double dD = g.inc[k] - g.ret[k];
          const double damp = sigma * atten * dp[k] - 2.0 * amp / D * dD;
          gp[k] += sum_amp * damp + amp * sum_tau * dD / (double)K_C;
        }
      }
    }
    for (int k = 0; k < 3; ++k) {
      g_normals[p * 3 + k] = gn[k] / (double)P;
      if (g_points) g_points[p * 3 + k] = gp[k] / (double)P;
    }
  }
}

void oracle_tracer_backward_f32(const float* gr, const float* gi, const float* normals,
                                const float* sigmas, const float* points, const float* tx,
                                const float* rx, const uint8_t* inb, int64_t A, int64_t S, int64_t P,
                                float fs, float f0, float As, float* g_normals, float* g_sigmas) {
  const float phase_base = 2.0f * K_PI * f0;
  const float phase_slope = 2.0f * K_PI * As;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t p = 0; p < P; ++p) {
    float gn[3] = {0.0f, 0.0f, 0.0f};
    const float* n = normals + p * 3;
    for (int64_t a = 0; a < A; ++a) {
      g_sigmas[a * P + p] = 0.0f;
      if (!inb[p]) continue;
      geo32 g;
      geometry_f32(tx + a * 3, rx + a * 3, n, points + p * 3, &g);
      if (g.align < 1.0e-6f || g.idn > 0.0f) continue;
      float J[9], M[9], gsa[3];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
          const float shared = -2.0f * n[r] * g.inc[c];
          J[r * 3 + c] = r == c ? shared - 2.0f * g.idn : shared;
        }
      const float inv = 1.0f / (sqrtf(dot3f(g.refl_raw, g.refl_raw)) + K_EPS);
      const float x = g.refl[0], y = g.refl[1], z = g.refl[2];
      const float R[9] = {1.0f - x * x, -x * y, -x * z, -y * x, 1.0f - y * y, -y * z,
                          -z * x, -z * y, 1.0f - z * z};
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
          M[r * 3 + c] = (R[r * 3 + 0] * J[0 * 3 + c] + R[r * 3 + 1] * J[1 * 3 + c] + R[r * 3 + 2] * J[2 * 3 + c]) * inv;
      for (int ax = 0; ax < 3; ++ax) {
        float v = 0.0f;
        for (int k = 0; k < 3; ++k) v += M[k * 3 + ax] * g.ret[k];
        gsa[ax] = v;
      }
      float d = path_distance_f32(tx + a * 3, rx + a * 3, points + p * 3);
      const float atten = 1.0f / sqf(d);
      const float sigma = sigmas[a * P + p];
      d += K_BIAS;
      const float tau = d / K_C;
      float acc_sigma = 0.0f;
      for (int64_t s = 0; s < S; ++s) {
        const float sample_time = (float)s / fs;
        const float phase = (phase_base + phase_slope * sample_time) * tau;
        const float pr = cosf(phase), pi = sinf(phase);
        const float grr = gr[a * S + s] * pr;
        const float gii = gi[a * S + s] * pi;
        const float ns = sigma * atten;
        gn[0] += ns * gsa[0] * (grr + gii);
        gn[1] += ns * gsa[1] * (grr + gii);
        gn[2] += ns * gsa[2] * (grr + gii);
        acc_sigma += atten * g.align * (grr + gii);
      }
      g_sigmas[a * P + p] = acc_sigma / (float)P;
    }
    for (int k = 0; k < 3; ++k) g_normals[p * 3 + k] = gn[k] / (float)P;
  }
}

/* ======================= along-ray resampler ============================
 * SignalTracer_cuda_kernel.cu:199-349, arithmetic in the element type. */

static inline int bracket_f32(const float* z, int S, float t) {
  int lo = 0, hi = S - 1;
  while (lo < hi - 1) {
    const int mid = (lo + hi) / 2;
    if (z[mid] <= t) lo = mid;
    else hi = mid;
  }
  return lo;
}

void oracle_bilinear_forward_f32(const float* normals, const float* sigmas, const float* z,
                                 const float* tz, int64_t A, int64_t R, int64_t S, int64_t T,
                                 float* out_n, float* out_s, uint8_t* out_inb) {
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < R; ++r) {
    const float* zr = z + r * S;
    for (int64_t t = 0; t < T; ++t) {
      const float target = tz[r * T + t];
      const int lo = bracket_f32(zr, (int)S, target);
      const float z0 = zr[lo], z1 = zr[lo + 1];
      const int oob = (target < z0) || (target > z1);
      out_inb[r * T + t] = oob ? 0 : 1;
      float* on = out_n + (r * T + t) * 3;
      if (oob) {
        on[0] = on[1] = on[2] = 0.0f;
        for (int64_t a = 0; a < A; ++a) out_s[(a * R + r) * T + t] = 0.0f;
        continue;
      }
      const float den = (z1 - z0) > 1.0e-6f ? (z1 - z0) : 1.0e-6f;
      const float wu = (target - z0) / den;
      const float wl = 1.0f - wu;
      for (int k = 0; k < 3; ++k) on[k] = wl * normals[(r * S + lo) * 3 + k] + wu * normals[(r * S + lo + 1) * 3 + k];
      for (int64_t a = 0; a < A; ++a) {
        const float* sg = sigmas + (a * R + r) * S;
        out_s[(a * R + r) * T + t] = wl * sg[lo] + wu * sg[lo + 1];
      }
    }
  }
}

/* Adds into grad_n [R,S,3] and grad_s [A,R,S], target order per element. */
void oracle_bilinear_backward_f32(const float* gon, const float* gos, const float* z, const float* tz,
                                  int64_t A, int64_t R, int64_t S, int64_t T, float* grad_n,
                                  float* grad_s) {
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < R; ++r) {
    const float* zr = z + r * S;
    for (int64_t t = 0; t < T; ++t) {
      const float target = tz[r * T + t];
      const int lo = bracket_f32(zr, (int)S, target);
      const float z0 = zr[lo], z1 = zr[lo + 1];
      if (target < z0 || target > z1) continue;
      const float den = (z1 - z0) > 1.0e-6f ? (z1 - z0) : 1.0e-6f;
      const float wu = (target - z0) / den;
      const float wl = 1.0f - wu;
      for (int64_t a = 0; a < A; ++a) {
        const float g = gos[(a * R + r) * T + t];
        grad_s[(a * R + r) * S + lo] += wl * g;
        grad_s[(a * R + r) * S + lo + 1] += wu * g;
      }
      for (int k = 0; k < 3; ++k) {
        const float g = gon[(r * T + t) * 3 + k];
        grad_n[(r * S + lo) * 3 + k] += wl * g;
        grad_n[(r * S + lo + 1) * 3 + k] += wu * g;
      }
    }
  }
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  extern int omp_get_max_threads(void);
  return omp_get_max_threads();
#else
  return 1;
#endif
}
