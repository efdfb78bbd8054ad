/*
 * geraf_rf.h -- C ABI of the B200 (sm_100a) RF operator library `libgeraf_rf.so`.
 *
 * The library implements GeRaF's two RF operators, the FMCW matched-filter
 * backprojection (RFMatchedFilter) and the lensless specular signal tracer
 * (RFSignalTracer), plus the along-ray resampler that ships in the same
 * extension.  Every entry point here replaces one function of the reference's
 * pybind `_C` modules; the reference file:line of that function is given above
 * each declaration.  Paths are relative to the GeRaF-SENS checkout.
 *
 * Conventions (the same as the reference's `_C` functions):
 *   - All tensor arguments are raw DEVICE pointers to contiguous row-major
 *     arrays owned by the caller; outputs are written in place ("out-parameter"
 *     style); nothing is allocated by the library.
 *   - `dtype` selects the element type of every floating-point array of the
 *     call (GERAF_DTYPE_*).  Boolean masks are one byte per element (0 / 1).
 *   - Work is enqueued on `stream` (a cudaStream_t; NULL = legacy default
 *     stream) and the call returns without synchronising.
 *   - Return value: GERAF_OK, or a GERAF_ERR_* code; `geraf_rf_last_error()`
 *     then holds a message for the calling thread.
 *   - Entry points that may use a workspace (reduction partials, the tracer's
 *     point list) take `workspace` /
 *     `workspace_bytes`; the matching `*_workspace_bytes` query returns the
 *     size needed for the same arguments (0 when none is needed, in which case
 *     `workspace` may be NULL).  A workspace must be 256-byte aligned device
 *     memory and must not be shared by calls that may overlap on the GPU.
 */
#ifndef GERAF_RF_H_
#define GERAF_RF_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define GERAF_OK 0
#define GERAF_ERR_INVALID_ARGUMENT 1 /* shape / size / pointer / dtype problem   */
#define GERAF_ERR_UNSUPPORTED 2      /* valid request this build does not serve  */
#define GERAF_ERR_WORKSPACE 3        /* workspace missing, short or misaligned   */
#define GERAF_ERR_CUDA 4             /* a CUDA runtime call or launch failed      */
#define GERAF_ERR_DEVICE_TIMEOUT 5   /* a bounded device-side wait gave up        */
#define GERAF_ERR_DEVICE_CHECK 6     /* a device-side consistency check failed    */

/* ---- element types (match the reference's AT_DISPATCH lists) ----------- */
#define GERAF_DTYPE_F32 0
#define GERAF_DTYPE_F64 1
#define GERAF_DTYPE_F16 2 /* matched filter only, as in the reference */

/* ---- arithmetic forms -------------------------------------------------- */
/* PLAIN: the reference's FP32 arithmetic, expression for expression: one
 *        accurate sinf/cosf per (voxel|point, antenna, sample) and the
 *        reference's summation order per output element.  Judged against the
 *        reference kernels (relative L2 <= 1e-5).
 * MIXED: carrier phase f0*tau reduced modulo one cycle in FP64, per-sample
 *        sums by FP32 recurrences (second-order Goertzel, three-term
 *        Chebyshev, packed Horner; a few phasors per (voxel|point, antenna)
 *        instead of one per sample), compensated
 *        (Kahan) accumulation across antennas.  Judged against an FP64 oracle
 *        (relative L2 <= 1e-4).                                              */
#define GERAF_MODE_PLAIN 0
#define GERAF_MODE_MIXED 1
/* NUFFT (matched filter and signal tracer; no reference counterpart): the
 *        MIXED phase model with the per-antenna sample sums evaluated through
 *        oversampled range FFTs and a W-point "exponential of semicircle"
 *        interpolation kernel, O(W) instead of O(S) work per
 *        (voxel|point, antenna).  A fast approximate form: relative L2
 *        against the FP64 oracle ~1e-6 at W = 8 (tuning.taps), ~1e-3 at
 *        W = 4.  Needs num_adc_samples <= 4096.  Each adjoint is the exact
 *        adjoint of its forward.  Not available for the ragged tracer.     */
#define GERAF_MODE_NUFFT 2

/* Launch shape.  Any field left 0 takes the library default for the call. */
typedef struct geraf_tuning {
  int32_t threads;          /* threads per block: 64, 128 or 256                       */
  int32_t items_per_thread; /* voxels (MF forward) or points (tracer adjoint): 1, 2, 4 */
  int32_t stage_rows;       /* antenna rows per shared-memory stage                     */
  int32_t splits;           /* partial-sum splits of the reduced dimension              */
  int32_t chunk;            /* samples per lane in the sample-major kernels: 8,16,32    */
  int32_t taps;             /* NUFFT interpolation width W: 4, 6, 8, 10 or 12           */
} geraf_tuning_t;

/* ---- library information ---------------------------------------------- */
/* Message of the last failed call on this thread ("" if none). */
const char* geraf_rf_last_error(void);
/* CUDART_VERSION the library was built with (reference: csrc/cuda_version.cu:8). */
int32_t geraf_rf_cudart_version(void);
/* Compiler and target description, e.g. "GCC 13.3; nvcc 12.9; sm_100a"
 * (reference: csrc/vision.cpp:47-68, get_compiler_version). */
const char* geraf_rf_build_info(void);
/* Reads, and with reset != 0 clears, the device status word of the current
 * device: GERAF_OK, or the code a kernel raised -- GERAF_ERR_DEVICE_TIMEOUT
 * (a bounded wait gave up), GERAF_ERR_INVALID_ARGUMENT (malformed ragged
 * point offsets), GERAF_ERR_DEVICE_CHECK (a NUFFT adjoint point fell outside
 * the band bounded from the voxels' bounding box; it was skipped).
 * Synchronises `stream`. */
int32_t geraf_rf_device_status(void* stream, int32_t reset, int32_t* status_out);

/* ---- RFMatchedFilter ---------------------------------------------------- */
/* y[v] = (1/A) sum_a sum_n (re + j im)[a,n] * exp(-j phi(a,v,n)),
 * phi = 2*pi*773.704*tau + 2*pi*As*(n/fs)*tau,  tau = (|tx_a-v| + |rx_a-v| + 0.15)/2.9979.
 * real, imag: [A,S]; tx_pos, rx_pos: [A,3]; voxel: [3,N] (x row, y row, z row);
 * output_real, output_imag: [N].
 * Replaces MatchedFilter::MatchedFilter_forward
 * (geraf/ops/RFMatchedFilter/csrc/matched_filter/MatchedFilter_cuda.cu:173-210,
 *  kernel MatchedFilter_cuda_kernel.cu:65-115). */
int32_t geraf_mf_forward_workspace_bytes(int64_t total_ant_size, int64_t num_adc_samples,
                                         int64_t num_voxels, int32_t dtype, int32_t mode,
                                         const geraf_tuning_t* tuning, size_t* bytes);
int32_t geraf_mf_forward(const void* real, const void* imag, const void* tx_pos,
                         const void* rx_pos, void* output_real, void* output_imag,
                         const void* voxel, int64_t total_ant_size, int64_t num_adc_samples,
                         float adc_sample_rate, float chirp_slope_scaled, int64_t num_voxels,
                         int32_t dtype, int32_t mode, const geraf_tuning_t* tuning,
                         void* workspace, size_t workspace_bytes, void* stream);

/* Exact adjoint of geraf_mf_forward with respect to (real, imag):
 * grad[a,n] = (1/A) sum_v (g_r + j g_i)[v] * exp(+j phi(a,v,n)).
 * grad_output_real/imag: [N]; grad_real, grad_imag: [A,S] (overwritten).
 * `real`/`imag` are accepted for signature parity and not read.
 * Replaces MatchedFilter::MatchedFilter_backward_realimag
 * (MatchedFilter_cuda.cu:253-297, kernel MatchedFilter_cuda_kernel.cu:171-220). */
int32_t geraf_mf_backward_workspace_bytes(int64_t total_ant_size, int64_t num_adc_samples,
                                          int64_t num_voxels, int32_t dtype, int32_t mode,
                                          const geraf_tuning_t* tuning, size_t* bytes);
int32_t geraf_mf_backward(const void* grad_output_real, const void* grad_output_imag,
                          const void* real, const void* imag, const void* tx_pos,
                          const void* rx_pos, void* grad_real, void* grad_imag,
                          const void* voxel, int64_t total_ant_size, int64_t num_adc_samples,
                          float adc_sample_rate, float chirp_slope_scaled, int64_t num_voxels,
                          int32_t dtype, int32_t mode, const geraf_tuning_t* tuning,
                          void* workspace, size_t workspace_bytes, void* stream);

/* Range-bin variant: per antenna, gather bin floor(d/fft_spacing/2) of the
 * [A,bins] spectrum (skipped when d > fft_spacing*bins) times exp(-j 2 pi 773.704 tau).
 * `flags`: 0 for the reference's behaviour; GERAF_FFT_CONSISTENT_BINS keeps
 * delays up to 2*fft_spacing*bins instead, the bound that matches the bin index
 * (the reference's bound reaches only the first half of the bins).
 * Replaces MatchedFilter::MatchedFilter_fft_forward (MatchedFilter_cuda.cu:212-251,
 * kernel MatchedFilter_cuda_kernel.cu:117-169). */
#define GERAF_FFT_CONSISTENT_BINS 1
int32_t geraf_mf_fft_forward(const void* real, const void* imag, const void* tx_pos,
                             const void* rx_pos, void* output_real, void* output_imag,
                             const void* voxel, int64_t total_ant_size, int64_t num_range_bins,
                             float fft_spacing, float adc_sample_rate, float chirp_slope_scaled,
                             int64_t num_voxels, int32_t dtype, int32_t flags, void* stream);
/* Adjoint of geraf_mf_fft_forward (same `flags`).  Replaces
 * MatchedFilter::MatchedFilter_fft_backward_realimag (MatchedFilter_cuda.cu:299-343,
 * kernel MatchedFilter_cuda_kernel.cu:222-279). */
int32_t geraf_mf_fft_backward(const void* grad_output_real, const void* grad_output_imag,
                              const void* real, const void* imag, const void* tx_pos,
                              const void* rx_pos, void* grad_real, void* grad_imag,
                              const void* voxel, int64_t total_ant_size, int64_t num_range_bins,
                              float fft_spacing, float adc_sample_rate, float chirp_slope_scaled,
                              int64_t num_voxels, int32_t dtype, int32_t flags, void* stream);

/* Matched-filter forward (MIXED form, FP32 arrays) that allocates nothing and
 * takes no workspace.  No counterpart in the reference.  It serves callers that
 * cannot allocate device memory: hosts that fix their device-memory budget at
 * start-up and own every buffer (e.g. a radar acquisition pipeline that may not
 * allocate once it runs) and so cannot provide the problem-sized workspace
 * geraf_mf_forward asks for.  The partial sums live in a 16 MiB array compiled
 * into this library, which every GPU that loads the library holds until the
 * process exits; hence num_voxels <= 1048576 (larger sizes return
 * GERAF_ERR_INVALID_ARGUMENT).  The first call on each device looks up that
 * array's device address (make it before any stream capture).  All calls share
 * the array: calls that may overlap on the GPU (other streams, other host
 * threads) race and must be serialised by the caller.  Arguments as for
 * geraf_mf_forward. */
int32_t geraf_mf_forward_noalloc(const void* real, const void* imag, const void* tx_pos,
                                 const void* rx_pos, void* output_real, void* output_imag,
                                 const void* voxel, int64_t total_ant_size,
                                 int64_t num_adc_samples, float adc_sample_rate,
                                 float chirp_slope_scaled, int64_t num_voxels, void* stream);

/* ---- RFSignalTracer ----------------------------------------------------- */
/* x[a,n] = (1/P) sum_{p in-bounds, not culled} sigma[a,p] * rho / D^2 * exp(+j (2 pi f0 + 2 pi As t_n) tau),
 * rho = <normalize(rx_a - p), normalize(i - 2 (i.n) n)>, i = normalize(p - tx_a),
 * culled when rho < 1e-6 or i.n > 0; D = |tx_a - p| + |rx_a - p|; tau = (D + 0.15)/2.9979.
 * normals, points: [P,3]; sigmas: [A,P]; tx_pos, rx_pos: [A,3]; inbounds: [P] (u8);
 * output_real, output_imag: [A,S].
 * In MIXED and NUFFT mode the forward and the adjoint first list, in their
 * workspace (about 4.3 bytes per point), the in-bounds points that a
 * conservative test cannot cull for every antenna of the call, and visit only
 * those; the workspace is therefore needed even without split partials.
 * Replaces SignalTracer::SignalTracer_forward
 * (geraf/ops/RFSignalTracer/csrc/signal_tracer/SignalTracer_cuda.cu:314-356,
 *  kernel SignalTracer_cuda_kernel.cu:351-450). */
int32_t geraf_tracer_forward_workspace_bytes(int64_t total_ant_size, int64_t num_adc_samples,
                                             int64_t total_point_size, int32_t dtype, int32_t mode,
                                             const geraf_tuning_t* tuning, size_t* bytes);
int32_t geraf_tracer_forward(const void* normals, const void* sigmas, const void* points,
                             const void* tx_pos, const void* rx_pos, const uint8_t* inbounds,
                             void* output_real, void* output_imag, int64_t num_adc_samples,
                             float adc_sample_rate, float start_frequency,
                             float chirp_slope_scaled, int64_t total_ant_size,
                             int64_t total_point_size, int32_t dtype, int32_t mode,
                             const geraf_tuning_t* tuning, void* workspace,
                             size_t workspace_bytes, void* stream);

/* Adjoint of geraf_tracer_forward: grad_sigmas [A,P], grad_normals [P,3] and,
 * when grad_points != NULL, grad_points [P,3] (the reference has no position
 * gradient).  Entries of out-of-bounds points are written as zero (the
 * reference leaves them unwritten).  grad_output_real/imag: [A,S].
 * Replaces SignalTracer::SignalTracer_backward_normal_sigma
 * (SignalTracer_cuda.cu:358-406, kernel SignalTracer_cuda_kernel.cu:452-587). */
int32_t geraf_tracer_backward_workspace_bytes(int64_t total_ant_size, int64_t num_adc_samples,
                                              int64_t total_point_size, int32_t dtype,
                                              int32_t mode, int32_t with_points,
                                              const geraf_tuning_t* tuning, size_t* bytes);
int32_t geraf_tracer_backward(const void* grad_output_real, const void* grad_output_imag,
                              const void* normals, const void* sigmas, const void* points,
                              const void* tx_pos, const void* rx_pos, const uint8_t* inbounds,
                              void* grad_normals, void* grad_sigmas, void* grad_points,
                              int64_t num_adc_samples, float adc_sample_rate,
                              float start_frequency, float chirp_slope_scaled,
                              int64_t total_ant_size, int64_t total_point_size, int32_t dtype,
                              int32_t mode, const geraf_tuning_t* tuning, void* workspace,
                              size_t workspace_bytes, void* stream);

/* Batched tracer over all antennas of a step, each with its own uneven set of
 * points (MIXED form).  Points of antenna 0 come first, then antenna 1, ...;
 * point_offsets [A+1] (int64, CSR, offsets[0] = 0, offsets[A] = P,
 * non-decreasing) delimits them.  normals, points: [P,3]; sigmas: [P] (each
 * point's amplitude weight for its own antenna); inbounds: [P] or NULL (all
 * in bounds); output [A,S]; S <= 1024.  Row a equals geraf_tracer_forward
 * over antenna a's points alone (normalised by that antenna's point count;
 * an antenna without points gives NaN, as 0/0 in the reference).  One
 * persistent launch load-balances the uneven antennas; malformed offsets are
 * detected on the device (no point is read; device status word = 1).
 * Replaces a loop of SignalTracer::SignalTracer_forward calls, one per antenna
 * (SignalTracer_cuda.cu:314-356): the batched entry point has no single
 * counterpart in the reference. */
/* Launch shape (`tuning`, may be NULL): threads (64, 128, 256), chunk =
 * samples per lane (8, 16, 32), items_per_thread = points per thread of one
 * work item (0: sized from the step); the workspace size depends on it. */
int32_t geraf_tracer_ragged_workspace_bytes(int64_t total_ant_size, int64_t num_adc_samples,
                                            int64_t total_point_size, int32_t dtype,
                                            const geraf_tuning_t* tuning, size_t* bytes);
int32_t geraf_tracer_forward_ragged(const void* normals, const void* sigmas, const void* points,
                                    const int64_t* point_offsets, const void* tx_pos,
                                    const void* rx_pos, const uint8_t* inbounds, void* output_real,
                                    void* output_imag, int64_t num_adc_samples,
                                    float adc_sample_rate, float start_frequency,
                                    float chirp_slope_scaled, int64_t total_ant_size,
                                    int64_t total_point_size, int32_t dtype,
                                    const geraf_tuning_t* tuning, void* workspace,
                                    size_t workspace_bytes, void* stream);
/* Adjoint of geraf_tracer_forward_ragged: grad_sigmas [P], grad_normals [P,3]
 * and, when non-NULL, grad_points [P,3]; out-of-bounds points get zeros.
 * `tuning` (may be NULL): stage_rows = residual rows staged per block (1..8). 
 * Replaces the per-antenna SignalTracer::SignalTracer_backward_normal_sigma
 * calls (SignalTracer_cuda.cu:358-406). */
int32_t geraf_tracer_backward_ragged(const void* grad_output_real, const void* grad_output_imag,
                                     const void* normals, const void* sigmas, const void* points,
                                     const int64_t* point_offsets, const void* tx_pos,
                                     const void* rx_pos, const uint8_t* inbounds,
                                     void* grad_normals, void* grad_sigmas, void* grad_points,
                                     int64_t num_adc_samples, float adc_sample_rate,
                                     float start_frequency, float chirp_slope_scaled,
                                     int64_t total_ant_size, int64_t total_point_size,
                                     int32_t dtype, const geraf_tuning_t* tuning, void* stream);

/* Linear resampling along rays: for each ray and target depth, bracket the
 * target in the ray's coarse depths by binary search and interpolate sigma
 * (all A rows) and normals; out-of-range targets give 0 and inbounds = 0.
 * normals [R,S,3], sigmas [A,R,S], z_vals [R,S], target_z_vals [R,T];
 * output_normals [R,T,3], output_sigmas [A,R,T], output_inbounds [R,T] (u8).
 * Replaces SignalTracer::BilinearRaysample_forward
 * (SignalTracer_cuda.cu:241-276, kernel SignalTracer_cuda_kernel.cu:199-279). */
int32_t geraf_bilinear_forward(const void* normals, const void* sigmas, const void* z_vals,
                               const void* target_z_vals, void* output_normals,
                               void* output_sigmas, uint8_t* output_inbounds,
                               int64_t num_antennas, int64_t num_rays, int64_t num_samples,
                               int64_t num_target_samples, int32_t dtype, void* stream);
/* Adjoint of geraf_bilinear_forward; ADDS into grad_normals [R,S,3] and
 * grad_sigmas [A,R,S] (the reference's callers pass zeroed buffers).
 * Replaces SignalTracer::BilinearRaysample_backward
 * (SignalTracer_cuda.cu:278-312, kernel SignalTracer_cuda_kernel.cu:281-349). */
int32_t geraf_bilinear_backward(const void* grad_output_normals, const void* grad_output_sigmas,
                                const void* z_vals, const void* target_z_vals,
                                void* grad_normals, void* grad_sigmas, int64_t num_antennas,
                                int64_t num_rays, int64_t num_samples,
                                int64_t num_target_samples, int32_t dtype, void* stream);

/* ---- matched-filter volume at target points ----------------------------- */
/* out[i] = the volume [nx, ny, nz] (float32, x slowest, as sarimage.bin) sampled
 * at points_norm[i] = (x, y, z) in normalised [-1, 1]^3 coordinates: trilinear
 * (mode GERAF_SAMPLE_TRILINEAR) or nearest-voxel (GERAF_SAMPLE_NEAREST, ties to
 * even), zero outside the volume, corners at +-1 when align_corners != 0.
 * points_norm [num_points, 3] and out [num_points] are float32.  The torch
 * grid_sample call of the reference's data workers: the volume as a
 * [1,1,nx,ny,nz] tensor with the grid given as (z, y, x), padding zeros.
 * Replaces _sample_volume / InterpolateMFAtTargets
 * (geraf/datasets/transforms/loading.py:20-25, 78-100), which run on the host. */
#define GERAF_SAMPLE_TRILINEAR 0
#define GERAF_SAMPLE_NEAREST 1
int32_t geraf_volume_sample(const void* volume, int64_t nx, int64_t ny, int64_t nz,
                            const void* points_norm, int64_t num_points, void* out, int32_t mode,
                            int32_t align_corners, void* stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* GERAF_RF_H_ */
