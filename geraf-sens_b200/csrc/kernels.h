// Internal launch interface between the C ABI layer (capi.cu) and the kernel
// translation units.  Sizes are validated by the caller before any launcher
// runs; launchers only pick launch shapes, enqueue kernels and report the
// launch status.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace geraf {

enum DType : int { kF32 = 0, kF64 = 1, kF16 = 2 };
enum Mode : int { kPlain = 0, kMixed = 1, kNufft = 2 };

struct Tuning {
  int threads = 0;
  int items = 0;       // voxels / points per thread
  int stage_rows = 0;  // antenna rows per shared-memory stage
  int splits = 0;      // partial-sum splits of the reduced dimension
  int chunk = 0;       // samples per lane (sample-major kernels)
  int taps = 0;        // interpolation kernel width (NUFFT matched filter)
};

struct DeviceInfo {
  int sm_count;
  int max_smem_optin;
};
DeviceInfo current_device_info();

// Device address of the library's status word on the current device
// (a successful lookup is cached per device; null while lookups fail).
int* device_status_ptr();

// Sets the calling thread's message returned by geraf_rf_last_error().
void set_last_error(const char* msg);

// The matched filter's size / dtype / mode validation of geraf_mf_forward
// (GERAF_OK or an error code, with the message set).
int32_t mf_check_sizes(int64_t A, int64_t S, int64_t N, int32_t dtype, int32_t mode);

// ---- matched filter ------------------------------------------------------
struct MfArgs {
  const void* real;
  const void* imag;
  const void* tx;
  const void* rx;
  void* out_real;
  void* out_imag;
  const void* voxel;  // [3, N]
  const void* grad_real_out;  // backward: [N]
  const void* grad_imag_out;
  int64_t A, S, N;
  float fs, As;
  int dtype, mode;
};

Tuning mf_forward_resolve(const MfArgs& a, const Tuning& req);
size_t mf_forward_workspace(const MfArgs& a, const Tuning& t);
cudaError_t mf_forward(const MfArgs& a, const Tuning& t, void* ws, cudaStream_t st);

// Fast approximate matched filter (MODE_NUFFT, nufft_kernels.cu); the generic
// mf_forward_* entry points dispatch here for that mode.
constexpr int64_t kNufftMaxSamples = 4096;
bool mf_nufft_supported(int64_t S);
Tuning mf_nufft_forward_resolve(const MfArgs& a, const Tuning& req);
size_t mf_nufft_forward_workspace(const MfArgs& a, const Tuning& t);
cudaError_t mf_nufft_forward(const MfArgs& a, const Tuning& t, void* ws, cudaStream_t st);
Tuning mf_nufft_backward_resolve(const MfArgs& a, const Tuning& req);
size_t mf_nufft_backward_workspace(const MfArgs& a, const Tuning& t);
cudaError_t mf_nufft_backward(const MfArgs& a, const Tuning& t, void* ws, cudaStream_t st);

// Sums `splits` float2 partials per element in split order (FP64), divides by
// `divisor` and stores in the element type.
cudaError_t launch_finalize_partials(int dtype, const float2* partial, int splits, int64_t count,
                                     float divisor, void* out_r, void* out_i, cudaStream_t st);

Tuning mf_backward_resolve(const MfArgs& a, const Tuning& req);
size_t mf_backward_workspace(const MfArgs& a, const Tuning& t);
cudaError_t mf_backward(const MfArgs& a, const Tuning& t, void* ws, cudaStream_t st);

struct MfFftArgs {
  const void* real;  // forward: [A, bins] spectrum; backward: unused
  const void* imag;
  const void* tx;
  const void* rx;
  void* out_real;  // forward: [N]; backward: [A, bins]
  void* out_imag;
  const void* voxel;
  const void* grad_real_out;  // backward: [N]
  const void* grad_imag_out;
  int64_t A, bins, N;
  float spacing;
  int dtype;
  // false: the reference's bound (a delay d is kept when d <= spacing * bins, though
  // its bin floor(d / spacing / 2) reaches only half the bins); true: the bound
  // matches the index (d <= 2 spacing bins), so every bin can be reached
  bool consistent_bins;
};
cudaError_t mf_fft_forward(const MfFftArgs& a, cudaStream_t st);
cudaError_t mf_fft_backward(const MfFftArgs& a, cudaStream_t st);

// ---- signal tracer ------------------------------------------------------
struct TracerArgs {
  const void* normals;  // [P,3]
  const void* sigmas;   // [A,P]
  const void* points;   // [P,3]
  const void* tx;       // [A,3]
  const void* rx;
  const uint8_t* inbounds;  // [P]
  void* out_real;  // forward: [A,S]
  void* out_imag;
  const void* grad_real_out;  // backward: [A,S]
  const void* grad_imag_out;
  void* grad_normals;  // backward: [P,3]
  void* grad_sigmas;   // backward: [A,P]
  void* grad_points;   // backward: [P,3] or null
  int64_t A, S, P;
  float fs, f0, As;
  int dtype, mode;
};

Tuning tracer_forward_resolve(const TracerArgs& a, const Tuning& req);
size_t tracer_forward_workspace(const TracerArgs& a, const Tuning& t);
cudaError_t tracer_forward(const TracerArgs& a, const Tuning& t, void* ws, cudaStream_t st);

Tuning tracer_backward_resolve(const TracerArgs& a, const Tuning& req);
size_t tracer_backward_workspace(const TracerArgs& a, const Tuning& t);
cudaError_t tracer_backward(const TracerArgs& a, const Tuning& t, void* ws, cudaStream_t st);

// Point pre-cull of the MIXED and NUFFT tracers (tracer_precull.cu): the in-bounds points
// that a conservative per-point test cannot cull for every antenna of the call,
// listed in ascending order in a workspace region of tracer_point_list_bytes(P)
// bytes, with their count on the device.  With zero_grads the adjoint's
// gradients of every point left out are written as zeros.
struct PointList {
  const int* list;
  const int* count;
};
bool tracer_point_list_applies(const TracerArgs& a);
size_t tracer_point_list_bytes(int64_t P);
PointList tracer_point_list_view(void* ws, int64_t P);
cudaError_t tracer_point_list(const TracerArgs& a, void* ws, bool zero_grads, cudaStream_t st);

// Fast approximate tracer (MODE_NUFFT, nufft_tracer_kernels.cu); the generic
// tracer_* entry points dispatch here for that mode.
Tuning tracer_nufft_forward_resolve(const TracerArgs& a, const Tuning& req);
size_t tracer_nufft_forward_workspace(const TracerArgs& a, const Tuning& t);
cudaError_t tracer_nufft_forward(const TracerArgs& a, const Tuning& t, void* ws, cudaStream_t st);
Tuning tracer_nufft_backward_resolve(const TracerArgs& a, const Tuning& req);
size_t tracer_nufft_backward_workspace(const TracerArgs& a, const Tuning& t);
cudaError_t tracer_nufft_backward(const TracerArgs& a, const Tuning& t, void* ws, cudaStream_t st);

// Sums `splits` [P][6] partial point gradients in split order and divides by P
// into grad_normals (and grad_points when non-null); with a point list, only
// the listed points'.
cudaError_t launch_tracer_bwd_finalize(int dtype, const float* partial, int splits, int64_t P, void* g_normals,
                                       void* g_points, cudaStream_t st, const int* plist = nullptr,
                                       const int* plist_count = nullptr);

// Batched tracer over antennas with uneven point sets (CSR point_offsets [A+1]).
struct RaggedArgs {
  const void* normals;      // [P,3]
  const void* sigmas;       // [P]
  const void* points;       // [P,3]
  const int64_t* offsets;   // [A+1]
  const void* tx;           // [A,3]
  const void* rx;
  const uint8_t* inbounds;  // [P] or null
  void* out_real;           // forward: [A,S]
  void* out_imag;
  const void* grad_real_out;  // backward: [A,S]
  const void* grad_imag_out;
  void* grad_normals;  // backward: [P,3]
  void* grad_sigmas;   // backward: [P]
  void* grad_points;   // backward: [P,3] or null
  int64_t A, S, P;
  float fs, f0, As;
  int dtype;
};
// Launch shapes of the batched tracer.  Forward: threads (64, 128, 256),
// chunk = samples per lane (8, 16, 32), items = points per thread of one work
// item (0: from the step's size).  Adjoint: stage_rows = residual rows staged
// per block (1..8; 0: the default of 4, fewer when the rows are long).
Tuning tracer_ragged_forward_resolve(const RaggedArgs& a, const Tuning& req);
Tuning tracer_ragged_backward_resolve(const RaggedArgs& a, const Tuning& req);
size_t tracer_ragged_workspace(int64_t A, int64_t S, int64_t P, const Tuning& t);
cudaError_t tracer_forward_ragged(const RaggedArgs& a, const Tuning& t, void* ws, cudaStream_t st);
cudaError_t tracer_backward_ragged(const RaggedArgs& a, const Tuning& t, cudaStream_t st);

struct BilinearArgs {
  const void* normals;  // fwd: [R,S,3] in; bwd: grad_output_normals [R,T,3]
  const void* sigmas;   // fwd: [A,R,S] in; bwd: grad_output_sigmas [A,R,T]
  const void* z_vals;   // [R,S]
  const void* tz_vals;  // [R,T]
  void* out_normals;    // fwd: [R,T,3]; bwd: grad_normals [R,S,3] (accumulated)
  void* out_sigmas;     // fwd: [A,R,T]; bwd: grad_sigmas [A,R,S] (accumulated)
  uint8_t* out_inbounds;  // fwd: [R,T]
  int64_t A, R, S, T;
  int dtype;
};
cudaError_t bilinear_forward(const BilinearArgs& a, cudaStream_t st);
cudaError_t bilinear_backward(const BilinearArgs& a, cudaStream_t st);

// ---- volume sampling at target points -----------------------------------------
struct VolumeSampleArgs {
  const void* volume;  // [nx, ny, nz] float32, x slowest
  const void* points;  // [num_points, 3] float32, normalised (x, y, z)
  void* out;           // [num_points] float32
  int64_t nx, ny, nz, num_points;
  bool nearest, align_corners;
};
cudaError_t volume_sample(const VolumeSampleArgs& a, cudaStream_t st);

// ---- shared host helpers -------------------------------------------------
// FP64 phase constants of the MIXED form for start frequency f0, chirp slope
// As, sample rate fs (see path_cycles in common.cuh).
struct PhaseConsts {
  double k0, b0, k1, b1;
};
PhaseConsts phase_consts(float f0, float As, float fs);

// Picks the number of splits of the reduced dimension so that
// `units * splits` blocks fill the GPU in near-whole waves.
int pick_splits(int64_t units, int blocks_per_sm, int sm_count, int64_t max_splits);

}  // namespace geraf
