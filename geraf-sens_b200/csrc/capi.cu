// extern "C" entry points of libgeraf_rf (declared in include/geraf_rf.h):
// argument validation with the reference's error wording, launch-shape
// resolution, workspace sizing, error reporting and the device status word.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/geraf_rf.h"
#include "common.cuh"
#include "kernels.h"

#define GERAF_EXPORT extern "C" __attribute__((visibility("default")))

namespace geraf {

__device__ int g_device_status = 0;

namespace {

thread_local std::string t_last_error;

int32_t fail(int32_t code, const std::string& msg) {
  t_last_error = msg;
  return code;
}

int32_t cuda_fail(cudaError_t err, const char* what) {
  t_last_error = std::string(what) + ": " + cudaGetErrorString(err);
  return GERAF_ERR_CUDA;
}

constexpr int kMaxDevices = 64;
std::once_flag g_dev_once[kMaxDevices];
DeviceInfo g_dev_info[kMaxDevices];
std::mutex g_status_mutex;
int* g_status_ptr[kMaxDevices];  // guarded by g_status_mutex; null until a lookup succeeds

int current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
  return dev;
}

void init_device(int dev) {
  DeviceInfo info{148, 227 * 1024};
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0)
    info.sm_count = v;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess && v > 0)
    info.max_smem_optin = v;
  g_dev_info[dev] = info;
}

void ensure_device(int dev) {
  std::call_once(g_dev_once[dev], init_device, dev);
}

Tuning to_tuning(const geraf_tuning_t* t) {
  Tuning out;
  if (t != nullptr) {
    out.threads = t->threads;
    out.items = t->items_per_thread;
    out.stage_rows = t->stage_rows;
    out.splits = t->splits;
    out.chunk = t->chunk;
    out.taps = t->taps;
  }
  return out;
}

bool valid_dtype(int32_t dtype, bool allow_half) {
  return dtype == GERAF_DTYPE_F32 || dtype == GERAF_DTYPE_F64 ||
         (allow_half && dtype == GERAF_DTYPE_F16);
}

const char* dtype_name(int32_t dtype) {
  return dtype == GERAF_DTYPE_F64 ? "Double" : dtype == GERAF_DTYPE_F16 ? "Half" : "Float";
}

constexpr int64_t kI32Max = 2147483647LL;

#define REQUIRE(cond, msg)                                      \
  do {                                                          \
    if (!(cond)) return fail(GERAF_ERR_INVALID_ARGUMENT, (msg)); \
  } while (0)

int32_t check_workspace(size_t need, void* ws, size_t bytes) {
  if (need == 0) return GERAF_OK;
  if (ws == nullptr || bytes < need) {
    return fail(GERAF_ERR_WORKSPACE, "workspace of " + std::to_string(need) +
                                         " bytes required, got " + std::to_string(bytes));
  }
  if ((reinterpret_cast<uintptr_t>(ws) & 255u) != 0) {
    return fail(GERAF_ERR_WORKSPACE, "workspace must be 256-byte aligned");
  }
  return GERAF_OK;
}

int32_t check_mf_sizes(int64_t A, int64_t S, int64_t N, int32_t dtype, int32_t mode) {
  REQUIRE(A >= 0 && S >= 0 && N >= 0, "sizes must be non-negative");
  REQUIRE(A <= kI32Max && S <= kI32Max && N <= kI32Max,
          "sizes must fit the reference's int arguments");
  REQUIRE(A * S <= (int64_t{1} << 40) && N <= (int64_t{1} << 31), "problem too large");
  if (!valid_dtype(dtype, true)) {
    return fail(GERAF_ERR_INVALID_ARGUMENT,
                std::string("\"matched_filter\" not implemented for '") + dtype_name(dtype) + "'");
  }
  REQUIRE(mode == GERAF_MODE_PLAIN || mode == GERAF_MODE_MIXED || mode == GERAF_MODE_NUFFT,
          "mode must be PLAIN, MIXED or NUFFT");
  if (mode == GERAF_MODE_NUFFT && !mf_nufft_supported(S)) {
    return fail(GERAF_ERR_UNSUPPORTED, "NUFFT matched filter needs num_adc_samples <= 4096");
  }
  return GERAF_OK;
}

int32_t check_tracer_sizes(int64_t A, int64_t S, int64_t P, int32_t dtype, int32_t mode) {
  REQUIRE(A >= 0 && S >= 0 && P >= 0, "sizes must be non-negative");
  REQUIRE(A <= kI32Max && S <= kI32Max && P <= kI32Max,
          "sizes must fit the reference's int arguments");
  if (!valid_dtype(dtype, false)) {
    return fail(GERAF_ERR_INVALID_ARGUMENT,
                std::string("\"signal_tracer\" not implemented for '") + dtype_name(dtype) + "'");
  }
  REQUIRE(mode == GERAF_MODE_PLAIN || mode == GERAF_MODE_MIXED || mode == GERAF_MODE_NUFFT,
          "mode must be PLAIN, MIXED or NUFFT");
  if (mode == GERAF_MODE_NUFFT && !mf_nufft_supported(S)) {
    return fail(GERAF_ERR_UNSUPPORTED, "NUFFT signal tracer needs num_adc_samples <= 4096");
  }
  return GERAF_OK;
}

int32_t finish_launch(cudaError_t err, const char* what) {
  if (err != cudaSuccess) return cuda_fail(err, what);
  return GERAF_OK;
}

MfArgs mf_args(int64_t A, int64_t S, int64_t N, float fs, float As, int32_t dtype, int32_t mode) {
  MfArgs a{};
  a.A = A;
  a.S = S;
  a.N = N;
  a.fs = fs;
  a.As = As;
  a.dtype = dtype;
  a.mode = mode;
  return a;
}

TracerArgs tracer_args(int64_t A, int64_t S, int64_t P, float fs, float f0, float As,
                       int32_t dtype, int32_t mode) {
  TracerArgs a{};
  a.A = A;
  a.S = S;
  a.P = P;
  a.fs = fs;
  a.f0 = f0;
  a.As = As;
  a.dtype = dtype;
  a.mode = mode;
  return a;
}

}  // namespace

void set_last_error(const char* msg) { t_last_error = msg; }

DeviceInfo current_device_info() {
  const int dev = current_device();
  ensure_device(dev);
  return g_dev_info[dev];
}

int* device_status_ptr() {
  const int dev = current_device();
  // A successful lookup is kept per device; a failed one (e.g. made before the
  // device could be used) is not, so the next call tries again.
  std::lock_guard<std::mutex> lock(g_status_mutex);
  if (g_status_ptr[dev] == nullptr) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_device_status) == cudaSuccess) {
      g_status_ptr[dev] = static_cast<int*>(ptr);
    } else {
      cudaGetLastError();
    }
  }
  return g_status_ptr[dev];
}

int32_t mf_check_sizes(int64_t A, int64_t S, int64_t N, int32_t dtype, int32_t mode) {
  return check_mf_sizes(A, S, N, dtype, mode);
}

PhaseConsts phase_consts(float f0, float As, float fs) {
  // pi_f / pi: the reference's 2*kPi factor is 2 * float(pi), not 2 pi.
  const double r = static_cast<double>(kPiF) / 3.14159265358979323846;
  const double c = static_cast<double>(kSpeedOfLight);
  PhaseConsts pc;
  pc.k0 = r * static_cast<double>(f0) / c;
  pc.b0 = static_cast<double>(kPathBias) * pc.k0;
  pc.k1 = r * static_cast<double>(As) / (static_cast<double>(fs) * c);
  pc.b1 = static_cast<double>(kPathBias) * pc.k1;
  return pc;
}

int pick_splits(int64_t units, int blocks_per_sm, int sm_count, int64_t max_splits) {
  const double slots = static_cast<double>(blocks_per_sm) * sm_count;
  if (units <= 0 || max_splits <= 1) return 1;
  if (static_cast<double>(units) >= 8.0 * slots) return 1;
  int best = 1;
  double best_score = -1.0;
  const int limit = static_cast<int>(std::min<int64_t>(max_splits, 256));
  for (int s = 1; s <= limit; ++s) {
    const double blocks = static_cast<double>(units) * s;
    const double waves = blocks / slots;
    const double eff = waves / std::ceil(waves);
    // Prefer full waves, then fewer splits (less partial-sum traffic).
    const double score = eff - 0.002 * s;
    if (waves >= 1.0 && score > best_score) {
      best_score = score;
      best = s;
    }
    if (blocks >= 16.0 * slots) break;
  }
  return best;
}

}  // namespace geraf

using namespace geraf;

// ===========================================================================
GERAF_EXPORT const char* geraf_rf_last_error(void) { return t_last_error.c_str(); }

GERAF_EXPORT int32_t geraf_rf_cudart_version(void) { return CUDART_VERSION; }

GERAF_EXPORT const char* geraf_rf_build_info(void) {
  static std::string info = [] {
    std::string s;
#if defined(__GNUC__) && !defined(__clang__)
    s += "GCC " + std::to_string(__GNUC__) + "." + std::to_string(__GNUC_MINOR__);
#endif
    s += "; nvcc " + std::to_string(__CUDACC_VER_MAJOR__) + "." + std::to_string(__CUDACC_VER_MINOR__);
    s += "; sm_100a";
    return s;
  }();
  return info.c_str();
}

GERAF_EXPORT int32_t geraf_rf_device_status(void* stream, int32_t reset, int32_t* status_out) {
  if (status_out == nullptr) return fail(GERAF_ERR_INVALID_ARGUMENT, "status_out is null");
  int* dptr = device_status_ptr();
  if (dptr == nullptr) return fail(GERAF_ERR_CUDA, "device status word unavailable");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int value = 0;
  cudaError_t err = cudaMemcpyAsync(&value, dptr, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  if (err == cudaSuccess && reset) {
    const int zero = 0;
    err = cudaMemcpyAsync(dptr, &zero, sizeof(int), cudaMemcpyHostToDevice, st);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  }
  if (err != cudaSuccess) return cuda_fail(err, "device status read");
  *status_out = value;
  return GERAF_OK;
}

// ---- matched filter --------------------------------------------------------
GERAF_EXPORT int32_t geraf_mf_forward_workspace_bytes(int64_t A, int64_t S, int64_t N, int32_t dtype,
                                                      int32_t mode, const geraf_tuning_t* tuning,
                                                      size_t* bytes) {
  if (bytes == nullptr) return fail(GERAF_ERR_INVALID_ARGUMENT, "bytes is null");
  if (int32_t rc = check_mf_sizes(A, S, N, dtype, mode)) return rc;
  const MfArgs a = mf_args(A, S, N, 1.0f, 0.0f, dtype, mode);
  *bytes = mf_forward_workspace(a, mf_forward_resolve(a, to_tuning(tuning)));
  return GERAF_OK;
}

GERAF_EXPORT int32_t geraf_mf_forward(const void* real, const void* imag, const void* tx_pos,
                                      const void* rx_pos, void* output_real, void* output_imag,
                                      const void* voxel, int64_t total_ant_size,
                                      int64_t num_adc_samples, float adc_sample_rate,
                                      float chirp_slope_scaled, int64_t num_voxels, int32_t dtype,
                                      int32_t mode, const geraf_tuning_t* tuning, void* workspace,
                                      size_t workspace_bytes, void* stream) {
  if (int32_t rc = check_mf_sizes(total_ant_size, num_adc_samples, num_voxels, dtype, mode)) return rc;
  if (num_voxels > 0) {
    REQUIRE(output_real != nullptr && output_imag != nullptr && voxel != nullptr,
            "output and voxel pointers must be non-null");
    if (total_ant_size > 0) {
      REQUIRE(tx_pos != nullptr && rx_pos != nullptr, "antenna position pointers must be non-null");
      if (num_adc_samples > 0) REQUIRE(real != nullptr && imag != nullptr, "sample pointers must be non-null");
    }
  }
  MfArgs a = mf_args(total_ant_size, num_adc_samples, num_voxels, adc_sample_rate,
                     chirp_slope_scaled, dtype, mode);
  a.real = real;
  a.imag = imag;
  a.tx = tx_pos;
  a.rx = rx_pos;
  a.out_real = output_real;
  a.out_imag = output_imag;
  a.voxel = voxel;
  const Tuning t = mf_forward_resolve(a, to_tuning(tuning));
  if (int32_t rc = check_workspace(mf_forward_workspace(a, t), workspace, workspace_bytes)) return rc;
  return finish_launch(mf_forward(a, t, workspace, static_cast<cudaStream_t>(stream)),
                       "matched_filter_forward launch");
}

GERAF_EXPORT int32_t geraf_mf_backward_workspace_bytes(int64_t A, int64_t S, int64_t N,
                                                       int32_t dtype, int32_t mode,
                                                       const geraf_tuning_t* tuning, size_t* bytes) {
  if (bytes == nullptr) return fail(GERAF_ERR_INVALID_ARGUMENT, "bytes is null");
  if (int32_t rc = check_mf_sizes(A, S, N, dtype, mode)) return rc;
  const MfArgs a = mf_args(A, S, N, 1.0f, 0.0f, dtype, mode);
  *bytes = mf_backward_workspace(a, mf_backward_resolve(a, to_tuning(tuning)));
  return GERAF_OK;
}

GERAF_EXPORT int32_t geraf_mf_backward(const void* grad_output_real, const void* grad_output_imag,
                                       const void* real, const void* imag, const void* tx_pos,
                                       const void* rx_pos, void* grad_real, void* grad_imag,
                                       const void* voxel, int64_t total_ant_size,
                                       int64_t num_adc_samples, float adc_sample_rate,
                                       float chirp_slope_scaled, int64_t num_voxels, int32_t dtype,
                                       int32_t mode, const geraf_tuning_t* tuning, void* workspace,
                                       size_t workspace_bytes, void* stream) {
  (void)real;
  (void)imag;
  if (int32_t rc = check_mf_sizes(total_ant_size, num_adc_samples, num_voxels, dtype, mode)) return rc;
  if (total_ant_size > 0 && num_adc_samples > 0) {
    REQUIRE(grad_real != nullptr && grad_imag != nullptr && tx_pos != nullptr && rx_pos != nullptr,
            "gradient and antenna pointers must be non-null");
    if (num_voxels > 0) {
      REQUIRE(grad_output_real != nullptr && grad_output_imag != nullptr && voxel != nullptr,
              "grad_output and voxel pointers must be non-null");
    }
  }
  MfArgs a = mf_args(total_ant_size, num_adc_samples, num_voxels, adc_sample_rate,
                     chirp_slope_scaled, dtype, mode);
  a.grad_real_out = grad_output_real;
  a.grad_imag_out = grad_output_imag;
  a.tx = tx_pos;
  a.rx = rx_pos;
  a.out_real = grad_real;
  a.out_imag = grad_imag;
  a.voxel = voxel;
  const Tuning t = mf_backward_resolve(a, to_tuning(tuning));
  if (int32_t rc = check_workspace(mf_backward_workspace(a, t), workspace, workspace_bytes)) return rc;
  return finish_launch(mf_backward(a, t, workspace, static_cast<cudaStream_t>(stream)),
                       "matched_filter_backward launch");
}

GERAF_EXPORT int32_t geraf_mf_fft_forward(const void* real, const void* imag, const void* tx_pos,
                                          const void* rx_pos, void* output_real, void* output_imag,
                                          const void* voxel, int64_t total_ant_size,
                                          int64_t num_range_bins, float fft_spacing,
                                          float adc_sample_rate, float chirp_slope_scaled,
                                          int64_t num_voxels, int32_t dtype, int32_t flags,
                                          void* stream) {
  (void)adc_sample_rate;
  (void)chirp_slope_scaled;
  if (int32_t rc = check_mf_sizes(total_ant_size, num_range_bins, num_voxels, dtype, GERAF_MODE_PLAIN)) return rc;
  REQUIRE((flags & ~GERAF_FFT_CONSISTENT_BINS) == 0, "unknown range-bin flags");
  MfFftArgs a{};
  a.consistent_bins = (flags & GERAF_FFT_CONSISTENT_BINS) != 0;
  a.real = real;
  a.imag = imag;
  a.tx = tx_pos;
  a.rx = rx_pos;
  a.out_real = output_real;
  a.out_imag = output_imag;
  a.voxel = voxel;
  a.A = total_ant_size;
  a.bins = num_range_bins;
  a.N = num_voxels;
  a.spacing = fft_spacing;
  a.dtype = dtype;
  return finish_launch(mf_fft_forward(a, static_cast<cudaStream_t>(stream)),
                       "matched_filter_fft_forward launch");
}

GERAF_EXPORT int32_t geraf_mf_fft_backward(const void* grad_output_real, const void* grad_output_imag,
                                           const void* real, const void* imag, const void* tx_pos,
                                           const void* rx_pos, void* grad_real, void* grad_imag,
                                           const void* voxel, int64_t total_ant_size,
                                           int64_t num_range_bins, float fft_spacing,
                                           float adc_sample_rate, float chirp_slope_scaled,
                                           int64_t num_voxels, int32_t dtype, int32_t flags,
                                           void* stream) {
  (void)real;
  (void)imag;
  (void)adc_sample_rate;
  (void)chirp_slope_scaled;
  if (int32_t rc = check_mf_sizes(total_ant_size, num_range_bins, num_voxels, dtype, GERAF_MODE_PLAIN)) return rc;
  REQUIRE((flags & ~GERAF_FFT_CONSISTENT_BINS) == 0, "unknown range-bin flags");
  MfFftArgs a{};
  a.consistent_bins = (flags & GERAF_FFT_CONSISTENT_BINS) != 0;
  a.tx = tx_pos;
  a.rx = rx_pos;
  a.out_real = grad_real;
  a.out_imag = grad_imag;
  a.voxel = voxel;
  a.grad_real_out = grad_output_real;
  a.grad_imag_out = grad_output_imag;
  a.A = total_ant_size;
  a.bins = num_range_bins;
  a.N = num_voxels;
  a.spacing = fft_spacing;
  a.dtype = dtype;
  return finish_launch(mf_fft_backward(a, static_cast<cudaStream_t>(stream)),
                       "matched_filter_fft_backward launch");
}

// ---- signal tracer ------------------------------------------------------------
GERAF_EXPORT int32_t geraf_tracer_forward_workspace_bytes(int64_t A, int64_t S, int64_t P,
                                                          int32_t dtype, int32_t mode,
                                                          const geraf_tuning_t* tuning,
                                                          size_t* bytes) {
  if (bytes == nullptr) return fail(GERAF_ERR_INVALID_ARGUMENT, "bytes is null");
  if (int32_t rc = check_tracer_sizes(A, S, P, dtype, mode)) return rc;
  const TracerArgs a = tracer_args(A, S, P, 1.0f, 0.0f, 0.0f, dtype, mode);
  *bytes = tracer_forward_workspace(a, tracer_forward_resolve(a, to_tuning(tuning)));
  return GERAF_OK;
}

GERAF_EXPORT int32_t geraf_tracer_forward(const void* normals, const void* sigmas, const void* points,
                                          const void* tx_pos, const void* rx_pos,
                                          const uint8_t* inbounds, void* output_real,
                                          void* output_imag, int64_t num_adc_samples,
                                          float adc_sample_rate, float start_frequency,
                                          float chirp_slope_scaled, int64_t total_ant_size,
                                          int64_t total_point_size, int32_t dtype, int32_t mode,
                                          const geraf_tuning_t* tuning, void* workspace,
                                          size_t workspace_bytes, void* stream) {
  if (int32_t rc = check_tracer_sizes(total_ant_size, num_adc_samples, total_point_size, dtype, mode)) return rc;
  if (total_ant_size > 0 && num_adc_samples > 0) {
    REQUIRE(output_real != nullptr && output_imag != nullptr && tx_pos != nullptr && rx_pos != nullptr,
            "output and antenna pointers must be non-null");
    if (total_point_size > 0) {
      REQUIRE(normals != nullptr && sigmas != nullptr && points != nullptr && inbounds != nullptr,
              "point pointers must be non-null");
    }
  }
  TracerArgs a = tracer_args(total_ant_size, num_adc_samples, total_point_size, adc_sample_rate,
                             start_frequency, chirp_slope_scaled, dtype, mode);
  a.normals = normals;
  a.sigmas = sigmas;
  a.points = points;
  a.tx = tx_pos;
  a.rx = rx_pos;
  a.inbounds = inbounds;
  a.out_real = output_real;
  a.out_imag = output_imag;
  const Tuning t = tracer_forward_resolve(a, to_tuning(tuning));
  if (int32_t rc = check_workspace(tracer_forward_workspace(a, t), workspace, workspace_bytes)) return rc;
  return finish_launch(tracer_forward(a, t, workspace, static_cast<cudaStream_t>(stream)),
                       "signal_tracer_forward launch");
}

GERAF_EXPORT int32_t geraf_tracer_backward_workspace_bytes(int64_t A, int64_t S, int64_t P,
                                                           int32_t dtype, int32_t mode,
                                                           int32_t with_points,
                                                           const geraf_tuning_t* tuning,
                                                           size_t* bytes) {
  (void)with_points;
  if (bytes == nullptr) return fail(GERAF_ERR_INVALID_ARGUMENT, "bytes is null");
  if (int32_t rc = check_tracer_sizes(A, S, P, dtype, mode)) return rc;
  const TracerArgs a = tracer_args(A, S, P, 1.0f, 0.0f, 0.0f, dtype, mode);
  *bytes = tracer_backward_workspace(a, tracer_backward_resolve(a, to_tuning(tuning)));
  return GERAF_OK;
}

GERAF_EXPORT int32_t geraf_tracer_backward(const void* grad_output_real, const void* grad_output_imag,
                                           const void* normals, const void* sigmas,
                                           const void* points, const void* tx_pos,
                                           const void* rx_pos, const uint8_t* inbounds,
                                           void* grad_normals, void* grad_sigmas, void* grad_points,
                                           int64_t num_adc_samples, float adc_sample_rate,
                                           float start_frequency, float chirp_slope_scaled,
                                           int64_t total_ant_size, int64_t total_point_size,
                                           int32_t dtype, int32_t mode,
                                           const geraf_tuning_t* tuning, void* workspace,
                                           size_t workspace_bytes, void* stream) {
  if (int32_t rc = check_tracer_sizes(total_ant_size, num_adc_samples, total_point_size, dtype, mode)) return rc;
  if (total_point_size > 0) {
    REQUIRE(grad_normals != nullptr && normals != nullptr && points != nullptr && inbounds != nullptr,
            "point pointers must be non-null");
    if (total_ant_size > 0) {
      REQUIRE(grad_sigmas != nullptr && sigmas != nullptr && tx_pos != nullptr && rx_pos != nullptr,
              "antenna pointers must be non-null");
      if (num_adc_samples > 0) {
        REQUIRE(grad_output_real != nullptr && grad_output_imag != nullptr,
                "grad_output pointers must be non-null");
      }
    }
  }
  TracerArgs a = tracer_args(total_ant_size, num_adc_samples, total_point_size, adc_sample_rate,
                             start_frequency, chirp_slope_scaled, dtype, mode);
  a.grad_real_out = grad_output_real;
  a.grad_imag_out = grad_output_imag;
  a.normals = normals;
  a.sigmas = sigmas;
  a.points = points;
  a.tx = tx_pos;
  a.rx = rx_pos;
  a.inbounds = inbounds;
  a.grad_normals = grad_normals;
  a.grad_sigmas = grad_sigmas;
  a.grad_points = grad_points;
  const Tuning t = tracer_backward_resolve(a, to_tuning(tuning));
  if (int32_t rc = check_workspace(tracer_backward_workspace(a, t), workspace, workspace_bytes)) return rc;
  return finish_launch(tracer_backward(a, t, workspace, static_cast<cudaStream_t>(stream)),
                       "signal_tracer_backward launch");
}

// ---- batched tracer over uneven per-antenna point sets ----------------------------
namespace {
int32_t check_ragged(int64_t A, int64_t S, int64_t P, int32_t dtype) {
  REQUIRE(A >= 0 && S >= 0 && P >= 0, "sizes must be non-negative");
  REQUIRE(A <= kI32Max && P <= (int64_t{1} << 40), "sizes out of range");
  REQUIRE(S <= 1024, "the batched tracer supports at most 1024 ADC samples");
  REQUIRE(!(A == 0 && P > 0), "points given but no antennas: point_offsets cannot be valid");
  if (!valid_dtype(dtype, false)) {
    return fail(GERAF_ERR_INVALID_ARGUMENT,
                std::string("\"signal_tracer_ragged\" not implemented for '") + dtype_name(dtype) + "'");
  }
  return GERAF_OK;
}
}  // namespace

GERAF_EXPORT int32_t geraf_tracer_ragged_workspace_bytes(int64_t A, int64_t S, int64_t P,
                                                         int32_t dtype, const geraf_tuning_t* tuning,
                                                         size_t* bytes) {
  if (bytes == nullptr) return fail(GERAF_ERR_INVALID_ARGUMENT, "bytes is null");
  if (int32_t rc = check_ragged(A, S, P, dtype)) return rc;
  RaggedArgs a{};
  a.A = A;
  a.S = S;
  a.P = P;
  *bytes = tracer_ragged_workspace(A, S, P, tracer_ragged_forward_resolve(a, to_tuning(tuning)));
  return GERAF_OK;
}

GERAF_EXPORT int32_t geraf_tracer_forward_ragged(
    const void* normals, const void* sigmas, const void* points, const int64_t* point_offsets,
    const void* tx_pos, const void* rx_pos, const uint8_t* inbounds, void* output_real,
    void* output_imag, int64_t num_adc_samples, float adc_sample_rate, float start_frequency,
    float chirp_slope_scaled, int64_t total_ant_size, int64_t total_point_size, int32_t dtype,
    const geraf_tuning_t* tuning, void* workspace, size_t workspace_bytes, void* stream) {
  if (int32_t rc = check_ragged(total_ant_size, num_adc_samples, total_point_size, dtype)) return rc;
  if (total_ant_size > 0 && num_adc_samples > 0) {
    REQUIRE(output_real && output_imag && tx_pos && rx_pos && point_offsets,
            "output, antenna and offset pointers must be non-null");
    if (total_point_size > 0) REQUIRE(normals && sigmas && points, "point pointers must be non-null");
  }
  RaggedArgs a{};
  a.normals = normals;
  a.sigmas = sigmas;
  a.points = points;
  a.offsets = point_offsets;
  a.tx = tx_pos;
  a.rx = rx_pos;
  a.inbounds = inbounds;
  a.out_real = output_real;
  a.out_imag = output_imag;
  a.A = total_ant_size;
  a.S = num_adc_samples;
  a.P = total_point_size;
  a.fs = adc_sample_rate;
  a.f0 = start_frequency;
  a.As = chirp_slope_scaled;
  a.dtype = dtype;
  const Tuning t = tracer_ragged_forward_resolve(a, to_tuning(tuning));
  if (int32_t rc = check_workspace(tracer_ragged_workspace(a.A, a.S, a.P, t), workspace, workspace_bytes)) return rc;
  return finish_launch(tracer_forward_ragged(a, t, workspace, static_cast<cudaStream_t>(stream)),
                       "signal_tracer_forward_ragged launch");
}

GERAF_EXPORT int32_t geraf_tracer_backward_ragged(
    const void* grad_output_real, const void* grad_output_imag, const void* normals,
    const void* sigmas, const void* points, const int64_t* point_offsets, const void* tx_pos,
    const void* rx_pos, const uint8_t* inbounds, void* grad_normals, void* grad_sigmas,
    void* grad_points, int64_t num_adc_samples, float adc_sample_rate, float start_frequency,
    float chirp_slope_scaled, int64_t total_ant_size, int64_t total_point_size, int32_t dtype,
    const geraf_tuning_t* tuning, void* stream) {
  if (int32_t rc = check_ragged(total_ant_size, num_adc_samples, total_point_size, dtype)) return rc;
  if (total_point_size > 0) {
    REQUIRE(grad_normals && grad_sigmas && normals && sigmas && points && point_offsets && tx_pos &&
                rx_pos && (num_adc_samples == 0 || (grad_output_real && grad_output_imag)),
            "pointers must be non-null");
  }
  RaggedArgs a{};
  a.grad_real_out = grad_output_real;
  a.grad_imag_out = grad_output_imag;
  a.normals = normals;
  a.sigmas = sigmas;
  a.points = points;
  a.offsets = point_offsets;
  a.tx = tx_pos;
  a.rx = rx_pos;
  a.inbounds = inbounds;
  a.grad_normals = grad_normals;
  a.grad_sigmas = grad_sigmas;
  a.grad_points = grad_points;
  a.A = total_ant_size;
  a.S = num_adc_samples;
  a.P = total_point_size;
  a.fs = adc_sample_rate;
  a.f0 = start_frequency;
  a.As = chirp_slope_scaled;
  a.dtype = dtype;
  return finish_launch(tracer_backward_ragged(a, tracer_ragged_backward_resolve(a, to_tuning(tuning)),
                                              static_cast<cudaStream_t>(stream)),
                       "signal_tracer_backward_ragged launch");
}

GERAF_EXPORT int32_t geraf_bilinear_forward(const void* normals, const void* sigmas,
                                            const void* z_vals, const void* target_z_vals,
                                            void* output_normals, void* output_sigmas,
                                            uint8_t* output_inbounds, int64_t num_antennas,
                                            int64_t num_rays, int64_t num_samples,
                                            int64_t num_target_samples, int32_t dtype,
                                            void* stream) {
  REQUIRE(num_antennas >= 0 && num_rays >= 0 && num_samples >= 0 && num_target_samples >= 0,
          "sizes must be non-negative");
  REQUIRE(num_antennas <= kI32Max && num_rays <= kI32Max && num_samples <= kI32Max &&
              num_target_samples <= kI32Max,
          "sizes must fit the reference's int arguments");
  if (!valid_dtype(dtype, false)) {
    return fail(GERAF_ERR_INVALID_ARGUMENT,
                std::string("\"bilinear_raysample_forward_cuda\" not implemented for '") +
                    dtype_name(dtype) + "'");
  }
  if (num_rays > 0 && num_target_samples > 0) {
    // The bracketing search reads samples lower and lower + 1 of every ray.
    REQUIRE(num_samples >= 2, "`z_vals` needs at least 2 samples per ray to bracket a target");
    REQUIRE(normals && z_vals && target_z_vals && output_normals && output_inbounds,
            "pointers must be non-null");
    REQUIRE(num_antennas == 0 || (sigmas && output_sigmas), "sigma pointers must be non-null");
  }
  BilinearArgs a{};
  a.normals = normals;
  a.sigmas = sigmas;
  a.z_vals = z_vals;
  a.tz_vals = target_z_vals;
  a.out_normals = output_normals;
  a.out_sigmas = output_sigmas;
  a.out_inbounds = output_inbounds;
  a.A = num_antennas;
  a.R = num_rays;
  a.S = num_samples;
  a.T = num_target_samples;
  a.dtype = dtype;
  return finish_launch(bilinear_forward(a, static_cast<cudaStream_t>(stream)),
                       "bilinear_raysample_forward launch");
}

GERAF_EXPORT int32_t geraf_bilinear_backward(const void* grad_output_normals,
                                             const void* grad_output_sigmas, const void* z_vals,
                                             const void* target_z_vals, void* grad_normals,
                                             void* grad_sigmas, int64_t num_antennas,
                                             int64_t num_rays, int64_t num_samples,
                                             int64_t num_target_samples, int32_t dtype,
                                             void* stream) {
  REQUIRE(num_antennas >= 0 && num_rays >= 0 && num_samples >= 0 && num_target_samples >= 0,
          "sizes must be non-negative");
  REQUIRE(num_antennas <= kI32Max && num_rays <= kI32Max && num_samples <= kI32Max &&
              num_target_samples <= kI32Max,
          "sizes must fit the reference's int arguments");
  if (!valid_dtype(dtype, false)) {
    return fail(GERAF_ERR_INVALID_ARGUMENT,
                std::string("\"bilinear_raysample_backward_cuda\" not implemented for '") +
                    dtype_name(dtype) + "'");
  }
  if (num_rays > 0 && num_target_samples > 0 && num_samples > 0) {
    REQUIRE(num_samples >= 2, "`z_vals` needs at least 2 samples per ray to bracket a target");
    REQUIRE(grad_output_normals && z_vals && target_z_vals && grad_normals,
            "pointers must be non-null");
    REQUIRE(num_antennas == 0 || (grad_output_sigmas && grad_sigmas), "sigma pointers must be non-null");
  }
  BilinearArgs a{};
  a.normals = grad_output_normals;
  a.sigmas = grad_output_sigmas;
  a.z_vals = z_vals;
  a.tz_vals = target_z_vals;
  a.out_normals = grad_normals;
  a.out_sigmas = grad_sigmas;
  a.A = num_antennas;
  a.R = num_rays;
  a.S = num_samples;
  a.T = num_target_samples;
  a.dtype = dtype;
  if (num_target_samples == 0) return GERAF_OK;
  return finish_launch(bilinear_backward(a, static_cast<cudaStream_t>(stream)),
                       "bilinear_raysample_backward launch");
}

// ---- matched-filter volume at target points --------------------------------
GERAF_EXPORT int32_t geraf_volume_sample(const void* volume, int64_t nx, int64_t ny, int64_t nz,
                                         const void* points_norm, int64_t num_points, void* out,
                                         int32_t mode, int32_t align_corners, void* stream) {
  REQUIRE(nx >= 0 && ny >= 0 && nz >= 0 && num_points >= 0, "sizes must be non-negative");
  REQUIRE(nx <= kI32Max && ny <= kI32Max && nz <= kI32Max, "volume dimensions must fit int32");
  REQUIRE(mode == GERAF_SAMPLE_TRILINEAR || mode == GERAF_SAMPLE_NEAREST,
          "mode must be GERAF_SAMPLE_TRILINEAR or GERAF_SAMPLE_NEAREST");
  const bool empty = nx == 0 || ny == 0 || nz == 0;
  if (num_points > 0) {
    REQUIRE(points_norm != nullptr && out != nullptr && (empty || volume != nullptr),
            "pointers must be non-null");
  }
  if (num_points == 0) return GERAF_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (empty) {  // an empty volume samples to zero everywhere
    return finish_launch(cudaMemsetAsync(out, 0, static_cast<size_t>(num_points) * sizeof(float), st),
                         "volume_sample fill");
  }
  VolumeSampleArgs a{};
  a.volume = volume;
  a.points = points_norm;
  a.out = out;
  a.nx = nx;
  a.ny = ny;
  a.nz = nz;
  a.num_points = num_points;
  a.nearest = mode == GERAF_SAMPLE_NEAREST;
  a.align_corners = align_corners != 0;
  return finish_launch(volume_sample(a, st), "volume_sample launch");
}
