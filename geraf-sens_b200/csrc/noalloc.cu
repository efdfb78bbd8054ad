// Matched-filter forward that allocates nothing: the mixed-form split kernel
// with its partial sums kept in a fixed device array that ships inside this
// library, for callers that cannot allocate device memory.
//
// Who needs it: C/C++ hosts that embed the library with a fixed device-memory
// budget decided at start-up -- e.g. a radar acquisition pipeline that owns all
// of its buffers and forbids allocation once it runs -- cannot hand the regular
// geraf_mf_forward a workspace of their own, because the workspace size depends
// on the problem and allocating it would break that budget.  This entry point
// takes only the inputs and outputs; its scratch is a file-scope __device__
// array of kMaxSlots float2 (16 MiB), which every GPU that loads the library
// holds until the process exits.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/geraf_rf.h"
#include "common.cuh"
#include "kernels.h"

#define GERAF_EXPORT extern "C" __attribute__((visibility("default")))

namespace geraf {
namespace {

// 2^21 partial-sum slots of 8 bytes = 16 MiB: splits x num_voxels must fit.
constexpr int64_t kMaxSlots = int64_t{1} << 21;
constexpr int kMinSplits = 2;

static __device__ __align__(256) float2 g_noalloc_scratch[kMaxSlots];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void* g_scratch_ptr[kMaxDevices];  // guarded by g_scratch_mutex; null until a lookup succeeds

// In host code `g_noalloc_scratch` names a host-side shadow, not device
// memory: the device address is looked up with the device current.  A
// successful lookup is kept per device; a failed one (e.g. made before the
// device could be used) is not, so the next call tries again.
void* scratch_address(int dev, cudaError_t* err) {
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  *err = cudaSuccess;
  if (g_scratch_ptr[dev] == nullptr) {
    void* p = nullptr;
    *err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (*err != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    g_scratch_ptr[dev] = p;
  }
  return g_scratch_ptr[dev];
}

int32_t fail(int32_t code, const std::string& msg) {
  set_last_error(msg.c_str());
  return code;
}

}  // namespace
}  // namespace geraf

using namespace geraf;

GERAF_EXPORT int32_t geraf_mf_forward_noalloc(const void* real, const void* imag,
                                              const void* tx_pos, const void* rx_pos,
                                              void* output_real, void* output_imag,
                                              const void* voxel, int64_t total_ant_size,
                                              int64_t num_adc_samples, float adc_sample_rate,
                                              float chirp_slope_scaled, int64_t num_voxels,
                                              void* stream) {
  if (int32_t rc = mf_check_sizes(total_ant_size, num_adc_samples, num_voxels, GERAF_DTYPE_F32,
                                  GERAF_MODE_MIXED)) {
    return rc;
  }
  if (num_voxels > kMaxSlots / kMinSplits) {
    return fail(GERAF_ERR_INVALID_ARGUMENT,
                "num_voxels " + std::to_string(num_voxels) +
                    " exceeds the fixed scratch of geraf_mf_forward_noalloc (at most " +
                    std::to_string(kMaxSlots / kMinSplits) +
                    " voxels); use geraf_mf_forward with a caller-provided workspace");
  }
  if (num_voxels == 0) return GERAF_OK;
  if (output_real == nullptr || output_imag == nullptr || voxel == nullptr ||
      (total_ant_size > 0 && (tx_pos == nullptr || rx_pos == nullptr)) ||
      (total_ant_size > 0 && num_adc_samples > 0 && (real == nullptr || imag == nullptr))) {
    return fail(GERAF_ERR_INVALID_ARGUMENT, "pointers must be non-null");
  }
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    return fail(GERAF_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(err));
  }
  void* scratch = scratch_address(dev, &err);
  if (scratch == nullptr) {
    return fail(GERAF_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(err));
  }

  MfArgs a{};
  a.real = real;
  a.imag = imag;
  a.tx = tx_pos;
  a.rx = rx_pos;
  a.out_real = output_real;
  a.out_imag = output_imag;
  a.voxel = voxel;
  a.A = total_ant_size;
  a.S = num_adc_samples;
  a.N = num_voxels;
  a.fs = adc_sample_rate;
  a.As = chirp_slope_scaled;
  a.dtype = kF32;
  a.mode = kMixed;
  Tuning t = mf_forward_resolve(a, Tuning{});
  // Always the split variant: at least two partial sums per voxel, as many as fit.
  const int64_t rows_total = std::max<int64_t>(1, (a.A + t.stage_rows - 1) / t.stage_rows);
  const int64_t fit = kMaxSlots / num_voxels;
  t.splits = static_cast<int>(std::max<int64_t>(kMinSplits, std::min<int64_t>({t.splits, fit, rows_total})));
  if (t.splits < kMinSplits) t.splits = kMinSplits;
  // Every (split, voxel) slot is written before the finishing pass reads it,
  // so the scratch needs no clearing between calls.
  err = mf_forward(a, t, scratch, static_cast<cudaStream_t>(stream));
  if (err != cudaSuccess) {
    return fail(GERAF_ERR_CUDA,
                std::string("matched_filter_forward_noalloc launch: ") + cudaGetErrorString(err));
  }
  return GERAF_OK;
}
