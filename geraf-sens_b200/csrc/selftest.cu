// Test hooks of libgeraf_rf (declared in include/geraf_rf_testing.h): the
// operators' bounded-wait error path, driven to its timeout without a fault.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/geraf_rf.h"
#include "../../include/geraf_rf_testing.h"
#include "common.cuh"
#include "kernels.h"

#define GERAF_EXPORT extern "C" __attribute__((visibility("default")))

namespace geraf {
namespace {

// The staging ring of the MF and tracer kernels in bulk mode, with nothing
// ever issued: both stage barriers are initialised for one arrival that never
// comes, so wait() gives up after `limit_ns` exactly as a kernel whose copy
// never landed would, and the block leaves through the same drain-and-return
// path.
__global__ void __launch_bounds__(128) wait_timeout_kernel(int* status, uint64_t limit_ns,
                                                           int* returned) {
  __shared__ __align__(16) float buf[2 * 2 * 4];
  __shared__ __align__(8) uint64_t bar[2];
  PairStager<float> stg{buf, bar, 4, 1, true};
  stg.wait_ns = limit_ns;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (!stg.wait(0, 0, status)) {
    stg.drain(1, 0, status);
    if (threadIdx.x == 0) atomicAdd(returned, 1);
    return;
  }
}

}  // namespace
}  // namespace geraf

GERAF_EXPORT int32_t geraf_rf_selftest_wait_timeout(int64_t limit_ns, int32_t blocks,
                                                    int32_t* returned_blocks, void* stream) {
  if (limit_ns <= 0 || limit_ns > static_cast<int64_t>(geraf::kWaitLimitNs) || blocks <= 0 ||
      blocks > 1024 || returned_blocks == nullptr) {
    return GERAF_ERR_INVALID_ARGUMENT;
  }
  int* status = geraf::device_status_ptr();
  if (status == nullptr) return GERAF_ERR_CUDA;
  geraf::wait_timeout_kernel<<<blocks, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      status, static_cast<uint64_t>(limit_ns), reinterpret_cast<int*>(returned_blocks));
  return cudaGetLastError() == cudaSuccess ? GERAF_OK : GERAF_ERR_CUDA;
}
