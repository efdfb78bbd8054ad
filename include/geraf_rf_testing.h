/*
 * geraf_rf_testing.h -- test hooks of `libgeraf_rf.so`.  Not operators and not
 * part of the drop-in interface (geraf_rf.h); no counterpart in the reference.
 * They exist so that the library's own device-side error paths can be
 * exercised on a GPU without faulting or hanging it.
 */
#ifndef GERAF_RF_TESTING_H_
#define GERAF_RF_TESTING_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Runs the operators' bounded-wait path to its timeout.  Enqueues `blocks`
 * blocks (1..1024) of 128 threads of the kernels' shared-memory staging code
 * (the double-buffered mbarrier ring) with a wait limit of `limit_ns`
 * (1 .. 2e9, the operators' own limit): every block waits on a stage barrier
 * that no copy or arrival ever completes, gives up after `limit_ns`, raises
 * GERAF_ERR_DEVICE_TIMEOUT in the device status word (read it with
 * geraf_rf_device_status), drains the other stage with the same bounded wait,
 * and returns.  Each block that returned this way adds 1 to *returned_blocks
 * (device memory, zeroed by the caller).  No memory access leaves the block's
 * own shared memory except those two words. */
int32_t geraf_rf_selftest_wait_timeout(int64_t limit_ns, int32_t blocks, int32_t* returned_blocks,
                                       void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GERAF_RF_TESTING_H_ */
