"""ctypes binding of ``libgeraf_probe.so`` (``benchkit/probe.cu``): the FP32
peak probes behind ``bench.py``'s roofline and the sincosf identity check.

Each probe enqueues work on a stream and returns a status code of
``include/geraf_rf.h`` (0 = ok); the caller times it with CUDA events.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgeraf_probe.so")

_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
SIGNATURES = {
    # blocks x threads (<= 256) threads of `iters` x 8 packed FMA pairs:
    # blocks * threads * iters * 32 flops
    "geraf_rf_fma_probe": (_i32, [_i32, _i32, _i32, _vp, _vp]),
    # blocks x threads (<= 128) threads of the MIXED forward's Horner loop over
    # `rows` rows of 256 samples x 8 voxels: blocks * threads * rows * 16384 flops
    "geraf_rf_horner_probe": (_i32, [_i32, _i32, _i32, _vp, _vp]),
    # the same sum by the second-order (Goertzel) recurrence, same flop count
    "geraf_rf_goertzel_probe": (_i32, [_i32, _i32, _i32, _vp, _vp]),
    # adds to *mismatches (device u64) the FP32 inputs where sincosf differs
    # from separate sinf / cosf calls in any bit (all 2^32 inputs)
    "geraf_rf_sincos_identity_check": (_i32, [_vp, _vp]),
}

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built (make -C benchkit)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, what: str) -> None:
    if status != 0:
        raise RuntimeError(f"{what} failed with status {status}")


def measure(name: str, blocks_per_sm: int, device=0) -> float:
    """Best-of-5 rate of one probe in TFLOP/s (CUDA events on the current stream)."""
    import torch

    dev = torch.device("cuda", device)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    if name == "fma":
        blocks, threads, arg, flops = sms * blocks_per_sm, 256, 1 << 12, 32
    else:
        blocks, threads, arg, flops = sms * blocks_per_sm, 128, 256, 16384
    fn = getattr(lib(), f"geraf_rf_{name}_probe")
    sink = torch.empty(blocks * threads, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        check(fn(blocks, threads, arg, sink.data_ptr(), stream), name)
        e.record()
        e.synchronize()
        best = max(best, blocks * threads * arg * flops / (s.elapsed_time(e) * 1e-3) / 1e12)
    return best


def main() -> int:
    """Prints the FP32 FMA rate and the two loop probes at 2-6 blocks per SM (JSON)."""
    import json

    res = {"fma_tflops": round(measure("fma", 8), 2)}
    for bps in (2, 3, 4, 6):
        for name in ("horner", "goertzel"):
            res[f"{name}_{bps}_blocks_per_sm_tflops"] = round(measure(name, bps), 2)
    print(json.dumps(res))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
