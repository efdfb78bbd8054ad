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
