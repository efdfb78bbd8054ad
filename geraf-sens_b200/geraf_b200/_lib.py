"""ctypes binding of ``libgeraf_rf.so`` (declarations in ``include/geraf_rf.h``).

The shared library is built in-tree (``make -C geraf-sens_b200/csrc``) and is the
only compute path of this package: there is no CPU or PyTorch fallback, and a
missing library raises ``ImportError`` at first use.
"""
from __future__ import annotations

import ctypes
import os
import threading

LIB_NAME = "libgeraf_rf.so"
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

GERAF_OK = 0
GERAF_ERR_INVALID_ARGUMENT = 1
GERAF_ERR_UNSUPPORTED = 2
GERAF_ERR_WORKSPACE = 3
GERAF_ERR_CUDA = 4
GERAF_ERR_DEVICE_TIMEOUT = 5
GERAF_ERR_DEVICE_CHECK = 6

DTYPE_F32 = 0
DTYPE_F64 = 1
DTYPE_F16 = 2

MODE_PLAIN = 0
MODE_MIXED = 1
MODE_NUFFT = 2

SAMPLE_TRILINEAR = 0
SAMPLE_NEAREST = 1

FFT_CONSISTENT_BINS = 1


class Tuning(ctypes.Structure):
    """``geraf_tuning_t``: launch shape; 0 in any field = library default."""

    _fields_ = [
        ("threads", ctypes.c_int32),
        ("items_per_thread", ctypes.c_int32),
        ("stage_rows", ctypes.c_int32),
        ("splits", ctypes.c_int32),
        ("chunk", ctypes.c_int32),
        ("taps", ctypes.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}

    @classmethod
    def from_dict(cls, d: dict | None) -> "Tuning":
        t = cls()
        for name, _ in cls._fields_:
            setattr(t, name, int((d or {}).get(name, 0)))
        return t


_vp = ctypes.c_void_p
_u8p = ctypes.c_void_p
_i64 = ctypes.c_int64
_i32 = ctypes.c_int32
_f32 = ctypes.c_float
_szp = ctypes.POINTER(ctypes.c_size_t)
_tp = ctypes.POINTER(Tuning)

# name -> (restype, argtypes); must match include/geraf_rf.h exactly.
SIGNATURES = {
    "geraf_rf_last_error": (ctypes.c_char_p, []),
    "geraf_rf_cudart_version": (_i32, []),
    "geraf_rf_build_info": (ctypes.c_char_p, []),
    "geraf_rf_device_status": (_i32, [_vp, _i32, ctypes.POINTER(_i32)]),
    "geraf_mf_forward_workspace_bytes": (_i32, [_i64, _i64, _i64, _i32, _i32, _tp, _szp]),
    "geraf_mf_forward": (
        _i32,
        [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _f32, _f32, _i64, _i32, _i32, _tp, _vp,
         ctypes.c_size_t, _vp],
    ),
    "geraf_mf_forward_noalloc": (
        _i32, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _f32, _f32, _i64, _vp]
    ),
    "geraf_mf_backward_workspace_bytes": (_i32, [_i64, _i64, _i64, _i32, _i32, _tp, _szp]),
    "geraf_mf_backward": (
        _i32,
        [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _f32, _f32, _i64, _i32, _i32,
         _tp, _vp, ctypes.c_size_t, _vp],
    ),
    "geraf_mf_fft_forward": (
        _i32, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _f32, _f32, _f32, _i64, _i32, _i32, _vp]
    ),
    "geraf_mf_fft_backward": (
        _i32,
        [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _f32, _f32, _f32, _i64, _i32,
         _i32, _vp],
    ),
    "geraf_tracer_forward_workspace_bytes": (_i32, [_i64, _i64, _i64, _i32, _i32, _tp, _szp]),
    "geraf_tracer_forward": (
        _i32,
        [_vp, _vp, _vp, _vp, _vp, _u8p, _vp, _vp, _i64, _f32, _f32, _f32, _i64, _i64, _i32, _i32,
         _tp, _vp, ctypes.c_size_t, _vp],
    ),
    "geraf_tracer_backward_workspace_bytes": (
        _i32, [_i64, _i64, _i64, _i32, _i32, _i32, _tp, _szp]
    ),
    "geraf_tracer_backward": (
        _i32,
        [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _u8p, _vp, _vp, _vp, _i64, _f32, _f32, _f32, _i64,
         _i64, _i32, _i32, _tp, _vp, ctypes.c_size_t, _vp],
    ),
    "geraf_tracer_ragged_workspace_bytes": (_i32, [_i64, _i64, _i64, _i32, _tp, _szp]),
    "geraf_tracer_forward_ragged": (
        _i32,
        [_vp, _vp, _vp, _vp, _vp, _vp, _u8p, _vp, _vp, _i64, _f32, _f32, _f32, _i64, _i64, _i32,
         _tp, _vp, ctypes.c_size_t, _vp],
    ),
    "geraf_tracer_backward_ragged": (
        _i32,
        [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _u8p, _vp, _vp, _vp, _i64, _f32, _f32, _f32, _i64,
         _i64, _i32, _tp, _vp],
    ),
    "geraf_bilinear_forward": (
        _i32, [_vp, _vp, _vp, _vp, _vp, _vp, _u8p, _i64, _i64, _i64, _i64, _i32, _vp]
    ),
    "geraf_bilinear_backward": (
        _i32, [_vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _i64, _i64, _i32, _vp]
    ),
    "geraf_volume_sample": (_i32, [_vp, _i64, _i64, _i64, _vp, _i64, _vp, _i32, _i32, _vp]),
}

# Test hooks (include/geraf_rf_testing.h): not operators, bound for the tests.
TEST_SIGNATURES = {
    "geraf_rf_selftest_wait_timeout": (_i32, [_i64, _i32, _vp, _vp]),
}

_lock = threading.Lock()
_lib = None


class GerafError(RuntimeError):
    """A failed library call; ``code`` is the GERAF_ERR_* status."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


def load() -> ctypes.CDLL:
    """Loads the library once (thread-safe) and binds every declared symbol."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_NAME} not found at {LIB_PATH}; build it with "
                "`make -C geraf-sens_b200/csrc` (or __graft_entry__.build())"
            )
        lib = ctypes.CDLL(LIB_PATH)
        for name, (restype, argtypes) in {**SIGNATURES, **TEST_SIGNATURES}.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
        return lib


def last_error() -> str:
    msg = load().geraf_rf_last_error()
    return msg.decode() if msg else ""


def check(rc: int, what: str) -> None:
    if rc != GERAF_OK:
        raise GerafError(rc, f"{what}: {last_error()}")


def call(name: str, *args) -> None:
    """Calls a status-returning entry point; raises GerafError on failure."""
    check(getattr(load(), name)(*args), name)


def workspace_bytes(name: str, *args) -> int:
    out = ctypes.c_size_t(0)
    call(name, *args, ctypes.byref(out))
    return int(out.value)


def device_status(stream_ptr: int = 0, reset: bool = True) -> int:
    """Reads (and clears) the device status word; synchronises the stream."""
    out = ctypes.c_int32(0)
    call("geraf_rf_device_status", stream_ptr, int(reset), ctypes.byref(out))
    return int(out.value)
