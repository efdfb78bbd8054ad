"""Host-side plumbing shared by the operator modules: tensor checks with the
reference's error wording, dtype / stream / workspace handling, the arithmetic
form (PLAIN / MIXED / NUFFT) selection and tuned launch shapes.

PyTorch supplies device memory (its caching allocator, so workspaces are
CUDA-graph safe), the current stream and autograd; every byte of compute runs
in ``libgeraf_rf.so``.
"""
from __future__ import annotations

import contextlib
import ctypes
import os
import threading

import torch

from . import _lib

_DTYPES = {
    torch.float32: _lib.DTYPE_F32,
    torch.float64: _lib.DTYPE_F64,
    torch.float16: _lib.DTYPE_F16,
}
_DTYPE_NAMES = {torch.float32: "Float", torch.float64: "Double", torch.float16: "Half"}

_state = threading.local()

PRECISIONS = ("mixed", "plain", "nufft")
_MODES = {"mixed": _lib.MODE_MIXED, "plain": _lib.MODE_PLAIN, "nufft": _lib.MODE_NUFFT}


def default_precision() -> str:
    """Arithmetic form used when a call does not name one.

    ``mixed`` (FP64 phase reduction, recurrence sample sums, compensated
    sums; checked against an FP64 oracle) unless ``GERAF_RF_PRECISION`` names
    ``plain`` (the reference's FP32 arithmetic, expression for expression) or
    ``nufft`` (the fast approximate form of the matched filter and the signal
    tracer: MIXED phases, the sample sums through oversampled range FFTs and a
    short interpolation kernel; operators without it run ``mixed`` under it),
    or a :func:`precision` context is active.
    """
    override = getattr(_state, "precision", None)
    if override is not None:
        return override
    env = os.environ.get("GERAF_RF_PRECISION", "mixed").strip().lower()
    return env if env in PRECISIONS else "mixed"


@contextlib.contextmanager
def precision(mode: str):
    """Selects the arithmetic form for RF operator calls on this thread."""
    if mode not in PRECISIONS:
        raise ValueError(f"precision must be one of {PRECISIONS}, got {mode!r}")
    prev = getattr(_state, "precision", None)
    _state.precision = mode
    try:
        yield
    finally:
        _state.precision = prev


def mode_code(precision_: str | None, allow_nufft: bool = False) -> int:
    """C-ABI arithmetic form of a call.  ``nufft`` exists for the matched
    filter and the signal tracer: named explicitly for another operator it is
    an error, as the ambient default it means ``mixed`` there."""
    p = precision_ or default_precision()
    if p not in PRECISIONS:
        raise ValueError(f"precision must be one of {PRECISIONS}, got {p!r}")
    if p == "nufft" and not allow_nufft:
        if precision_ is not None:
            raise ValueError("precision 'nufft' is only available for the matched filter and the signal tracer")
        p = "mixed"
    return _MODES[p]


def dtype_code(t: torch.Tensor, op: str, allow_half: bool) -> int:
    code = _DTYPES.get(t.dtype)
    if code is None or (code == _lib.DTYPE_F16 and not allow_half):
        name = _DTYPE_NAMES.get(t.dtype, str(t.dtype).replace("torch.", ""))
        raise RuntimeError(f'"{op}" not implemented for \'{name}\'')
    return code


def torch_check(cond: bool, msg: str) -> None:
    """Mirror of TORCH_CHECK: raises RuntimeError with the reference's message."""
    if not cond:
        raise RuntimeError(msg)


def check_cuda_contig(t: torch.Tensor, name: str) -> None:
    torch_check(t.is_cuda, f"`{name}` must be a CUDA tensor.")
    torch_check(t.is_contiguous(), f"`{name}` must be contiguous.")


def check_same_dtype(ref: torch.Tensor, *named: tuple[torch.Tensor, str]) -> None:
    """The reference reads every array through one scalar_t; mixed dtypes are refused."""
    for t, name in named:
        torch_check(t.dtype == ref.dtype, f"`{name}` must have dtype {ref.dtype}, got {t.dtype}.")


def ptr(t: torch.Tensor | None) -> int | None:
    if t is None or t.numel() == 0:
        return None
    return t.data_ptr()


def stream_ptr(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def workspace(nbytes: int, device: torch.device) -> torch.Tensor | None:
    if nbytes <= 0:
        return None
    # The caching allocator returns blocks aligned to at least 512 bytes.
    return torch.empty(nbytes, dtype=torch.uint8, device=device)


def tuning_struct(op: str, sizes: tuple, mode: int, tuning: dict | None) -> _lib.Tuning | None:
    """Explicit tuning wins; otherwise the autotuner cache; otherwise library defaults."""
    if tuning is None:
        from . import autotune

        tuning = autotune.lookup(op, sizes, mode)
    if not tuning:
        return None
    return _lib.Tuning.from_dict(tuning)


def tuning_ref(t: _lib.Tuning | None):
    return ctypes.byref(t) if t is not None else None


class device_guard:
    """Makes ``device`` current for the call (the reference's CUDAGuard)."""

    def __init__(self, device: torch.device):
        self._ctx = torch.cuda.device(device)

    def __enter__(self):
        self._ctx.__enter__()
        return self

    def __exit__(self, *exc):
        return self._ctx.__exit__(*exc)
