"""Launch-shape autotuner for the RF kernels.

For a given operator, problem size and arithmetic form, every candidate
``geraf_tuning_t`` is timed on the current device with CUDA events (after a
warm-up launch) and the fastest is remembered -- in memory and, when
``GERAF_RF_TUNE_CACHE`` names a file, in that JSON file -- keyed by
(operator, form, sizes, device name).  The operator modules consult
:func:`lookup` on every call; with no entry the library's own defaults apply.
"""
from __future__ import annotations

import json
import os
import threading
from typing import Callable, Iterable

import torch

_lock = threading.Lock()
_cache: dict[str, dict] = {}
_loaded_from: str | None = None


def _device_name() -> str:
    try:
        return torch.cuda.get_device_name(torch.cuda.current_device())
    except Exception:  # noqa: BLE001 - no device: the key only needs to be stable
        return "cpu"


def _key(op: str, sizes: tuple, mode: int) -> str:
    return f"{op}|{mode}|{'x'.join(str(int(s)) for s in sizes)}|{_device_name()}"


def _cache_file() -> str | None:
    return os.environ.get("GERAF_RF_TUNE_CACHE") or None


def _maybe_load() -> None:
    global _loaded_from
    path = _cache_file()
    if path is None or path == _loaded_from:
        return
    _loaded_from = path
    if os.path.exists(path):
        with open(path) as f:
            _cache.update(json.load(f))


def lookup(op: str, sizes: tuple, mode: int) -> dict | None:
    with _lock:
        _maybe_load()
        return _cache.get(_key(op, sizes, mode))


def record(op: str, sizes: tuple, mode: int, tuning: dict) -> None:
    with _lock:
        _maybe_load()
        _cache[_key(op, sizes, mode)] = dict(tuning)
        path = _cache_file()
        if path:
            os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
            tmp = path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(_cache, f, indent=1, sort_keys=True)
            os.replace(tmp, path)


def clear() -> None:
    with _lock:
        _cache.clear()


def time_call(fn: Callable[[], None], iters: int = 3, warmup: int = 1) -> float:
    """Mean milliseconds of ``fn`` on the current stream (CUDA events)."""
    for _ in range(warmup):
        fn()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    for _ in range(iters):
        fn()
    stop.record()
    stop.synchronize()
    return start.elapsed_time(stop) / iters


def tune(op: str, sizes: tuple, mode: int, run: Callable[[dict], None],
         candidates: Iterable[dict], iters: int = 3) -> tuple[dict, list[tuple[dict, float]]]:
    """Times ``run(candidate)`` for each candidate, records and returns the fastest."""
    results = []
    for cand in candidates:
        try:
            ms = time_call(lambda: run(cand), iters=iters)
        except RuntimeError:
            continue
        results.append((dict(cand), ms))
    if not results:
        raise RuntimeError(f"no tuning candidate of {op} ran")
    best = min(results, key=lambda r: r[1])[0]
    record(op, sizes, mode, best)
    return best, results


def mf_forward_candidates(mode: int) -> list[dict]:
    out = []
    for threads in (64, 128, 256):
        for items in ((2, 4, 8) if mode == 1 else (1, 2)):
            for rows in (4, 8, 16):
                out.append({"threads": threads, "items_per_thread": items, "stage_rows": rows})
    return out


def sample_major_candidates() -> list[dict]:
    """MF adjoint / tracer forward: threads x samples-per-lane."""
    return [{"threads": t, "chunk": c} for t in (64, 128, 256) for c in (8, 16, 32)]


def tracer_backward_candidates() -> list[dict]:
    return [{"threads": t, "stage_rows": r} for t in (64, 128) for r in (4, 8, 16)]


def ragged_forward_candidates() -> list[dict]:
    """Batched tracer forward: threads x samples-per-lane x points per thread of a work item."""
    return [{"threads": t, "chunk": c, "items_per_thread": i}
            for t in (64, 128, 256) for c in (8, 16) for i in (16, 32)]


def ragged_backward_candidates() -> list[dict]:
    """Batched tracer adjoint: residual rows staged per block."""
    return [{"stage_rows": r} for r in (1, 2, 4, 8)]

