"""Batched signal tracer over all antennas of a step with uneven per-antenna
point sets -- one persistent launch instead of one ``signal_tracer_cuda`` call
per antenna.

Layout: the points of antenna 0, then antenna 1, ...; ``point_offsets`` [A+1]
(int64, CSR) delimits them.  ``normals``/``points`` [P,3], ``sigmas`` [P] (each
point's amplitude for its own antenna), ``inbounds`` [P] bool or None.  Row a of
the result equals the reference tracer over antenna a's points alone
(``geraf/ops/RFSignalTracer/signal_tracer_cuda.py:152-188`` with
``total_point_size`` = that antenna's point count).  MIXED arithmetic only.
Gradients flow to ``normals``, ``sigmas`` and ``points``.
"""
from __future__ import annotations

import torch
from torch.autograd import Function
from torch.autograd.function import once_differentiable

from ... import _lib
from ...runtime import (check_cuda_contig, device_guard, dtype_code, ptr, stream_ptr, torch_check, tuning_ref,
                        tuning_struct, workspace)


def _check(normals, sigmas, points, point_offsets, tx, rx, inbounds, S):
    for t, n in ((normals, "normals"), (sigmas, "sigmas"), (points, "points"),
                 (point_offsets, "point_offsets"), (tx, "antenna_t"), (rx, "antenna_r")):
        check_cuda_contig(t, n)
    P = points.shape[0]
    A = tx.shape[0]
    torch_check(normals.dim() == 2 and normals.shape == (P, 3), "`normals` must have shape [P, 3].")
    torch_check(points.dim() == 2 and points.size(1) == 3, "`points` must have shape [P, 3].")
    torch_check(sigmas.dim() == 1 and sigmas.size(0) == P, "`sigmas` must have shape [P].")
    torch_check(point_offsets.dtype == torch.int64 and point_offsets.dim() == 1
                and point_offsets.size(0) == A + 1, "`point_offsets` must be int64 [A + 1].")
    torch_check(tx.dim() == 2 and tx.size(1) == 3 and rx.shape == tx.shape,
                "`antenna_t` / `antenna_r` must have shape [A, 3].")
    if inbounds is not None:
        check_cuda_contig(inbounds, "inbounds")
        torch_check(inbounds.dtype == torch.bool and inbounds.shape == (P,), "`inbounds` must be bool [P].")
    for t, n in ((sigmas, "sigmas"), (points, "points"), (tx, "antenna_t"), (rx, "antenna_r")):
        torch_check(t.dtype == normals.dtype, f"`{n}` must have dtype {normals.dtype}.")
    return A, P


class _RaggedTracer(Function):
    @staticmethod
    def forward(ctx, normals, sigmas, points, point_offsets, antenna_t, antenna_r, inbounds,
                numADCSample, adcSampleRate, fc_start, As_sci, tuning, tuning_backward):
        normals, sigmas, points = normals.contiguous(), sigmas.contiguous(), points.contiguous()
        antenna_t, antenna_r = antenna_t.contiguous(), antenna_r.contiguous()
        point_offsets = point_offsets.contiguous()
        inbounds = inbounds.contiguous() if inbounds is not None else None
        S = int(numADCSample)
        A, P = _check(normals, sigmas, points, point_offsets, antenna_t, antenna_r, inbounds, S)
        dt = dtype_code(normals, "signal_tracer_ragged", allow_half=False)
        out_r = torch.empty((A, S), dtype=normals.dtype, device=normals.device)
        out_i = torch.empty_like(out_r)
        tun = tuning_struct("tracer_ragged_forward", (A, S, P), _lib.MODE_MIXED, tuning)
        with device_guard(normals.device):
            nbytes = _lib.workspace_bytes("geraf_tracer_ragged_workspace_bytes", A, S, P, dt, tuning_ref(tun))
            ws = workspace(nbytes, normals.device)
            _lib.call("geraf_tracer_forward_ragged", ptr(normals), ptr(sigmas), ptr(points),
                      ptr(point_offsets), ptr(antenna_t), ptr(antenna_r), ptr(inbounds), ptr(out_r),
                      ptr(out_i), S, float(adcSampleRate), float(fc_start), float(As_sci), A, P, dt,
                      tuning_ref(tun), ptr(ws), nbytes, stream_ptr(normals.device))
        ctx.save_for_backward(normals, sigmas, points, point_offsets, antenna_t, antenna_r,
                              inbounds if inbounds is not None else torch.empty(0, device=normals.device))
        ctx.has_inb = inbounds is not None
        ctx.scalars = (S, float(adcSampleRate), float(fc_start), float(As_sci), A, P, dt)
        ctx.tuning_backward = tuning_backward
        return out_r, out_i

    @staticmethod
    @once_differentiable
    def backward(ctx, g_r, g_i):
        normals, sigmas, points, offsets, tx, rx, inb = ctx.saved_tensors
        S, fs, f0, As, A, P, dt = ctx.scalars
        inb = inb if ctx.has_inb else None
        g_r, g_i = g_r.contiguous(), g_i.contiguous()
        gn = torch.empty_like(normals)
        gs = torch.empty_like(sigmas)
        gp = torch.empty_like(points) if ctx.needs_input_grad[2] else None
        tun = tuning_struct("tracer_ragged_backward", (A, S, P), _lib.MODE_MIXED, ctx.tuning_backward)
        with device_guard(normals.device):
            _lib.call("geraf_tracer_backward_ragged", ptr(g_r), ptr(g_i), ptr(normals), ptr(sigmas),
                      ptr(points), ptr(offsets), ptr(tx), ptr(rx), ptr(inb), ptr(gn), ptr(gs), ptr(gp),
                      S, fs, f0, As, A, P, dt, tuning_ref(tun), stream_ptr(normals.device))
        return (gn if ctx.needs_input_grad[0] else None, gs if ctx.needs_input_grad[1] else None,
                gp) + (None,) * 10


def signal_tracer_ragged(normals: torch.Tensor, sigmas: torch.Tensor, points: torch.Tensor,
                         point_offsets: torch.Tensor, antenna_t: torch.Tensor, antenna_r: torch.Tensor,
                         numADCSample: int, adcSampleRate: float, fc_start: float, As_sci: float,
                         inbounds: torch.Tensor | None = None, *, tuning: dict | None = None,
                         tuning_backward: dict | None = None):
    """IF [A, S] (real, imag) of every antenna from its own points.  ``tuning`` /
    ``tuning_backward``: launch shapes of the forward and the adjoint (default:
    the autotuner cache, else the library's)."""
    if not all(t.is_cuda for t in (normals, sigmas, points, point_offsets, antenna_t, antenna_r)):
        raise ValueError("All signal tracer inputs must be CUDA tensors.")
    return _RaggedTracer.apply(normals, sigmas, points, point_offsets, antenna_t, antenna_r, inbounds,
                               numADCSample, adcSampleRate, fc_start, As_sci, tuning, tuning_backward)
