"""Autograd wrapper of the specular signal tracer, call-compatible with the
reference's ``geraf.ops.RFSignalTracer.signal_tracer_cuda``
(``geraf/ops/RFSignalTracer/signal_tracer_cuda.py:17-188``).

Kept from the reference: ``use_diff=False`` raises ``ValueError``; malformed
shapes raise ``ValueError`` with the same conditions; non-CUDA inputs raise
``ValueError``; the misspelt keyword ``nomralization`` is accepted (and, as in
the reference, has no effect); gradients for ``normals`` and ``sigmas``.
Added: when ``points`` requires grad, the adjoint also returns its gradient
(the reference returns ``None`` there), plus keyword ``precision`` / ``tuning``.
"""
from __future__ import annotations

import torch
from torch.autograd import Function
from torch.autograd.function import once_differentiable

from ...runtime import default_precision
from . import _C


def _ensure_contiguous(tensor: torch.Tensor) -> torch.Tensor:
    return tensor if tensor.is_contiguous() else tensor.contiguous()


class _SignalTracerFunction(Function):
    @staticmethod
    def forward(ctx, normals, sigmas, points, antenna_t, antenna_r, inbounds, numADCSample,
                adcSampleRate, fc_start, As_sci, total_ant_size, total_point_size, use_diff,
                nomralization, precision=None, tuning=None):
        if not use_diff:
            raise ValueError("The standalone signal tracer retains only the differentiable CUDA path.")
        if normals.dim() != 2 or normals.size(1) != 3:
            raise ValueError(f"`normals` must have shape [num_points, 3], got {tuple(normals.shape)}.")
        if points.dim() != 2 or points.size(1) != 3:
            raise ValueError(f"`points` must have shape [num_points, 3], got {tuple(points.shape)}.")
        if sigmas.dim() != 2:
            raise ValueError(f"`sigmas` must have shape [num_antennas, num_points], got {tuple(sigmas.shape)}.")
        if antenna_t.dim() != 2 or antenna_t.size(1) != 3:
            raise ValueError(f"`antenna_t` must have shape [num_antennas, 3], got {tuple(antenna_t.shape)}.")
        if antenna_r.dim() != 2 or antenna_r.size(1) != 3:
            raise ValueError(f"`antenna_r` must have shape [num_antennas, 3], got {tuple(antenna_r.shape)}.")
        if inbounds.dim() != 1:
            raise ValueError(f"`inbounds` must have shape [num_points], got {tuple(inbounds.shape)}.")

        normals = _ensure_contiguous(normals)
        sigmas = _ensure_contiguous(sigmas)
        points = _ensure_contiguous(points)
        antenna_t = _ensure_contiguous(antenna_t)
        antenna_r = _ensure_contiguous(antenna_r)
        inbounds = _ensure_contiguous(inbounds)

        output_real = torch.empty((total_ant_size, numADCSample), dtype=normals.dtype,
                                  device=normals.device)
        output_imag = torch.empty_like(output_real)
        _C.SignalTracer_forward(normals, sigmas, points, antenna_t, antenna_r, inbounds,
                                output_real, output_imag, numADCSample, adcSampleRate, fc_start,
                                As_sci, total_ant_size, total_point_size, precision=precision,
                                tuning=tuning)

        ctx.save_for_backward(normals, sigmas, points, antenna_t, antenna_r, inbounds)
        ctx.scalars = (numADCSample, adcSampleRate, fc_start, As_sci, total_ant_size,
                       total_point_size)
        ctx.nomralization = nomralization
        # the backward runs the form (and NUFFT width) of the forward that ran
        ctx.precision = precision or default_precision()
        ctx.taps = (tuning or {}).get("taps")
        return output_real, output_imag

    @staticmethod
    @once_differentiable
    def backward(ctx, grad_output_real, grad_output_imag):
        normals, sigmas, points, antenna_t, antenna_r, inbounds = ctx.saved_tensors
        numADCSample, adcSampleRate, fc_start, As_sci, A, P = ctx.scalars
        grad_output_real = _ensure_contiguous(grad_output_real)
        grad_output_imag = _ensure_contiguous(grad_output_imag)

        grad_normals = grad_sigmas = grad_points = None
        want_n, want_s, want_p = ctx.needs_input_grad[0], ctx.needs_input_grad[1], ctx.needs_input_grad[2]
        if want_n or want_s or want_p:
            full_grad_normals = torch.empty_like(normals)
            full_grad_sigmas = torch.empty_like(sigmas)
            full_grad_points = torch.empty_like(points) if want_p else None
            _C.SignalTracer_backward_normal_sigma(
                grad_output_real, grad_output_imag, normals, sigmas, points, antenna_t, antenna_r,
                inbounds, full_grad_normals, full_grad_sigmas, numADCSample, adcSampleRate,
                fc_start, As_sci, A, P, grad_points=full_grad_points, precision=ctx.precision,
                tuning={"taps": ctx.taps} if ctx.taps else None)
            grad_normals = full_grad_normals if want_n else None
            grad_sigmas = full_grad_sigmas if want_s else None
            grad_points = full_grad_points
        return (grad_normals, grad_sigmas, grad_points) + (None,) * 13


def signal_tracer_cuda(normals: torch.Tensor, sigmas: torch.Tensor, points: torch.Tensor,
                       antenna_t: torch.Tensor, antenna_r: torch.Tensor, inbounds: torch.Tensor,
                       numADCSample: int, adcSampleRate: float, fc_start: float, As_sci: float,
                       total_ant_size: int, total_point_size: int, use_diff: bool = True,
                       nomralization: bool = True, *, precision: str | None = None,
                       tuning: dict | None = None) -> tuple[torch.Tensor, torch.Tensor]:
    """Renders IF samples [A, S] (real, imag) from specular points."""
    if not all(t.is_cuda for t in (normals, sigmas, points, antenna_t, antenna_r, inbounds)):
        raise ValueError("All signal tracer inputs must be CUDA tensors.")
    return _SignalTracerFunction.apply(normals, sigmas, points, antenna_t, antenna_r, inbounds,
                                       numADCSample, adcSampleRate, fc_start, As_sci,
                                       total_ant_size, total_point_size, use_diff, nomralization,
                                       precision, tuning)
