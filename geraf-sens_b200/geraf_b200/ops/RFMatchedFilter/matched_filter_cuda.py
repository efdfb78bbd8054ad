"""Autograd wrapper of the matched filter, call-compatible with the reference's
``geraf.ops.RFMatchedFilter.matched_filter_cuda``
(``geraf/ops/RFMatchedFilter/matched_filter_cuda.py:12-255``).

Semantics kept from the reference:
  * ``voxel`` is given as [N, 3] and handed to the kernel as a contiguous [3, N]
    (x row, y row, z row) copy (``matched_filter_cuda.py:89``);
  * shape problems raise ``AssertionError``; non-CUDA inputs raise ``AssertionError``;
  * the backward pass produces gradients for ``real`` and ``image`` only, and
    only when both require grad (``matched_filter_cuda.py:175``); it is
    once-differentiable.
Addition: keyword ``precision`` ("mixed" / "plain" / "nufft"; default from
``geraf_b200.runtime.default_precision``) and ``tuning``.  The form is fixed
when the forward runs; the backward uses the same form and, for "nufft", the
same interpolation width (``tuning["taps"]``), so it is the adjoint of the
forward that ran.
"""
from __future__ import annotations

from typing import Tuple

import torch
from torch.autograd import Function
from torch.autograd.function import once_differentiable

from ...runtime import default_precision
from . import _C


def _as_contiguous(t: torch.Tensor) -> torch.Tensor:
    return t if t.is_contiguous() else t.contiguous()


class _MatchedFilterKernel(Function):
    @staticmethod
    def forward(ctx, real, image, tpos, rpos, voxel, total_ant_size, numADCSample, adcSampleRate,
                As_sci, N, precision=None, tuning=None):
        assert real.dim() == 2, f"`real` must be 2-D [total_ant_size, numADCSample], got {real.dim()}-D"
        assert image.dim() == 2, f"`image` must be 2-D [total_ant_size, numADCSample], got {image.dim()}-D"
        assert tpos.dim() == 2, f"`tpos` must be 2-D [total_ant_size, 3], got {tpos.dim()}-D"
        assert rpos.dim() == 2, f"`rpos` must be 2-D [total_ant_size, 3], got {rpos.dim()}-D"
        assert voxel.dim() == 2, f"`voxel` must be 2-D [N, 3], got {voxel.dim()}-D"
        assert tuple(real.shape) == (total_ant_size, numADCSample), (
            f"`real` has shape {tuple(real.shape)}, expected ({total_ant_size}, {numADCSample})")
        assert tuple(image.shape) == (total_ant_size, numADCSample), (
            f"`image` has shape {tuple(image.shape)}, expected ({total_ant_size}, {numADCSample})")
        assert tuple(tpos.shape) == (total_ant_size, 3), (
            f"`tpos` has shape {tuple(tpos.shape)}, expected ({total_ant_size}, 3)")
        assert tuple(rpos.shape) == (total_ant_size, 3), (
            f"`rpos` has shape {tuple(rpos.shape)}, expected ({total_ant_size}, 3)")
        assert tuple(voxel.shape) == (N, 3), f"`voxel` has shape {tuple(voxel.shape)}, expected ({N}, 3)"

        voxel_soa = _as_contiguous(voxel.transpose(0, 1))
        real = _as_contiguous(real)
        image = _as_contiguous(image)
        tpos = _as_contiguous(tpos)
        rpos = _as_contiguous(rpos)

        output_real = torch.empty((N,), dtype=real.dtype, device=real.device)
        output_image = torch.empty((N,), dtype=real.dtype, device=real.device)
        _C.MatchedFilter_forward(real, image, tpos, rpos, output_real, output_image, voxel_soa,
                                 total_ant_size, numADCSample, adcSampleRate, As_sci, N,
                                 precision=precision, tuning=tuning)

        ctx.save_for_backward(real, image, tpos, rpos, voxel_soa)
        ctx.sizes = (total_ant_size, numADCSample, adcSampleRate, As_sci, N)
        ctx.precision = precision or default_precision()
        ctx.taps = (tuning or {}).get("taps")
        return output_real, output_image

    @staticmethod
    @once_differentiable
    def backward(ctx, grad_output_real, grad_output_image):
        real, image, tpos, rpos, voxel_soa = ctx.saved_tensors
        total_ant_size, numADCSample, adcSampleRate, As_sci, N = ctx.sizes
        assert grad_output_real.is_cuda and grad_output_image.is_cuda, \
            "grad_output_real and grad_output_image must be CUDA tensors."
        grad_output_real = _as_contiguous(grad_output_real)
        grad_output_image = _as_contiguous(grad_output_image)

        grad_real = grad_image = None
        if ctx.needs_input_grad[0] and ctx.needs_input_grad[1]:
            grad_real = torch.empty_like(real)
            grad_image = torch.empty_like(image)
            _C.MatchedFilter_backward_realimag(
                grad_output_real, grad_output_image, real, image, tpos, rpos, grad_real,
                grad_image, voxel_soa, total_ant_size, numADCSample, adcSampleRate, As_sci, N,
                precision=ctx.precision, tuning={"taps": ctx.taps} if ctx.taps else None)
        return (grad_real, grad_image) + (None,) * 10


def matched_filter_cuda(real: torch.Tensor, image: torch.Tensor, tpos: torch.Tensor,
                        rpos: torch.Tensor, voxel: torch.Tensor, total_ant_size: int,
                        numADCSample: int, adcSampleRate: float, As_sci: float, N: int, *,
                        precision: str | None = None,
                        tuning: dict | None = None) -> Tuple[torch.Tensor, torch.Tensor]:
    """Matched-filter backprojection of IF samples ``real + j image`` [A, S] onto
    ``voxel`` [N, 3]; returns ``(out_real, out_imag)`` [N]."""
    assert real.is_cuda and image.is_cuda and tpos.is_cuda and rpos.is_cuda and voxel.is_cuda, \
        "All tensors must be on CUDA."
    return _MatchedFilterKernel.apply(real, image, tpos, rpos, voxel, total_ant_size, numADCSample,
                                      adcSampleRate, As_sci, N, precision, tuning)
