"""Selected / unselected antenna split of the matched filter, call-compatible with
the reference's ``faster_matched_filter_cuda``
(``geraf/ops/RFMatchedFilter/faster_matched_filter_cuda.py:12-319``).

The forward pass filters the concatenation [selected; unselected] of the IF
rows and antenna positions (normalised by all ``total_ant_size`` antennas).
The backward pass runs the adjoint over the selected antennas only, as a
``num_sel``-antenna filter, then rescales by ``num_sel / total_ant_size`` so the
result carries the same 1/total normalisation
(``faster_matched_filter_cuda.py:229-238``).  Gradients flow to
``real_sel`` / ``image_sel`` only, when both require grad.
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


class _FasterMatchedFilterKernel(Function):
    @staticmethod
    def forward(ctx, real_sel, image_sel, real_unsel, image_unsel, tpos_sel, rpos_sel, tpos_unsel,
                rpos_unsel, voxel, total_ant_size, num_sel, numADCSample, adcSampleRate, As_sci, N,
                precision=None, tuning=None):
        for name, t in (("real_sel", real_sel), ("image_sel", image_sel), ("real_unsel", real_unsel),
                        ("image_unsel", image_unsel), ("tpos_sel", tpos_sel), ("rpos_sel", rpos_sel),
                        ("tpos_unsel", tpos_unsel), ("rpos_unsel", rpos_unsel), ("voxel", voxel)):
            assert t.dim() == 2, f"`{name}` must be 2-D, got {t.dim()}-D"
        num_unsel = total_ant_size - num_sel
        for name, t, rows, cols in (("real_sel", real_sel, num_sel, numADCSample),
                                    ("image_sel", image_sel, num_sel, numADCSample),
                                    ("tpos_sel", tpos_sel, num_sel, 3),
                                    ("rpos_sel", rpos_sel, num_sel, 3),
                                    ("real_unsel", real_unsel, num_unsel, numADCSample),
                                    ("image_unsel", image_unsel, num_unsel, numADCSample),
                                    ("tpos_unsel", tpos_unsel, num_unsel, 3),
                                    ("rpos_unsel", rpos_unsel, num_unsel, 3),
                                    ("voxel", voxel, N, 3)):
            assert tuple(t.shape) == (rows, cols), (
                f"`{name}` has shape {tuple(t.shape)}, expected ({rows}, {cols})")

        voxel_soa = _as_contiguous(voxel.transpose(0, 1))
        real = torch.cat([_as_contiguous(real_sel), _as_contiguous(real_unsel)], dim=0)
        image = torch.cat([_as_contiguous(image_sel), _as_contiguous(image_unsel)], dim=0)
        tpos = torch.cat([_as_contiguous(tpos_sel), _as_contiguous(tpos_unsel)], dim=0)
        rpos = torch.cat([_as_contiguous(rpos_sel), _as_contiguous(rpos_unsel)], dim=0)

        output_real = torch.empty((N,), dtype=real_sel.dtype, device=real_sel.device)
        output_image = torch.empty((N,), dtype=real_sel.dtype, device=real_sel.device)
        _C.MatchedFilter_forward(real, image, tpos, rpos, output_real, output_image, voxel_soa,
                                 total_ant_size, numADCSample, adcSampleRate, As_sci, N,
                                 precision=precision, tuning=tuning)

        ctx.save_for_backward(_as_contiguous(real_sel), _as_contiguous(image_sel),
                              _as_contiguous(tpos_sel), _as_contiguous(rpos_sel), voxel_soa)
        ctx.sizes = (total_ant_size, num_sel, numADCSample, adcSampleRate, As_sci, N)
        # the backward runs the form (and NUFFT width) of the forward that ran
        ctx.precision = precision or default_precision()
        ctx.taps = (tuning or {}).get("taps")
        return output_real, output_image

    @staticmethod
    @once_differentiable
    def backward(ctx, grad_output_real, grad_output_image):
        real_sel, image_sel, tpos_sel, rpos_sel, voxel_soa = ctx.saved_tensors
        total_ant_size, num_sel, numADCSample, adcSampleRate, As_sci, N = ctx.sizes
        assert grad_output_real.is_cuda and grad_output_image.is_cuda, \
            "grad_output_real and grad_output_image must be CUDA tensors."
        grad_output_real = _as_contiguous(grad_output_real)
        grad_output_image = _as_contiguous(grad_output_image)
        grad_real = grad_image = None
        if ctx.needs_input_grad[0] and ctx.needs_input_grad[1]:
            grad_real = torch.empty_like(real_sel)
            grad_image = torch.empty_like(image_sel)
            _C.MatchedFilter_backward_realimag(
                grad_output_real, grad_output_image, real_sel, image_sel, tpos_sel, rpos_sel,
                grad_real, grad_image, voxel_soa, num_sel, numADCSample, adcSampleRate, As_sci, N,
                precision=ctx.precision, tuning={"taps": ctx.taps} if ctx.taps else None)
            grad_real = grad_real * num_sel / total_ant_size
            grad_image = grad_image * num_sel / total_ant_size
        return (grad_real, grad_image) + (None,) * 15


def faster_matched_filter_cuda(real_sel, image_sel, real_unsel, image_unsel, tpos_sel, rpos_sel,
                               tpos_unsel, rpos_unsel, voxel, total_ant_size: int, num_sel: int,
                               numADCSample: int, adcSampleRate: float, As_sci: float, N: int, *,
                               precision: str | None = None,
                               tuning: dict | None = None) -> Tuple[torch.Tensor, torch.Tensor]:
    """Matched filter over [selected; unselected] antennas with gradients for the selected rows."""
    assert real_sel.is_cuda and image_sel.is_cuda and tpos_sel.is_cuda and rpos_sel.is_cuda \
        and voxel.is_cuda, "All tensors must be on CUDA."
    assert real_unsel.is_cuda and image_unsel.is_cuda and tpos_unsel.is_cuda and rpos_unsel.is_cuda, \
        "All tensors must be on CUDA."
    return _FasterMatchedFilterKernel.apply(real_sel, image_sel, real_unsel, image_unsel, tpos_sel,
                                            rpos_sel, tpos_unsel, rpos_unsel, voxel,
                                            total_ant_size, num_sel, numADCSample, adcSampleRate,
                                            As_sci, N, precision, tuning)
