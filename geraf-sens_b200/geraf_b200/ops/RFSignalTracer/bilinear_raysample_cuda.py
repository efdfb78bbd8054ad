"""Autograd wrapper of the along-ray linear resampler, call-compatible with the
reference's ``bilinear_raysample_cuda``
(``geraf/ops/RFSignalTracer/bilinear_raysample_cuda.py:12-145``): outputs
``(normals [R,T,3], sigmas [A,R,T], inbounds [R,T] bool)``; the backward pass
scatters into zero-initialised gradients of ``normals`` and ``sigmas``.
"""
from __future__ import annotations

from typing import Tuple

import torch
from torch.autograd import Function
from torch.autograd.function import once_differentiable

from . import _C


class BilinearRaysampleKernel(Function):
    @staticmethod
    def forward(ctx, normals, sigmas, z_vals, tgt_z_vals, N_ant, N_ray, Nz, Nz_tgt):
        normals = normals.contiguous()
        sigmas = sigmas.contiguous()
        z_vals = z_vals.contiguous()
        tgt_z_vals = tgt_z_vals.contiguous()
        output_normals = torch.empty((N_ray, Nz_tgt, 3), dtype=normals.dtype, device=normals.device)
        output_sigmas = torch.empty((N_ant, N_ray, Nz_tgt), dtype=sigmas.dtype, device=sigmas.device)
        output_inbounds = torch.empty((N_ray, Nz_tgt), dtype=torch.bool, device=sigmas.device)
        _C.BilinearRaysample_forward(normals, sigmas, z_vals, tgt_z_vals, output_normals,
                                     output_sigmas, output_inbounds, N_ant, N_ray, Nz, Nz_tgt)
        ctx.save_for_backward(z_vals, tgt_z_vals)
        ctx.sizes = (N_ant, N_ray, Nz, Nz_tgt)
        ctx.mark_non_differentiable(output_inbounds)
        return output_normals, output_sigmas, output_inbounds

    @staticmethod
    @once_differentiable
    def backward(ctx, grad_output_normals, grad_output_sigmas, _grad_inbounds):
        z_vals, tgt_z_vals = ctx.saved_tensors
        N_ant, N_ray, Nz, Nz_tgt = ctx.sizes
        grad_output_normals = grad_output_normals.contiguous()
        grad_output_sigmas = grad_output_sigmas.contiguous()
        normals_grad = torch.zeros((N_ray, Nz, 3), dtype=grad_output_normals.dtype,
                                   device=grad_output_normals.device)
        sigmas_grad = torch.zeros((N_ant, N_ray, Nz), dtype=grad_output_sigmas.dtype,
                                  device=grad_output_sigmas.device)
        _C.BilinearRaysample_backward(grad_output_normals, grad_output_sigmas, z_vals, tgt_z_vals,
                                      normals_grad, sigmas_grad, N_ant, N_ray, Nz, Nz_tgt)
        return normals_grad, sigmas_grad, None, None, None, None, None, None


def bilinear_raysample_cuda(normals: torch.Tensor, sigmas: torch.Tensor, z_vals: torch.Tensor,
                            tgt_z_vals: torch.Tensor, N_ant: int, N_ray: int, Nz: int,
                            Nz_tgt: int) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """Interpolates normals [N_ray, Nz, 3] and sigmas [N_ant, N_ray, Nz] at ``tgt_z_vals``
    [N_ray, Nz_tgt]; returns (normals, sigmas, inbounds)."""
    return BilinearRaysampleKernel.apply(normals, sigmas, z_vals, tgt_z_vals, N_ant, N_ray, Nz,
                                         Nz_tgt)
