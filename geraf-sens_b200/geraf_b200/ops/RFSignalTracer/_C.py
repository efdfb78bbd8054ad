"""Drop-in replacement of the reference's ``geraf.ops.RFSignalTracer._C`` module.

Same function names, positional arguments, out-parameter convention and
``RuntimeError`` messages as ``geraf/ops/RFSignalTracer/csrc/vision.cpp:70-97``
and ``csrc/signal_tracer/SignalTracer_cuda.cu:10-406``.  Calls run on the
current torch stream of the input's device and do not synchronise.

Differences, all additive:
  * ``SignalTracer_backward_normal_sigma`` accepts ``grad_points=`` ([P,3],
    overwritten) to also return the gradient with respect to point positions,
    which the reference does not provide;
  * entries of ``grad_normals`` / ``grad_sigmas`` belonging to out-of-bounds
    points are written as 0 (the reference leaves them unwritten);
  * keyword-only ``precision`` / ``tuning`` as in the matched filter.
"""
from __future__ import annotations

import torch

from ... import _lib
from ...runtime import (
    check_cuda_contig,
    check_same_dtype,
    device_guard,
    dtype_code,
    mode_code,
    ptr,
    stream_ptr,
    torch_check,
    tuning_ref,
    tuning_struct,
    workspace,
)


def _check_tracer(normals, sigmas, points, tx_pos, rx_pos, inbounds, output_real, output_imag,
                  S, A, P):
    # SignalTracer_cuda.cu:100-140
    for t, n in ((normals, "normals"), (sigmas, "sigmas"), (points, "points"), (tx_pos, "tx_pos"),
                 (rx_pos, "rx_pos"), (inbounds, "inbounds"), (output_real, "output_real"),
                 (output_imag, "output_imag")):
        check_cuda_contig(t, n)
    torch_check(inbounds.dtype == torch.bool, "`inbounds` must be bool.")
    torch_check(normals.dim() == 2 and normals.size(1) == 3, "`normals` must have shape [P, 3].")
    torch_check(points.dim() == 2 and points.size(1) == 3, "`points` must have shape [P, 3].")
    torch_check(sigmas.dim() == 2, "`sigmas` must have shape [A, P].")
    torch_check(tx_pos.dim() == 2 and tx_pos.size(1) == 3, "`tx_pos` must have shape [A, 3].")
    torch_check(rx_pos.dim() == 2 and rx_pos.size(1) == 3, "`rx_pos` must have shape [A, 3].")
    torch_check(inbounds.dim() == 1, "`inbounds` must have shape [P].")
    torch_check(output_real.dim() == 2, "`output_real` must have shape [A, S].")
    torch_check(output_imag.dim() == 2, "`output_imag` must have shape [A, S].")
    torch_check(normals.size(0) == P, "`normals` point dimension mismatch.")
    torch_check(points.size(0) == P, "`points` point dimension mismatch.")
    torch_check(sigmas.size(0) == A and sigmas.size(1) == P, "`sigmas` shape mismatch.")
    torch_check(tx_pos.size(0) == A, "`tx_pos` antenna dimension mismatch.")
    torch_check(rx_pos.size(0) == A, "`rx_pos` antenna dimension mismatch.")
    torch_check(inbounds.size(0) == P, "`inbounds` point dimension mismatch.")
    torch_check(output_real.size(0) == A and output_real.size(1) == S, "`output_real` shape mismatch.")
    torch_check(output_imag.size(0) == A and output_imag.size(1) == S, "`output_imag` shape mismatch.")
    check_same_dtype(normals, (sigmas, "sigmas"), (points, "points"), (tx_pos, "tx_pos"),
                     (rx_pos, "rx_pos"), (output_real, "output_real"), (output_imag, "output_imag"))


def SignalTracer_forward(normals, sigmas, points, tx_pos, rx_pos, inbounds, output_real,
                         output_imag, num_adc_samples, adc_sample_rate, start_frequency,
                         chirp_slope_scaled, total_ant_size, total_point_size, *, precision=None,
                         tuning=None):
    """Renders IF samples ``output_{real,imag}`` [A, S] from specular points."""
    S, A, P = int(num_adc_samples), int(total_ant_size), int(total_point_size)
    _check_tracer(normals, sigmas, points, tx_pos, rx_pos, inbounds, output_real, output_imag,
                  S, A, P)
    dt = dtype_code(normals, "signal_tracer_forward_cuda", allow_half=False)
    mode = mode_code(precision, allow_nufft=True)
    tun = tuning_struct("tracer_forward", (A, S, P), mode, tuning)
    with device_guard(normals.device):
        nbytes = _lib.workspace_bytes("geraf_tracer_forward_workspace_bytes", A, S, P, dt, mode,
                                      tuning_ref(tun))
        ws = workspace(nbytes, normals.device)
        _lib.call("geraf_tracer_forward", ptr(normals), ptr(sigmas), ptr(points), ptr(tx_pos),
                  ptr(rx_pos), ptr(inbounds), ptr(output_real), ptr(output_imag), S,
                  float(adc_sample_rate), float(start_frequency), float(chirp_slope_scaled), A, P,
                  dt, mode, tuning_ref(tun), ptr(ws), nbytes, stream_ptr(normals.device))


def SignalTracer_backward_normal_sigma(grad_output_real, grad_output_imag, normals, sigmas, points,
                                       tx_pos, rx_pos, inbounds, grad_normals, grad_sigmas,
                                       num_adc_samples, adc_sample_rate, start_frequency,
                                       chirp_slope_scaled, total_ant_size, total_point_size, *,
                                       grad_points=None, precision=None, tuning=None):
    """Adjoint of :func:`SignalTracer_forward` into ``grad_normals`` [P,3], ``grad_sigmas``
    [A,P] and, if given, ``grad_points`` [P,3]."""
    S, A, P = int(num_adc_samples), int(total_ant_size), int(total_point_size)
    # SignalTracer_cuda.cu:142-178: the forward checks with grad_output in the output slots.
    _check_tracer(normals, sigmas, points, tx_pos, rx_pos, inbounds, grad_output_real,
                  grad_output_imag, S, A, P)
    check_cuda_contig(grad_normals, "grad_normals")
    check_cuda_contig(grad_sigmas, "grad_sigmas")
    torch_check(grad_normals.dim() == 2 and grad_normals.size(1) == 3,
                "`grad_normals` must have shape [P, 3].")
    torch_check(grad_sigmas.dim() == 2, "`grad_sigmas` must have shape [A, P].")
    torch_check(grad_normals.size(0) == P, "`grad_normals` point dimension mismatch.")
    torch_check(grad_sigmas.size(0) == A and grad_sigmas.size(1) == P, "`grad_sigmas` shape mismatch.")
    check_same_dtype(normals, (grad_normals, "grad_normals"), (grad_sigmas, "grad_sigmas"))
    if grad_points is not None:
        check_cuda_contig(grad_points, "grad_points")
        torch_check(grad_points.dim() == 2 and grad_points.size(0) == P and grad_points.size(1) == 3,
                    "`grad_points` must have shape [P, 3].")
        check_same_dtype(normals, (grad_points, "grad_points"))
    dt = dtype_code(grad_output_real, "signal_tracer_backward_normal_sigma_cuda", allow_half=False)
    mode = mode_code(precision, allow_nufft=True)
    tun = tuning_struct("tracer_backward", (A, S, P), mode, tuning)
    with device_guard(grad_output_real.device):
        nbytes = _lib.workspace_bytes("geraf_tracer_backward_workspace_bytes", A, S, P, dt, mode,
                                      int(grad_points is not None), tuning_ref(tun))
        ws = workspace(nbytes, normals.device)
        gp = ptr(grad_points) if grad_points is not None and grad_points.numel() > 0 else None
        _lib.call("geraf_tracer_backward", ptr(grad_output_real), ptr(grad_output_imag),
                  ptr(normals), ptr(sigmas), ptr(points), ptr(tx_pos), ptr(rx_pos), ptr(inbounds),
                  ptr(grad_normals), ptr(grad_sigmas), gp, S, float(adc_sample_rate),
                  float(start_frequency), float(chirp_slope_scaled), A, P, dt, mode,
                  tuning_ref(tun), ptr(ws), nbytes, stream_ptr(normals.device))


def _check_bilinear_fwd(normals, sigmas, z_vals, tz, out_n, out_s, out_inb, A, R, S, T):
    # SignalTracer_cuda.cu:15-57
    for t, n in ((normals, "normals"), (sigmas, "sigmas"), (z_vals, "z_vals"), (tz, "target_z_vals"),
                 (out_n, "output_normals"), (out_s, "output_sigmas"), (out_inb, "output_inbounds")):
        check_cuda_contig(t, n)
    torch_check(normals.dim() == 3, "`normals` must have shape [R, S, 3].")
    torch_check(sigmas.dim() == 3, "`sigmas` must have shape [A, R, S].")
    torch_check(z_vals.dim() == 2, "`z_vals` must have shape [R, S].")
    torch_check(tz.dim() == 2, "`target_z_vals` must have shape [R, T].")
    torch_check(out_n.dim() == 3, "`output_normals` must have shape [R, T, 3].")
    torch_check(out_s.dim() == 3, "`output_sigmas` must have shape [A, R, T].")
    torch_check(out_inb.dim() == 2, "`output_inbounds` must have shape [R, T].")
    torch_check(out_inb.dtype == torch.bool, "`output_inbounds` must be bool.")
    torch_check(tuple(normals.shape) == (R, S, 3), "`normals` shape mismatch.")
    torch_check(tuple(sigmas.shape) == (A, R, S), "`sigmas` shape mismatch.")
    torch_check(tuple(z_vals.shape) == (R, S), "`z_vals` shape mismatch.")
    torch_check(tuple(tz.shape) == (R, T), "`target_z_vals` shape mismatch.")
    torch_check(tuple(out_n.shape) == (R, T, 3), "`output_normals` shape mismatch.")
    torch_check(tuple(out_s.shape) == (A, R, T), "`output_sigmas` shape mismatch.")
    torch_check(tuple(out_inb.shape) == (R, T), "`output_inbounds` shape mismatch.")
    check_same_dtype(normals, (sigmas, "sigmas"), (z_vals, "z_vals"), (tz, "target_z_vals"),
                     (out_n, "output_normals"), (out_s, "output_sigmas"))


def BilinearRaysample_forward(normals, sigmas, z_vals, target_z_vals, output_normals,
                              output_sigmas, output_inbounds, num_antennas, num_rays, num_samples,
                              num_target_samples):
    """Linear resampling of normals [R,S,3] and sigmas [A,R,S] at target depths [R,T]."""
    A, R, S, T = int(num_antennas), int(num_rays), int(num_samples), int(num_target_samples)
    _check_bilinear_fwd(normals, sigmas, z_vals, target_z_vals, output_normals, output_sigmas,
                        output_inbounds, A, R, S, T)
    dt = dtype_code(normals, "bilinear_raysample_forward_cuda", allow_half=False)
    with device_guard(normals.device):
        _lib.call("geraf_bilinear_forward", ptr(normals), ptr(sigmas), ptr(z_vals),
                  ptr(target_z_vals), ptr(output_normals), ptr(output_sigmas),
                  ptr(output_inbounds), A, R, S, T, dt, stream_ptr(normals.device))


def BilinearRaysample_backward(grad_output_normals, grad_output_sigmas, z_vals, target_z_vals,
                               grad_normals, grad_sigmas, num_antennas, num_rays, num_samples,
                               num_target_samples):
    """Adjoint of the resampler; ADDS into ``grad_normals`` [R,S,3] and ``grad_sigmas`` [A,R,S]."""
    A, R, S, T = int(num_antennas), int(num_rays), int(num_samples), int(num_target_samples)
    # SignalTracer_cuda.cu:59-98
    for t, n in ((grad_output_normals, "grad_output_normals"),
                 (grad_output_sigmas, "grad_output_sigmas"), (z_vals, "z_vals"),
                 (target_z_vals, "target_z_vals"), (grad_normals, "grad_normals"),
                 (grad_sigmas, "grad_sigmas")):
        check_cuda_contig(t, n)
    torch_check(grad_output_normals.dim() == 3, "`grad_output_normals` must have shape [R, T, 3].")
    torch_check(grad_output_sigmas.dim() == 3, "`grad_output_sigmas` must have shape [A, R, T].")
    torch_check(grad_normals.dim() == 3, "`grad_normals` must have shape [R, S, 3].")
    torch_check(grad_sigmas.dim() == 3, "`grad_sigmas` must have shape [A, R, S].")
    torch_check(tuple(grad_output_normals.shape) == (R, T, 3), "`grad_output_normals` shape mismatch.")
    torch_check(tuple(grad_output_sigmas.shape) == (A, R, T), "`grad_output_sigmas` shape mismatch.")
    torch_check(tuple(z_vals.shape) == (R, S), "`z_vals` shape mismatch.")
    torch_check(tuple(target_z_vals.shape) == (R, T), "`target_z_vals` shape mismatch.")
    torch_check(tuple(grad_normals.shape) == (R, S, 3), "`grad_normals` shape mismatch.")
    torch_check(tuple(grad_sigmas.shape) == (A, R, S), "`grad_sigmas` shape mismatch.")
    check_same_dtype(grad_output_normals, (grad_output_sigmas, "grad_output_sigmas"),
                     (z_vals, "z_vals"), (target_z_vals, "target_z_vals"),
                     (grad_normals, "grad_normals"), (grad_sigmas, "grad_sigmas"))
    dt = dtype_code(grad_output_normals, "bilinear_raysample_backward_cuda", allow_half=False)
    with device_guard(grad_output_normals.device):
        _lib.call("geraf_bilinear_backward", ptr(grad_output_normals), ptr(grad_output_sigmas),
                  ptr(z_vals), ptr(target_z_vals), ptr(grad_normals), ptr(grad_sigmas), A, R, S, T,
                  dt, stream_ptr(grad_output_normals.device))


from ..RFMatchedFilter._C import get_compiler_version, get_cuda_version, has_cuda  # noqa: E402,F401
