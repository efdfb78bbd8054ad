"""Drop-in replacement of the reference's ``geraf.ops.RFMatchedFilter._C`` module.

Same function names, positional arguments, out-parameter convention (outputs are
allocated by the caller and filled in place; the functions return ``None``) and
error behaviour (``RuntimeError`` with the reference's TORCH_CHECK messages) as
``geraf/ops/RFMatchedFilter/csrc/vision.cpp:70-97`` and
``csrc/matched_filter/MatchedFilter_cuda.cu:10-343``.  Each call runs on the
current torch stream of the input's device and does not synchronise.

Extra keyword-only arguments (not in the reference): ``precision`` ("mixed",
"plain" or "nufft", default from :func:`geraf_b200.runtime.default_precision`)
and ``tuning`` (a launch-shape dict, default from the autotuner cache; for
"nufft" its ``taps`` key sets the interpolation width, 4 to 12, default 8).
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


def _check_common(real, imag, tx_pos, rx_pos, voxel):
    # MatchedFilter_cuda.cu:10-37
    for t, n in ((real, "real"), (imag, "imag"), (tx_pos, "tx_pos"), (rx_pos, "rx_pos"), (voxel, "voxel")):
        torch_check(t.is_cuda, f"`{n}` must be a CUDA tensor.")
    for t, n in ((real, "real"), (imag, "imag"), (tx_pos, "tx_pos"), (rx_pos, "rx_pos"), (voxel, "voxel")):
        torch_check(t.is_contiguous(), f"`{n}` must be contiguous.")
    torch_check(real.dim() == 2, "`real` must have shape [A, S].")
    torch_check(imag.dim() == 2, "`imag` must have shape [A, S].")
    torch_check(tx_pos.dim() == 2, "`tx_pos` must have shape [A, 3].")
    torch_check(rx_pos.dim() == 2, "`rx_pos` must have shape [A, 3].")
    torch_check(voxel.dim() == 2, "`voxel` must have shape [3, N].")
    torch_check(real.shape == imag.shape, "`real` and `imag` must match.")
    torch_check(tx_pos.size(1) == 3, "`tx_pos` must store XYZ triplets.")
    torch_check(rx_pos.size(1) == 3, "`rx_pos` must store XYZ triplets.")


def _check_forward(real, imag, tx_pos, rx_pos, output_real, output_imag, voxel, A, S, N):
    # MatchedFilter_cuda.cu:39-69
    _check_common(real, imag, tx_pos, rx_pos, voxel)
    torch_check(output_real.is_cuda, "`output_real` must be a CUDA tensor.")
    torch_check(output_imag.is_cuda, "`output_imag` must be a CUDA tensor.")
    torch_check(output_real.is_contiguous(), "`output_real` must be contiguous.")
    torch_check(output_imag.is_contiguous(), "`output_imag` must be contiguous.")
    torch_check(output_real.dim() == 1, "`output_real` must have shape [N].")
    torch_check(output_imag.dim() == 1, "`output_imag` must have shape [N].")
    torch_check(real.size(0) == A, "`real` antenna dimension mismatch.")
    torch_check(real.size(1) == S, "`real` sample dimension mismatch.")
    torch_check(imag.size(0) == A, "`imag` antenna dimension mismatch.")
    torch_check(imag.size(1) == S, "`imag` sample dimension mismatch.")
    torch_check(tx_pos.size(0) == A, "`tx_pos` antenna dimension mismatch.")
    torch_check(rx_pos.size(0) == A, "`rx_pos` antenna dimension mismatch.")
    torch_check(voxel.size(0) == 3, "`voxel` must be laid out as [3, N].")
    torch_check(voxel.size(1) == N, "`voxel` count mismatch.")
    torch_check(output_real.size(0) == N, "`output_real` voxel dimension mismatch.")
    torch_check(output_imag.size(0) == N, "`output_imag` voxel dimension mismatch.")
    check_same_dtype(real, (imag, "imag"), (tx_pos, "tx_pos"), (rx_pos, "rx_pos"),
                     (voxel, "voxel"), (output_real, "output_real"), (output_imag, "output_imag"))


def _check_backward(gr, gi, real, imag, tx_pos, rx_pos, grad_real, grad_imag, voxel, A, S, N):
    # MatchedFilter_cuda.cu:71-107
    _check_common(real, imag, tx_pos, rx_pos, voxel)
    for t, n in ((gr, "grad_output_real"), (gi, "grad_output_imag"), (grad_real, "grad_real"),
                 (grad_imag, "grad_imag")):
        torch_check(t.is_cuda, f"`{n}` must be a CUDA tensor.")
    for t, n in ((gr, "grad_output_real"), (gi, "grad_output_imag"), (grad_real, "grad_real"),
                 (grad_imag, "grad_imag")):
        torch_check(t.is_contiguous(), f"`{n}` must be contiguous.")
    torch_check(gr.dim() == 1, "`grad_output_real` must have shape [N].")
    torch_check(gi.dim() == 1, "`grad_output_imag` must have shape [N].")
    torch_check(grad_real.dim() == 2, "`grad_real` must have shape [A, S].")
    torch_check(grad_imag.dim() == 2, "`grad_imag` must have shape [A, S].")
    torch_check(gr.size(0) == N, "`grad_output_real` voxel dimension mismatch.")
    torch_check(gi.size(0) == N, "`grad_output_imag` voxel dimension mismatch.")
    torch_check(grad_real.size(0) == A, "`grad_real` antenna dimension mismatch.")
    torch_check(grad_real.size(1) == S, "`grad_real` sample dimension mismatch.")
    torch_check(grad_imag.size(0) == A, "`grad_imag` antenna dimension mismatch.")
    torch_check(grad_imag.size(1) == S, "`grad_imag` sample dimension mismatch.")
    check_same_dtype(real, (gi, "grad_output_imag"), (gr, "grad_output_real"), (tx_pos, "tx_pos"),
                     (rx_pos, "rx_pos"), (voxel, "voxel"), (grad_real, "grad_real"),
                     (grad_imag, "grad_imag"))


def MatchedFilter_forward(real, imag, tx_pos, rx_pos, output_real, output_imag, voxel,
                          total_ant_size, num_adc_samples, adc_sample_rate, chirp_slope_scaled,
                          num_voxels, *, precision=None, tuning=None):
    """Matched-filter backprojection of raw ADC samples into ``output_{real,imag}`` [N]."""
    A, S, N = int(total_ant_size), int(num_adc_samples), int(num_voxels)
    _check_forward(real, imag, tx_pos, rx_pos, output_real, output_imag, voxel, A, S, N)
    dt = dtype_code(real, "matched_filter_forward_cuda", allow_half=True)
    mode = mode_code(precision, allow_nufft=True)
    tun = tuning_struct("mf_forward", (A, S, N), mode, tuning)
    with device_guard(real.device):
        nbytes = _lib.workspace_bytes("geraf_mf_forward_workspace_bytes", A, S, N, dt, mode,
                                      tuning_ref(tun))
        ws = workspace(nbytes, real.device)
        _lib.call("geraf_mf_forward", ptr(real), ptr(imag), ptr(tx_pos), ptr(rx_pos),
                  ptr(output_real), ptr(output_imag), ptr(voxel), A, S, float(adc_sample_rate),
                  float(chirp_slope_scaled), N, dt, mode, tuning_ref(tun), ptr(ws), nbytes,
                  stream_ptr(real.device))


def MatchedFilter_backward_realimag(grad_output_real, grad_output_imag, real, imag, tx_pos, rx_pos,
                                    grad_real, grad_imag, voxel, total_ant_size, num_adc_samples,
                                    adc_sample_rate, chirp_slope_scaled, num_voxels, *,
                                    precision=None, tuning=None):
    """Exact adjoint of :func:`MatchedFilter_forward` into ``grad_{real,imag}`` [A, S]."""
    A, S, N = int(total_ant_size), int(num_adc_samples), int(num_voxels)
    _check_backward(grad_output_real, grad_output_imag, real, imag, tx_pos, rx_pos, grad_real,
                    grad_imag, voxel, A, S, N)
    dt = dtype_code(real, "matched_filter_backward_realimag_cuda", allow_half=True)
    mode = mode_code(precision, allow_nufft=True)
    tun = tuning_struct("mf_backward", (A, S, N), mode, tuning)
    with device_guard(real.device):
        nbytes = _lib.workspace_bytes("geraf_mf_backward_workspace_bytes", A, S, N, dt, mode,
                                      tuning_ref(tun))
        ws = workspace(nbytes, real.device)
        _lib.call("geraf_mf_backward", ptr(grad_output_real), ptr(grad_output_imag), ptr(real),
                  ptr(imag), ptr(tx_pos), ptr(rx_pos), ptr(grad_real), ptr(grad_imag), ptr(voxel),
                  A, S, float(adc_sample_rate), float(chirp_slope_scaled), N, dt, mode,
                  tuning_ref(tun), ptr(ws), nbytes, stream_ptr(real.device))


def MatchedFilter_fft_forward(real, imag, tx_pos, rx_pos, output_real, output_imag, voxel,
                              total_ant_size, num_range_bins, fft_spacing, adc_sample_rate,
                              chirp_slope_scaled, num_voxels, *, consistent_bins=False):
    """Range-bin matched filter (reference: MatchedFilter_cuda_kernel.cu:117-169).

    ``consistent_bins=True`` keeps path delays up to 2 * fft_spacing * bins, the
    bound that matches the bin index floor(d / fft_spacing / 2); the default is
    the reference's bound fft_spacing * bins (:143-148), which reaches only the
    first half of the bins."""
    A, B, N = int(total_ant_size), int(num_range_bins), int(num_voxels)
    _check_forward(real, imag, tx_pos, rx_pos, output_real, output_imag, voxel, A, B, N)
    dt = dtype_code(real, "matched_filter_fft_forward_cuda", allow_half=True)
    flags = _lib.FFT_CONSISTENT_BINS if consistent_bins else 0
    with device_guard(real.device):
        _lib.call("geraf_mf_fft_forward", ptr(real), ptr(imag), ptr(tx_pos), ptr(rx_pos),
                  ptr(output_real), ptr(output_imag), ptr(voxel), A, B, float(fft_spacing),
                  float(adc_sample_rate), float(chirp_slope_scaled), N, dt, flags,
                  stream_ptr(real.device))


def MatchedFilter_fft_backward_realimag(grad_output_real, grad_output_imag, real, imag, tx_pos,
                                        rx_pos, grad_real, grad_imag, voxel, total_ant_size,
                                        num_range_bins, fft_spacing, adc_sample_rate,
                                        chirp_slope_scaled, num_voxels, *, consistent_bins=False):
    """Adjoint of :func:`MatchedFilter_fft_forward` (MatchedFilter_cuda_kernel.cu:222-279),
    with the same ``consistent_bins``."""
    A, B, N = int(total_ant_size), int(num_range_bins), int(num_voxels)
    _check_backward(grad_output_real, grad_output_imag, real, imag, tx_pos, rx_pos, grad_real,
                    grad_imag, voxel, A, B, N)
    dt = dtype_code(real, "matched_filter_fft_backward_realimag_cuda", allow_half=True)
    flags = _lib.FFT_CONSISTENT_BINS if consistent_bins else 0
    with device_guard(real.device):
        _lib.call("geraf_mf_fft_backward", ptr(grad_output_real), ptr(grad_output_imag),
                  ptr(real), ptr(imag), ptr(tx_pos), ptr(rx_pos), ptr(grad_real), ptr(grad_imag),
                  ptr(voxel), A, B, float(fft_spacing), float(adc_sample_rate),
                  float(chirp_slope_scaled), N, dt, flags, stream_ptr(real.device))


def get_cuda_version() -> str:
    """"CUDA <major>.<minor>" of the runtime the library was built with (vision.cpp:16-39)."""
    v = int(_lib.load().geraf_rf_cudart_version())
    s = f"CUDA {v // 1000}.{v // 10 % 100}"
    if v % 10:
        s += f".{v % 10}"
    return s


def has_cuda() -> bool:
    return True


def get_compiler_version() -> str:
    info = _lib.load().geraf_rf_build_info().decode()
    return info.split(";")[0].strip()
