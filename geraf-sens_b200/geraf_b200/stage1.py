"""The RF part of GeRaF's stage-1 loss on the device, in one capturable sequence.

``GeRaFStage1.loss`` (``geraf/models/rendering/rf_rendering.py:721-820``) turns
the SDF network's output at a ray's coarse samples into predicted
matched-filter magnitudes at the ray's target samples:

1. normals = normalised SDF gradients; the amplitudes and normals are resampled
   from the coarse depths to the target depths (``_sample_tgt_normals_and_sigmas``
   :622-645, the along-ray resampler), the resampled normals normalised again;
2. the tracer renders the IF of the current antenna chunk from the target
   points (``lensless_ray_tracer`` :769-780), out-of-range targets masked;
3. the render is mixed with the other chunks' cached IF and matched-filtered at
   the target points (``_gather_unselected_adc`` / ``_matched_filter_prediction``
   :655-716, :783-803); the prediction is the magnitude.

:func:`stage1_rf_prediction` runs that sequence on this library's operators.
One difference keeps every shape fixed from step to step (so a whole training
step can be captured in a CUDA graph): the reference matched-filters only the
in-bounds target points (``tgt_sampled_poses_glb[inbounds]``, :696-697), this
function matched-filters all of them and returns the in-bounds mask with the
prediction; averaging the caller's loss over the masked points gives the
reference's loss.  The bank of cached chunks is an :class:`AntennaBank` in
device memory.
"""
from __future__ import annotations

import torch
import torch.nn.functional as F

from .bank import AntennaBank
from .ops.RFSignalTracer.bilinear_raysample_cuda import bilinear_raysample_cuda
from .ops.RFSignalTracer.signal_tracer_cuda import signal_tracer_cuda


def stage1_rf_prediction(gradients: torch.Tensor, sigmas: torch.Tensor, z_vals: torch.Tensor,
                         tgt_z_vals: torch.Tensor, tgt_points: torch.Tensor, bank: AntennaBank,
                         radar_cfg: dict, precision: str | None = None,
                         mf_precision: str | None = None) -> tuple[torch.Tensor, torch.Tensor]:
    """Predicted |MF| [R*T] at the target points and their in-bounds mask [R*T].

    gradients [R, S_c, 3] (SDF gradients at the coarse samples), sigmas [R, S_c]
    (their amplitudes), z_vals [R, S_c] and tgt_z_vals [R, T] (depths along each
    ray), tgt_points [R, T, 3] (world positions of the target samples).
    ``precision`` selects the tracer's arithmetic form, ``mf_precision`` the
    matched filter's (default: the same)."""
    R, Sc = z_vals.shape
    T = tgt_z_vals.shape[1]
    P = R * T
    normals = F.normalize(gradients, dim=-1)
    tgt_normals, tgt_sigmas, inbounds = bilinear_raysample_cuda(normals.contiguous(), sigmas.reshape(1, R, Sc),
                                                                z_vals, tgt_z_vals, 1, R, Sc, T)
    tgt_normals = F.normalize(tgt_normals, dim=-1).reshape(P, 3)
    inbounds = inbounds.reshape(P)
    C = bank.chunk
    tx_s, rx_s = bank.selected_positions()
    points = tgt_points.reshape(P, 3)
    xr, xi = signal_tracer_cuda(tgt_normals, tgt_sigmas.reshape(1, P).expand(C, P).contiguous(), points,
                                tx_s, rx_s, inbounds, radar_cfg["numADCSample"], radar_cfg["adcSampleRate"],
                                radar_cfg["fc_start"], radar_cfg["As_sci"], C, P, precision=precision)
    yr, yi = bank.matched_filter(xr, xi, points, radar_cfg, precision=mf_precision or precision)
    return torch.sqrt(yr * yr + yi * yi + 1e-20), inbounds
