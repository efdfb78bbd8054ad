"""Op adapters with the call contract of the reference's ``geraf.models.model_utils``
(``matched_filter.py:7-108``, ``ray_tracer.py:7-58``, ``ray_sampler.py:7-66``):
they read the radar constants from a ``radar_cfg`` dict and reject any backend
but ``"cuda"`` with ``ValueError``.  Renderers written against the reference
can import these instead and run unchanged.
"""
from __future__ import annotations

from typing import Dict

import torch


def base_matched_filter(real: torch.Tensor, image: torch.Tensor, t_pos: torch.Tensor,
                        r_pos: torch.Tensor, points: torch.Tensor, radar_cfg: Dict[str, float],
                        backend: str = "cuda", **kw):
    """Matched filter of IF [A,S] onto ``points`` [N,3] -> (real [N], imag [N])."""
    if backend != "cuda":
        raise ValueError(f"Unsupported matched filter backend: {backend!r}. Only 'cuda' is retained.")
    from .ops.RFMatchedFilter.matched_filter_cuda import matched_filter_cuda

    return matched_filter_cuda(real, image, t_pos, r_pos, points, t_pos.shape[0],
                               radar_cfg["numADCSample"], radar_cfg["adcSampleRate"],
                               radar_cfg["As_sci"], points.shape[0], **kw)


def faster_matched_filter(real_sel, image_sel, real_unsel, image_unsel, tpos_sel, rpos_sel,
                          tpos_unsel, rpos_unsel, points, radar_cfg: Dict[str, float],
                          backend: str = "cuda", **kw):
    """Matched filter over [selected; unselected] antennas, gradients to the selected rows."""
    if backend != "cuda":
        raise ValueError(
            f"Unsupported faster matched filter backend: {backend!r}. Only 'cuda' is retained.")
    from .ops.RFMatchedFilter.faster_matched_filter_cuda import faster_matched_filter_cuda

    num_sel = tpos_sel.shape[0]
    total = num_sel + tpos_unsel.shape[0]
    return faster_matched_filter_cuda(real_sel, image_sel, real_unsel, image_unsel, tpos_sel,
                                      rpos_sel, tpos_unsel, rpos_unsel, points, total, num_sel,
                                      radar_cfg["numADCSample"], radar_cfg["adcSampleRate"],
                                      radar_cfg["As_sci"], points.shape[0], **kw)


def lensless_ray_tracer(normals: torch.Tensor, sigmas: torch.Tensor, points: torch.Tensor,
                        antenna_t: torch.Tensor, antenna_r: torch.Tensor,
                        radar_cfg: Dict[str, float], backend: str = "cuda",
                        inbounds: torch.Tensor | None = None, use_diff: bool = True,
                        nomralization: bool = True, **kw):
    """Specular IF rendering -> (real [A,S], imag [A,S]); ``inbounds`` defaults to all points."""
    num_points = normals.shape[0]
    if inbounds is None:
        inbounds = torch.ones(num_points, dtype=torch.bool, device=points.device)
    if backend != "cuda":
        raise ValueError(f"Unsupported ray tracer backend: {backend!r}. Only 'cuda' is retained.")
    from .ops.RFSignalTracer.signal_tracer_cuda import signal_tracer_cuda

    return signal_tracer_cuda(normals=normals, sigmas=sigmas, points=points, antenna_t=antenna_t,
                              antenna_r=antenna_r, inbounds=inbounds,
                              numADCSample=radar_cfg["numADCSample"],
                              adcSampleRate=radar_cfg["adcSampleRate"],
                              fc_start=radar_cfg["fc_start"], As_sci=radar_cfg["As_sci"],
                              total_ant_size=antenna_t.shape[0], total_point_size=num_points,
                              use_diff=use_diff, nomralization=nomralization, **kw)


def bilinear_ray_sampler(normals: torch.Tensor, sigmas: torch.Tensor, z_vals: torch.Tensor,
                         tgt_z_vals: torch.Tensor, backend: str = "cuda"):
    """Resamples normals [R,S,3] / sigmas [A,R,S] at ``tgt_z_vals`` [R,T]."""
    N_ray, Nz, _ = normals.shape
    N_ant = sigmas.shape[0]
    Nz_tgt = tgt_z_vals.shape[1]
    if backend != "cuda":
        raise ValueError(f"Unsupported backend: {backend}. Use 'cuda' or 'torch'.")
    from .ops.RFSignalTracer.bilinear_raysample_cuda import bilinear_raysample_cuda

    return bilinear_raysample_cuda(normals=normals, sigmas=sigmas, z_vals=z_vals,
                                   tgt_z_vals=tgt_z_vals, N_ant=N_ant, N_ray=N_ray, Nz=Nz,
                                   Nz_tgt=Nz_tgt)
