"""Differentiable pure-PyTorch restatement of the specular signal tracer.

TEST INFRASTRUCTURE ONLY: the autograd cross-check of the hand-written
adjoint (normals, sigmas and -- with no reference counterpart -- points).
Follows ``geraf/ops/RFSignalTracer/csrc/signal_tracer/SignalTracer_cuda_kernel.cu``
lines 172-197 (geometry), 58-76 (distance, amplitude) and 351-450 (forward),
evaluated in whatever dtype the inputs carry (float64 for the checks).
Culling masks are computed without gradient, like the kernel's ``continue``.
"""
from __future__ import annotations

import math

import torch

K_C = float(torch.tensor(2.9979, dtype=torch.float32))
K_BIAS = float(torch.tensor(0.15, dtype=torch.float32))
K_EPS = float(torch.tensor(1e-7, dtype=torch.float32))
K_PI = float(torch.tensor(math.pi, dtype=torch.float32))


def _normalize(v: torch.Tensor) -> torch.Tensor:
    return v / (torch.linalg.norm(v, dim=-1, keepdim=True) + K_EPS)


def _amp_tau(normals, sigmas, points, tx, rx, inbounds):
    """Specular amplitude and delay of every (antenna, point) pair [A,P], and
    the pairs that survive culling."""
    inc_raw = points[None, :, :] - tx[:, None, :]          # [A,P,3]
    ret_raw = rx[:, None, :] - points[None, :, :]
    inc = _normalize(inc_raw)
    idn = (inc * normals[None]).sum(-1)
    refl_raw = inc - 2.0 * idn[..., None] * normals[None]
    refl = _normalize(refl_raw)
    ret = _normalize(ret_raw)
    align = (ret * refl).sum(-1)
    with torch.no_grad():
        live = (align >= 1e-6) & (idn <= 0.0) & inbounds[None, :]
    D = torch.linalg.norm(inc_raw, dim=-1) + torch.linalg.norm(ret_raw, dim=-1)
    amp = sigmas * align / (D * D)
    amp = torch.where(live, amp, torch.zeros_like(amp))
    tau = (D + K_BIAS) / K_C
    return amp, tau, live


def _rates(S: int, fs: float, f0: float, As: float, like: torch.Tensor) -> torch.Tensor:
    """Per-sample phase rate 2 pi f0 + 2 pi As t_n [S].  The scalars are rounded
    to FP32 first: the operator receives them as C floats."""
    fs, f0, As = (float(torch.tensor(v, dtype=torch.float32)) for v in (fs, f0, As))
    n = torch.arange(S, dtype=like.dtype, device=like.device)
    return 2.0 * K_PI * f0 + 2.0 * K_PI * As * (n / fs)


def tracer_forward(normals, sigmas, points, tx, rx, inbounds, S: int, fs: float, f0: float,
                   As: float):
    """normals/points [P,3], sigmas [A,P], tx/rx [A,3], inbounds [P] -> (re, im) [A,S]."""
    P = points.shape[0]
    amp, tau, _ = _amp_tau(normals, sigmas, points, tx, rx, inbounds)
    phase = tau[..., None] * _rates(S, fs, f0, As, points)  # [A,P,S]
    re = (amp[..., None] * torch.cos(phase)).sum(1) / P
    im = (amp[..., None] * torch.sin(phase)).sum(1) / P
    return re, im


def point_losses(normals, sigmas, points, tx, rx, S: int, fs: float, f0: float, As: float, gr, gi):
    """Each point's share of L = sum_{a,n} (g_r x_r + g_i x_i) before the 1/P
    normalisation, [P], for residual rows gr, gi [A,S]; and the culling mask
    [A,P] it was formed with.  All points are taken as in bounds."""
    inb = torch.ones(points.shape[0], dtype=torch.bool, device=points.device)
    amp, tau, live = _amp_tau(normals, sigmas, points, tx, rx, inb)
    phase = tau[..., None] * _rates(S, fs, f0, As, points)  # [A,P,S]
    per_pair = (torch.cos(phase) * gr[:, None, :] + torch.sin(phase) * gi[:, None, :]).sum(-1)
    return (amp * per_pair).sum(0), live
