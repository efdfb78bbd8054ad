"""Random-initialised SDF field used to synthesise realistic tracer inputs.

The tracer's inputs in a GeRaF training step come from a NeuS-style SDF MLP
evaluated on ray samples: unit normals are the normalised SDF gradient and the
per-sample amplitudes are alpha-composited weights times a reflectance in
[0, 1] times a scalar power.  This module builds such inputs from a freshly
initialised network of the published architecture -- 8 hidden layers of 256,
softplus (beta = 100), 6-frequency positional encoding, skip connection into
layer 4, geometric (sphere) initialisation, weight normalisation -- so the
benchmarks see the same value distributions without a trained checkpoint.
The network stays in PyTorch; it is input generation, not the hot path.
"""
from __future__ import annotations

import math

import numpy as np
import torch
from torch import nn


class PositionalEncoding(nn.Module):
    def __init__(self, multires: int = 6):
        super().__init__()
        self.freqs = [2.0 ** i for i in range(multires)]
        self.out_dim = 3 + 3 * 2 * multires

    def forward(self, x):
        parts = [x]
        for f in self.freqs:
            parts += [torch.sin(f * x), torch.cos(f * x)]
        return torch.cat(parts, -1)


class SDFNetwork(nn.Module):
    """sdf(x) and a 256-d feature; geometric init makes sdf ~ |x| - bias."""

    def __init__(self, d_hidden=256, n_layers=8, skip_in=(4,), multires=6, bias=0.5, d_feature=256):
        super().__init__()
        self.embed = PositionalEncoding(multires)
        dims = [self.embed.out_dim] + [d_hidden] * n_layers + [1 + d_feature]
        self.skip_in = set(skip_in)
        self.layers = nn.ModuleList()
        for i in range(len(dims) - 1):
            out_dim = dims[i + 1] - dims[0] if (i + 1) in self.skip_in else dims[i + 1]
            lin = nn.Linear(dims[i], out_dim)
            if i == len(dims) - 2:  # last layer: sdf ~ |x| - bias
                nn.init.normal_(lin.weight, mean=math.sqrt(math.pi) / math.sqrt(dims[i]), std=1e-4)
                nn.init.constant_(lin.bias, -bias)
            elif i == 0:  # only the raw xyz inputs drive the first layer
                nn.init.constant_(lin.bias, 0.0)
                nn.init.constant_(lin.weight[:, 3:], 0.0)
                nn.init.normal_(lin.weight[:, :3], 0.0, math.sqrt(2) / math.sqrt(out_dim))
            elif i in self.skip_in:  # the re-injected encoding starts at zero weight
                nn.init.constant_(lin.bias, 0.0)
                nn.init.normal_(lin.weight, 0.0, math.sqrt(2) / math.sqrt(out_dim))
                nn.init.constant_(lin.weight[:, -(dims[0] - 3):], 0.0)
            else:
                nn.init.constant_(lin.bias, 0.0)
                nn.init.normal_(lin.weight, 0.0, math.sqrt(2) / math.sqrt(out_dim))
            self.layers.append(nn.utils.parametrizations.weight_norm(lin))
        self.act = nn.Softplus(beta=100)

    def forward(self, x):
        e = self.embed(x)
        h = e
        for i, lin in enumerate(self.layers):
            if i in self.skip_in:
                h = torch.cat([h, e], -1) / math.sqrt(2)
            h = lin(h)
            if i < len(self.layers) - 1:
                h = self.act(h)
        return h[..., :1], h[..., 1:]


def tracer_workload(num_antennas=64, num_rays=4096, samples_per_ray=128, num_adc=128, seed=0,
                    device="cuda", center=(0.0, 0.0, 0.4), scale=0.2, near=0.22, far=0.58,
                    inv_s=math.exp(10 * 0.3), power=1.0):
    """Tracer inputs of one step: ``num_antennas`` array positions looking at a
    random-init SDF scene, ``num_rays`` rays x ``samples_per_ray`` samples
    shared by all antennas (the reference layout: points [P,3], sigmas [A,P]).
    Returns a dict of device tensors and the radar config."""
    from . import scenes

    g = torch.Generator(device="cpu").manual_seed(seed)
    torch.manual_seed(seed)
    tx_np, rx_np = scenes.virtual_array(16)
    pick = np.random.default_rng(seed).choice(tx_np.shape[0], num_antennas, replace=False)
    tx = torch.tensor(tx_np[np.sort(pick)], device=device)
    rx = torch.tensor(rx_np[np.sort(pick)], device=device)
    origin = rx.mean(0)
    c = torch.tensor(center, device=device)
    # rays through a disk of radius `scale` around the scene centre
    u = torch.rand(num_rays, generator=g).to(device)
    th = 2 * math.pi * torch.rand(num_rays, generator=g).to(device)
    aim = c + torch.stack([scale * torch.sqrt(u) * torch.cos(th), scale * torch.sqrt(u) * torch.sin(th),
                           torch.zeros_like(u)], -1)
    dirs = aim - origin
    dirs = dirs / dirs.norm(dim=-1, keepdim=True)
    t = torch.linspace(near, far, samples_per_ray, device=device)
    t = t[None, :] + (far - near) / samples_per_ray * torch.rand(num_rays, samples_per_ray, generator=g).to(device)
    t, _ = torch.sort(t, dim=1)
    pts = origin + dirs[:, None, :] * t[..., None]                      # [R,T,3]
    net = SDFNetwork().to(device)
    head = nn.Linear(256, 1).to(device)
    x = ((pts - c) / scale).reshape(-1, 3).requires_grad_(True)
    sdf, feat = net(x)
    grad, = torch.autograd.grad(sdf.sum(), x)
    with torch.no_grad():
        sdf = sdf.reshape(num_rays, samples_per_ray)
        cdf = torch.sigmoid(sdf * inv_s)
        alpha = ((cdf[:, :-1] - cdf[:, 1:]) / (cdf[:, :-1] + 1e-5)).clamp(0.0, 1.0)
        alpha = torch.cat([alpha, alpha[:, -1:]], 1)
        trans = torch.cumprod(torch.cat([torch.ones_like(alpha[:, :1]), 1.0 - alpha + 1e-7], 1), 1)[:, :-1]
        weights = alpha * trans
        refl = torch.sigmoid(head(feat)).reshape(num_rays, samples_per_ray)
        sig = (weights * refl * power).reshape(1, -1)
        normals = grad / (grad.norm(dim=-1, keepdim=True) + 1e-12)
    P = num_rays * samples_per_ray
    ch = scenes.chirp(num_adc)
    return dict(normals=normals.detach().contiguous(), sigmas=sig.repeat(num_antennas, 1).contiguous(),
                points=pts.reshape(P, 3).detach().contiguous(), tx=tx.contiguous(), rx=rx.contiguous(),
                inbounds=torch.ones(P, dtype=torch.bool, device=device), chirp=ch,
                radar_cfg=ch.radar_cfg(fc_start=770.0), rays=num_rays, P=P, A=num_antennas)
