"""A GeRaF stage-1 RF training step on synthetic data (benchmark support).

The reference's stage-1 loss (``geraf/models/rendering/rf_rendering.py:721-820``)
with a random-initialised NeuS SDF network (``benchkit.sdf``):

* rays from the array's centre through a disk around the scene, ``coarse``
  stratified samples per ray for the SDF network and ``samples_per_ray``
  target samples per ray for the renderer (the reference's UniformRaySampler /
  TargetRaySampler; some targets fall outside the coarse depth range);
* the SDF network at the coarse samples (FP16 autocast, as the reference),
  NeuS alpha compositing, a sigmoid reflectance head times a fixed power (the
  reference config's FixedPowerNetwork) give each coarse sample's amplitude;
  normals are the normalised SDF gradients (differentiable: double backward);
* this library's stage-1 RF path (:func:`geraf_b200.stage1.stage1_rf_prediction`):
  resample to the targets, render the current antenna chunk, matched-filter the
  mix with the antenna bank's other chunks at the target points;
* the reference's "charbonier" loss sqrt((pred - gt)^2 + 1e-3) averaged over the
  in-bounds targets, gt being a matched-filter volume sampled at the target
  points (the reference's InterpolateMFAtTargets, here this library's
  ``geraf_b200.volume.sample_volume``), plus the eikonal term 0.1 mean(|grad| - 1)^2;
* backward and Adam.

Out of scope (renderer details of the reference, not its RF operators): the
transmission calibration against the unit sphere (``_calibrate_transmission``),
the inv_s annealing schedule and the dynamic loss mask.

``capture()`` / ``run()`` come from :class:`geraf_b200.step.GraphedStep`; with
``bank_size`` > 1 each step renders one chunk of the antennas (round-robin).
"""
from __future__ import annotations

import math

import torch
from torch import nn

from geraf_b200.bank import AntennaBank
from geraf_b200.stage1 import stage1_rf_prediction
from geraf_b200.step import GraphedStep
from geraf_b200.volume import sample_volume

SCENE_CENTER = (0.0, 0.0, 0.4)
SDF_RADIUS = 0.3   # m: the reference's unit-sphere normalisation radius (sample_cfg["radius"])


class Stage1RFStep(GraphedStep):
    """One stage-1 step: SDF network -> amplitudes -> RF prediction -> loss -> Adam."""

    def __init__(self, num_antennas=128, num_rays=2048, samples_per_ray=128, coarse_samples=None,
                 num_adc=256, precision: str = "mixed", mf_precision: str | None = None, bank_size: int = 1,
                 device="cuda", seed=0, lr=5e-4, grad_regression: float = 0.1, sdf_fp16: bool = True,
                 target_volume: torch.Tensor | None = None, volume_half: float = 0.16,
                 power: float | None = None):
        from . import scenes
        from .sdf import SDFNetwork

        torch.manual_seed(seed)
        self.device = torch.device(device)
        self.precision = precision
        self.mf_precision = mf_precision or precision
        # eikonal regulariser weight (with_grad_regression, 0.1 in
        # configs/geraf/bunnyboxv1/geraf2_bunnyboxv1_stage1.py:62)
        self.grad_regression = grad_regression
        self.sdf_fp16 = sdf_fp16
        self.net = SDFNetwork().to(self.device)
        self.head = nn.Linear(256, 1).to(self.device)
        self.log_inv_s = nn.Parameter(torch.tensor(10 * 0.3, device=self.device))  # inv_s = e^3
        params = list(self.net.parameters()) + list(self.head.parameters()) + [self.log_inv_s]
        self.opt = torch.optim.Adam(params, lr=lr, capturable=True)
        # the frame's antennas (all chunks of the bank): a seeded subset of the
        # 64 x 64 x 3TX4RX array; each step renders num_antennas / bank_size of them
        tx, rx = scenes.virtual_array(64)
        g = torch.Generator().manual_seed(seed)
        pick = torch.randperm(tx.shape[0], generator=g)[:num_antennas].sort().values
        self.tx = torch.tensor(tx, device=self.device)[pick].contiguous()
        self.rx = torch.tensor(rx, device=self.device)[pick].contiguous()
        self.chirp = scenes.chirp(num_adc)
        self.cfg = self.chirp.radar_cfg(fc_start=scenes.MF_CARRIER)
        self.center = torch.tensor(SCENE_CENTER, device=self.device)
        self.R, self.T = num_rays, samples_per_ray
        self.Sc = coarse_samples or max(2, samples_per_ray // 2)
        self.gen = torch.Generator(device=self.device).manual_seed(seed + 1)
        # static ray buffers, refilled by resample() outside any graph
        self.z_vals = torch.empty((self.R, self.Sc), device=self.device)
        self.tgt_z_vals = torch.empty((self.R, self.T), device=self.device)
        self.coarse_points = torch.empty((self.R, self.Sc, 3), device=self.device)
        self.tgt_points = torch.empty((self.R, self.T, 3), device=self.device)
        self.gt = torch.ones(self.R * self.T, device=self.device)
        self.target_volume = target_volume
        self.volume_half = volume_half
        self.bank_size = bank_size
        self.bank = AntennaBank(self.tx, self.rx, bank_size, num_adc)
        self.resample()
        self.power = 1.0 if power is None else float(power)
        if bank_size > 1:
            self._fill_bank()
        self.bank.select(bank_size - 1)   # the first step's advance() moves to chunk 0

    # -- inputs -----------------------------------------------------------------
    def resample(self) -> None:
        """New rays and samples (in place) and the target magnitudes at the targets."""
        R, T, Sc = self.R, self.T, self.Sc
        dev = self.device
        origin = self.rx.mean(0)
        u = torch.rand(R, device=dev, generator=self.gen)
        th = 2 * math.pi * torch.rand(R, device=dev, generator=self.gen)
        aim = self.center + torch.stack([0.2 * torch.sqrt(u) * torch.cos(th), 0.2 * torch.sqrt(u) * torch.sin(th),
                                         torch.zeros_like(u)], -1)
        d = aim - origin
        d = d / d.norm(dim=-1, keepdim=True)
        near, far = 0.22, 0.58
        z = torch.linspace(near, far, Sc, device=dev)[None, :] + (far - near) / Sc * torch.rand(
            R, Sc, device=dev, generator=self.gen)
        self.z_vals.copy_(torch.sort(z, dim=1).values)
        # the target pass spans a slightly wider range: its ends fall outside the coarse samples
        tn, tf = 0.21, 0.59
        zt = torch.linspace(tn, tf, T, device=dev)[None, :] + (tf - tn) / T * torch.rand(
            R, T, device=dev, generator=self.gen)
        self.tgt_z_vals.copy_(torch.sort(zt, dim=1).values)
        self.coarse_points.copy_(origin + d[:, None, :] * self.z_vals[..., None])
        self.tgt_points.copy_(origin + d[:, None, :] * self.tgt_z_vals[..., None])
        if self.target_volume is not None:
            norm = (self.tgt_points.reshape(-1, 3) - self.center) / self.volume_half
            self.gt.copy_(sample_volume(self.target_volume, norm))

    def _sdf(self, points, create_graph: bool):
        """SDF, feature vector and SDF gradient (with respect to the normalised
        coordinates (p - centre) / 0.3 m) at world points, as FP32."""
        x = ((points - self.center) / SDF_RADIUS).reshape(-1, 3).requires_grad_(True)
        with torch.autocast("cuda", dtype=torch.float16, enabled=self.sdf_fp16 and x.is_cuda):
            sdf, feat = self.net(x)
            grad, = torch.autograd.grad(sdf.sum(), x, create_graph=create_graph)
        return sdf.float(), feat.float(), grad.float()

    def _amplitudes(self, sdf, feat):
        """Coarse-sample amplitudes [R, Sc]: NeuS alpha x transmittance x reflectance x power."""
        inv_s = torch.exp(self.log_inv_s)
        cdf = torch.sigmoid(sdf.reshape(self.R, self.Sc) * inv_s)
        alpha = ((cdf[:, :-1] - cdf[:, 1:]) / (cdf[:, :-1] + 1e-5)).clamp(0.0, 1.0)
        alpha = torch.cat([alpha, alpha[:, -1:]], 1)
        # transmittance prod_{j<i} (1 - alpha_j), as exp(cumsum(log)): the backward of
        # cumprod synchronises with the host, which stream capture forbids
        log_t = torch.log(1.0 - alpha + 1e-7)
        trans = torch.exp(torch.cumsum(log_t, 1) - log_t)
        refl = torch.sigmoid(self.head(feat)).reshape(self.R, self.Sc)
        return alpha * trans * refl * self.power

    def predict(self, create_graph: bool):
        """(predicted |MF| [R*T], in-bounds mask [R*T], SDF gradients [R*Sc, 3])."""
        sdf, feat, grad = self._sdf(self.coarse_points, create_graph)
        sig = self._amplitudes(sdf, feat)
        pred, inb = stage1_rf_prediction(grad.reshape(self.R, self.Sc, 3), sig, self.z_vals, self.tgt_z_vals,
                                         self.tgt_points, self.bank, self.cfg, precision=self.precision,
                                         mf_precision=self.mf_precision)
        return pred, inb, grad

    def _fill_bank(self) -> None:
        """Renders every chunk once with the current network (``_ensure_cached_adc``)."""
        from geraf_b200.ops.RFSignalTracer.bilinear_raysample_cuda import bilinear_raysample_cuda
        from geraf_b200.ops.RFSignalTracer.signal_tracer_cuda import signal_tracer_cuda

        sdf, feat, grad = self._sdf(self.coarse_points, create_graph=False)
        with torch.no_grad():
            sig = self._amplitudes(sdf.detach(), feat.detach())
            R, Sc, T = self.R, self.Sc, self.T
            P = R * T
            n = torch.nn.functional.normalize(grad.reshape(R, Sc, 3), dim=-1)
            tn, ts, inb = bilinear_raysample_cuda(n.contiguous(), sig.reshape(1, R, Sc), self.z_vals,
                                                  self.tgt_z_vals, 1, R, Sc, T)
            tn = torch.nn.functional.normalize(tn, dim=-1).reshape(P, 3)
            C = self.bank.chunk
            cfg = self.cfg

            def render(tx, rx):
                return signal_tracer_cuda(tn, ts.reshape(1, P).expand(C, P).contiguous(),
                                          self.tgt_points.reshape(P, 3), tx, rx, inb.reshape(P),
                                          cfg["numADCSample"], cfg["adcSampleRate"], cfg["fc_start"],
                                          cfg["As_sci"], C, P, precision=self.precision)

            self.bank.fill(render)

    @torch.no_grad()
    def calibrate_power(self) -> float:
        """Sets the fixed power so that the initial prediction's mean over the in-bounds
        targets equals the target's (the role of the reference's light_power /
        trans_power normalisation); returns it."""
        self.power = 1.0
        with torch.enable_grad():
            pred, inb, _ = self.predict(create_graph=False)
        m = inb.float()
        mean_pred = float((pred * m).sum() / m.sum().clamp_min(1.0))
        mean_gt = float((self.gt * m).sum() / m.sum().clamp_min(1.0))
        self.power = mean_gt / max(mean_pred, 1e-30)
        if self.bank_size > 1:
            self._fill_bank()
            self.bank.select(self.bank_size - 1)
        return self.power

    # -- the step -----------------------------------------------------------------
    def _advance(self) -> None:
        if self.bank_size > 1:
            self.bank.advance()

    def _step_eager(self) -> torch.Tensor:
        self.opt.zero_grad(set_to_none=False)
        pred, inb, grad = self.predict(create_graph=True)
        m = inb.float()
        per_point = torch.sqrt((pred - self.gt) ** 2 + 1e-3)   # the reference's "charbonier" loss
        loss = (per_point * m).sum() / m.sum().clamp_min(1.0)
        if self.grad_regression:
            # mean (|grad sdf| - 1)^2 over the coarse samples (rf_rendering.py:647-650, 818-819)
            loss = loss + self.grad_regression * ((grad.norm(dim=-1) - 1.0) ** 2).mean()
        loss.backward()
        self.opt.step()
        return loss.detach()
