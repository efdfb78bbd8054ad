"""RF training steps built from the operators, eager or captured in a CUDA graph.

Two step shapes that a GeRaF training loop runs:

* :class:`RaggedRFStep` -- every antenna of a step renders IF from its own
  uneven set of points (one persistent launch, ``signal_tracer_ragged``), the
  IF of all antennas is matched-filtered onto a voxel set, and an L1 loss on
  the magnitude against a target volume is back-propagated through the matched
  filter adjoint and the tracer adjoint onto the points' amplitudes, normals
  and positions.
* :class:`Stage1RFStep` -- a GeRaF stage-1 RF step on synthetic data: a
  random-init NeuS SDF MLP evaluated on ray samples (under FP16 autocast, as
  the reference) gives normals (SDF gradient, differentiable) and amplitudes
  (alpha-composited weights x reflectance); the tracer renders the IF of a bank of antennas from the shared
  points, the matched filter images it onto target voxels, an L1 loss on the
  magnitude against a target volume, plus the eikonal regulariser on the SDF
  gradient, is back-propagated (double backward through the SDF gradient) and
  Adam updates the network.

``capture()`` records one whole step (forward, backward and, for the stage-1
step, the optimizer update) into a CUDA graph over static input buffers;
``run()`` replays it.  The stage-1 step can also keep the reference's antenna
bank (``bank_size`` > 1): each step renders one chunk of the antennas and
matched-filters it with the other chunks' last renders, all in device memory.
All operator calls enqueue on the current stream and allocate through
PyTorch's caching allocator, which the graph's private pool serves during
capture.
"""
from __future__ import annotations

import math

import torch
from torch import nn

from .ops.RFMatchedFilter.faster_matched_filter_cuda import faster_matched_filter_cuda
from .ops.RFMatchedFilter.matched_filter_cuda import matched_filter_cuda
from .ops.RFSignalTracer.ragged import signal_tracer_ragged
from .ops.RFSignalTracer.signal_tracer_cuda import signal_tracer_cuda


class _Graphable:
    graph: torch.cuda.CUDAGraph | None = None

    def _step_eager(self) -> torch.Tensor:  # pragma: no cover - abstract
        raise NotImplementedError

    def _advance(self) -> None:
        """Per-step host-side set-up before a step runs (none by default)."""

    def warmup(self, iters: int = 2) -> None:
        """Eager steps on a side stream (autograd and allocator warm-up before capture)."""
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            for _ in range(iters):
                self._advance()
                self._step_eager()
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()

    def capture(self) -> None:
        self.warmup()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.static_loss = self._step_eager()
        torch.cuda.synchronize()

    def run(self) -> torch.Tensor:
        """One step: graph replay when captured, else eager."""
        self._advance()
        if self.graph is not None:
            self.graph.replay()
            return self.static_loss
        return self._step_eager()


class RaggedRFStep(_Graphable):
    """Ragged tracer -> matched filter -> L1(|y|, target) -> adjoints.

    Inputs (device tensors): normals/points [P,3], sigmas [P], point_offsets
    [A+1] (int64), tx/rx [A,3], voxels [N,3], target magnitudes [N].
    Gradients are left in ``.grad`` of normals, sigmas and points.
    """

    def __init__(self, normals, sigmas, points, point_offsets, tx, rx, voxels, target_mag, radar_cfg,
                 precision: str = "mixed"):
        self.normals = normals.detach().clone().requires_grad_(True)
        self.sigmas = sigmas.detach().clone().requires_grad_(True)
        self.points = points.detach().clone().requires_grad_(True)
        self.offsets, self.tx, self.rx = point_offsets, tx, rx
        self.voxels, self.target = voxels, target_mag
        self.cfg = radar_cfg
        self.precision = precision

    def _step_eager(self) -> torch.Tensor:
        for t in (self.normals, self.sigmas, self.points):
            t.grad = None
        cfg = self.cfg
        A, S = self.tx.shape[0], cfg["numADCSample"]
        xr, xi = signal_tracer_ragged(self.normals, self.sigmas, self.points, self.offsets, self.tx, self.rx,
                                      S, cfg["adcSampleRate"], cfg["fc_start"], cfg["As_sci"])
        yr, yi = matched_filter_cuda(xr, xi, self.tx, self.rx, self.voxels, A, S, cfg["adcSampleRate"],
                                     cfg["As_sci"], self.voxels.shape[0], precision=self.precision)
        loss = (torch.sqrt(yr * yr + yi * yi + 1e-20) - self.target).abs().mean()
        loss.backward()
        return loss.detach()


class Stage1RFStep(_Graphable):
    """A stage-1 GeRaF RF step with a random-init NeuS SDF MLP (see ``geraf_b200.sdf``)."""

    def __init__(self, num_antennas=128, num_rays=2048, samples_per_ray=128, num_adc=128, voxels=None,
                 target_mag=None, precision: str = "mixed", device="cuda", seed=0, lr=5e-4,
                 mf_precision: str | None = None, grad_regression: float = 0.1, bank_size: int = 1,
                 sdf_fp16: bool = True):
        from . import scenes
        from .sdf import SDFNetwork

        torch.manual_seed(seed)
        self.device = torch.device(device)
        self.precision = precision
        # the matched filter may run a form of its own ("nufft"); the tracer runs `precision`
        self.mf_precision = mf_precision or precision
        # eikonal regulariser weight (the reference's `with_grad_regression`, 0.1 in
        # configs/geraf/bunnyboxv1/geraf2_bunnyboxv1_stage1.py:62)
        self.grad_regression = grad_regression
        # the SDF network and its gradient run under FP16 autocast, as the reference's
        # stage-1 loss does (rf_rendering.py:742-749); the RF operators get FP32
        self.sdf_fp16 = sdf_fp16
        self.net = SDFNetwork().to(self.device)
        self.head = nn.Linear(256, 1).to(self.device)
        self.log_inv_s = nn.Parameter(torch.tensor(10 * 0.3, device=self.device))  # inv_s = e^3
        params = list(self.net.parameters()) + list(self.head.parameters()) + [self.log_inv_s]
        self.opt = torch.optim.Adam(params, lr=lr, capturable=True)
        tx, rx = scenes.virtual_array(16)
        g = torch.Generator().manual_seed(seed)
        pick = torch.randperm(tx.shape[0], generator=g)[:num_antennas].sort().values
        self.tx = torch.tensor(tx, device=self.device)[pick].contiguous()
        self.rx = torch.tensor(rx, device=self.device)[pick].contiguous()
        self.chirp = scenes.chirp(num_adc)
        self.cfg = self.chirp.radar_cfg(fc_start=scenes.MF_CARRIER)
        self.center = torch.tensor([0.0, 0.0, 0.4], device=self.device)
        self.scale = 0.2
        self.R, self.T = num_rays, samples_per_ray
        # static ray-sample buffer, refilled by resample() outside the graph
        self.points = torch.empty((num_rays * samples_per_ray, 3), device=self.device)
        self.inbounds = torch.ones(num_rays * samples_per_ray, dtype=torch.bool, device=self.device)
        self.gen = torch.Generator(device=self.device).manual_seed(seed + 1)
        self.resample()
        if voxels is None:
            voxels = torch.tensor(scenes.voxel_grid(32, size=0.3).T.copy(), device=self.device)
        self.voxels = voxels.contiguous()
        self.target = (target_mag if target_mag is not None
                       else torch.ones(self.voxels.shape[0], device=self.device))
        # Antenna bank (rf_rendering.py:558-604, 682-683, 718-800): the antennas are
        # split into `bank_size` chunks; a step renders one chunk with gradients and
        # matched-filters it together with the other chunks' IF from their last
        # render.  The bank lives in device memory and the chunk's antenna indices in
        # static index buffers, so a step is one graph replay with no host copies.
        A = self.tx.shape[0]
        if bank_size < 1 or A % bank_size:
            raise ValueError(f"bank_size must divide the {A} antennas, got {bank_size}")
        self.bank_size = bank_size
        self.chunk = A // bank_size
        self._chunk_id = -1
        if bank_size > 1:
            self.sel_idx = torch.empty(self.chunk, dtype=torch.int64, device=self.device)
            self.unsel_idx = torch.empty(A - self.chunk, dtype=torch.int64, device=self.device)
            S = self.chirp.num_samples
            self.bank_re = torch.zeros((A, S), device=self.device)
            self.bank_im = torch.zeros((A, S), device=self.device)
            self._fill_bank()
            self._set_chunk(0)   # valid indices from the start; the first step still takes chunk 0
            self._chunk_id = -1

    def _set_chunk(self, c: int) -> None:
        """Points the static index buffers at chunk ``c`` (outside any graph)."""
        A = self.tx.shape[0]
        ids = torch.arange(A, device=self.device)
        sel = (ids // self.chunk) == c
        self.sel_idx.copy_(ids[sel])
        self.unsel_idx.copy_(ids[~sel])
        self._chunk_id = c

    def _render_inputs(self, sdf, feat, grad):
        """Unit normals [P, 3] and amplitudes [1, P] of the ray samples from the SDF."""
        normals = grad / (grad.norm(dim=-1, keepdim=True) + 1e-12)
        inv_s = torch.exp(self.log_inv_s)
        sdf = sdf.reshape(self.R, self.T)
        cdf = torch.sigmoid(sdf * inv_s)
        alpha = ((cdf[:, :-1] - cdf[:, 1:]) / (cdf[:, :-1] + 1e-5)).clamp(0.0, 1.0)
        alpha = torch.cat([alpha, alpha[:, -1:]], 1)
        # transmittance prod_{j<i} (1 - alpha_j); formed as exp(cumsum(log)) because the
        # backward of cumprod synchronises with the host, which stream capture forbids
        log_t = torch.log(1.0 - alpha + 1e-7)
        trans = torch.exp(torch.cumsum(log_t, 1) - log_t)
        sig = (alpha * trans * torch.sigmoid(self.head(feat)).reshape(self.R, self.T)).reshape(1, -1)
        return normals, sig

    def _sdf(self, x, create_graph: bool):
        """SDF, feature vector and SDF gradient at normalised points x, as FP32."""
        with torch.autocast("cuda", dtype=torch.float16, enabled=self.sdf_fp16 and x.is_cuda):
            sdf, feat = self.net(x)
            grad, = torch.autograd.grad(sdf.sum(), x, create_graph=create_graph)
        return sdf.float(), feat.float(), grad.float()

    def _fill_bank(self) -> None:
        """Renders every chunk once with the current network (rf_rendering.py:558-604)."""
        x = ((self.points - self.center) / self.scale).requires_grad_(True)
        sdf, feat, grad = self._sdf(x, create_graph=False)
        with torch.no_grad():
            normals, sig = self._render_inputs(sdf.detach(), feat.detach(), grad)
            P = self.R * self.T
            S = self.chirp.num_samples
            for c in range(self.bank_size):
                rows = slice(c * self.chunk, (c + 1) * self.chunk)
                xr, xi = signal_tracer_cuda(normals, sig.expand(self.chunk, P).contiguous(), self.points,
                                            self.tx[rows].contiguous(), self.rx[rows].contiguous(),
                                            self.inbounds, S, self.cfg["adcSampleRate"], self.cfg["fc_start"],
                                            self.cfg["As_sci"], self.chunk, P, precision=self.precision)
                self.bank_re[rows] = xr
                self.bank_im[rows] = xi

    def _advance(self) -> None:
        """With an antenna bank, every step moves on to the next chunk (round-robin)."""
        if self.bank_size > 1:
            self._set_chunk((self._chunk_id + 1) % self.bank_size)

    def resample(self) -> None:
        """New rays through the scene disk, stratified samples along each (in place)."""
        R, T = self.R, self.T
        origin = self.rx.mean(0)
        u = torch.rand(R, device=self.device, generator=self.gen)
        th = 2 * math.pi * torch.rand(R, device=self.device, generator=self.gen)
        aim = self.center + torch.stack([self.scale * torch.sqrt(u) * torch.cos(th),
                                         self.scale * torch.sqrt(u) * torch.sin(th), torch.zeros_like(u)], -1)
        d = aim - origin
        d = d / d.norm(dim=-1, keepdim=True)
        near, far = 0.22, 0.58
        t = torch.linspace(near, far, T, device=self.device)[None, :] + (far - near) / T * torch.rand(
            R, T, device=self.device, generator=self.gen)
        t, _ = torch.sort(t, dim=1)
        self.points.copy_((origin + d[:, None, :] * t[..., None]).reshape(-1, 3))

    def _step_eager(self) -> torch.Tensor:
        self.opt.zero_grad(set_to_none=False)
        A, S = self.tx.shape[0], self.chirp.num_samples
        x = ((self.points - self.center) / self.scale).requires_grad_(True)
        sdf, feat, grad = self._sdf(x, create_graph=True)
        normals, sig = self._render_inputs(sdf, feat, grad)
        P = self.R * self.T
        N = self.voxels.shape[0]
        fs, As = self.cfg["adcSampleRate"], self.cfg["As_sci"]
        if self.bank_size > 1:
            C = self.chunk
            tx_s, rx_s = self.tx.index_select(0, self.sel_idx), self.rx.index_select(0, self.sel_idx)
            tx_u, rx_u = self.tx.index_select(0, self.unsel_idx), self.rx.index_select(0, self.unsel_idx)
            xr, xi = signal_tracer_cuda(normals, sig.expand(C, P).contiguous(), self.points, tx_s, rx_s,
                                        self.inbounds, S, fs, self.cfg["fc_start"], As, C, P,
                                        precision=self.precision)
            # [rendered chunk; cached chunks], adjoint over the rendered chunk only
            yr, yi = faster_matched_filter_cuda(xr, xi, self.bank_re.index_select(0, self.unsel_idx),
                                                self.bank_im.index_select(0, self.unsel_idx), tx_s, rx_s,
                                                tx_u, rx_u, self.voxels, A, C, S, fs, As, N,
                                                precision=self.mf_precision)
            self.bank_re.index_copy_(0, self.sel_idx, xr.detach())
            self.bank_im.index_copy_(0, self.sel_idx, xi.detach())
        else:
            xr, xi = signal_tracer_cuda(normals, sig.expand(A, P).contiguous(), self.points, self.tx, self.rx,
                                        self.inbounds, S, fs, self.cfg["fc_start"], As, A, P,
                                        precision=self.precision)
            yr, yi = matched_filter_cuda(xr, xi, self.tx, self.rx, self.voxels, A, S, fs, As, N,
                                         precision=self.mf_precision)
        mag = torch.sqrt(yr * yr + yi * yi + 1e-20)
        loss = (mag / (mag.detach().mean() + 1e-20) - self.target).abs().mean()
        if self.grad_regression:
            # mean (|grad sdf| - 1)^2 over the samples (rf_rendering.py:647-650, 818-819)
            loss = loss + self.grad_regression * ((grad.norm(dim=-1) - 1.0) ** 2).mean()
        loss.backward()
        self.opt.step()
        return loss.detach()
