"""RF training steps built from the operators, eager or captured in a CUDA graph.

* :class:`GraphedStep` -- the capture / replay frame: ``capture()`` records one
  whole step (forward, backward and any optimizer update) into a CUDA graph over
  static input buffers after an eager warm-up on a side stream; ``run()``
  replays it.  All operator calls enqueue on the current stream and allocate
  through PyTorch's caching allocator, which the graph's private pool serves
  during capture.
* :class:`RaggedRFStep` -- every antenna of a step renders IF from its own
  uneven set of points (one persistent launch, ``signal_tracer_ragged``), the
  IF of all antennas is matched-filtered onto a voxel set, and an L1 loss on
  the magnitude against a target volume is back-propagated through the matched
  filter adjoint and the tracer adjoint onto the points' amplitudes, normals
  and positions.
"""
from __future__ import annotations

import torch

from .ops.RFMatchedFilter.matched_filter_cuda import matched_filter_cuda
from .ops.RFSignalTracer.ragged import signal_tracer_ragged


class GraphedStep:
    """Subclasses implement ``_step_eager`` (one step, returning the loss)."""

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


class RaggedRFStep(GraphedStep):
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
