"""Multi-GPU sharding of the RF operators over ``torch.distributed`` (NCCL).

One process per GPU.  The operators partition naturally:

* matched filter -- voxels are split into contiguous slabs, one per rank.  The
  forward pass needs no communication (each rank backprojects its slab from a
  replicated copy of the IF samples and antenna positions); the slabs are
  gathered only when the caller asks for the whole volume.  The adjoint is a
  sum over voxels, so each rank's slab adjoint [A, S] is summed with one
  all-reduce.
* signal tracer -- antennas are split across ranks.  The forward pass is
  independent per antenna; in the adjoint, ``grad_sigmas`` [A_rank, P] stays
  local and the per-point gradients (normals, positions) [P, 3] are summed with
  one all-reduce.

Every rank takes the same collective steps in the same order.  The compute
callables are injectable so the communication logic can be exercised with the
``gloo`` backend on CPU; by default they are this library's CUDA kernels.
"""
from __future__ import annotations

from typing import Callable

import torch
import torch.distributed as dist


def shard_range(total: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous near-equal slab [start, end) of ``total`` items for ``rank``."""
    base, rem = divmod(total, world)
    start = rank * base + min(rank, rem)
    return start, start + base + (1 if rank < rem else 0)


def _world(group) -> tuple[int, int]:
    if not dist.is_available() or not dist.is_initialized():
        return 1, 0
    return dist.get_world_size(group), dist.get_rank(group)


# ---- default CUDA compute ----------------------------------------------------
def _cuda_mf_forward(real, imag, tpos, rpos, voxel_3n, fs, As, precision):
    from .ops.RFMatchedFilter import _C

    N = voxel_3n.shape[1]
    out_r = torch.empty(N, dtype=real.dtype, device=real.device)
    out_i = torch.empty(N, dtype=real.dtype, device=real.device)
    _C.MatchedFilter_forward(real, imag, tpos, rpos, out_r, out_i, voxel_3n, real.shape[0],
                             real.shape[1], fs, As, N, precision=precision)
    return out_r, out_i


def _cuda_mf_backward(gr, gi, real, imag, tpos, rpos, voxel_3n, fs, As, precision):
    from .ops.RFMatchedFilter import _C

    grad_r = torch.empty_like(real)
    grad_i = torch.empty_like(imag)
    _C.MatchedFilter_backward_realimag(gr, gi, real, imag, tpos, rpos, grad_r, grad_i, voxel_3n,
                                       real.shape[0], real.shape[1], fs, As, voxel_3n.shape[1],
                                       precision=precision)
    return grad_r, grad_i


class _ShardedMF(torch.autograd.Function):
    @staticmethod
    def forward(ctx, real, imag, tpos, rpos, voxel_slab_3n, fs, As, precision, group, fwd, bwd):
        out_r, out_i = fwd(real, imag, tpos, rpos, voxel_slab_3n, fs, As, precision)
        ctx.save_for_backward(real, imag, tpos, rpos, voxel_slab_3n)
        ctx.cfg = (fs, As, precision, group, bwd)
        return out_r, out_i

    @staticmethod
    def backward(ctx, g_r, g_i):
        real, imag, tpos, rpos, vox = ctx.saved_tensors
        fs, As, precision, group, bwd = ctx.cfg
        grad_r = grad_i = None
        if ctx.needs_input_grad[0] and ctx.needs_input_grad[1]:
            grad_r, grad_i = bwd(g_r.contiguous(), g_i.contiguous(), real, imag, tpos, rpos, vox, fs,
                                 As, precision)
            world, _ = _world(group)
            if world > 1:
                both = torch.stack([grad_r, grad_i])
                dist.all_reduce(both, op=dist.ReduceOp.SUM, group=group)
                grad_r, grad_i = both[0], both[1]
        return (grad_r, grad_i) + (None,) * 9


class _GatherSlabs(torch.autograd.Function):
    """All-gather of the ranks' (real, imag) slabs into the whole volume.

    Backward: this rank's slice of the incoming gradient.  That is the gradient
    of a loss every rank computes identically from the gathered volume (the
    replicated-loss pattern ``gather=True`` serves); the slab adjoints are then
    summed across ranks by the matched filter's own backward all-reduce."""

    @staticmethod
    def forward(ctx, out_r, out_i, start, end, N, group):
        world, _ = _world(group)
        sizes = [shard_range(N, world, r) for r in range(world)]
        width = max(e - s for s, e in sizes)
        pad = torch.zeros((2, width), dtype=out_r.dtype, device=out_r.device)
        pad[0, : end - start] = out_r
        pad[1, : end - start] = out_i
        parts = [torch.empty_like(pad) for _ in range(world)]
        dist.all_gather(parts, pad, group=group)
        ctx.span = (start, end)
        full_r = torch.cat([p[0, : e - s] for p, (s, e) in zip(parts, sizes)])
        full_i = torch.cat([p[1, : e - s] for p, (s, e) in zip(parts, sizes)])
        return full_r, full_i

    @staticmethod
    def backward(ctx, g_r, g_i):
        s, e = ctx.span
        return g_r[s:e], g_i[s:e], None, None, None, None


def sharded_matched_filter(real: torch.Tensor, image: torch.Tensor, tpos: torch.Tensor,
                           rpos: torch.Tensor, voxel: torch.Tensor, adcSampleRate: float,
                           As_sci: float, *, precision: str | None = None, group=None,
                           gather: bool = False,
                           forward_fn: Callable | None = None,
                           backward_fn: Callable | None = None):
    """Matched filter of replicated IF [A,S] onto this rank's slab of ``voxel`` [N,3].

    Returns this rank's slab ``(out_real, out_imag)`` and its voxel range, or
    with ``gather=True`` the whole volume on every rank (one all-gather).  The
    gradient with respect to (real, image) is the sum of all ranks' slab
    adjoints (one all-reduce in the backward pass).  With ``gather=True`` every
    rank must compute the same loss from the gathered volume: the gather's
    backward takes each rank's own slice of that loss's gradient.
    """
    world, rank = _world(group)
    N = voxel.shape[0]
    start, end = shard_range(N, world, rank)
    slab = voxel[start:end].t().contiguous()
    out_r, out_i = _ShardedMF.apply(real.contiguous(), image.contiguous(), tpos.contiguous(),
                                    rpos.contiguous(), slab, adcSampleRate, As_sci, precision, group,
                                    forward_fn or _cuda_mf_forward, backward_fn or _cuda_mf_backward)
    if not gather or world == 1:
        return out_r, out_i, (start, end)
    full_r, full_i = _GatherSlabs.apply(out_r, out_i, start, end, N, group)
    return full_r, full_i, (0, N)


# ---- tracer ----------------------------------------------------------------------
def _cuda_tracer_forward(normals, sigmas, points, tx, rx, inbounds, S, fs, f0, As, precision):
    from .ops.RFSignalTracer import _C

    A, P = sigmas.shape
    out_r = torch.empty((A, S), dtype=normals.dtype, device=normals.device)
    out_i = torch.empty_like(out_r)
    _C.SignalTracer_forward(normals, sigmas, points, tx, rx, inbounds, out_r, out_i, S, fs, f0, As, A,
                            P, precision=precision)
    return out_r, out_i


def _cuda_tracer_backward(gr, gi, normals, sigmas, points, tx, rx, inbounds, S, fs, f0, As,
                          precision, want_points):
    from .ops.RFSignalTracer import _C

    A, P = sigmas.shape
    gn = torch.empty_like(normals)
    gs = torch.empty_like(sigmas)
    gp = torch.empty_like(points) if want_points else None
    _C.SignalTracer_backward_normal_sigma(gr, gi, normals, sigmas, points, tx, rx, inbounds, gn, gs,
                                          S, fs, f0, As, A, P, grad_points=gp, precision=precision)
    return gn, gs, gp


class _ShardedTracer(torch.autograd.Function):
    @staticmethod
    def forward(ctx, normals, sigmas_local, points, tx_local, rx_local, inbounds, S, fs, f0, As,
                precision, group, fwd, bwd):
        out_r, out_i = fwd(normals, sigmas_local, points, tx_local, rx_local, inbounds, S, fs, f0, As,
                           precision)
        ctx.save_for_backward(normals, sigmas_local, points, tx_local, rx_local, inbounds)
        ctx.cfg = (S, fs, f0, As, precision, group, bwd)
        return out_r, out_i

    @staticmethod
    def backward(ctx, g_r, g_i):
        normals, sigmas, points, tx, rx, inb = ctx.saved_tensors
        S, fs, f0, As, precision, group, bwd = ctx.cfg
        want_p = ctx.needs_input_grad[2]
        gn, gs, gp = bwd(g_r.contiguous(), g_i.contiguous(), normals, sigmas, points, tx, rx, inb, S,
                         fs, f0, As, precision, want_p)
        world, _ = _world(group)
        if world > 1:
            # per-point gradients are sums over antennas: one all-reduce of [P, 3] (x2)
            flat = torch.cat([gn.reshape(-1)] + ([gp.reshape(-1)] if want_p else []))
            dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
            gn = flat[: gn.numel()].view_as(gn)
            if want_p:
                gp = flat[gn.numel():].view_as(points)
        return (gn if ctx.needs_input_grad[0] else None, gs if ctx.needs_input_grad[1] else None,
                gp) + (None,) * 11


def sharded_signal_tracer(normals: torch.Tensor, sigmas: torch.Tensor, points: torch.Tensor,
                          antenna_t: torch.Tensor, antenna_r: torch.Tensor, inbounds: torch.Tensor,
                          numADCSample: int, adcSampleRate: float, fc_start: float, As_sci: float,
                          *, precision: str | None = None, group=None,
                          forward_fn: Callable | None = None, backward_fn: Callable | None = None):
    """Renders this rank's antenna slab [A_rank, S] of the tracer.

    ``sigmas`` / ``antenna_t`` / ``antenna_r`` are the full [A, ...] tensors
    (or already-sliced local rows when their first dimension equals the
    slab).  Points and normals are replicated.  The normalisation is by the
    total point count, as in the unsharded operator.
    """
    world, rank = _world(group)
    A = antenna_t.shape[0]
    start, end = shard_range(A, world, rank)
    sig = sigmas[start:end] if sigmas.shape[0] == A else sigmas
    tx = antenna_t[start:end] if antenna_t.shape[0] == A else antenna_t
    rx = antenna_r[start:end] if antenna_r.shape[0] == A else antenna_r
    out_r, out_i = _ShardedTracer.apply(normals.contiguous(), sig.contiguous(), points.contiguous(),
                                        tx.contiguous(), rx.contiguous(), inbounds.contiguous(),
                                        numADCSample, adcSampleRate, fc_start, As_sci, precision,
                                        group, forward_fn or _cuda_tracer_forward,
                                        backward_fn or _cuda_tracer_backward)
    return out_r, out_i, (start, end)
