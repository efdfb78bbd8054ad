"""GeRaF's stage-1 antenna bank, kept in device memory.

The reference renders only one chunk of a frame's antennas per training step
and matched-filters it together with the other chunks' IF from their last
render, which it keeps on the host (``geraf/models/rendering/rf_rendering.py``:
chunks ``generate_series`` :275-276, the first fill ``_ensure_cached_adc``
:558-604, the per-step gather and refresh ``_gather_unselected_adc`` :655-683,
the round-robin pointer ``_update_chunk_pointer`` :718-719).  Every step there
copies the cached chunks host -> device and the new render device -> host.

:class:`AntennaBank` keeps the cached IF in device memory and the current
chunk's antenna indices in static index buffers, so one step is a fixed
sequence of device operations with no host copies -- it can be captured in a
CUDA graph and replayed; :meth:`advance` (outside any graph) moves the buffers
to the next chunk.  Chunks are the reference's strided ones: chunk ``g`` holds
antennas ``g, g + bank_size, g + 2 bank_size, ...``.
"""
from __future__ import annotations

from typing import Callable

import torch

from .ops.RFMatchedFilter.faster_matched_filter_cuda import faster_matched_filter_cuda


class AntennaBank:
    """IF cache of ``bank_size`` antenna chunks for one frame (tx, rx [A, 3])."""

    def __init__(self, tx: torch.Tensor, rx: torch.Tensor, bank_size: int, num_adc: int):
        A = tx.shape[0]
        if bank_size < 1 or A % bank_size:
            raise ValueError(f"bank_size must divide the {A} antennas, got {bank_size} "
                             "(equal chunks keep every step's shapes fixed)")
        self.tx, self.rx = tx.contiguous(), rx.contiguous()
        self.bank_size = bank_size
        self.chunk = A // bank_size
        dev = tx.device
        self.real = torch.zeros((A, num_adc), dtype=tx.dtype, device=dev)
        self.imag = torch.zeros_like(self.real)
        self.sel_idx = torch.empty(self.chunk, dtype=torch.int64, device=dev)
        self.unsel_idx = torch.empty(A - self.chunk, dtype=torch.int64, device=dev)
        self.chunk_id = -1
        self.select(0)

    def chunk_indices(self, c: int) -> torch.Tensor:
        """Antennas of chunk ``c`` (the reference's ``generate_series``)."""
        return torch.arange(c, self.tx.shape[0], self.bank_size, device=self.tx.device)

    def select(self, c: int) -> None:
        """Points the static index buffers at chunk ``c`` (host side, outside any graph)."""
        ids = torch.arange(self.tx.shape[0], device=self.tx.device)
        sel = (ids % self.bank_size) == c
        self.sel_idx.copy_(ids[sel])
        self.unsel_idx.copy_(ids[~sel])
        self.chunk_id = c

    def advance(self) -> None:
        """Moves to the next chunk, round-robin (``_update_chunk_pointer``)."""
        self.select((self.chunk_id + 1) % self.bank_size)

    def selected_positions(self) -> tuple[torch.Tensor, torch.Tensor]:
        """(tx, rx) [chunk, 3] of the current chunk, gathered on the device."""
        return self.tx.index_select(0, self.sel_idx), self.rx.index_select(0, self.sel_idx)

    @torch.no_grad()
    def fill(self, render: Callable[[torch.Tensor, torch.Tensor], tuple[torch.Tensor, torch.Tensor]]) -> None:
        """Renders every chunk once (``_ensure_cached_adc``): ``render(tx_c, rx_c)``
        returns the chunk's IF (real, imag) [chunk, S]."""
        for c in range(self.bank_size):
            ids = self.chunk_indices(c)
            re, im = render(self.tx.index_select(0, ids), self.rx.index_select(0, ids))
            self.real.index_copy_(0, ids, re.detach())
            self.imag.index_copy_(0, ids, im.detach())

    def matched_filter(self, real: torch.Tensor, imag: torch.Tensor, points: torch.Tensor, radar_cfg: dict,
                       precision: str | None = None) -> tuple[torch.Tensor, torch.Tensor]:
        """The matched filter of [this step's render of the current chunk; the other
        chunks' cached IF] at ``points`` [N, 3], with gradients to the render only
        (the reference's mix + ``base_matched_filter``, rf_rendering.py:783-803);
        then stores the render in the bank."""
        tx_s, rx_s = self.selected_positions()
        tx_u, rx_u = self.tx.index_select(0, self.unsel_idx), self.rx.index_select(0, self.unsel_idx)
        re_u, im_u = self.real.index_select(0, self.unsel_idx), self.imag.index_select(0, self.unsel_idx)
        A, C, N = self.tx.shape[0], self.chunk, points.shape[0]
        yr, yi = faster_matched_filter_cuda(real, imag, re_u, im_u, tx_s, rx_s, tx_u, rx_u, points, A, C,
                                            radar_cfg["numADCSample"], radar_cfg["adcSampleRate"],
                                            radar_cfg["As_sci"], N, precision=precision)
        self.real.index_copy_(0, self.sel_idx, real.detach())
        self.imag.index_copy_(0, self.sel_idx, imag.detach())
        return yr, yi
