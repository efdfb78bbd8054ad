"""The stage-1 RF path on the device (geraf_b200.stage1, geraf_b200.bank): the
prediction against the reference's own sequence of operator calls, including
its matched filter over the in-bounds target points only, and the antenna
bank's chunks, fill and round-robin against the reference's generate_series
and mix (rf_rendering.py:275-276, 558-604, 655-716, 761-803)."""
import numpy as np
import pytest
import torch
import torch.nn.functional as F

from benchkit import scenes
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _rays(seed, R=96, Sc=24, T=40, A=12, S=64):
    g = torch.Generator(device="cuda").manual_seed(seed)
    tx, rx = scenes.virtual_array(2)
    tx = torch.tensor(tx[:A], device="cuda")
    rx = torch.tensor(rx[:A], device="cuda")
    origin = rx.mean(0)
    aim = torch.tensor([0.0, 0.0, 0.4], device="cuda") + 0.1 * (torch.rand((R, 3), device="cuda", generator=g) - 0.5)
    d = F.normalize(aim - origin, dim=-1)
    z = torch.sort(0.3 + 0.2 * torch.rand((R, Sc), device="cuda", generator=g), dim=1).values
    tz = torch.sort(0.28 + 0.24 * torch.rand((R, T), device="cuda", generator=g), dim=1).values
    grads = torch.randn((R, Sc, 3), device="cuda", generator=g) - 2.0 * d[:, None, :]
    sig = torch.rand((R, Sc), device="cuda", generator=g)
    pts = origin + d[:, None, :] * tz[..., None]
    cfg = scenes.chirp(S).radar_cfg(fc_start=770.0)
    return dict(tx=tx, rx=rx, z=z, tz=tz, grads=grads, sig=sig, pts=pts, cfg=cfg)


def _reference_sequence(c, tx_sel, rx_sel, mix_real, mix_imag, mix_tx, mix_rx, precision):
    """The reference's calls in order, the MF over in-bounds targets only."""
    from geraf_b200.ops.RFMatchedFilter.matched_filter_cuda import matched_filter_cuda
    from geraf_b200.ops.RFSignalTracer.bilinear_raysample_cuda import bilinear_raysample_cuda
    from geraf_b200.ops.RFSignalTracer.signal_tracer_cuda import signal_tracer_cuda

    R, Sc = c["z"].shape
    T = c["tz"].shape[1]
    P = R * T
    n = F.normalize(c["grads"], dim=-1)
    tn, ts, inb = bilinear_raysample_cuda(n, c["sig"].reshape(1, R, Sc), c["z"], c["tz"], 1, R, Sc, T)
    tn = F.normalize(tn, dim=-1)
    C = tx_sel.shape[0]
    cfg = c["cfg"]
    xr, xi = signal_tracer_cuda(tn.reshape(P, 3), ts.repeat(C, 1, 1).reshape(C, P), c["pts"].reshape(P, 3),
                                tx_sel, rx_sel, inb.reshape(P), cfg["numADCSample"], cfg["adcSampleRate"],
                                cfg["fc_start"], cfg["As_sci"], C, P, precision=precision)
    re, im = mix_real(xr), mix_imag(xi)
    inb = inb.reshape(P)
    pts = c["pts"].reshape(P, 3)[inb]
    yr, yi = matched_filter_cuda(re, im, mix_tx, mix_rx, pts, mix_tx.shape[0], cfg["numADCSample"],
                                 cfg["adcSampleRate"], cfg["As_sci"], pts.shape[0], precision=precision)
    return torch.hypot(yr, yi), inb, xr, xi


@pytest.mark.parametrize("precision", ["mixed", "plain"])
def test_prediction_matches_the_reference_sequence(cuda, precision):
    from geraf_b200.bank import AntennaBank
    from geraf_b200.stage1 import stage1_rf_prediction

    c = _rays(0)
    A, S = c["tx"].shape[0], c["cfg"]["numADCSample"]
    bank = AntennaBank(c["tx"], c["rx"], 1, S)
    pred, inb = stage1_rf_prediction(c["grads"], c["sig"], c["z"], c["tz"], c["pts"], bank, c["cfg"],
                                     precision=precision)
    ref, ref_inb, _, _ = _reference_sequence(c, c["tx"], c["rx"], lambda x: x, lambda x: x, c["tx"], c["rx"],
                                             precision)
    assert torch.equal(inb, ref_inb)
    assert 0 < int(inb.sum()) < inb.numel()   # some targets fall outside the coarse samples
    # per-point matched filter: the out-of-bounds points change nothing at the others
    assert rel_l2(pred[inb].double().cpu().numpy(), ref.double().cpu().numpy()) < 2e-6


def test_antenna_bank_chunks_fill_and_mix(cuda):
    """Strided chunks as generate_series; a banked prediction, with every chunk
    cached from the same inputs, equals the unbanked one; advance() is round-robin
    and each step refreshes its chunk's rows."""
    from geraf_b200.bank import AntennaBank
    from geraf_b200.ops.RFSignalTracer.bilinear_raysample_cuda import bilinear_raysample_cuda
    from geraf_b200.ops.RFSignalTracer.signal_tracer_cuda import signal_tracer_cuda
    from geraf_b200.stage1 import stage1_rf_prediction

    c = _rays(1)
    A, S = c["tx"].shape[0], c["cfg"]["numADCSample"]
    bank = AntennaBank(c["tx"], c["rx"], 3, S)
    for g in range(3):
        assert torch.equal(bank.chunk_indices(g).cpu(), torch.arange(g, A, 3))
    with pytest.raises(ValueError):
        AntennaBank(c["tx"], c["rx"], 5, S)
    R, Sc = c["z"].shape
    T = c["tz"].shape[1]
    P = R * T
    tn, ts, inb = bilinear_raysample_cuda(F.normalize(c["grads"], dim=-1), c["sig"].reshape(1, R, Sc), c["z"],
                                          c["tz"], 1, R, Sc, T)
    tn = F.normalize(tn, dim=-1).reshape(P, 3)
    cfg = c["cfg"]

    def render(tx, rx):
        C = tx.shape[0]
        return signal_tracer_cuda(tn, ts.reshape(1, P).expand(C, P).contiguous(), c["pts"].reshape(P, 3), tx, rx,
                                  inb.reshape(P), cfg["numADCSample"], cfg["adcSampleRate"], cfg["fc_start"],
                                  cfg["As_sci"], C, P)

    bank.fill(render)
    full = AntennaBank(c["tx"], c["rx"], 1, S)
    ref, _ = stage1_rf_prediction(c["grads"], c["sig"], c["z"], c["tz"], c["pts"], full, cfg)
    seen = []
    for step in range(4):
        bank.advance()
        seen.append(bank.chunk_id)
        pred, _ = stage1_rf_prediction(c["grads"], c["sig"], c["z"], c["tz"], c["pts"], bank, cfg)
        # [chunk; others] is the whole array in another order: the same volume to rounding
        assert rel_l2(pred.double().cpu().numpy(), ref.double().cpu().numpy()) < 2e-6
    assert seen == [1, 2, 0, 1]
    whole_r, whole_i = render(c["tx"], c["rx"])
    assert rel_l2(bank.real.cpu().numpy(), whole_r.cpu().numpy()) < 1e-6
    assert rel_l2(bank.imag.cpu().numpy(), whole_i.cpu().numpy()) < 1e-6
