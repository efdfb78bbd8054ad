"""Batched tracer over uneven per-antenna point sets: each row vs the regular
tracer over that antenna's points, the FP64 oracle, autograd, empty antennas,
absent inbounds, malformed offsets (detected on the device) and adjoint tiles that
span more antennas than they stage."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from benchkit import scenes
from geraf_b200 import _lib
from oracle import rf_oracle as orc

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-4


def ragged_case(seed=0, A=7, S=48, counts=None):
    rng = np.random.default_rng(seed)
    tx, rx = scenes.virtual_array(2)
    tx = (tx[:A] + rng.normal(0, 0.01, (A, 3))).astype(np.float32)
    rx = (rx[:A] + rng.normal(0, 0.01, (A, 3))).astype(np.float32)
    if counts is None:
        counts = rng.integers(1, 3000, A)
    counts = np.asarray(counts, np.int64)
    P = int(counts.sum())
    d = rng.normal(0, 1, (P, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pts = (np.array([0, 0, 0.4]) + 0.08 * d).astype(np.float32)
    nrm = d - rng.uniform(0.5, 1.2, (P, 1)) * np.array([0, 0, 1.0])
    nrm = (nrm / np.linalg.norm(nrm, axis=1, keepdims=True)).astype(np.float32)
    ch = scenes.chirp(S)
    return dict(tx=tx, rx=rx, pts=pts, nrm=nrm, sig=rng.uniform(0, 1, P).astype(np.float32),
                inb=rng.uniform(0, 1, P) < 0.9, off=np.concatenate([[0], np.cumsum(counts)]).astype(np.int64),
                ch=ch, f0=770.0, S=S)


def run(c, with_inb=True):
    from geraf_b200.ops.RFSignalTracer.ragged import signal_tracer_ragged

    t = {k: torch.tensor(c[k], device="cuda") for k in ("tx", "rx", "pts", "nrm", "sig", "off")}
    inb = torch.tensor(c["inb"], device="cuda") if with_inb else None
    ch = c["ch"]
    return signal_tracer_ragged(t["nrm"], t["sig"], t["pts"], t["off"], t["tx"], t["rx"], c["S"],
                                ch.adc_sample_rate, c["f0"], ch.As_sci, inbounds=inb)


def test_rows_match_per_antenna_oracle(cuda):
    c = ragged_case()
    xr, xi = run(c)
    x = xr.double().cpu().numpy() + 1j * xi.double().cpu().numpy()
    ch = c["ch"]
    for a in range(c["tx"].shape[0]):
        s, e = c["off"][a], c["off"][a + 1]
        rr, ri = orc.tracer_forward(c["nrm"][s:e], c["sig"][None, s:e], c["pts"][s:e], c["tx"][a:a + 1],
                                    c["rx"][a:a + 1], c["inb"][s:e], c["S"], ch.adc_sample_rate, c["f0"],
                                    ch.As_sci)
        assert rel_l2(x[a], rr[0] + 1j * ri[0]) < MIXED_TOL, a


def test_rows_match_regular_tracer(cuda):
    from geraf_b200.ops.RFSignalTracer import _C

    c = ragged_case(seed=3, A=5, counts=[4000, 700, 1, 5000, 2049])
    xr, xi = run(c)
    ch = c["ch"]
    for a in range(5):
        s, e = int(c["off"][a]), int(c["off"][a + 1])
        P = e - s
        out_r = torch.empty((1, c["S"]), device="cuda")
        out_i = torch.empty((1, c["S"]), device="cuda")
        _C.SignalTracer_forward(torch.tensor(c["nrm"][s:e], device="cuda"),
                                torch.tensor(c["sig"][None, s:e], device="cuda"),
                                torch.tensor(c["pts"][s:e], device="cuda"),
                                torch.tensor(c["tx"][a:a + 1], device="cuda"),
                                torch.tensor(c["rx"][a:a + 1], device="cuda"),
                                torch.tensor(c["inb"][s:e], device="cuda"), out_r, out_i, c["S"],
                                ch.adc_sample_rate, c["f0"], ch.As_sci, 1, P, precision="mixed")
        assert rel_l2(xr[a].double().cpu().numpy() + 1j * xi[a].double().cpu().numpy(),
                      out_r[0].double().cpu().numpy() + 1j * out_i[0].double().cpu().numpy()) < 2e-6


def test_adjoint_matches_per_antenna_oracle(cuda):
    from geraf_b200.ops.RFSignalTracer.ragged import signal_tracer_ragged

    c = ragged_case(seed=5, A=4)
    ch = c["ch"]
    t = {k: torch.tensor(c[k], device="cuda") for k in ("tx", "rx", "off")}
    nrm = torch.tensor(c["nrm"], device="cuda", requires_grad=True)
    sig = torch.tensor(c["sig"], device="cuda", requires_grad=True)
    pts = torch.tensor(c["pts"], device="cuda", requires_grad=True)
    xr, xi = signal_tracer_ragged(nrm, sig, pts, t["off"], t["tx"], t["rx"], c["S"], ch.adc_sample_rate,
                                  c["f0"], ch.As_sci, inbounds=torch.tensor(c["inb"], device="cuda"))
    rng = np.random.default_rng(1)
    gr = rng.standard_normal(xr.shape).astype(np.float32)
    gi = rng.standard_normal(xr.shape).astype(np.float32)
    ((xr * torch.tensor(gr, device="cuda")).sum() + (xi * torch.tensor(gi, device="cuda")).sum()).backward()
    for a in range(4):
        s, e = c["off"][a], c["off"][a + 1]
        gn, gs, gp = orc.tracer_backward(gr[a:a + 1], gi[a:a + 1], c["nrm"][s:e], c["sig"][None, s:e],
                                         c["pts"][s:e], c["tx"][a:a + 1], c["rx"][a:a + 1], c["inb"][s:e],
                                         ch.adc_sample_rate, c["f0"], ch.As_sci)
        assert rel_l2(sig.grad[s:e].double().cpu().numpy(), gs[0]) < MIXED_TOL
        assert rel_l2(nrm.grad[s:e].double().cpu().numpy(), gn) < MIXED_TOL
        assert rel_l2(pts.grad[s:e].double().cpu().numpy(), gp) < MIXED_TOL


def test_empty_antenna_and_no_inbounds_mask(cuda):
    c = ragged_case(seed=2, A=4, counts=[300, 0, 500, 64])
    xr, _ = run(c, with_inb=False)
    x = xr.cpu().numpy()
    assert np.isnan(x[1]).all()          # no points: 0/0 as in the reference
    assert np.isfinite(x[[0, 2, 3]]).all()
    c["inb"][:] = True
    xr2, _ = run(c, with_inb=True)
    np.testing.assert_array_equal(np.nan_to_num(xr2.cpu().numpy()), np.nan_to_num(x))


def test_malformed_offsets_are_detected_without_reading_points(cuda):
    from geraf_b200.ops.RFSignalTracer.ragged import signal_tracer_ragged

    c = ragged_case(seed=4, A=3, counts=[100, 100, 100])
    _lib.device_status(torch.cuda.current_stream().cuda_stream, reset=True)
    bad = np.array([0, 250, 120, 300], np.int64)  # decreasing
    t = {k: torch.tensor(c[k], device="cuda") for k in ("tx", "rx", "pts", "nrm", "sig")}
    ch = c["ch"]
    xr, xi = signal_tracer_ragged(t["nrm"], t["sig"], t["pts"], torch.tensor(bad, device="cuda"), t["tx"],
                                  t["rx"], c["S"], ch.adc_sample_rate, c["f0"], ch.As_sci)
    status = _lib.device_status(torch.cuda.current_stream().cuda_stream, reset=True)
    assert status == 1
    # no work item was formed, so every row is 0 / P_a
    assert (xr == 0).all() and (xi == 0).all()


def test_mixed_scale_workload_balances(cuda):
    """Ray counts U[512, 8192] x samples U[64, 192] on 16 antennas: rows still match."""
    rng = np.random.default_rng(11)
    counts = rng.integers(512, 8193, 16) * rng.integers(64, 193, 16) // 64
    c = ragged_case(seed=11, A=16, S=64, counts=counts)
    xr, xi = run(c)
    ch = c["ch"]
    for a in (0, 7, 15):
        s, e = c["off"][a], c["off"][a + 1]
        rr, ri = orc.tracer_forward(c["nrm"][s:e], c["sig"][None, s:e], c["pts"][s:e], c["tx"][a:a + 1],
                                    c["rx"][a:a + 1], c["inb"][s:e], c["S"], ch.adc_sample_rate, c["f0"],
                                    ch.As_sci)
        assert rel_l2(xr[a].double().cpu().numpy() + 1j * xi[a].double().cpu().numpy(), rr[0] + 1j * ri[0]) < MIXED_TOL


def test_adjoint_with_tiles_spanning_many_antennas(cuda):
    """24 antennas of 0-90 points: each 1024-point tile of the adjoint spans more
    antennas than it stages in shared memory, so the residual rows come from global
    memory; the gradients still match the per-antenna oracle."""
    from geraf_b200.ops.RFSignalTracer.ragged import signal_tracer_ragged

    rng = np.random.default_rng(21)
    counts = rng.integers(0, 91, 24)
    counts[3] = 0
    c = ragged_case(seed=21, A=24, counts=counts)
    ch = c["ch"]
    t = {k: torch.tensor(c[k], device="cuda") for k in ("tx", "rx", "off")}
    nrm = torch.tensor(c["nrm"], device="cuda", requires_grad=True)
    sig = torch.tensor(c["sig"], device="cuda", requires_grad=True)
    pts = torch.tensor(c["pts"], device="cuda", requires_grad=True)
    xr, xi = signal_tracer_ragged(nrm, sig, pts, t["off"], t["tx"], t["rx"], c["S"], ch.adc_sample_rate,
                                  c["f0"], ch.As_sci, inbounds=torch.tensor(c["inb"], device="cuda"))
    gr = rng.standard_normal(xr.shape).astype(np.float32)
    gi = rng.standard_normal(xr.shape).astype(np.float32)
    ((xr * torch.tensor(gr, device="cuda")).sum() + (xi * torch.tensor(gi, device="cuda")).sum()).backward()
    for a in range(24):
        s, e = c["off"][a], c["off"][a + 1]
        if e == s:
            continue
        gn, gs, gp = orc.tracer_backward(gr[a:a + 1], gi[a:a + 1], c["nrm"][s:e], c["sig"][None, s:e],
                                         c["pts"][s:e], c["tx"][a:a + 1], c["rx"][a:a + 1], c["inb"][s:e],
                                         ch.adc_sample_rate, c["f0"], ch.As_sci)
        if np.linalg.norm(gs) == 0:
            assert np.all(sig.grad[s:e].cpu().numpy() == 0)
            continue
        assert rel_l2(sig.grad[s:e].double().cpu().numpy(), gs[0]) < MIXED_TOL, a
        assert rel_l2(nrm.grad[s:e].double().cpu().numpy(), gn) < MIXED_TOL, a
        assert rel_l2(pts.grad[s:e].double().cpu().numpy(), gp) < MIXED_TOL, a


@pytest.mark.parametrize("fwd_tuning,bwd_tuning", [
    ({"threads": 64, "chunk": 8, "items_per_thread": 4}, {"stage_rows": 1}),
    ({"threads": 256, "chunk": 32, "items_per_thread": 16}, {"stage_rows": 8}),
    ({"threads": 128, "chunk": 8}, {"stage_rows": 2}),
])
def test_launch_shapes_agree(cuda, fwd_tuning, bwd_tuning):
    """Every tuned launch shape gives the library default's results (sums in
    other orders only) for the forward and the adjoint, S above one block's
    8-sample-chunk reach included."""
    from geraf_b200.ops.RFSignalTracer.ragged import signal_tracer_ragged

    for S in (48, 600):
        c = ragged_case(seed=6, A=6, S=S, counts=[1500, 1, 2600, 0, 700, 3100])
        ch = c["ch"]
        outs = []
        for ft, bt in ((None, None), (fwd_tuning, bwd_tuning)):
            t = {k: torch.tensor(c[k], device="cuda") for k in ("tx", "rx", "pts", "nrm", "sig", "off")}
            for k in ("pts", "nrm", "sig"):
                t[k].requires_grad_(True)
            xr, xi = signal_tracer_ragged(t["nrm"], t["sig"], t["pts"], t["off"], t["tx"], t["rx"], S,
                                          ch.adc_sample_rate, c["f0"], ch.As_sci,
                                          inbounds=torch.tensor(c["inb"], device="cuda"), tuning=ft,
                                          tuning_backward=bt)
            g = torch.Generator(device="cuda").manual_seed(1)
            gr = torch.randn(xr.shape, device="cuda", generator=g)
            gi = torch.randn(xr.shape, device="cuda", generator=g)
            keep = torch.isfinite(xr[:, 0])  # antenna 3 has no points: 0/0
            ((xr[keep] * gr[keep]).sum() + (xi[keep] * gi[keep]).sum()).backward()
            outs.append([torch.complex(xr, xi)[keep].detach().cpu().numpy()] +
                        [t[k].grad.double().cpu().numpy() for k in ("sig", "nrm", "pts")])
        # work items of other sizes group the per-antenna partial sums differently
        for a, b in zip(outs[0], outs[1]):
            assert rel_l2(b, a) < 5e-6
