"""The multi-GPU sharding logic on CPU: world size 2 over the gloo backend, with
the compute injected from the CPU oracle, against the unsharded oracle."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from conftest import PKG_DIR, ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _np(t):
    return t.detach().cpu().numpy()


def oracle_mf_fwd(real, imag, tpos, rpos, vox_3n, fs, As, precision):
    from oracle import rf_oracle as orc

    r, i = orc.mf_forward(_np(real), _np(imag), _np(tpos), _np(rpos), _np(vox_3n), fs, As, "f64")
    return torch.tensor(r), torch.tensor(i)


def oracle_mf_bwd(gr, gi, real, imag, tpos, rpos, vox_3n, fs, As, precision):
    from oracle import rf_oracle as orc

    A, S = real.shape
    r, i = orc.mf_backward(_np(gr), _np(gi), _np(tpos), _np(rpos), _np(vox_3n), A, S, fs, As, "f64")
    return torch.tensor(r), torch.tensor(i)


def oracle_tr_fwd(normals, sigmas, points, tx, rx, inb, S, fs, f0, As, precision):
    from oracle import rf_oracle as orc

    r, i = orc.tracer_forward(_np(normals), _np(sigmas), _np(points), _np(tx), _np(rx), _np(inb), S,
                              fs, f0, As, "f64")
    return torch.tensor(r), torch.tensor(i)


def oracle_tr_bwd(gr, gi, normals, sigmas, points, tx, rx, inb, S, fs, f0, As, precision, want_p):
    from oracle import rf_oracle as orc

    gn, gs, gp = orc.tracer_backward(_np(gr), _np(gi), _np(normals), _np(sigmas), _np(points), _np(tx),
                                     _np(rx), _np(inb), fs, f0, As, "f64", with_points=want_p)
    return torch.tensor(gn), torch.tensor(gs), (torch.tensor(gp) if gp is not None else None)


def make_inputs():
    from benchkit import scenes

    rng = np.random.default_rng(0)
    tx, rx = scenes.virtual_array(3)
    ch = scenes.chirp(16)
    pos, amp = scenes.point_scene(rng, 4, size=0.1)
    re, im = scenes.synthesize_if_numpy(tx, rx, pos, amp, ch, snr_db=None)
    vox = scenes.voxel_grid(5, size=0.1).T.copy()  # [N, 3]
    gr = rng.standard_normal(vox.shape[0])
    gi = rng.standard_normal(vox.shape[0])
    P, A = 60, tx.shape[0]
    d = rng.normal(0, 1, (P, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pts = (np.array([0, 0, 0.4]) + 0.08 * d).astype(np.float32)
    nrm = d - np.array([0, 0, 0.9])
    nrm = (nrm / np.linalg.norm(nrm, axis=1, keepdims=True)).astype(np.float32)
    sig = rng.uniform(0, 1, (A, P)).astype(np.float32)
    hr = rng.standard_normal((A, 16))
    hi = rng.standard_normal((A, 16))
    return dict(tx=tx, rx=rx, ch=ch, re=re, im=im, vox=vox, gr=gr, gi=gi, pts=pts, nrm=nrm, sig=sig,
                hr=hr, hi=hi)


def _worker(rank, world, port, outdir):
    sys.path[:0] = [ROOT, PKG_DIR]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    from geraf_b200 import distributed as gd

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        c = make_inputs()
        ch = c["ch"]
        re = torch.tensor(c["re"], dtype=torch.float64, requires_grad=True)
        im = torch.tensor(c["im"], dtype=torch.float64, requires_grad=True)
        yr, yi, (s, e) = gd.sharded_matched_filter(
            re, im, torch.tensor(c["tx"]), torch.tensor(c["rx"]), torch.tensor(c["vox"]),
            ch.adc_sample_rate, ch.As_sci, forward_fn=oracle_mf_fwd, backward_fn=oracle_mf_bwd)
        loss = (yr * torch.tensor(c["gr"][s:e])).sum() + (yi * torch.tensor(c["gi"][s:e])).sum()
        loss.backward()
        # the gathered volume is differentiable: the same loss on every rank from the whole volume
        re2 = re.detach().clone().requires_grad_(True)
        im2 = im.detach().clone().requires_grad_(True)
        full_r, full_i, _ = gd.sharded_matched_filter(
            re2, im2, torch.tensor(c["tx"]), torch.tensor(c["rx"]), torch.tensor(c["vox"]),
            ch.adc_sample_rate, ch.As_sci, gather=True, forward_fn=oracle_mf_fwd, backward_fn=oracle_mf_bwd)
        ((full_r * torch.tensor(c["gr"])).sum() + (full_i * torch.tensor(c["gi"])).sum()).backward()
        # tracer, antenna-sharded
        n = torch.tensor(c["nrm"], dtype=torch.float64, requires_grad=True)
        sg = torch.tensor(c["sig"], dtype=torch.float64, requires_grad=True)
        p = torch.tensor(c["pts"], dtype=torch.float64, requires_grad=True)
        inb = torch.ones(p.shape[0], dtype=torch.bool)
        xr, xi, (a0, a1) = gd.sharded_signal_tracer(
            n, sg, p, torch.tensor(c["tx"]), torch.tensor(c["rx"]), inb, 16, ch.adc_sample_rate, 770.0,
            ch.As_sci, forward_fn=oracle_tr_fwd, backward_fn=oracle_tr_bwd)
        ((xr * torch.tensor(c["hr"][a0:a1])).sum() + (xi * torch.tensor(c["hi"][a0:a1])).sum()).backward()
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), yr=_np(yr), yi=_np(yi), s=s, e=e,
                 gre=_np(re.grad), gim=_np(im.grad), full_r=_np(full_r), full_i=_np(full_i),
                 gre2=_np(re2.grad), gim2=_np(im2.grad), xr=_np(xr),
                 xi=_np(xi), a0=a0, a1=a1, gn=_np(n.grad), gs=_np(sg.grad), gp=_np(p.grad))
    finally:
        dist.destroy_process_group()


def test_shard_ranges_cover_exactly():
    from geraf_b200.distributed import shard_range

    for total in (0, 1, 7, 128):
        for world in (1, 2, 3, 8):
            spans = [shard_range(total, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == total
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            assert max(e - s for s, e in spans) - min(e - s for s, e in spans) <= 1


def test_two_rank_gloo_matches_unsharded(tmp_path):
    from oracle import rf_oracle as orc

    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(timeout=240)
        assert pr.exitcode == 0
    c = make_inputs()
    ch = c["ch"]
    A, S = c["re"].shape
    ref_r, ref_i = orc.mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"].T.copy(), ch.adc_sample_rate,
                                  ch.As_sci)
    ref_gr, ref_gi = orc.mf_backward(c["gr"], c["gi"], c["tx"], c["rx"], c["vox"].T.copy(), A, S,
                                     ch.adc_sample_rate, ch.As_sci)
    tr_r, tr_i = orc.tracer_forward(c["nrm"], c["sig"], c["pts"], c["tx"], c["rx"], np.ones(60, bool), 16,
                                    ch.adc_sample_rate, 770.0, ch.As_sci)
    gn, gs, gp = orc.tracer_backward(c["hr"], c["hi"], c["nrm"], c["sig"], c["pts"], c["tx"], c["rx"],
                                     np.ones(60, bool), ch.adc_sample_rate, 770.0, ch.As_sci)
    got_gs = np.zeros_like(gs)
    for r in range(world):
        d = np.load(tmp_path / f"rank{r}.npz")
        s, e = int(d["s"]), int(d["e"])
        np.testing.assert_allclose(d["yr"], ref_r[s:e], rtol=1e-6, atol=1e-9)
        np.testing.assert_allclose(d["yi"], ref_i[s:e], rtol=1e-6, atol=1e-9)
        np.testing.assert_allclose(d["full_r"], ref_r, rtol=1e-6, atol=1e-9)
        np.testing.assert_allclose(d["full_i"], ref_i, rtol=1e-6, atol=1e-9)
        # the all-reduced slab adjoints equal the unsharded adjoint on every rank
        np.testing.assert_allclose(d["gre"], ref_gr, rtol=1e-6, atol=1e-9)
        np.testing.assert_allclose(d["gim"], ref_gi, rtol=1e-6, atol=1e-9)
        # and through the gathered volume
        np.testing.assert_allclose(d["gre2"], ref_gr, rtol=1e-6, atol=1e-9)
        np.testing.assert_allclose(d["gim2"], ref_gi, rtol=1e-6, atol=1e-9)
        a0, a1 = int(d["a0"]), int(d["a1"])
        np.testing.assert_allclose(d["xr"], tr_r[a0:a1], rtol=1e-6, atol=1e-12)
        np.testing.assert_allclose(d["xi"], tr_i[a0:a1], rtol=1e-6, atol=1e-12)
        np.testing.assert_allclose(d["gn"], gn, rtol=1e-6, atol=1e-12)
        np.testing.assert_allclose(d["gp"], gp, rtol=1e-6, atol=1e-12)
        got_gs[a0:a1] = d["gs"][a0:a1]
    np.testing.assert_allclose(got_gs, gs, rtol=1e-6, atol=1e-12)
