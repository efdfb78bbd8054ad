"""Generates the golden vectors in tests/golden/*.npz from the REFERENCE's own CUDA
kernels: the unmodified GeRaF ``_C`` extensions compiled for sm_100a by
``oracle/build_ref.py`` into ``oracle/_ref/`` (run that first, where the
reference checkout exists; the built modules then travel with the tree).

Needs a CUDA GPU.  Every case stores its seeded inputs and the reference's
outputs; outputs are pre-filled with NaN so entries the reference leaves
unwritten stay NaN (the tracer adjoint skips out-of-bounds points).  The
resampler's adjoint accumulates, so its gradient buffers start from a stored
non-zero pattern.

    python tests/golden/make_golden.py --out tests/golden
    python tests/golden/make_golden.py --only fullsize_mf3072ch_f32   # one case
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [ROOT, os.path.join(ROOT, "geraf-sens_b200")]

from benchkit import scenes  # noqa: E402
from oracle import build_ref  # noqa: E402


def mf_inputs(seed, scan, S, k, n, noise=True):
    rng = np.random.default_rng(seed)
    tx, rx = scenes.virtual_array(scan)
    pos, amp = scenes.point_scene(rng, k, size=0.12)
    ch = scenes.chirp(S)
    re, im = scenes.synthesize_if_numpy(tx, rx, pos, amp, ch, snr_db=20.0 if noise else None, rng=rng)
    vox = scenes.voxel_grid(n, size=0.12)
    return dict(real=re, imag=im, tx=tx, rx=rx, voxel=vox, fs=np.float32(ch.adc_sample_rate),
                As=np.float32(ch.As_sci))


def tracer_inputs(seed, A, P, S, f0=770.0, inb_frac=0.85):
    rng = np.random.default_rng(seed)
    tx, rx = scenes.virtual_array(2)
    tx = (tx[:A] + rng.normal(0, 0.01, (A, 3))).astype(np.float32)
    rx = (rx[:A] + rng.normal(0, 0.01, (A, 3))).astype(np.float32)
    d = rng.normal(0, 1, (P, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    points = (np.array([0, 0, 0.4]) + 0.08 * d).astype(np.float32)
    nrm = d - rng.uniform(0.5, 1.2, (P, 1)) * np.array([0, 0, 1.0])
    nrm = (nrm / np.linalg.norm(nrm, axis=1, keepdims=True)).astype(np.float32)
    sig = rng.uniform(0, 1, (A, P)).astype(np.float32)
    inb = rng.uniform(0, 1, P) < inb_frac
    ch = scenes.chirp(S)
    return dict(normals=nrm, sigmas=sig, points=points, tx=tx, rx=rx, inbounds=inb,
                fs=np.float32(ch.adc_sample_rate), f0=np.float32(f0), As=np.float32(ch.As_sci))


def bilinear_inputs(seed, A, R, S, T):
    rng = np.random.default_rng(seed)
    z = np.sort(rng.uniform(0.2, 0.6, (R, S)), axis=1).astype(np.float32)
    z[0, 3] = z[0, 4]  # a repeated depth exercises the 1e-6 denominator clamp
    tz = rng.uniform(0.15, 0.65, (R, T)).astype(np.float32)
    tz[1, :4] = z[1, :4]  # targets exactly on coarse samples
    return dict(normals=rng.standard_normal((R, S, 3)).astype(np.float32),
                sigmas=rng.uniform(0, 1, (A, R, S)).astype(np.float32), z_vals=z, tgt_z_vals=tz,
                grad_out_normals=rng.standard_normal((R, T, 3)).astype(np.float32),
                grad_out_sigmas=rng.standard_normal((A, R, T)).astype(np.float32),
                grad_normals_init=(0.01 * rng.standard_normal((R, S, 3))).astype(np.float32),
                grad_sigmas_init=(0.01 * rng.standard_normal((A, R, S))).astype(np.float32))


def cu(x, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    return t.to(dtype) if dtype is not None else t


def run_mf(mod, inp, dtype, grad_seed):
    A, S = inp["real"].shape
    N = inp["voxel"].shape[1]
    args = [cu(inp[k], dtype) for k in ("real", "imag", "tx", "rx")]
    out_r = torch.full((N,), float("nan"), dtype=dtype, device="cuda")
    out_i = torch.full((N,), float("nan"), dtype=dtype, device="cuda")
    vox = cu(inp["voxel"], dtype)
    mod.MatchedFilter_forward(*args, out_r, out_i, vox, A, S, float(inp["fs"]), float(inp["As"]), N)
    rng = np.random.default_rng(grad_seed)
    gr = rng.standard_normal(N).astype(np.float32)
    gi = rng.standard_normal(N).astype(np.float32)
    g_r = torch.full((A, S), float("nan"), dtype=dtype, device="cuda")
    g_i = torch.full((A, S), float("nan"), dtype=dtype, device="cuda")
    mod.MatchedFilter_backward_realimag(cu(gr, dtype), cu(gi, dtype), *args, g_r, g_i, vox, A, S,
                                        float(inp["fs"]), float(inp["As"]), N)
    torch.cuda.synchronize()
    return dict(out_real=out_r.float().cpu().numpy(), out_imag=out_i.float().cpu().numpy(),
                grad_output_real=gr, grad_output_imag=gi, grad_real=g_r.float().cpu().numpy(),
                grad_imag=g_i.float().cpu().numpy())


def run_mf_fft(mod, inp, bins, spacing, grad_seed):
    rng = np.random.default_rng(grad_seed)
    A = inp["tx"].shape[0]
    N = inp["voxel"].shape[1]
    spec_r = rng.standard_normal((A, bins)).astype(np.float32)
    spec_i = rng.standard_normal((A, bins)).astype(np.float32)
    out_r = torch.full((N,), float("nan"), device="cuda")
    out_i = torch.full((N,), float("nan"), device="cuda")
    args = [cu(spec_r), cu(spec_i), cu(inp["tx"]), cu(inp["rx"])]
    vox = cu(inp["voxel"])
    mod.MatchedFilter_fft_forward(*args, out_r, out_i, vox, A, bins, spacing, float(inp["fs"]),
                                  float(inp["As"]), N)
    gr = rng.standard_normal(N).astype(np.float32)
    gi = rng.standard_normal(N).astype(np.float32)
    g_r = torch.full((A, bins), float("nan"), device="cuda")
    g_i = torch.full((A, bins), float("nan"), device="cuda")
    mod.MatchedFilter_fft_backward_realimag(cu(gr), cu(gi), *args, g_r, g_i, vox, A, bins, spacing,
                                            float(inp["fs"]), float(inp["As"]), N)
    torch.cuda.synchronize()
    return dict(spec_real=spec_r, spec_imag=spec_i, bins=np.int64(bins), spacing=np.float32(spacing),
                out_real=out_r.cpu().numpy(), out_imag=out_i.cpu().numpy(), grad_output_real=gr,
                grad_output_imag=gi, grad_real=g_r.cpu().numpy(), grad_imag=g_i.cpu().numpy())


def run_tracer(mod, inp, dtype, grad_seed):
    A, P = inp["sigmas"].shape
    S = int(inp["S"])
    t = {k: cu(inp[k], dtype) for k in ("normals", "sigmas", "points", "tx", "rx")}
    inb = cu(inp["inbounds"])
    out_r = torch.full((A, S), float("nan"), dtype=dtype, device="cuda")
    out_i = torch.full((A, S), float("nan"), dtype=dtype, device="cuda")
    sc = (S, float(inp["fs"]), float(inp["f0"]), float(inp["As"]), A, P)
    mod.SignalTracer_forward(t["normals"], t["sigmas"], t["points"], t["tx"], t["rx"], inb, out_r,
                             out_i, *sc)
    rng = np.random.default_rng(grad_seed)
    gr = rng.standard_normal((A, S)).astype(np.float32)
    gi = rng.standard_normal((A, S)).astype(np.float32)
    gn = torch.full((P, 3), float("nan"), dtype=dtype, device="cuda")
    gs = torch.full((A, P), float("nan"), dtype=dtype, device="cuda")
    mod.SignalTracer_backward_normal_sigma(cu(gr, dtype), cu(gi, dtype), t["normals"], t["sigmas"],
                                           t["points"], t["tx"], t["rx"], inb, gn, gs, *sc)
    torch.cuda.synchronize()
    return dict(out_real=out_r.cpu().numpy(), out_imag=out_i.cpu().numpy(), grad_output_real=gr,
                grad_output_imag=gi, grad_normals=gn.cpu().numpy(), grad_sigmas=gs.cpu().numpy())


def run_bilinear(mod, inp):
    A, R, S = inp["sigmas"].shape
    T = inp["tgt_z_vals"].shape[1]
    on = torch.full((R, T, 3), float("nan"), device="cuda")
    os_ = torch.full((A, R, T), float("nan"), device="cuda")
    ob = torch.zeros((R, T), dtype=torch.bool, device="cuda")
    mod.BilinearRaysample_forward(cu(inp["normals"]), cu(inp["sigmas"]), cu(inp["z_vals"]),
                                  cu(inp["tgt_z_vals"]), on, os_, ob, A, R, S, T)
    gn = cu(inp["grad_normals_init"]).clone()
    gs = cu(inp["grad_sigmas_init"]).clone()
    mod.BilinearRaysample_backward(cu(inp["grad_out_normals"]), cu(inp["grad_out_sigmas"]),
                                   cu(inp["z_vals"]), cu(inp["tgt_z_vals"]), gn, gs, A, R, S, T)
    torch.cuda.synchronize()
    return dict(out_normals=on.cpu().numpy(), out_sigmas=os_.cpu().numpy(),
                out_inbounds=ob.cpu().numpy(), grad_normals=gn.cpu().numpy(),
                grad_sigmas=gs.cpu().numpy())


def run_mf_3072ch(mod):
    """The reference's kernels on the full 3072-channel workload (3072 x 128 x 48^3).
    The inputs are regenerated by the tests from their seed, so the fixture
    keeps only checksums of them, the forward at the 4096-voxel subset and the
    adjoint (of a seeded output gradient) at the 96-row subset."""
    from oracle import workload_parity as wp

    w = wp.mf3072_inputs(0)
    A, S = w["re"].shape
    N = w["vox"].shape[1]
    args = [cu(w[k]) for k in ("re", "im", "tx", "rx")]
    vox = cu(w["vox"])
    out_r = torch.full((N,), float("nan"), device="cuda")
    out_i = torch.full((N,), float("nan"), device="cuda")
    mod.MatchedFilter_forward(*args, out_r, out_i, vox, A, S, float(w["fs"]), float(w["As"]), N)
    g = wp.adjoint_grad(N, 21)
    g_r = torch.full((A, S), float("nan"), device="cuda")
    g_i = torch.full((A, S), float("nan"), device="cuda")
    mod.MatchedFilter_backward_realimag(cu(g.real.copy()), cu(g.imag.copy()), *args, g_r, g_i, vox, A, S,
                                        float(w["fs"]), float(w["As"]), N)
    torch.cuda.synchronize()
    vi, rows = wp.MF3072_VOXELS, wp.MF3072_ROWS
    return dict(input_abs_sums=np.array([np.abs(w["re"].astype(np.float64)).sum(),
                                         np.abs(w["im"].astype(np.float64)).sum()]),
                voxel_ids=vi, rows=rows, grad_seed=np.int64(21),
                out_real=out_r.cpu().numpy()[vi], out_imag=out_i.cpu().numpy()[vi],
                grad_real=g_r.cpu().numpy()[rows], grad_imag=g_i.cpu().numpy()[rows])


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("--only", default=None, help="comma list of case names to (re)generate")
    args = ap.parse_args(argv)
    os.makedirs(args.out, exist_ok=True)
    mf = build_ref.load("RFMatchedFilter")
    st = build_ref.load("RFSignalTracer")
    only = set(args.only.split(",")) if args.only else None

    def save(name, d):
        np.savez_compressed(os.path.join(args.out, name + ".npz"), **d)
        print("wrote", name)

    if only is not None:
        cases = {"fullsize_mf3072ch_f32": lambda: run_mf_3072ch(mf)}
        unknown = only - set(cases)
        if unknown:
            raise SystemExit(f"--only supports {sorted(cases)}, not {sorted(unknown)}")
        for name in sorted(only):
            save(name, cases[name]())
        return

    # matched filter: a physical scene, odd sizes, and the f16 / f64 dispatch paths
    inp = mf_inputs(1, scan=4, S=64, k=8, n=7)
    save("mf_scene_f32", {**inp, **run_mf(mf, inp, torch.float32, 11)})
    inp = mf_inputs(2, scan=2, S=37, k=3, n=5)
    save("mf_odd_f32", {**inp, **run_mf(mf, inp, torch.float32, 12)})
    inp = mf_inputs(3, scan=2, S=32, k=4, n=4)
    save("mf_scene_f16", {**inp, **run_mf(mf, inp, torch.float16, 13)})
    inp = mf_inputs(4, scan=2, S=16, k=4, n=4)
    save("mf_scene_f64", {**inp, **run_mf(mf, inp, torch.float64, 14)})
    inp = mf_inputs(5, scan=2, S=8, k=2, n=6)
    save("mf_fft_f32", {**inp, **run_mf_fft(mf, inp, bins=40, spacing=0.03, grad_seed=15)})

    # tracer: culling, out-of-bounds points, f64 dispatch
    inp = tracer_inputs(6, A=8, P=700, S=32)
    inp["S"] = np.int64(32)
    save("tracer_f32", {**inp, **run_tracer(st, inp, torch.float32, 16)})
    inp = tracer_inputs(7, A=3, P=130, S=20, f0=773.704)
    inp["S"] = np.int64(20)
    save("tracer_f64", {**inp, **run_tracer(st, inp, torch.float64, 17)})

    inp = bilinear_inputs(8, A=2, R=12, S=16, T=24)
    save("bilinear_f32", {**inp, **run_bilinear(st, inp)})

    # the reference's kernels at the full 3072-channel workload size
    save("fullsize_mf3072ch_f32", run_mf_3072ch(mf))


if __name__ == "__main__":
    main()
