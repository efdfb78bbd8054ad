#!/usr/bin/env python
"""Benchmark of the GeRaF RF operators on B200.

Headline (one JSON line on rank 0): matched-filter backprojection throughput in
G (voxel x antenna x sample) per second on the full-size workload -- 49152
virtual channels (64 x 64 scan x 3TX4RX), 256 ADC samples per chirp, a 128^3
voxel volume over a cube-shell + torus scene of 30k point scatterers at 20 dB
SNR (synthetic: the reference's RF data is not released) -- in the MIXED
arithmetic form (FP64 phase reduction, FP32 Horner phasors, compensated sums).

One step = one backprojection of the whole volume with inputs resident in HBM
(``value``); ``e2e`` repeats it through the public ``matched_filter_cuda`` call
from pinned host buffers with the host->device copies and the result read-back
inside the timed region.  Under torchrun each rank backprojects its own 128^3
slab of a taller volume (weak scaling, no collective on the data path).

Also reported: the FP32-pipe roofline of the kernel (algorithmic 8 flops per
voxel-antenna-sample over the measured FP32 FMA rate) with the measured ceiling
of its Horner loop, and clocks during the timed region.  At N = 1 the line adds
the extras: the PLAIN forward and adjoint, the MIXED MF adjoint, the NUFFT form,
the tracer forward + adjoint in rays/s, the ragged and stage-1 steps, relative
L2 errors against the FP64 oracle, and the CPU baseline (the reference-order
FP32 oracle port on the host cores).

``--impl reference`` times the reference's CPU path -- here the FP32
reference-order restatement in oracle/ (the reference has no CPU code) -- on a
bounded voxel sample of the same workload, and adds the reference's own CUDA
kernels (rebuilt for sm_100a into oracle/_ref) timed on this GPU.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "geraf-sens_b200")]

METRIC = "MF backprojection Gvox·ant·samp/s; tracer fwd+bwd rays/s; rel err vs FP64"
UNIT = "Gvox·ant·samp/s"
FLOPS_PER_TRIPLE = 8  # one complex multiply-accumulate of an IF sample by a unit phasor
L2_FLUSH_BYTES = 256 << 20


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["mf-full", "mf-small"], default="mf-full")
    ap.add_argument("--precision", choices=["mixed", "plain"], default="mixed")
    ap.add_argument("--no-extras", action="store_true", help="headline only (for profiling)")
    ap.add_argument("--extras", default="plain,adjoint,nufft,tracer,ragged,stage1,cpu",
                    help="comma list of secondary measurements: plain, adjoint, nufft, tracer, "
                         "ragged, stage1, cpu")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--ragged-antennas", type=int, default=256,
                    help="antennas of the ragged-step extra (fewer for a small profiling case)")
    ap.add_argument("--no-tune", action="store_true", help="skip the launch-shape autotuner")
    ap.add_argument("--stage1-steps", type=int, default=160,
                    help="training steps per form of the stage-1 equal-error comparison")
    return ap.parse_args(argv)


# ---------------------------------------------------------------------------
def dist_setup():
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi sampling of SM clock, power and throttle reasons every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "-i", str(gpu_index),
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        rows = []
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(dict(sm=float(parts[1]), max=float(parts[2]),
                                 power=float(parts[3]) if parts[3] not in ("[N/A]", "N/A") else 0.0,
                                 hw=parts[5], hwt=parts[6], swt=parts[7], swp=parts[8]))
            except ValueError:
                continue
        if not rows:
            return None
        loaded = [r for r in rows if r["power"] > 250.0] or rows
        sm = sorted(r["sm"] for r in loaded)
        reasons = set()
        for r in loaded:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"),
                              ("swt", "sw_thermal_slowdown"), ("swp", "sw_power_cap")):
                if r[key].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(r["max"] for r in rows),
                "reasons": sorted(reasons), "samples": len(rows), "samples_under_load": len(loaded),
                "power_w_max": max(r["power"] for r in rows)}


# ---------------------------------------------------------------------------
def fp32_peak_tflops(dev) -> float:
    """Measured FP32 FMA rate of this GPU (the roofline denominator)."""
    import torch

    from benchkit import probes

    lib = probes.lib()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    blocks, threads, iters = sms * 8, 256, 1 << 12
    sink = torch.empty(blocks * threads, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    best = 0.0
    for _ in range(4):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        probes.check(lib.geraf_rf_fma_probe(blocks, threads, iters, sink.data_ptr(), stream), "probe")
        e.record()
        e.synchronize()
        ms = s.elapsed_time(e)
        best = max(best, blocks * threads * iters * 32 / (ms * 1e-3) / 1e12)
    return best


def loop_ceiling_tflops(dev) -> float:
    """Measured rate of the MIXED forward's sample loop alone (geraf_rf_goertzel_probe:
    the second-order recurrence on packed complex samples, 4 blocks per SM, no
    per-(voxel, antenna) set-up), the ceiling of that loop's instruction form."""
    from benchkit import probes

    return probes.measure("goertzel", 4, dev.index or 0)


def make_mf_workload(name, rank, world, dev, seed):
    import numpy as np
    import torch

    from benchkit import scenes

    w = scenes.mf_full_workload(seed) if name == "mf-full" else scenes.mf_small_workload(seed)
    vox = w["voxel"].copy()
    span = float(vox[2].max() - vox[2].min()) + (vox[2, 1] - vox[2, 0] if vox.shape[1] > 1 else 0.0)
    vox[2] += rank * (span if span > 0 else 0.0)  # rank r backprojects slab r of a taller volume
    tx = torch.tensor(w["tx"], device=dev)
    rx = torch.tensor(w["rx"], device=dev)
    gen = torch.Generator(device=dev).manual_seed(seed + 1)
    re, im = scenes.synthesize_if(tx, rx, torch.tensor(w["positions"]), torch.tensor(w["amplitudes"]),
                                  w["chirp"], snr_db=w["snr_db"], generator=gen)
    return dict(tx=tx, rx=rx, real=re, imag=im, voxel=torch.tensor(vox, device=dev), chirp=w["chirp"],
                A=tx.shape[0], S=w["chirp"].num_samples, N=vox.shape[1], positions=w["positions"])


def workload_config(name: str, A: int, S: int, N: int) -> dict:
    """The workload as both arms name it (identical dicts, so the two lines
    describe the same job); the arithmetic form and launch shape are reported
    beside it under ``form``."""
    return {"workload": f"{name}: {A} virtual channels x {S} ADC samples x {N} voxels per GPU",
            "antennas": A, "samples": S, "voxels_per_gpu": N,
            "l2": ("GPU arm: flushed between timed steps (256 MiB write); CPU arm: the host "
                   "path has no device L2 to flush")}


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform

    return platform.processor() or "unknown"


def spec_fp32_tflops(dev, sm_mhz: float | None) -> float | None:
    """The FP32 FMA issue rate the SM count and a clock imply: SMs x 128 lanes x
    2 flops x clock (the sampled median clock under load)."""
    import torch

    if not sm_mhz:
        return None
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    return sms * 128 * 2 * sm_mhz * 1e6 / 1e12


def mf_call(wl, out_r, out_i, precision, voxel=None, N=None, tuning=None):
    from geraf_b200.ops.RFMatchedFilter import _C

    ch = wl["chirp"]
    vox = wl["voxel"] if voxel is None else voxel
    n = wl["N"] if N is None else N
    _C.MatchedFilter_forward(wl["real"], wl["imag"], wl["tx"], wl["rx"], out_r, out_i, vox, wl["A"],
                             wl["S"], ch.adc_sample_rate, ch.As_sci, n, precision=precision, tuning=tuning)


def autotune_mf_forward(wl, precision, dev, antenna_fraction=8):
    """Runs the autotuner for the headline call (untimed).  Launch shapes are timed
    on every voxel and a leading 1/8 of the antennas, so the grid, the waves per
    SM and the antenna split match the full call while each candidate takes an
    eighth of its time; the winner is recorded under the full problem's key."""
    import torch

    from geraf_b200 import _lib, autotune

    mode = _lib.MODE_MIXED if precision == "mixed" else _lib.MODE_PLAIN
    sub = antenna_subset(wl, max(1, wl["A"] // antenna_fraction))
    yr = torch.empty(wl["N"], device=dev)
    yi = torch.empty(wl["N"], device=dev)
    cands = [c for c in autotune.mf_forward_candidates(mode)
             if c["threads"] >= 128 and c["stage_rows"] in ((4, 8) if precision == "mixed" else (8, 16))]
    best, results = autotune.tune("mf_forward", (wl["A"], wl["S"], wl["N"]), mode,
                                  lambda t: mf_call(sub, yr, yi, precision, tuning=t), cands, iters=1)
    return best, len(results)


def launches_per_mf_call(wl, precision) -> int:
    from geraf_b200 import _lib

    mode = _lib.MODE_MIXED if precision == "mixed" else _lib.MODE_PLAIN
    ws = _lib.workspace_bytes("geraf_mf_forward_workspace_bytes", wl["A"], wl["S"], wl["N"],
                              _lib.DTYPE_F32, mode, None)
    return 2 if ws > 0 else 1


def read_profile_traffic(workload: str):
    """DRAM bytes per launch of the MF forward from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"mf_forward_mixed_{workload.replace('-', '_')}.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.strip().startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ---------------------------------------------------------------------------
def run_ours(args):
    import numpy as np
    import torch

    world, rank, local = dist_setup()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    from geraf_b200 import _lib

    _lib.load()
    wl = make_mf_workload(args.workload, rank, world, dev, args.seed)
    A, S, N = wl["A"], wl["S"], wl["N"]
    triples = float(A) * S * N
    out_r = torch.empty(N, device=dev)
    out_i = torch.empty(N, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, device=dev)
    stream = torch.cuda.current_stream(dev)

    tuned, n_cands = (autotune_mf_forward(wl, args.precision, dev) if args.precision == "mixed" and
                      not args.no_tune else ({}, 0))
    # warm-up (also resolves launch shapes, module loading and the status word)
    for _ in range(max(args.warmup, 1)):
        mf_call(wl, out_r, out_i, args.precision)
    torch.cuda.synchronize(dev)

    clocks = ClockSampler(local)
    kernel_ms = []
    barrier(world)
    torch.cuda.synchronize(dev)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        flush.fill_(1.0)  # L2 flush between steps (256 MiB write)
        ks, ke = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ks.record(stream)
        mf_call(wl, out_r, out_i, args.precision)
        ke.record(stream)
        kernel_ms.append((ks, ke))
    t1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(world)
    clock_info = clocks.stop()
    total_ms = max_over_ranks(t0.elapsed_time(t1), world)
    kms = float(np.mean([a.elapsed_time(b) for a, b in kernel_ms]))
    value = world * triples / (total_ms * 1e-3 / args.steps) / 1e9

    # end to end through the public API, host buffers in, host result out
    from geraf_b200.ops.RFMatchedFilter import matched_filter_cuda

    ch = wl["chirp"]
    h_re = wl["real"].cpu().pin_memory()
    h_im = wl["imag"].cpu().pin_memory()
    h_tx = wl["tx"].cpu().pin_memory()
    h_rx = wl["rx"].cpu().pin_memory()
    h_vox = wl["voxel"].t().contiguous().cpu().pin_memory()  # the API takes [N, 3]
    h_out_r = torch.empty(N, pin_memory=True)
    h_out_i = torch.empty(N, pin_memory=True)
    h2d = sum(t.numel() * t.element_size() for t in (h_re, h_im, h_tx, h_rx, h_vox))
    d2h = 2 * N * 4

    def e2e_step():
        yr, yi = matched_filter_cuda(h_re.to(dev, non_blocking=True), h_im.to(dev, non_blocking=True),
                                     h_tx.to(dev, non_blocking=True), h_rx.to(dev, non_blocking=True),
                                     h_vox.to(dev, non_blocking=True), A, S, ch.adc_sample_rate,
                                     ch.As_sci, N, precision=args.precision)
        h_out_r.copy_(yr, non_blocking=True)
        h_out_i.copy_(yi, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize(dev)
    e2e_steps = max(1, min(args.steps, 3))
    barrier(world)
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(world)
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world) / e2e_steps
    e2e_value = world * triples / (e2e_ms * 1e-3) / 1e9

    peak = fp32_peak_tflops(dev)
    ceiling = loop_ceiling_tflops(dev) if args.precision == "mixed" else None
    achieved = FLOPS_PER_TRIPLE * triples / (kms * 1e-3) / 1e12
    traffic = read_profile_traffic(args.workload)
    launches = launches_per_mf_call(wl, args.precision) * args.steps

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded point-scatterer scene; reference RF data not released)",
        "config": workload_config(args.workload, A, S, N),
        "form": {
            "precision": args.precision,
            "phase_reduction": "f64" if args.precision == "mixed" else "f32 (reference order)",
            "launch_shape": tuned or "library default",
            "autotuned_candidates": n_cands,
        },
        "parallelism": f"voxel slabs x{world}, no collective",
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps": e2e_steps},
        "roofline": {"bound": "fp32", "achieved": round(achieved, 3), "peak": round(peak, 3),
                     "unit": "TFLOP/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                     "flops_per_launch": FLOPS_PER_TRIPLE * triples,
                     "peak_source": "measured FP32 FMA rate (geraf_rf_fma_probe, packed FMA chains) in this process",
                     "kernel_ms": round(kms, 3)},
        "gpu_launches": launches,
        "clocks": clock_info,
    }
    spec = spec_fp32_tflops(dev, (clock_info or {}).get("sm_mhz"))
    if spec is not None:
        line["roofline"]["spec_fp32_at_clock"] = {
            "value": round(spec, 3), "unit": "TFLOP/s", "frac": round(achieved / spec, 4),
            "source": "SMs x 128 FP32 lanes x 2 flops x the median SM clock sampled in the timed region"}
    if ceiling is not None:
        # The sample loop alone, without the per-(voxel, antenna) set-up: the ceiling of
        # the kernel's instruction form, below the FMA-rate peak (operand fetch).
        line["roofline"]["loop_ceiling"] = {
            "value": round(ceiling, 3), "unit": "TFLOP/s", "frac_of_peak": round(ceiling / peak, 4),
            "kernel_frac_of_ceiling": round(achieved / ceiling, 4),
            "source": "geraf_rf_goertzel_probe (the forward's second-order recurrence loop alone, "
                      "4 blocks per SM) in this process"}

    # The extras are single-GPU measurements: under torchrun (N > 1) they would only hold
    # every GPU while rank 0 repeats them, so they run at N = 1 alone.
    wanted = set() if args.no_extras or world > 1 else {x.strip() for x in args.extras.split(",") if x.strip()}
    if rank == 0 and wanted:
        art = {"fp32_peak": peak}  # and the outputs the extras keep for the FP64 comparison
        line.update(extras(args, wl, dev, out_r, out_i, wanted, art))
        if "cpu" in wanted:
            line["cpu_baseline"], line["rel_err_vs_fp64"] = cpu_leg(args, wl, out_r, out_i, dev, art)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def extras(args, wl, dev, out_r, out_i, wanted, art) -> dict:
    """Secondary measurements: PLAIN form, MF adjoint, NUFFT form, tracer
    fwd+adjoint, ragged and stage-1 steps.  ``art`` collects outputs for the
    FP64 comparison of the CPU leg."""
    res = {}
    if "plain" in wanted:
        res.update(_plain_extra(wl, dev))
    if "adjoint" in wanted:
        res.update(_adjoint_extra(args, wl, dev, art))
    if "nufft" in wanted:
        res.update(_nufft_extra(wl, dev, out_r, out_i, art))
    if "tracer" in wanted:
        res.update(_tracer_extra(args, dev, art))
    if "ragged" in wanted:
        res.update(_ragged_extra(args, dev))
    if "stage1" in wanted:
        res.update(_stage1_extra(args, dev))
    return res


def ragged_workload(dev, seed=0, num_antennas=256, S=256):
    """256 antennas of the 64x64x12 array, each with U[512, 8192] rays x U[64, 192]
    samples (its own points) on the cube-shell + torus scene region, S = 256."""
    import numpy as np
    import torch

    from benchkit import scenes

    rng = np.random.default_rng(seed)
    tx, rx = scenes.virtual_array(64)
    pick = np.sort(rng.choice(tx.shape[0], num_antennas, replace=False))
    rays = rng.integers(512, 8193, num_antennas)
    spr = rng.integers(64, 193, num_antennas)
    counts = rays * spr
    P = int(counts.sum())
    g = torch.Generator(device=dev).manual_seed(seed)
    ant = torch.repeat_interleave(torch.arange(num_antennas, device=dev), torch.tensor(counts, device=dev))
    txd = torch.tensor(tx[pick], device=dev)
    rxd = torch.tensor(rx[pick], device=dev)
    aim = torch.tensor([0.0, 0.0, 0.4], device=dev) + (torch.rand((P, 3), device=dev, generator=g) - 0.5) * 0.3
    org = rxd[ant]
    pts = org + (aim - org) * (0.85 + 0.3 * torch.rand((P, 1), device=dev, generator=g))
    nrm = torch.randn((P, 3), device=dev, generator=g)
    nrm = nrm - 1.5 * (pts - org) / (pts - org).norm(dim=1, keepdim=True)  # mostly facing the radar
    nrm = nrm / nrm.norm(dim=1, keepdim=True)
    sig = torch.rand(P, device=dev, generator=g)
    offs = torch.tensor(np.concatenate([[0], np.cumsum(counts)]).astype(np.int64), device=dev)
    return dict(normals=nrm.contiguous(), sigmas=sig, points=pts.contiguous(), point_offsets=offs, tx=txd,
                rx=rxd, rays=int(rays.sum()), P=P, S=S)


def _ragged_extra(args, dev) -> dict:
    """Batched uneven tracer + matched filter step (forward and adjoint), graph-captured."""
    import torch

    from benchkit import scenes
    from geraf_b200 import autotune
    from geraf_b200.step import RaggedRFStep

    w = ragged_workload(dev, args.seed, num_antennas=args.ragged_antennas)
    ch = scenes.chirp(w["S"])
    cfg = ch.radar_cfg(fc_start=770.0)
    vox = torch.tensor(scenes.voxel_grid(64, size=0.32).T.copy(), device=dev)
    A, S, P = w["tx"].shape[0], w["S"], w["P"]

    def make_step():
        return RaggedRFStep(w["normals"], w["sigmas"], w["points"], w["point_offsets"], w["tx"], w["rx"], vox,
                            torch.full((vox.shape[0],), 1e-4, device=dev), cfg)

    tuned = {}
    if not args.no_tune:
        # the batched tracer's forward and adjoint launch shapes, timed on the step's own inputs
        from geraf_b200 import _lib
        from geraf_b200.ops.RFSignalTracer.ragged import signal_tracer_ragged

        nrm = w["normals"].detach().clone().requires_grad_(True)
        g = torch.Generator(device=dev).manual_seed(args.seed + 9)
        gx = (torch.randn((A, S), device=dev, generator=g), torch.randn((A, S), device=dev, generator=g))

        def fwd(t=None):
            return signal_tracer_ragged(nrm, w["sigmas"], w["points"], w["point_offsets"], w["tx"], w["rx"], S,
                                        cfg["adcSampleRate"], cfg["fc_start"], cfg["As_sci"], tuning=t)

        # the adjoint is timed together with the (already tuned) forward that produces its graph
        default_f = autotune.time_call(lambda: fwd(), iters=3, warmup=1)
        best_f, res_f = autotune.tune("tracer_ragged_forward", (A, S, P), _lib.MODE_MIXED, fwd,
                                      autotune.ragged_forward_candidates(), iters=3)

        def run_bwd(t):
            xr, xi = signal_tracer_ragged(nrm, w["sigmas"], w["points"], w["point_offsets"], w["tx"], w["rx"],
                                          S, cfg["adcSampleRate"], cfg["fc_start"], cfg["As_sci"],
                                          tuning_backward=t)
            torch.autograd.backward([xr, xi], [gx[0], gx[1]])

        default_b = autotune.time_call(lambda: run_bwd(None), iters=3, warmup=1)
        best_b, res_b = autotune.tune("tracer_ragged_backward", (A, S, P), _lib.MODE_MIXED, run_bwd,
                                      autotune.ragged_backward_candidates(), iters=3)
        tuned = {"forward": {"launch_shape": best_f, "candidates": len(res_f),
                             "tuned_speedup_vs_default": round(default_f / min(m for _, m in res_f), 4)},
                 "forward_plus_adjoint": {"launch_shape": best_b, "candidates": len(res_b),
                                          "tuned_speedup_vs_default": round(default_b / min(m for _, m in res_b),
                                                                            4)}}
    step = make_step()
    step.capture()
    ms = autotune.time_call(step.run, iters=3, warmup=1)
    return {"ragged_step": {
        "workload": (f"{A} antennas, rays U[512,8192] x samples U[64,192] per antenna "
                     f"({w['rays']} rays, {P} points), S={S}, MF onto 64^3 voxels"),
        "ms": round(ms, 3), "rays_per_s": round(w["rays"] / (ms * 1e-3), 1),
        "point_samples_per_s_G": round(float(P) * S / (ms * 1e-3) / 1e9, 2),
        "graph": True, "autotune": tuned or "not run"}}


def _stage1_extra(args, dev) -> dict:
    """End-to-end stage-1 RF training step (the reference's loss shape): its forms'
    step times, then the equal-error comparison of MIXED + graph against PLAIN
    eager (benchkit.stage1_eval: both train from the same initialisation on the
    shell + torus target; Chamfer distance to the analytic surfaces at checkpoints)."""
    from benchkit import stage1_eval
    from benchkit.stage1 import Stage1RFStep
    from geraf_b200 import autotune

    res = {}
    for name, prec, mf_prec, bank, graph, iters in (("mixed_graph", "mixed", "mixed", 1, True, 5),
                                                    ("mixed_nufft_mf_graph", "mixed", "nufft", 1, True, 5),
                                                    ("nufft_graph", "nufft", "nufft", 1, True, 5),
                                                    ("mixed_bank2_graph", "mixed", "mixed", 2, True, 5),
                                                    ("plain_eager", "plain", "plain", 1, False, 2)):
        st = Stage1RFStep(num_antennas=128, num_rays=2048, samples_per_ray=128, num_adc=256, precision=prec,
                          device=dev, seed=args.seed, mf_precision=mf_prec, bank_size=bank)
        if graph:
            st.capture()
        ms = autotune.time_call(st.run, iters=iters, warmup=1)
        res[name] = {"ms": round(ms, 2), "it_per_s": round(1e3 / ms, 2)}
    eq = stage1_eval.compare(steps=args.stage1_steps, seed=args.seed, checkpoints=8)
    for form in ("mixed_graph", "plain_eager"):
        eq[form].pop("loss_every_10", None)
    return {"stage1_step": {"workload": ("128 antennas x 2048 rays x 128 target samples (64 coarse), S=256, "
                                         "random-init SDF MLP (FP16 autocast), resample -> tracer -> MF at "
                                         "the target points, charbonier loss + eikonal, Adam; bank2: the "
                                         "reference's 2-chunk antenna bank, one chunk rendered per step, the "
                                         "bank kept on the GPU"),
                            **res, "equal_error": eq}}


def antenna_subset(wl, a_sub):
    """The workload restricted to its leading ``a_sub`` antennas (all voxels)."""
    return dict(wl, A=a_sub, real=wl["real"][:a_sub], imag=wl["imag"][:a_sub], tx=wl["tx"][:a_sub],
                rx=wl["rx"][:a_sub])


def _plain_extra(wl, dev) -> dict:
    """PLAIN form (the reference's FP32 expressions, one sincos per triple) on every
    voxel and a leading antenna subset sized to about 1.5 s, so the grid is the
    full call's; forward and adjoint (the adjoint on every antenna and sample and
    a voxel subset: its threads are the (antenna, sample) pairs)."""
    import torch

    from geraf_b200 import autotune
    from geraf_b200.ops.RFMatchedFilter import _C as mfc

    res = {}
    A, S, N = wl["A"], wl["S"], wl["N"]
    ch = wl["chirp"]
    pr = torch.empty(N, device=dev)
    pi = torch.empty(N, device=dev)
    a_cal = min(A, 16)
    ms = autotune.time_call(lambda: mf_call(antenna_subset(wl, a_cal), pr, pi, "plain"), iters=1, warmup=1)
    a_sub = int(min(A, max(a_cal, a_cal * 1500.0 / max(ms, 1e-3))))
    sub = antenna_subset(wl, a_sub)
    ms = autotune.time_call(lambda: mf_call(sub, pr, pi, "plain"), iters=1, warmup=0)
    res["plain_form"] = {"value": round(float(a_sub) * S * N / (ms * 1e-3) / 1e9, 3), "unit": UNIT,
                         "sample": f"{N} voxels x {a_sub} antennas x {S} samples", "ms": round(ms, 2)}
    g_r = torch.randn(N, device=dev)
    g_i = torch.randn(N, device=dev)
    h_r = torch.empty((A, S), device=dev)
    h_i = torch.empty((A, S), device=dev)

    def adj(n_sub):
        v = wl["voxel"][:, :n_sub].contiguous()
        return lambda: mfc.MatchedFilter_backward_realimag(g_r[:n_sub], g_i[:n_sub], wl["real"], wl["imag"],
                                                           wl["tx"], wl["rx"], h_r, h_i, v, A, S,
                                                           ch.adc_sample_rate, ch.As_sci, n_sub,
                                                           precision="plain")

    n_cal = min(N, 64)
    ms = autotune.time_call(adj(n_cal), iters=1, warmup=1)
    n_sub = int(min(N, max(n_cal, n_cal * 1500.0 / max(ms, 1e-3))))
    ms = autotune.time_call(adj(n_sub), iters=1, warmup=0)
    res["plain_adjoint"] = {"value": round(float(A) * S * n_sub / (ms * 1e-3) / 1e9, 3), "unit": UNIT,
                            "sample": f"{A} antennas x {S} samples x {n_sub} voxels", "ms": round(ms, 2)}
    return res


def _adjoint_extra(args, wl, dev, art) -> dict:
    """MIXED MF adjoint on the full workload, with its launch shape autotuned
    first (every antenna x sample row block, a leading eighth of the voxels, so
    the grid is the full call's)."""
    import torch

    from geraf_b200 import _lib, autotune
    from geraf_b200.ops.RFMatchedFilter import _C as mfc

    res = {}
    A, S, N = wl["A"], wl["S"], wl["N"]
    ch = wl["chirp"]
    gen = torch.Generator(device=dev).manual_seed(args.seed + 5)
    g_r = torch.randn(N, device=dev, generator=gen)
    g_i = torch.randn(N, device=dev, generator=gen)
    h_r = torch.empty((A, S), device=dev)
    h_i = torch.empty((A, S), device=dev)

    def adj(n=N, tuning=None):
        mfc.MatchedFilter_backward_realimag(g_r[:n], g_i[:n], wl["real"], wl["imag"], wl["tx"], wl["rx"], h_r,
                                            h_i, wl["voxel"][:, :n].contiguous() if n < N else wl["voxel"],
                                            A, S, ch.adc_sample_rate, ch.As_sci, n, precision="mixed",
                                            tuning=tuning)

    shape, n_cands = "library default", 0
    if not args.no_tune:
        n_sub = max(1, N // 8)
        default_ms = autotune.time_call(lambda: adj(n_sub), iters=1, warmup=1)
        best, results = autotune.tune("mf_backward", (A, S, N), _lib.MODE_MIXED,
                                      lambda t: adj(n_sub, t), autotune.sample_major_candidates(), iters=1)
        shape, n_cands = best, len(results)
        gain = default_ms / min(ms for _, ms in results)
    ms = autotune.time_call(adj, iters=1, warmup=1)
    res["mf_adjoint"] = {"value": round(float(A) * S * N / (ms * 1e-3) / 1e9, 3), "unit": UNIT,
                         "ms": round(ms, 2), "precision": "mixed", "launch_shape": shape,
                         "autotuned_candidates": n_cands}
    if n_cands:
        res["mf_adjoint"]["tuned_speedup_vs_default"] = round(gain, 4)
    art["mf_adjoint"] = (torch.complex(g_r, g_i).cpu().numpy(), torch.complex(h_r, h_i).cpu().numpy())
    return res


def _nufft_extra(wl, dev, out_r, out_i, art) -> dict:
    """The matched filter's fast approximate form (oversampled range FFT + 8-point
    ES interpolation) on the full workload: forward and adjoint times, in the
    headline's unit (the same voxel x antenna x sample sums, evaluated in O(W)
    per voxel-antenna pair), and their relative L2 against the MIXED form over
    every output element (the MIXED form is itself ~2e-7 from FP64)."""
    import torch

    from geraf_b200 import autotune
    from geraf_b200.ops.RFMatchedFilter import _C as mfc

    A, S, N = wl["A"], wl["S"], wl["N"]
    ch = wl["chirp"]
    yr = torch.empty(N, device=dev)
    yi = torch.empty(N, device=dev)
    ms = autotune.time_call(lambda: mf_call(wl, yr, yi, "nufft"), iters=2, warmup=1)
    ref = torch.complex(out_r.double(), out_i.double())
    err = float((torch.complex(yr.double(), yi.double()) - ref).norm() / ref.norm())
    res = {"mf_forward_nufft": {"value": round(float(A) * S * N / (ms * 1e-3) / 1e9, 3), "unit": UNIT,
                                "ms": round(ms, 2), "taps": 8, "rel_l2_vs_mixed": err}}
    g_r = torch.randn(N, device=dev)
    g_i = torch.randn(N, device=dev)
    h_r = torch.empty((A, S), device=dev)
    h_i = torch.empty((A, S), device=dev)
    m_r = torch.empty((A, S), device=dev)
    m_i = torch.empty((A, S), device=dev)

    def adj(prec, hr, hi):
        mfc.MatchedFilter_backward_realimag(g_r, g_i, wl["real"], wl["imag"], wl["tx"], wl["rx"], hr, hi,
                                            wl["voxel"], A, S, ch.adc_sample_rate, ch.As_sci, N, precision=prec)

    art["mf_forward_nufft"] = torch.complex(yr, yi).cpu().numpy()
    ms_b = autotune.time_call(lambda: adj("nufft", h_r, h_i), iters=2, warmup=1)
    art["mf_adjoint_nufft"] = (torch.complex(g_r, g_i).cpu().numpy(), torch.complex(h_r, h_i).cpu().numpy())
    adj("mixed", m_r, m_i)
    ref_b = torch.complex(m_r.double(), m_i.double())
    err_b = float((torch.complex(h_r.double(), h_i.double()) - ref_b).norm() / ref_b.norm())
    res["mf_adjoint_nufft"] = {"value": round(float(A) * S * N / (ms_b * 1e-3) / 1e9, 3), "unit": UNIT,
                               "ms": round(ms_b, 2), "taps": 8, "rel_l2_vs_mixed": err_b}
    return res


def tracer_live_pairs(tw, chunk: int = 8) -> int:
    """(point, antenna) pairs of the tracer workload that survive the specular
    culling (the reference's FP32 geometry, SignalTracer_cuda_kernel.cu:172-197,
    restated in torch on the device): the pairs whose samples the kernels sum."""
    import torch

    def nrm(v):
        return v / (v.norm(dim=-1, keepdim=True) + 1e-7)

    pts, n, inb = tw["points"], tw["normals"], tw["inbounds"]
    live = 0
    for a0 in range(0, tw["tx"].shape[0], chunk):
        tx = tw["tx"][a0:a0 + chunk, None, :]
        rx = tw["rx"][a0:a0 + chunk, None, :]
        inc = nrm(pts[None] - tx)
        idn = (inc * n[None]).sum(-1)
        refl = nrm(inc - 2.0 * idn[..., None] * n[None])
        align = (nrm(rx - pts[None]) * refl).sum(-1)
        live += int(((align >= 1e-6) & (idn <= 0.0) & inb[None]).sum())
    return live


def tracer_listed_points(tw) -> int:
    """Points that the MIXED tracer's per-point pre-cull keeps (the in-bounds
    points it cannot cull for every antenna; csrc/tracer_precull.cu), restated in
    torch FP64 on the device."""
    import torch

    d = torch.float64
    tx, rx = tw["tx"].to(d), tw["rx"].to(d)
    ct, cr = tx.mean(0), rx.mean(0)
    rt = (tx - ct).norm(dim=1).max()
    rr = (rx - cr).norm(dim=1).max()
    rt = rt + 1e-12 * (rt + ct.abs().sum())
    rr = rr + 1e-12 * (rr + cr.abs().sum())
    n, p = tw["normals"].to(d), tw["points"].to(d)
    ic, oc = p - ct, cr - p
    nn = (n * n).sum(1)
    nrm, m = nn.sqrt(), 1.0 + 2.0 * nn
    icn = (ic * n).sum(1)
    ni, no = ic.norm(dim=1), oc.norm(dim=1)
    back = icn - rt * nrm > 1e-4 * (ni + rt) * nrm
    hi = ic - 2.0 * icn[:, None] * n
    ho = oc - 2.0 * (oc * n).sum(1)[:, None] * n
    bound = (oc * hi).sum(1) + rr * hi.norm(dim=1) + rt * ho.norm(dim=1) + m * rr * rt
    away = bound < -1e-4 * (no + rr) * (ni + rt) * m
    return int((tw["inbounds"] & ~(back | away)).sum())


def _tracer_extra(args, dev, art) -> dict:
    """Tracer forward + adjoint (with position gradients) on the 64-antenna x
    4096-ray x 128-sample workload of a random-init SDF network: MIXED (launch
    shapes autotuned first), NUFFT and PLAIN, in rays/s; the roofline of the
    MIXED pair over all (point, antenna, sample) triples and over the triples of
    live (not culled) pairs."""
    import torch

    from benchkit.sdf import tracer_workload
    from geraf_b200 import _lib, autotune
    from geraf_b200.ops.RFSignalTracer import _C as trc

    res = {}
    tw = tracer_workload(device=dev, seed=args.seed)
    At, P, St = tw["A"], tw["P"], tw["chirp"].num_samples
    cfg = tw["radar_cfg"]
    xr = torch.empty((At, St), device=dev)
    xi = torch.empty((At, St), device=dev)
    gen = torch.Generator(device=dev).manual_seed(args.seed + 7)
    gxr = torch.randn((At, St), device=dev, generator=gen)
    gxi = torch.randn((At, St), device=dev, generator=gen)
    gn = torch.empty((P, 3), device=dev)
    gs = torch.empty((At, P), device=dev)
    gp = torch.empty((P, 3), device=dev)

    def fwd(prec, tuning=None):
        trc.SignalTracer_forward(tw["normals"], tw["sigmas"], tw["points"], tw["tx"], tw["rx"],
                                 tw["inbounds"], xr, xi, St, cfg["adcSampleRate"], cfg["fc_start"],
                                 cfg["As_sci"], At, P, precision=prec, tuning=tuning)

    def bwd(prec, tuning=None):
        trc.SignalTracer_backward_normal_sigma(gxr, gxi, tw["normals"], tw["sigmas"], tw["points"],
                                               tw["tx"], tw["rx"], tw["inbounds"], gn, gs, St,
                                               cfg["adcSampleRate"], cfg["fc_start"], cfg["As_sci"],
                                               At, P, grad_points=gp if prec != "plain" else None,
                                               precision=prec, tuning=tuning)

    tuned = {}
    if not args.no_tune:
        for op, run, cands in (("tracer_forward", fwd, autotune.sample_major_candidates()),
                               ("tracer_backward", bwd, autotune.tracer_backward_candidates())):
            default_ms = autotune.time_call(lambda run=run: run("mixed"), iters=5, warmup=2)
            best, results = autotune.tune(op, (At, St, P), _lib.MODE_MIXED,
                                          lambda t, run=run: run("mixed", t), cands, iters=5)
            tuned[op] = {"launch_shape": best, "candidates": len(results),
                         "tuned_speedup_vs_default": round(default_ms / min(ms for _, ms in results), 4)}
    tr = {}
    outs = {}
    for prec in ("mixed", "nufft", "plain"):
        def step(prec=prec):
            fwd(prec)
            bwd(prec)
        ms = autotune.time_call(step, iters=5 if prec != "plain" else 1, warmup=1)
        tr[prec] = {"rays_per_s": round(At * tw["rays"] / (ms * 1e-3), 1), "ms": round(ms, 3),
                    "gpts_per_s": round(float(At) * P * St / (ms * 1e-3) / 1e9, 2)}
        outs[prec] = [torch.complex(xr, xi).to(torch.complex128)] + [t.double().clone() for t in (gs, gn, gp)]

    def rel(a, b):
        return float((a - b).norm() / b.norm())

    tr["nufft"]["rel_l2_vs_mixed"] = {k: rel(outs["nufft"][i], outs["mixed"][i])
                                      for i, k in enumerate(("signal", "grad_sigmas", "grad_normals",
                                                             "grad_points"))}
    # roofline of the MIXED forward + adjoint: 12 flops per (point, antenna, sample)
    live = tracer_live_pairs(tw)
    peak = art.get("fp32_peak")
    flops_all = 12.0 * At * P * St
    flops_live = 12.0 * live * St
    ms_m = tr["mixed"]["ms"]
    roof = {"flops_per_triple": 12, "live_pair_fraction": round(live / (At * P), 4),
            "listed_point_fraction": round(tracer_listed_points(tw) / P, 4),
            "achieved_all_tflops": round(flops_all / (ms_m * 1e-3) / 1e12, 3),
            "achieved_live_tflops": round(flops_live / (ms_m * 1e-3) / 1e12, 3)}
    if peak:
        roof["peak"] = round(peak, 3)
        roof["frac_all"] = round(flops_all / (ms_m * 1e-3) / 1e12 / peak, 4)
        roof["frac_live"] = round(flops_live / (ms_m * 1e-3) / 1e12 / peak, 4)
        roof["note"] = ("frac_live is the roofline: culled pairs carry no samples to sum; frac_all "
                        "counts every triple as the reference's kernels visit them.  The kernels form "
                        "the geometry of every pair of the points the per-point pre-cull keeps "
                        "(listed_point_fraction) and sum the samples of live pairs only")
    res["tracer"] = {"workload": f"{At} antennas x {tw['rays']} rays x {P // tw['rays']} samples, S={St}",
                     "unit": "rays/s (ray = ray x antenna pair)", "mixed_with_point_grads": tr["mixed"],
                     "nufft_with_point_grads": tr["nufft"], "plain": tr["plain"], "roofline": roof,
                     "autotune": tuned or "not run"}
    # the MIXED outputs, for the FP64 comparison in the CPU leg
    m = outs["mixed"]
    art["tracer"] = dict(
        w=dict(normals=tw["normals"].cpu().numpy(), sigmas=tw["sigmas"].cpu().numpy(),
               points=tw["points"].cpu().numpy(), tx=tw["tx"].cpu().numpy(), rx=tw["rx"].cpu().numpy(),
               inbounds=tw["inbounds"].cpu().numpy(), S=St, fs=cfg["adcSampleRate"], f0=cfg["fc_start"],
               As=cfg["As_sci"], rays=tw["rays"], samples_per_ray=P // tw["rays"]),
        g=torch.complex(gxr, gxi).cpu().numpy(), x=m[0].cpu().numpy(),
        grads={"sigmas": m[1].cpu().numpy(), "normals": m[2].cpu().numpy(), "points": m[3].cpu().numpy()})
    return res


def cpu_leg(args, wl, out_r, out_i, dev, art):
    """CPU baseline (reference-order FP32 oracle port, all host threads) on a
    bounded voxel sample, and the FP64-oracle errors of every output the run
    produced, on the fixed subsets of oracle/workload_parity.py."""
    import numpy as np
    import torch

    from oracle import rf_oracle as orc
    from oracle import workload_parity as wp

    ch = wl["chirp"]
    A, S, N = wl["A"], wl["S"], wl["N"]
    re = wl["real"].cpu().numpy()
    im = wl["imag"].cpu().numpy()
    tx = wl["tx"].cpu().numpy()
    rx = wl["rx"].cpu().numpy()
    vox = wl["voxel"].cpu().numpy()
    # calibrate a sample that takes ~10 s (the first call also starts the thread pool)
    rng = np.random.default_rng(7)
    n0 = orc.num_threads()
    idx = rng.choice(N, n0, replace=False)
    for _ in range(2):
        t = time.perf_counter()
        orc.mf_forward(re, im, tx, rx, vox[:, idx], ch.adc_sample_rate, ch.As_sci, "f32")
        dt0 = time.perf_counter() - t
    n = int(max(n0, min(4096, n0 * 10.0 / max(dt0, 1e-3))))
    for _ in range(2):  # small samples are dominated by start-up: resize once from a real run
        n = max(orc.num_threads(), (n // orc.num_threads()) * orc.num_threads())
        idx = rng.choice(N, n, replace=False)
        t = time.perf_counter()
        orc.mf_forward(re, im, tx, rx, vox[:, idx], ch.adc_sample_rate, ch.As_sci, "f32")
        dt = time.perf_counter() - t
        if dt >= 8.0 or n >= 16384:
            break
        n = int(min(16384, n * 12.0 / max(dt, 1e-3)))
    cpu = {"value": round(float(A) * S * n / dt / 1e9, 4), "unit": UNIT, "cores": orc.num_threads(),
           "kind": "port", "cpu_model": cpu_model(),
           "sample": (f"{n} random voxels x {A} antennas x {S} samples ({dt:.1f} s), FP32 reference "
                      f"order; extrapolated to the whole volume (the cost is linear in voxels)")}

    # ---- FP64 errors of every output (complex relative L2 on fixed subsets) ----
    t_err = time.perf_counter()
    w = dict(re=re, im=im, tx=tx, rx=rx, vox=vox, fs=ch.adc_sample_rate, As=ch.As_sci, S=S)
    full = args.workload == "mf-full"
    vi = wp.MF49152_VOXELS if full else wp.MF3072_VOXELS
    rows = wp.MF49152_ROWS if full else wp.MF3072_ROWS
    ref_f = wp.mf_forward_ref(w, vi)
    ours = out_r.cpu().numpy() + 1j * out_i.cpu().numpy()
    pr = torch.empty(len(vi), device=dev)
    pi = torch.empty(len(vi), device=dev)
    mf_call(wl, pr, pi, "plain", voxel=wl["voxel"][:, torch.tensor(vi, device=dev)].contiguous(), N=len(vi))
    errs = {"mf_forward": {"mixed": wp.rel(ours[vi], ref_f),
                           "plain": wp.rel(pr.cpu().numpy() + 1j * pi.cpu().numpy(), ref_f)}}
    if "mf_forward_nufft" in art:
        errs["mf_forward"]["nufft"] = wp.rel(art["mf_forward_nufft"][vi], ref_f)
    if "mf_adjoint" in art:
        g, h = art["mf_adjoint"]
        ref_b = wp.mf_adjoint_ref(g, w, rows)
        errs["mf_adjoint"] = {"mixed": wp.rel(h[rows], ref_b)}
        if "mf_adjoint_nufft" in art and np.array_equal(art["mf_adjoint_nufft"][0], g):
            errs["mf_adjoint"]["nufft"] = wp.rel(art["mf_adjoint_nufft"][1][rows], ref_b)
        elif "mf_adjoint_nufft" in art:
            g2, h2 = art["mf_adjoint_nufft"]
            errs["mf_adjoint"]["nufft"] = wp.rel(h2[rows], wp.mf_adjoint_ref(g2, w, rows))
    if "tracer" in art:
        tr = art["tracer"]
        tw = tr["w"]
        rays = wp.fd_rays(tw)
        pts = wp.ray_points(tw, rays)
        adj = wp.tracer_adjoint_errors(tr["grads"], tr["g"], tw, pts)
        errs["tracer_mixed"] = {"signal": wp.tracer_forward_error(tr["x"], tw, wp.TRACER_ROWS),
                                "grad_sigmas": adj["sigma"], "grad_normals": adj["normal"],
                                "grad_points": adj["position"]}
        fd = wp.tracer_fd_errors(tr["grads"], tr["g"], tw, rays)
        errs["tracer_mixed_vs_central_differences"] = {
            "grad_sigmas": fd["sigma"], "grad_normals": fd["normal"], "grad_points": fd["position"],
            "how": "largest per-ray |FD - analytic| / sum |analytic| over 256 random rays, FP64 "
                   "central differences of the pure-torch tracer"}
    subsets = (f"MF forward: {len(vi)} voxels ({'16^3 lattice of the 32^3 subset' if full else 'every 27th'}); "
               f"MF adjoint: {len(rows)} antenna rows over all voxels; tracer: 16 antenna rows (signal) "
               f"and the 32768 points of 256 random rays (gradients)")
    errs["how"] = "complex relative L2 vs the FP64 oracle; " + subsets
    errs["oracle_s"] = round(time.perf_counter() - t_err, 1)
    return cpu, errs


# ---------------------------------------------------------------------------
def reference_cuda_leg(args, w) -> dict:
    """The reference's own CUDA kernels -- the unmodified extensions, built for
    sm_100a into oracle/_ref by oracle/build_ref.py -- timed with CUDA events on
    this GPU, through their own ``_C`` entry points:

    - MF forward (one thread per voxel looping over antennas x samples,
      MatchedFilter_cuda_kernel.cu:65-115): every voxel of the workload and a
      leading subset of its antennas, so the grid is the full call's and the cost
      per voxel-antenna-sample is unchanged;
    - MF adjoint (one thread per antenna x sample looping over voxels, :171-220):
      every antenna and sample and a voxel subset, for the same reason;
    - tracer forward + adjoint onto normals and sigmas (SignalTracer_cuda_kernel.cu:
      351-587) on the 64-antenna x 4096-ray x 128-sample tracer workload, as is.

    Inputs are seeded Gaussian IF and gradients (the cost does not depend on the
    values) and the random-init SDF tracer scene."""
    import torch

    from benchkit.sdf import tracer_workload
    from oracle import build_ref

    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    try:
        mf = build_ref.load("RFMatchedFilter")
        st = build_ref.load("RFSignalTracer")
    except Exception as exc:  # noqa: BLE001 - reported, not fatal to the CPU arm
        return {"unavailable": f"reference extensions not loadable: {exc}"}
    dev = torch.device("cuda", torch.cuda.current_device())
    ch = w["chirp"]
    A, S, N = w["tx"].shape[0], ch.num_samples, w["voxel"].shape[1]
    gen = torch.Generator(device=dev).manual_seed(args.seed)
    re = torch.randn((A, S), device=dev, generator=gen)
    im = torch.randn((A, S), device=dev, generator=gen)
    tx = torch.tensor(w["tx"], device=dev, dtype=torch.float32)
    rx = torch.tensor(w["rx"], device=dev, dtype=torch.float32)
    vox = torch.tensor(w["voxel"], device=dev, dtype=torch.float32).contiguous()

    def timed(fn, iters=1):
        fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(iters):
            fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / iters

    out = {"build": "oracle/build_ref.py: the reference's _C sources, unmodified, -gencode sm_100a",
           "unit": UNIT}
    # MF forward: all N voxels, a_sub antennas (sized from a short calibration to ~2 s)
    yr = torch.empty(N, device=dev)
    yi = torch.empty(N, device=dev)

    def fwd(a_sub):
        return lambda: mf.MatchedFilter_forward(re[:a_sub], im[:a_sub], tx[:a_sub], rx[:a_sub], yr, yi, vox,
                                                a_sub, S, ch.adc_sample_rate, ch.As_sci, N)

    a_cal = min(A, 8)
    ms = timed(fwd(a_cal))
    a_sub = int(min(A, max(a_cal, a_cal * 2000.0 / max(ms, 1e-3))))
    ms = timed(fwd(a_sub))
    out["mf_forward"] = {"value": round(float(a_sub) * S * N / (ms * 1e-3) / 1e9, 3), "ms": round(ms, 2),
                         "sample": f"{N} voxels x {a_sub} antennas x {S} samples"}
    # MF adjoint: all A x S threads, n_sub voxels
    gr = torch.randn(N, device=dev, generator=gen)
    gi = torch.randn(N, device=dev, generator=gen)
    hr = torch.empty((A, S), device=dev)
    hi = torch.empty((A, S), device=dev)

    def adj(n_sub):
        v = vox[:, :n_sub].contiguous()
        return lambda: mf.MatchedFilter_backward_realimag(gr[:n_sub], gi[:n_sub], re, im, tx, rx, hr, hi, v,
                                                          A, S, ch.adc_sample_rate, ch.As_sci, n_sub)

    n_cal = min(N, 64)
    ms = timed(adj(n_cal))
    n_sub = int(min(N, max(n_cal, n_cal * 2000.0 / max(ms, 1e-3))))
    ms = timed(adj(n_sub))
    out["mf_adjoint"] = {"value": round(float(A) * S * n_sub / (ms * 1e-3) / 1e9, 3), "ms": round(ms, 2),
                         "sample": f"{A} antennas x {S} samples x {n_sub} voxels"}
    # tracer forward + adjoint (normals, sigmas) on the tracer workload
    tw = tracer_workload(device=dev, seed=args.seed)
    At, P, St = tw["A"], tw["P"], tw["chirp"].num_samples
    cfg = tw["radar_cfg"]
    xr = torch.empty((At, St), device=dev)
    xi = torch.empty((At, St), device=dev)
    gxr = torch.randn((At, St), device=dev, generator=gen)
    gxi = torch.randn((At, St), device=dev, generator=gen)
    gn = torch.empty((P, 3), device=dev)
    gs = torch.empty((At, P), device=dev)

    def tr_step():
        st.SignalTracer_forward(tw["normals"], tw["sigmas"], tw["points"], tw["tx"], tw["rx"], tw["inbounds"],
                                xr, xi, St, cfg["adcSampleRate"], cfg["fc_start"], cfg["As_sci"], At, P)
        st.SignalTracer_backward_normal_sigma(gxr, gxi, tw["normals"], tw["sigmas"], tw["points"], tw["tx"],
                                              tw["rx"], tw["inbounds"], gn, gs, St, cfg["adcSampleRate"],
                                              cfg["fc_start"], cfg["As_sci"], At, P)

    ms = timed(tr_step)
    out["tracer"] = {"workload": f"{At} antennas x {tw['rays']} rays x {P // tw['rays']} samples, S={St}",
                     "rays_per_s": round(At * tw["rays"] / (ms * 1e-3), 1), "ms": round(ms, 3),
                     "unit": "rays/s (ray = ray x antenna pair), forward + adjoint onto normals and sigmas"}
    return out


def run_reference(args):
    """Times the reference's arithmetic on the host cores (the FP32
    reference-order oracle port; the reference ships no CPU implementation)."""
    import numpy as np

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from benchkit import scenes
    from oracle import rf_oracle as orc

    w = scenes.mf_full_workload(args.seed) if args.workload == "mf-full" else scenes.mf_small_workload(args.seed)
    ch = w["chirp"]
    A, S = w["tx"].shape[0], ch.num_samples
    N = w["voxel"].shape[1]
    rng = np.random.default_rng(args.seed)
    # the cost is independent of the sample values: seeded Gaussian IF of the workload's shape
    re = rng.standard_normal((A, S)).astype(np.float32)
    im = rng.standard_normal((A, S)).astype(np.float32)
    idx = rng.choice(N, 8, replace=False)
    t = time.perf_counter()
    orc.mf_forward(re, im, w["tx"], w["rx"], w["voxel"][:, idx], ch.adc_sample_rate, ch.As_sci, "f32")
    dt0 = time.perf_counter() - t
    threads = orc.num_threads()
    n = int(max(threads, min(2048, 8 * 8.0 / max(dt0, 1e-3))))
    n = max(threads, (n // threads) * threads)
    times = []
    for step in range(args.warmup + args.steps):
        idx = rng.choice(N, n, replace=False)
        t = time.perf_counter()
        orc.mf_forward(re, im, w["tx"], w["rx"], w["voxel"][:, idx], ch.adc_sample_rate, ch.As_sci, "f32")
        if step >= args.warmup:
            times.append(time.perf_counter() - t)
    sec = float(np.mean(times))
    value = float(A) * S * n / sec / 1e9
    sample = (f"{n} random voxels of {N} x {A} antennas x {S} samples per step, "
              f"FP32 reference-order port, {threads} threads; extrapolated to the whole volume "
              f"(the cost is linear in voxels)")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(sec * 1e3, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": workload_config(args.workload, A, S, N),
        "form": {"precision": "plain", "phase_reduction": "f32 (reference order)", "host": "CPU"},
        "parallelism": "rank 0 host threads",
        "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": threads, "kind": "port",
                         "cpu_model": cpu_model(), "sample": sample},
        "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_extras:
        line["reference_cuda"] = reference_cuda_leg(args, w)
    print(json.dumps(line), flush=True)


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
