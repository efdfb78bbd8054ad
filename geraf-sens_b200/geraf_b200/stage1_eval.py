"""Equal-error comparison of RF training-step forms on the shell + torus scene.

The stage-1 RF step (:class:`geraf_b200.step.Stage1RFStep`) is trained for the
same number of steps, from the same initialisation, data and ray samples, in
two forms:

* ``mixed`` arithmetic with the whole step captured in one CUDA graph;
* ``plain`` arithmetic (the reference's FP32 expressions) run eagerly.

The target is the matched-filter magnitude of the cube-shell + torus scene
(point scatterers, 20 dB SNR) seen by the step's own antennas, on the step's
voxel grid.  After training, the SDF's zero level set is extracted on a grid
(sign changes between neighbouring grid points, linearly interpolated) and
compared with points sampled on the analytic surfaces by the symmetric Chamfer
distance; the network's mean |SDF| at those surface points is reported beside it
(it is defined even when the level set leaves the extraction box).  Equal
errors at equal step counts make the two forms' iterations/s directly
comparable.

    python -m geraf_b200.stage1_eval --steps 100
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np
import torch


def analytic_surface_points(n: int, rng: np.random.Generator, cube: float = 0.3, R: float = 0.08,
                            r: float = 0.03, center=(0.0, 0.0, 0.4)) -> np.ndarray:
    """Area-uniform samples of the cube's outer surface and the torus surface [n, 3]."""
    a_cube = 6 * cube * cube
    a_torus = 4 * math.pi * math.pi * R * r
    n_cube = int(round(n * a_cube / (a_cube + a_torus)))
    face = rng.integers(0, 6, n_cube)
    uv = rng.uniform(-cube / 2, cube / 2, (n_cube, 2))
    pts = np.empty((n_cube, 3))
    for ax in range(3):
        m = face // 2 == ax
        others = [o for o in range(3) if o != ax]
        pts[m, ax] = np.where(face[m] % 2 == 0, 1.0, -1.0) * cube / 2
        pts[m, others[0]] = uv[m, 0]
        pts[m, others[1]] = uv[m, 1]
    tor = []
    n_t = n - n_cube
    while sum(t.shape[0] for t in tor) < n_t:
        th = rng.uniform(0, 2 * np.pi, 2 * n_t)
        ph = rng.uniform(0, 2 * np.pi, 2 * n_t)
        keep = rng.uniform(0, 1, 2 * n_t) < (R + r * np.cos(ph)) / (R + r)
        th, ph = th[keep], ph[keep]
        tor.append(np.stack([(R + r * np.cos(ph)) * np.cos(th), (R + r * np.cos(ph)) * np.sin(th),
                             r * np.sin(ph)], 1))
    pts = np.concatenate([pts, np.concatenate(tor, 0)[:n_t]], 0)
    return (pts + np.asarray(center)).astype(np.float32)


@torch.no_grad()
def sdf_surface_points(net, center: torch.Tensor, scale: float, half: float = 0.3, res: int = 128,
                       chunk: int = 1 << 18) -> torch.Tensor:
    """Zero crossings of the SDF on a res^3 grid over center +- half (world coordinates)."""
    dev = center.device
    ax = torch.linspace(-half, half, res, device=dev)
    gx, gy, gz = torch.meshgrid(ax, ax, ax, indexing="ij")
    world = torch.stack([gx, gy, gz], -1).reshape(-1, 3) + center
    vals = torch.cat([net((world[i:i + chunk] - center) / scale)[0].reshape(-1)
                      for i in range(0, world.shape[0], chunk)]).reshape(res, res, res)
    world = world.reshape(res, res, res, 3)
    out = []
    for d in range(3):
        a = vals.narrow(d, 0, res - 1)
        b = vals.narrow(d, 1, res - 1)
        pa = world.narrow(d, 0, res - 1)
        pb = world.narrow(d, 1, res - 1)
        m = (a * b) < 0
        t = (a[m] / (a[m] - b[m])).unsqueeze(-1)
        out.append(pa[m] + t * (pb[m] - pa[m]))
    return torch.cat(out, 0)


@torch.no_grad()
def chamfer(a: torch.Tensor, b: torch.Tensor, chunk: int = 4096) -> float:
    """Symmetric Chamfer distance: mean nearest-neighbour distance a->b plus b->a (metres)."""
    if a.shape[0] == 0 or b.shape[0] == 0:
        return float("inf")

    def one_way(x, y):
        return torch.cat([torch.cdist(x[i:i + chunk], y, compute_mode="donot_use_mm_for_euclid_dist").min(1).values
                          for i in range(0, x.shape[0], chunk)]).mean()

    return float(one_way(a, b) + one_way(b, a))


@torch.no_grad()
def sdf_on_surface(net, center: torch.Tensor, scale: float, surface: torch.Tensor) -> float:
    """Mean |SDF| (metres) of the network at points of the analytic surface: how far,
    to first order, its zero level set lies from the true surface."""
    return float((net((surface - center) / scale)[0].abs() * scale).mean())


def scene_target(step, seed: int = 0) -> torch.Tensor:
    """|MF| of the shell + torus scene seen by ``step``'s antennas on its voxels, mean-normalised."""
    from . import scenes
    from .ops.RFMatchedFilter.matched_filter_cuda import matched_filter_cuda

    rng = np.random.default_rng(seed)
    pos, amp = scenes.shell_torus_scene(rng)
    g = torch.Generator(device=step.device).manual_seed(seed)
    re, im = scenes.synthesize_if(step.tx, step.rx, torch.tensor(pos), torch.tensor(amp), step.chirp,
                                  snr_db=20.0, generator=g)
    A, S = re.shape
    yr, yi = matched_filter_cuda(re, im, step.tx, step.rx, step.voxels, A, S, step.chirp.adc_sample_rate,
                                 step.chirp.As_sci, step.voxels.shape[0], precision="mixed")
    mag = torch.sqrt(yr * yr + yi * yi)
    return mag / mag.mean()


def train(precision: str, graph: bool, steps: int, seed: int = 0, voxels_per_axis: int = 128,
          device="cuda") -> dict:
    """Trains one form; returns its step time, losses and the final Chamfer distance."""
    from . import scenes
    from .step import Stage1RFStep

    dev = torch.device(device)
    vox = torch.tensor(scenes.voxel_grid(voxels_per_axis, size=0.32).T.copy(), device=dev)
    st = Stage1RFStep(num_antennas=128, num_rays=2048, samples_per_ray=128, num_adc=256, voxels=vox,
                      precision=precision, device=dev, seed=seed)
    st.target = scene_target(st, seed)
    ref = torch.tensor(analytic_surface_points(20000, np.random.default_rng(seed + 7)), device=dev)
    sdf_init = sdf_on_surface(st.net, st.center, st.scale, ref)
    if graph:
        st.capture()
    # a fixed schedule of ray resamplings, identical for both forms
    st.gen.manual_seed(seed + 1)
    losses = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(steps):
        st.resample()
        losses.append(st.run().clone())
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    surf = sdf_surface_points(st.net, st.center, st.scale)
    loss = torch.stack(losses).cpu().numpy()
    return {"precision": precision, "graph": graph, "steps": steps, "ms_per_step": 1e3 * secs / steps,
            "it_per_s": steps / secs, "loss_first": float(loss[0]), "loss_last": float(loss[-1]),
            "loss_every_10": [float(v) for v in loss[::10]],
            "chamfer_m": chamfer(surf, ref), "surface_points": int(surf.shape[0]),
            "sdf_on_surface_init_m": sdf_init,
            "sdf_on_surface_m": sdf_on_surface(st.net, st.center, st.scale, ref)}


def compare(steps: int = 100, seed: int = 0) -> dict:
    fast = train("mixed", True, steps, seed)
    ref = train("plain", False, steps, seed)
    return {"workload": ("stage-1 RF step, 128 antennas x 2048 rays x 128 samples, S = 256, MF onto "
                         "128^3 voxels, target |MF| of the shell + torus scene"),
            "mixed_graph": fast, "plain_eager": ref,
            "speedup_at_equal_steps": fast["it_per_s"] / ref["it_per_s"],
            "chamfer_ratio": fast["chamfer_m"] / ref["chamfer_m"],
            "sdf_on_surface_ratio": fast["sdf_on_surface_m"] / ref["sdf_on_surface_m"]}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args(argv)
    print(json.dumps(compare(args.steps, args.seed), indent=1))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
