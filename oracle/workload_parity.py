"""FP64 parity of the RF operators on the full-size workloads, evaluated on
subsets that the CPU oracle finishes in seconds.

TEST INFRASTRUCTURE ONLY: ``tests/test_gpu_configs.py`` asserts bounds on these
figures and ``bench.py`` reports them; nothing in the library imports this.

Workloads (seeded synthetic inputs; the reference's RF data is not released):

* ``mf3072``: 16 x 16 scan x 3TX4RX = 3072 channels, S = 128 at 5 Msps over
  4 GHz, 64 Rayleigh point scatterers in a 0.2 m cube at 0.4 m, 20 dB SNR,
  48^3 = 110592 voxels.  IF synthesised in FP64 on the CPU.
* ``mf49152``: 64 x 64 scan x 3TX4RX = 49152 channels, S = 256, a 0.3 m cube
  shell (20k scatterers) around a torus (10k), 20 dB SNR, 128^3 voxels over
  0.32 m.  IF synthesised on the GPU (the scatterer sum evaluated by the
  library's adjoint); the figures compare outputs computed from the same FP32
  inputs, so they do not depend on how the inputs were made.
* ``tracer``: 64 antennas x 4096 rays x 128 samples (P = 524288), S = 128, the
  tracer inputs of a random-initialised NeuS SDF network (``benchkit.sdf``).

Subsets (deterministic):

* MF forward: every 27th voxel of 48^3 (4096 voxels); of 128^3, every 8th
  voxel along each axis from index 4 (16^3 = 4096 voxels, a sub-lattice of the
  every-4th 32^3 subset).
* MF adjoint: antenna rows, every 32nd of 3072 (96 rows) or every 3072nd of
  49152 (16 rows), each summed over all voxels.
* Tracer forward: every 4th antenna (16 rows) over all points.  Tracer adjoint:
  the 32768 points of 256 random rays, over all antennas.  Finite differences:
  the same 256 rays.

The MF checks of the 49152-channel workload and every adjoint use the FP64
rotation form of the oracle (``form="f64r"``, equal to the per-sample FP64
form to ~1e-13); the 3072-channel forward uses the per-sample form itself.
Forward errors are complex relative L2 over the subset; adjoint errors are
relative L2 of each gradient over its subset.
"""
from __future__ import annotations

import numpy as np

from . import rf_oracle as orc
from . import torch_tracer

MF3072_VOXELS = np.arange(0, 48 ** 3, 27)
MF3072_ROWS = np.arange(0, 3072, 32)
MF49152_ROWS = np.arange(0, 49152, 3072)
TRACER_ROWS = np.arange(0, 64, 4)
FD_RAYS = 256


def lattice_subset(n: int, step: int, offset: int) -> np.ndarray:
    """Flat indices of the sub-lattice (offset + k step) of an n^3 grid laid
    out like ``benchkit.scenes.voxel_grid`` (x fastest)."""
    ax = np.arange(offset, n, step)
    iz, iy, ix = np.meshgrid(ax, ax, ax, indexing="ij")
    return ((iz * n + iy) * n + ix).ravel()


MF49152_VOXELS = lattice_subset(128, 8, 4)


def rel(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


# ---- workloads --------------------------------------------------------------
def mf3072_inputs(seed: int = 0) -> dict:
    """IF, geometry and voxels of the 3072-channel workload (numpy, CPU)."""
    from benchkit import scenes

    w = scenes.mf_small_workload(seed)
    rng = np.random.default_rng(seed + 1000)
    re, im = scenes.synthesize_if_numpy(w["tx"], w["rx"], w["positions"], w["amplitudes"], w["chirp"],
                                        snr_db=w["snr_db"], rng=rng)
    ch = w["chirp"]
    return dict(re=re, im=im, tx=w["tx"], rx=w["rx"], vox=w["voxel"], fs=ch.adc_sample_rate,
                As=ch.As_sci, S=ch.num_samples)


def mf49152_inputs(dev, seed: int = 0) -> dict:
    """The 49152-channel workload: device tensors (``t``) and numpy copies."""
    import torch

    from benchkit import scenes

    w = scenes.mf_full_workload(seed)
    ch = w["chirp"]
    tx = torch.tensor(w["tx"], device=dev)
    rx = torch.tensor(w["rx"], device=dev)
    g = torch.Generator(device=dev).manual_seed(seed)
    re, im = scenes.synthesize_if(tx, rx, torch.tensor(w["positions"]), torch.tensor(w["amplitudes"]), ch,
                                  snr_db=w["snr_db"], generator=g)
    vox = torch.tensor(w["voxel"], device=dev)
    torch.cuda.synchronize(dev)
    return dict(t=dict(re=re, im=im, tx=tx, rx=rx, vox=vox), re=re.cpu().numpy(), im=im.cpu().numpy(),
                tx=w["tx"], rx=w["rx"], vox=w["voxel"], fs=ch.adc_sample_rate, As=ch.As_sci,
                S=ch.num_samples)


def adjoint_grad(N: int, seed: int) -> np.ndarray:
    """The seeded complex output gradient fed to the MF adjoint checks [N]."""
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)


# ---- matched filter -----------------------------------------------------------
def mf_forward_ref(w: dict, voxels: np.ndarray, form: str = "f64r") -> np.ndarray:
    yr, yi = orc.mf_forward(w["re"], w["im"], w["tx"], w["rx"], w["vox"][:, voxels], w["fs"], w["As"], form)
    return yr + 1j * yi


def mf_forward_error(y: np.ndarray, w: dict, voxels: np.ndarray, form: str = "f64r") -> float:
    """Relative L2 of the complex volume ``y`` [N] at ``voxels`` against FP64."""
    return rel(np.asarray(y)[voxels], mf_forward_ref(w, voxels, form))


def mf_adjoint_ref(g: np.ndarray, w: dict, rows: np.ndarray) -> np.ndarray:
    A = w["tx"].shape[0]
    hr, hi = orc.mf_backward(g.real, g.imag, w["tx"][rows], w["rx"][rows], w["vox"], len(rows), w["S"],
                             w["fs"], w["As"], "f64r")
    # the oracle divides by the rows it was given; the operator by all A antennas
    return (hr + 1j * hi) * (len(rows) / A)


def mf_adjoint_error(h: np.ndarray, g: np.ndarray, w: dict, rows: np.ndarray) -> float:
    """Relative L2 of the complex adjoint ``h`` [A, S] on ``rows`` against FP64."""
    return rel(np.asarray(h)[rows], mf_adjoint_ref(g, w, rows))


# ---- signal tracer ----------------------------------------------------------
def tracer_inputs(dev, seed: int = 0, num_antennas: int = 64, num_rays: int = 4096,
                  samples_per_ray: int = 128, num_adc: int = 128) -> dict:
    """The tracer workload: device tensors (``t``) and numpy copies."""
    from benchkit.sdf import tracer_workload

    w = tracer_workload(num_antennas, num_rays, samples_per_ray, num_adc, seed=seed, device=dev)
    ch = w["chirp"]
    np_ = {k: w[k].detach().cpu().numpy() for k in ("normals", "sigmas", "points", "tx", "rx", "inbounds")}
    return dict(t=w, **np_, S=ch.num_samples, fs=ch.adc_sample_rate, f0=w["radar_cfg"]["fc_start"],
                As=ch.As_sci, rays=num_rays, samples_per_ray=samples_per_ray)


def ray_points(w: dict, rays: np.ndarray) -> np.ndarray:
    T = w["samples_per_ray"]
    return (np.asarray(rays)[:, None] * T + np.arange(T)[None, :]).ravel()


def fd_rays(w: dict, seed: int = 0, count: int = FD_RAYS) -> np.ndarray:
    return np.sort(np.random.default_rng(seed + 77).choice(w["rays"], count, replace=False))


def residual(A: int, S: int, seed: int) -> np.ndarray:
    """The seeded complex residual fed to the tracer adjoint checks [A, S]."""
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((A, S)) + 1j * rng.standard_normal((A, S))).astype(np.complex64)


def tracer_forward_error(x: np.ndarray, w: dict, rows: np.ndarray) -> float:
    """Relative L2 of the complex IF ``x`` [A, S] on antenna ``rows`` against FP64."""
    fr, fi = orc.tracer_forward(w["normals"], w["sigmas"][rows], w["points"], w["tx"][rows], w["rx"][rows],
                                w["inbounds"], w["S"], w["fs"], w["f0"], w["As"])
    return rel(np.asarray(x)[rows], fr + 1j * fi)


def tracer_adjoint_errors(grads: dict, g: np.ndarray, w: dict, pts: np.ndarray) -> dict:
    """Relative L2 of the sigma [A, P], normal [P, 3] and position [P, 3]
    gradients at points ``pts`` against the FP64 adjoint."""
    P = w["points"].shape[0]
    gn, gs, gp = orc.tracer_backward(g.real, g.imag, w["normals"][pts], w["sigmas"][:, pts], w["points"][pts],
                                     w["tx"], w["rx"], w["inbounds"][pts], w["fs"], w["f0"], w["As"])
    scale = len(pts) / P  # the oracle normalises by the points it was given
    return {"sigma": rel(np.asarray(grads["sigmas"])[:, pts], gs * scale),
            "normal": rel(np.asarray(grads["normals"])[pts], gn * scale),
            "position": rel(np.asarray(grads["points"])[pts], gp * scale)}


def tracer_fd_errors(grads: dict, g: np.ndarray, w: dict, rays: np.ndarray, seed: int = 0,
                     steps=(1e-3, 1e-6, 1e-7), chunk_points: int = 2048) -> dict:
    """Directional derivatives of L = sum_{a,n} Re(conj(g) x) along random
    directions of each ray's sigmas, normals and positions: the operator's
    gradient against FP64 central differences of the pure-torch tracer.

    Per ray the error is |FD - analytic| / sum_p |analytic_p| (the ray's
    directional derivative against the scale of its points' terms).  Returns
    the largest error over the rays for each of sigma, normal and position, and
    the number of points left out because a culling decision changed inside
    the difference step."""
    import torch

    P = w["points"].shape[0]
    T = w["samples_per_ray"]
    pts = ray_points(w, rays)
    rng = np.random.default_rng(seed + 99)
    A = w["tx"].shape[0]
    dirs = {"sigma": rng.standard_normal((A, len(pts))), "normal": rng.standard_normal((len(pts), 3)),
            "position": rng.standard_normal((len(pts), 3))}
    analytic = {"sigma": (np.asarray(grads["sigmas"], np.float64)[:, pts] * dirs["sigma"]).sum(0),
                "normal": (np.asarray(grads["normals"], np.float64)[pts] * dirs["normal"]).sum(1),
                "position": (np.asarray(grads["points"], np.float64)[pts] * dirs["position"]).sum(1)}
    d64 = lambda a: torch.tensor(np.asarray(a), dtype=torch.float64)  # noqa: E731
    tx, rx = d64(w["tx"]), d64(w["rx"])
    gr, gi = d64(g.real), d64(g.imag)
    base = {"sigma": d64(w["sigmas"][:, pts]), "normal": d64(w["normals"][pts]),
            "position": d64(w["points"][pts])}
    fd = {}
    dropped = 0
    for kind, h in zip(("sigma", "normal", "position"), steps):
        v = d64(dirs[kind])
        out = np.zeros(len(pts))
        for c0 in range(0, len(pts), chunk_points):
            sl = slice(c0, c0 + chunk_points)
            losses, lives = [], []
            for sign in (1.0, -1.0):
                args = {k: (base[k][:, sl] if k == "sigma" else base[k][sl]) for k in base}
                args[kind] = args[kind] + sign * h * (v[:, sl] if kind == "sigma" else v[sl])
                loss, live = torch_tracer.point_losses(args["normal"], args["sigma"], args["position"], tx, rx,
                                                       w["S"], w["fs"], w["f0"], w["As"], gr, gi)
                losses.append(loss)
                lives.append(live)
            same = (lives[0] == lives[1]).all(0).numpy()
            dropped += int((~same).sum())
            out[sl] = np.where(same, ((losses[0] - losses[1]) / (2 * h)).numpy() / P, np.nan)
        fd[kind] = out
    errs = {}
    for kind in fd:
        worst = 0.0
        for r in range(len(rays)):
            sl = slice(r * T, (r + 1) * T)
            keep = np.isfinite(fd[kind][sl])
            an = analytic[kind][sl][keep]
            scale = np.abs(an).sum()
            if scale == 0.0:
                continue
            worst = max(worst, abs(fd[kind][sl][keep].sum() - an.sum()) / scale)
        errs[kind] = worst
    errs["dropped_points"] = dropped
    return errs
