"""Seeded synthetic radar scenes for the RF operators.

The reference's RF dataset is not released, so benchmarks and tests run on
synthetic inputs with the shapes and value distributions of the workloads:

* FMCW chirps: ``B`` Hz swept over ``S`` samples at ``fs`` -> slope ``B fs / S``
  (``As_sci`` = slope / 1e8, the reference's scaled unit).  The matched filter
  always demodulates at 773.704e8 Hz (77.3704 GHz), so scenes are synthesised
  at that carrier.
* Virtual arrays: a ``scan_n x scan_n`` planar raster at ``pitch`` in the z = 0
  plane, each position carrying a 3 TX x 4 RX cascade (TX spaced 2 lambda, RX
  spaced lambda/2 along x, the layout of common 77 GHz single-chip radars):
  16 x 16 x 12 = 3072 channels or 64 x 64 x 12 = 49152 channels.
* Point-scatterer scenes in front of the array (+z), complex Rayleigh
  amplitudes with uniform phase, and the IF signal
  s[a,n] = sum_k a_k exp(+j phi(a,k,n)) plus complex Gaussian noise at a given
  SNR.  The synthesis runs on the GPU through this library's matched-filter
  adjoint (A * MF^H applied to the scatterer amplitudes), which is that sum
  exactly.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

MF_CARRIER = 773.704  # 1e8 Hz, fixed by the reference's matched filter
C_SCALED = 2.9979     # 1e8 m/s
WAVELENGTH = C_SCALED / MF_CARRIER  # m


@dataclass(frozen=True)
class Chirp:
    num_samples: int
    adc_sample_rate: float  # Hz
    bandwidth: float        # Hz

    @property
    def slope(self) -> float:
        return self.bandwidth * self.adc_sample_rate / self.num_samples

    @property
    def As_sci(self) -> float:
        return self.slope / 1e8

    def radar_cfg(self, fc_start: float = MF_CARRIER) -> dict:
        """The four keys the reference's op adapters read (configs/_base_/radar/radar_setup.py)."""
        return {"numADCSample": self.num_samples, "adcSampleRate": self.adc_sample_rate,
                "As_sci": self.As_sci, "fc_start": fc_start}


def chirp(num_samples: int, fs: float = 5e6, bandwidth: float = 4e9) -> Chirp:
    return Chirp(num_samples, fs, bandwidth)


def virtual_array(scan_n: int, pitch: float = 1e-3, n_tx: int = 3, n_rx: int = 4,
                  z: float = 0.0) -> tuple[np.ndarray, np.ndarray]:
    """(tx [A,3], rx [A,3]) float32, A = scan_n^2 * n_tx * n_rx, scan-major order."""
    lam = WAVELENGTH
    tx_off = np.stack([np.arange(n_tx) * 2.0 * lam, np.zeros(n_tx), np.zeros(n_tx)], 1)
    rx_off = np.stack([np.arange(n_rx) * 0.5 * lam + 0.5 * lam * n_rx, np.full(n_rx, 2.0 * lam),
                       np.zeros(n_rx)], 1)
    c = (np.arange(scan_n) - (scan_n - 1) / 2.0) * pitch
    gy, gx = np.meshgrid(c, c, indexing="ij")
    scan = np.stack([gx.ravel(), gy.ravel(), np.full(gx.size, z)], 1)
    tx = scan[:, None, None, :] + tx_off[None, :, None, :]
    rx = scan[:, None, None, :] + rx_off[None, None, :, :]
    tx = np.broadcast_to(tx, (scan.shape[0], n_tx, n_rx, 3)).reshape(-1, 3)
    rx = np.broadcast_to(rx, (scan.shape[0], n_tx, n_rx, 3)).reshape(-1, 3)
    return np.ascontiguousarray(tx, np.float32), np.ascontiguousarray(rx, np.float32)


def voxel_grid(n: int, center=(0.0, 0.0, 0.4), size: float = 0.2) -> np.ndarray:
    """Regular n^3 grid over a cube, as the matched filter's [3, N] (x, y, z rows) float32."""
    c = np.asarray(center, np.float64)
    ax = np.linspace(-size / 2, size / 2, n)
    gz, gy, gx = np.meshgrid(ax + c[2], ax + c[1], ax + c[0], indexing="ij")
    return np.ascontiguousarray(np.stack([gx.ravel(), gy.ravel(), gz.ravel()], 0), np.float32)


def rayleigh_amplitudes(rng: np.random.Generator, k: int) -> np.ndarray:
    mag = rng.rayleigh(1.0, k)
    ph = rng.uniform(0.0, 2.0 * np.pi, k)
    return (mag * np.exp(1j * ph)).astype(np.complex64)


def point_scene(rng: np.random.Generator, k: int = 64, center=(0.0, 0.0, 0.4),
                size: float = 0.2) -> tuple[np.ndarray, np.ndarray]:
    """k scatterers uniform in a cube: (positions [k,3] float32, amplitudes [k] complex64)."""
    pos = rng.uniform(-size / 2, size / 2, (k, 3)) + np.asarray(center)
    return pos.astype(np.float32), rayleigh_amplitudes(rng, k)


def shell_torus_scene(rng: np.random.Generator, n_shell: int = 20000, n_torus: int = 10000,
                      cube: float = 0.3, wall: float = 0.003, R: float = 0.08, r: float = 0.03,
                      center=(0.0, 0.0, 0.4)) -> tuple[np.ndarray, np.ndarray]:
    """Cube shell (edge ``cube``, walls ``wall`` thick) enclosing a torus, as point scatterers."""
    c = np.asarray(center, np.float64)
    face = rng.integers(0, 6, n_shell)
    uv = rng.uniform(-cube / 2, cube / 2, (n_shell, 2))
    depth = cube / 2 - rng.uniform(0.0, wall, n_shell)
    shell = np.empty((n_shell, 3))
    axis = face // 2
    sign = np.where(face % 2 == 0, 1.0, -1.0)
    for ax in range(3):
        m = axis == ax
        others = [o for o in range(3) if o != ax]
        shell[m, ax] = sign[m] * depth[m]
        shell[m, others[0]] = uv[m, 0]
        shell[m, others[1]] = uv[m, 1]
    # torus: area-uniform sampling by rejection on the tube angle
    pts = []
    while sum(p.shape[0] for p in pts) < n_torus:
        th = rng.uniform(0, 2 * np.pi, 2 * n_torus)
        ph = rng.uniform(0, 2 * np.pi, 2 * n_torus)
        keep = rng.uniform(0, 1, 2 * n_torus) < (R + r * np.cos(ph)) / (R + r)
        th, ph = th[keep], ph[keep]
        pts.append(np.stack([(R + r * np.cos(ph)) * np.cos(th), (R + r * np.cos(ph)) * np.sin(th),
                             r * np.sin(ph)], 1))
    torus = np.concatenate(pts, 0)[:n_torus]
    pos = np.concatenate([shell, torus], 0) + c
    return pos.astype(np.float32), rayleigh_amplitudes(rng, pos.shape[0])


def synthesize_if(tx: torch.Tensor, rx: torch.Tensor, positions: torch.Tensor,
                  amplitudes: torch.Tensor, ch: Chirp, snr_db: float | None = 20.0,
                  generator: torch.Generator | None = None) -> tuple[torch.Tensor, torch.Tensor]:
    """IF samples (real, imag) [A, S] float32 on the device of ``tx``.

    ``positions`` [K,3], ``amplitudes`` [K] complex.  Noise power is the mean
    signal power over 10^(snr_db/10).
    """
    from geraf_b200.ops.RFMatchedFilter import _C

    A, K, S = tx.shape[0], positions.shape[0], ch.num_samples
    dev = tx.device
    vox = positions.to(dev, torch.float32).t().contiguous()
    amp_r = amplitudes.real.to(dev, torch.float32).contiguous()
    amp_i = amplitudes.imag.to(dev, torch.float32).contiguous()
    real = torch.empty((A, S), dtype=torch.float32, device=dev)
    imag = torch.empty_like(real)
    dummy = torch.empty((A, S), dtype=torch.float32, device=dev)
    _C.MatchedFilter_backward_realimag(amp_r, amp_i, dummy, dummy, tx.contiguous(), rx.contiguous(),
                                       real, imag, vox, A, S, ch.adc_sample_rate, ch.As_sci, K,
                                       precision="mixed")
    real.mul_(A)
    imag.mul_(A)
    if snr_db is not None:
        p_sig = (real.square() + imag.square()).mean()
        sigma = torch.sqrt(p_sig / (10.0 ** (snr_db / 10.0)) / 2.0)
        real.add_(torch.randn(real.shape, device=dev, generator=generator) * sigma)
        imag.add_(torch.randn(imag.shape, device=dev, generator=generator) * sigma)
    return real, imag


def synthesize_if_numpy(tx, rx, positions, amplitudes, ch: Chirp, snr_db=20.0,
                        rng: np.random.Generator | None = None):
    """CPU (numpy, FP64) version of :func:`synthesize_if` for small cases and tests
    (antennas in chunks of 256, so the [A, K, S] phase array stays small)."""
    lam_f0 = 2.0 * float(np.float32(np.pi)) * float(np.float32(MF_CARRIER))
    w1 = 2.0 * float(np.float32(np.pi)) * float(np.float32(ch.As_sci))
    t = np.arange(ch.num_samples) / float(np.float32(ch.adc_sample_rate))
    s = np.empty((tx.shape[0], ch.num_samples), np.complex128)
    for a0 in range(0, tx.shape[0], 256):
        txc, rxc = tx[a0:a0 + 256], rx[a0:a0 + 256]
        d = (np.linalg.norm(txc[:, None, :].astype(np.float64) - positions[None], axis=-1)
             + np.linalg.norm(rxc[:, None, :].astype(np.float64) - positions[None], axis=-1)
             + float(np.float32(0.15)))
        tau = d / float(np.float32(C_SCALED))  # [a,K]
        ph = tau[:, :, None] * (lam_f0 + w1 * t)[None, None, :]
        s[a0:a0 + 256] = (amplitudes[None, :, None] * np.exp(1j * ph)).sum(1)
    if snr_db is not None:
        rng = rng or np.random.default_rng(0)
        p = np.mean(np.abs(s) ** 2)
        sig = np.sqrt(p / 10 ** (snr_db / 10) / 2)
        s = s + sig * (rng.standard_normal(s.shape) + 1j * rng.standard_normal(s.shape))
    return s.real.astype(np.float32), s.imag.astype(np.float32)


# ---- workloads named by what they are ---------------------------------------
def mf_small_workload(seed: int = 0):
    """3072-channel array (16x16 scan x 3TX4RX), S=128 at 5 Msps over 4 GHz,
    64 Rayleigh point scatterers in a 0.2 m cube at 0.4 m, 48^3 voxels."""
    rng = np.random.default_rng(seed)
    tx, rx = virtual_array(16)
    pos, amp = point_scene(rng, 64)
    return dict(tx=tx, rx=rx, positions=pos, amplitudes=amp, chirp=chirp(128),
                voxel=voxel_grid(48), snr_db=20.0, seed=seed)


def mf_full_workload(seed: int = 0):
    """49152-channel array (64x64 scan x 3TX4RX), S=256 at 5 Msps over 4 GHz,
    0.3 m cube shell (20k) + torus (10k) scatterers, 128^3 voxels over 0.32 m."""
    rng = np.random.default_rng(seed)
    tx, rx = virtual_array(64)
    pos, amp = shell_torus_scene(rng)
    return dict(tx=tx, rx=rx, positions=pos, amplitudes=amp, chirp=chirp(256),
                voxel=voxel_grid(128, size=0.32), snr_db=20.0, seed=seed)
