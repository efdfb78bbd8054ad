"""Offline matched-filter volume builder for GeRaF's RF data layout, and GPU
sampling of such volumes at target points.

On-disk format (the reference's loader, ``geraf/datasets/transforms/loading.py:28-61``,
and ``docs/PrepareData.md``): each radar frame folder holds ``adcr.npy`` /
``adci.npy`` (raw IF samples, [M, S]), ``tpos.npy`` / ``rpos.npy`` ([M, 3]) and
``sarimage.bin`` -- the matched-filter magnitude as raw float32 of shape
(Nx, Ny, Nz), C order, x outermost; an object folder holds the frames under
``mf/`` and ``<obj>.npy``, the sum of all frame volumes.  The grid spans
``bound = [xmin, xmax, ymin, ymax, zmin, zmax]`` at ``mf_res = [rx, ry, rz]``
with ``round((max - min) / res) + 1`` points per axis
(``geraf/utils/matched_filter/cuda_tools.py:4-29``).

The reference ships no builder for these files; this one backprojects every
voxel with this library's matched filter, in voxel chunks so a 601^3 frame
grid fits any memory budget.  Usage::

    python -m geraf_b200.volume FRAME_OR_OBJECT_DIR --bound 0.5 1.1 -0.37 0.23 -0.15 0.45 \\
        --mf-res 0.001 0.001 0.001 --adc-sample-rate 10e6 --slope 70.15e12
"""
from __future__ import annotations

import argparse
import os

import numpy as np
import torch


def grid_num(max_val: float, min_val: float, res: float) -> int:
    """Grid points from min to max inclusive at spacing res (the reference's ``grid_num``)."""
    if res <= 0:
        raise ValueError("Resolution 'res' must be greater than zero.")
    return int(round((max_val - min_val) / res)) + 1


def grid_shape(bound, mf_res) -> tuple[int, int, int]:
    return (grid_num(bound[1], bound[0], mf_res[0]), grid_num(bound[3], bound[2], mf_res[1]),
            grid_num(bound[5], bound[4], mf_res[2]))


def grid_voxels(bound, mf_res, start: int = 0, count: int | None = None, device="cpu") -> torch.Tensor:
    """Voxel centres [count, 3] of the flattened (x, y, z) C-order grid, from flat index ``start``."""
    nx, ny, nz = grid_shape(bound, mf_res)
    total = nx * ny * nz
    count = total - start if count is None else min(count, total - start)
    idx = torch.arange(start, start + count, device=device, dtype=torch.int64)
    iz = idx % nz
    iy = (idx // nz) % ny
    ix = idx // (nz * ny)
    return torch.stack([bound[0] + ix.to(torch.float64) * mf_res[0],
                        bound[2] + iy.to(torch.float64) * mf_res[1],
                        bound[4] + iz.to(torch.float64) * mf_res[2]], 1).to(torch.float32)


def build_mf_volume(adc_real, adc_imag, tpos, rpos, adc_sample_rate: float, As_sci: float, bound, mf_res,
                    precision: str = "mixed", chunk: int = 1 << 22, device="cuda") -> torch.Tensor:
    """|matched filter| on the (Nx, Ny, Nz) grid, float32 on ``device``."""
    from .ops.RFMatchedFilter import _C

    dev = torch.device(device)

    def dev_f32(x):  # numpy arrays or tensors on any device
        t = x if isinstance(x, torch.Tensor) else torch.as_tensor(np.asarray(x, np.float32))
        return t.to(device=dev, dtype=torch.float32).contiguous()

    re, im = dev_f32(adc_real), dev_f32(adc_imag)
    tx, rx = dev_f32(tpos).reshape(-1, 3), dev_f32(rpos).reshape(-1, 3)
    A, S = re.shape
    if tx.shape[0] != A or rx.shape[0] != A:
        raise ValueError(f"antenna count mismatch: IF has {A} rows, positions {tx.shape[0]}/{rx.shape[0]}")
    shape = grid_shape(bound, mf_res)
    total = shape[0] * shape[1] * shape[2]
    out = torch.empty(total, dtype=torch.float32, device=dev)
    yr = torch.empty(min(chunk, total), dtype=torch.float32, device=dev)
    yi = torch.empty_like(yr)
    for start in range(0, total, chunk):
        vox = grid_voxels(bound, mf_res, start, chunk, device=dev).t().contiguous()
        n = vox.shape[1]
        _C.MatchedFilter_forward(re, im, tx, rx, yr[:n], yi[:n], vox, A, S, float(adc_sample_rate),
                                 float(As_sci), n, precision=precision)
        torch.hypot(yr[:n], yi[:n], out=out[start:start + n])
    return out.view(shape)


def write_sarimage(path: str, volume) -> None:
    np.ascontiguousarray(torch.as_tensor(volume).detach().cpu().numpy(), dtype=np.float32).tofile(path)


def read_sarimage(path: str, shape) -> np.ndarray:
    return np.fromfile(path, dtype=np.float32).reshape(shape)


def process_frame(frame_dir: str, adc_sample_rate: float, As_sci: float, bound, mf_res,
                  precision: str = "mixed", device="cuda") -> torch.Tensor:
    """Builds ``frame_dir/sarimage.bin`` from the frame's ADC and antenna files."""
    vol = build_mf_volume(np.load(os.path.join(frame_dir, "adcr.npy")),
                          np.load(os.path.join(frame_dir, "adci.npy")),
                          np.load(os.path.join(frame_dir, "tpos.npy")),
                          np.load(os.path.join(frame_dir, "rpos.npy")), adc_sample_rate, As_sci, bound,
                          mf_res, precision=precision, device=device)
    write_sarimage(os.path.join(frame_dir, "sarimage.bin"), vol)
    return vol


def process_object(obj_dir: str, adc_sample_rate: float, As_sci: float, bound, mf_res,
                   precision: str = "mixed", device="cuda") -> str:
    """Every frame under ``obj_dir/mf/``, then ``obj_dir/<obj>.npy`` = sum of the frame volumes."""
    mf_dir = os.path.join(obj_dir, "mf")
    acc = None
    for name in sorted(os.listdir(mf_dir)):
        frame = os.path.join(mf_dir, name)
        if not os.path.isfile(os.path.join(frame, "adcr.npy")):
            continue
        vol = process_frame(frame, adc_sample_rate, As_sci, bound, mf_res, precision, device)
        acc = vol.clone() if acc is None else acc.add_(vol)
    if acc is None:
        raise FileNotFoundError(f"no frames with adcr.npy under {mf_dir}")
    out = os.path.join(obj_dir, os.path.basename(os.path.normpath(obj_dir)) + ".npy")
    np.save(out, acc.cpu().numpy().astype(np.float32))
    return out


def sample_volume(volume: torch.Tensor, points_norm: torch.Tensor, mode: str = "bilinear",
                  align_corners: bool = True) -> torch.Tensor:
    """Samples an (Nx, Ny, Nz) volume at points in normalised [-1, 1]^3 (x, y, z)
    coordinates on the GPU -- the reference's ``_sample_volume`` /
    ``InterpolateMFAtTargets`` (``geraf/datasets/transforms/loading.py:20-25,
    78-100``), which run torch grid_sample on the host in the data workers,
    moved next to the matched-filter output.  ``mode`` "bilinear" (trilinear)
    or "nearest", zeros outside the volume.  Both tensors must be CUDA tensors
    on one device; returns float32 [P] there (the library kernel
    ``geraf_volume_sample``: no PyTorch fallback)."""
    from . import _lib
    from .runtime import device_guard, ptr, stream_ptr

    modes = {"bilinear": _lib.SAMPLE_TRILINEAR, "nearest": _lib.SAMPLE_NEAREST}
    if mode not in modes:
        raise ValueError(f"sample_volume supports modes {sorted(modes)}, not {mode!r}")
    if volume.dim() != 3:
        raise ValueError(f"`volume` must have shape [Nx, Ny, Nz], got {tuple(volume.shape)}")
    if not (volume.is_cuda and points_norm.is_cuda) or volume.device != points_norm.device:
        raise ValueError("`volume` and `points_norm` must be CUDA tensors on the same device")
    vol = volume.to(torch.float32).contiguous()
    pts = points_norm.to(torch.float32).reshape(-1, 3).contiguous()
    out = torch.empty(pts.shape[0], dtype=torch.float32, device=vol.device)
    nx, ny, nz = vol.shape
    with device_guard(vol.device):
        _lib.call("geraf_volume_sample", ptr(vol), nx, ny, nz, ptr(pts), pts.shape[0], ptr(out), modes[mode],
                  int(bool(align_corners)), stream_ptr(vol.device))
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("path", help="a frame folder (with adcr.npy) or an object folder (with mf/)")
    ap.add_argument("--bound", type=float, nargs=6, required=True)
    ap.add_argument("--mf-res", type=float, nargs=3, required=True)
    ap.add_argument("--adc-sample-rate", type=float, required=True, help="Hz")
    ap.add_argument("--slope", type=float, required=True, help="chirp slope in Hz/s")
    ap.add_argument("--precision", choices=["mixed", "plain"], default="mixed")
    args = ap.parse_args(argv)
    As_sci = args.slope / 1e8
    if os.path.isfile(os.path.join(args.path, "adcr.npy")):
        process_frame(args.path, args.adc_sample_rate, As_sci, args.bound, args.mf_res, args.precision)
        print(os.path.join(args.path, "sarimage.bin"))
    else:
        print(process_object(args.path, args.adc_sample_rate, As_sci, args.bound, args.mf_res, args.precision))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
