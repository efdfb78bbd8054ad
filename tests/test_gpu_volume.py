"""Offline matched-filter volume builder on the GPU: files in the reference's
layout, values against the FP64 oracle, the aggregated object volume, and GPU
sampling at target points."""
import os

import numpy as np
import pytest
import torch

from benchkit import scenes
from geraf_b200 import volume
from oracle import rf_oracle as orc

pytestmark = pytest.mark.gpu


def test_object_folder_build(cuda, tmp_path):
    rng = np.random.default_rng(0)
    bound = [0.35, 0.45, -0.05, 0.05, -0.04, 0.04]
    res = [0.005, 0.005, 0.004]
    ch = scenes.chirp(32)
    tx, rx = scenes.virtual_array(3)
    obj = tmp_path / "toy_sub2"
    vols = []
    for k in range(2):
        frame = obj / "mf" / f"{k}_0_{k}"
        os.makedirs(frame)
        pos = np.array([[0.4 + 0.01 * k, 0.0, 0.01]], np.float32)
        re, im = scenes.synthesize_if_numpy(tx, rx, pos, np.array([1.0 + 0j], np.complex64), ch, snr_db=None)
        re = re + 0.01 * rng.standard_normal(re.shape).astype(np.float32)
        np.save(frame / "adcr.npy", re)
        np.save(frame / "adci.npy", im)
        np.save(frame / "tpos.npy", tx)
        np.save(frame / "rpos.npy", rx)
        vols.append((re, im))
    out = volume.process_object(str(obj), ch.adc_sample_rate, ch.As_sci, bound, res)
    shape = volume.grid_shape(bound, res)
    acc = np.load(out)
    assert acc.shape == shape
    grid = volume.grid_voxels(bound, res).numpy()
    pick = rng.choice(grid.shape[0], 40, replace=False)
    total = np.zeros(len(pick))
    for k, (re, im) in enumerate(vols):
        frame_vol = volume.read_sarimage(str(obj / "mf" / f"{k}_0_{k}" / "sarimage.bin"), shape).reshape(-1)
        yr, yi = orc.mf_forward(re, im, tx, rx, grid[pick].T.copy(), ch.adc_sample_rate, ch.As_sci)
        mag = np.hypot(yr, yi)
        np.testing.assert_allclose(frame_vol[pick], mag, rtol=1e-4, atol=1e-6 * mag.max())
        total += frame_vol[pick]
    np.testing.assert_allclose(acc.reshape(-1)[pick], total, rtol=1e-6)


@pytest.mark.parametrize("mode,align", [("bilinear", True), ("bilinear", False), ("nearest", True)])
def test_sample_volume_kernel_matches_the_reference_host_sampling(cuda, mode, align):
    """The library's target-point sampling against the reference's host path
    (torch grid_sample on the CPU, loading.py:20-25) and the FP64 restatement:
    a ragged volume, points inside, on faces and corners, outside, and NaN."""
    import torch.nn.functional as F

    rng = np.random.default_rng(1)
    vol = rng.standard_normal((37, 41, 29)).astype(np.float32)
    pts = rng.uniform(-1.15, 1.15, (20000, 3)).astype(np.float32)
    pts[:8] = np.array([[sx, sy, sz] for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)], np.float32)
    pts[8:40, 2] = 1.0
    pts[40:44] = [[2.5, 0, 0], [0, -2.5, 0], [0, 0, 3e30], [-2.5, 2.5, 0]]
    grid = torch.tensor(np.stack([pts[:, 2], pts[:, 1], pts[:, 0]], -1)).view(1, 1, 1, -1, 3)
    host = F.grid_sample(torch.tensor(vol)[None, None], grid, mode=mode, align_corners=align).reshape(-1).numpy()
    got = volume.sample_volume(torch.tensor(vol, device="cuda"), torch.tensor(pts, device="cuda"), mode,
                               align).cpu().numpy()
    scale = np.abs(vol).max()
    assert np.max(np.abs(got - host)) < 1e-6 * scale
    # against exact arithmetic: the FP32 source index (up to ~40 here) is rounded to
    # ~4e-6, which moves the interpolation weights by as much -- for torch as well
    assert np.max(np.abs(got - orc.sample_volume(vol, pts, mode, align))) < 2e-5 * scale
    assert np.max(np.abs(host - orc.sample_volume(vol, pts, mode, align))) < 2e-5 * scale
    assert np.all(got[40:44] == 0.0)
    nan_pts = torch.tensor([[np.nan, 0.0, 0.0], [0.0, 0.0, 0.0]], device="cuda")
    out = volume.sample_volume(torch.tensor(vol, device="cuda"), nan_pts, mode, align).cpu().numpy()
    assert out[0] == 0.0 and np.isfinite(out[1])


def test_sample_volume_rejects_bad_arguments(cuda):
    vol = torch.zeros((4, 4, 4), device="cuda")
    with pytest.raises(ValueError):
        volume.sample_volume(vol, torch.zeros((3, 3), device="cuda"), "bicubic")
    with pytest.raises(ValueError):
        volume.sample_volume(vol.cpu(), torch.zeros((3, 3)))
    empty = volume.sample_volume(torch.zeros((0, 4, 4), device="cuda"), torch.zeros((5, 3), device="cuda"))
    assert torch.equal(empty.cpu(), torch.zeros(5))
