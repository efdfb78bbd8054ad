"""Offline matched-filter volume builder on the GPU: files in the reference's
layout, values against the FP64 oracle, the aggregated object volume, and GPU
sampling at target points."""
import os

import numpy as np
import pytest
import torch

from geraf_b200 import scenes, volume
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


def test_sample_volume_on_gpu_matches_cpu(cuda):
    rng = np.random.default_rng(1)
    vol = torch.tensor(rng.standard_normal((9, 7, 5)).astype(np.float32))
    pts = torch.tensor(rng.uniform(-1, 1, (100, 3)).astype(np.float32))
    cpu = volume.sample_volume(vol, pts)
    gpu = volume.sample_volume(vol.cuda(), pts.cuda())
    assert torch.allclose(gpu.cpu(), cpu, atol=1e-6)
