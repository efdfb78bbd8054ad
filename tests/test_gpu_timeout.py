"""The operators' bounded device-side wait, driven to its timeout on the GPU.

Every kernel that waits on a shared-memory barrier (the TMA staging ring) gives
up after a wall-time limit, raises GERAF_ERR_DEVICE_TIMEOUT in the library's
device status word and returns, so a copy that never lands cannot hang the GPU.
The test hook ``geraf_rf_selftest_wait_timeout`` runs that staging code with a
1 ms limit on barriers that nothing completes (no copy is issued): the blocks
must come back, the status word must hold the timeout, and the library must
work normally afterwards."""
import ctypes
import time

import numpy as np
import pytest
import torch

from benchkit import scenes
from conftest import rel_l2
from gpu_helpers import mf_forward
from oracle import rf_oracle as orc

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_the_library_recovers(cuda):
    from geraf_b200 import _lib

    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    _lib.device_status(stream, reset=True)
    returned = torch.zeros(1, dtype=torch.int32, device="cuda")
    blocks = 4
    t0 = time.perf_counter()
    _lib.check(lib.geraf_rf_selftest_wait_timeout(1_000_000, blocks, ctypes.c_void_p(returned.data_ptr()),
                                                  stream), "selftest")
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    assert int(returned.item()) == blocks            # every block left through the timeout path
    assert elapsed < 1.0                             # ~2 ms of bounded waits, not the 2 s default
    assert _lib.device_status(stream, reset=True) == _lib.GERAF_ERR_DEVICE_TIMEOUT
    assert _lib.device_status(stream, reset=True) == _lib.GERAF_OK

    # the context is intact: an operator call right after matches the FP64 oracle
    rng = np.random.default_rng(0)
    tx, rx = scenes.virtual_array(2)
    ch = scenes.chirp(64)
    pos, amp = scenes.point_scene(rng, 4, size=0.1)
    re, im = scenes.synthesize_if_numpy(tx, rx, pos, amp, ch, snr_db=20.0, rng=rng)
    vox = scenes.voxel_grid(6, size=0.1)
    yr, yi = mf_forward(re, im, tx, rx, vox, ch.adc_sample_rate, ch.As_sci, "mixed")
    ref = orc.mf_forward(re, im, tx, rx, vox, ch.adc_sample_rate, ch.As_sci)
    assert rel_l2(yr + 1j * yi, ref[0] + 1j * ref[1]) < 1e-4
    assert _lib.device_status(stream, reset=True) == _lib.GERAF_OK
