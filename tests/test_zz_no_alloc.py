"""The matched-filter forward that allocates nothing (geraf_mf_forward_noalloc),
called through the C ABI and checked against the regular geraf_mf_forward.

That entry point exists for callers that cannot allocate device memory -- hosts
with a device-memory budget fixed at start-up that cannot hand the library a
problem-sized workspace -- and keeps its partial sums in an array compiled into
the library.  This file is named to be collected last, so a run that stops at
the first failure has run every other test before it."""
import ctypes

import numpy as np
import pytest
import torch

from conftest import rel_l2
from benchkit import scenes
from geraf_b200 import _lib

pytestmark = pytest.mark.gpu

TOL = 2e-6  # the tolerance between launch shapes of the mixed forward elsewhere in the suite


def _case(seed, scan, S, n, n_tx=3, n_rx=4):
    rng = np.random.default_rng(seed)
    tx, rx = scenes.virtual_array(scan, n_tx=n_tx, n_rx=n_rx)
    pos, amp = scenes.point_scene(rng, 6, size=0.12)
    ch = scenes.chirp(S)
    re, im = scenes.synthesize_if_numpy(tx, rx, pos, amp, ch, snr_db=20.0, rng=rng)
    dev = torch.device("cuda:0")
    t = {k: torch.tensor(v, device=dev) for k, v in
         dict(re=re, im=im, tx=tx, rx=rx, vox=scenes.voxel_grid(n, size=0.12)).items()}
    return t, ch


def _regular(t, ch):
    lib = _lib.load()
    A, S = t["re"].shape
    N = t["vox"].shape[1]
    out_r = torch.full((N,), float("nan"), device="cuda")
    out_i = torch.full((N,), float("nan"), device="cuda")
    need = ctypes.c_size_t(0)
    _lib.check(lib.geraf_mf_forward_workspace_bytes(A, S, N, _lib.DTYPE_F32, _lib.MODE_MIXED, None,
                                                    ctypes.byref(need)), "workspace query")
    ws = torch.empty(max(int(need.value), 1), dtype=torch.uint8, device="cuda")
    _lib.check(lib.geraf_mf_forward(t["re"].data_ptr(), t["im"].data_ptr(), t["tx"].data_ptr(),
                                    t["rx"].data_ptr(), out_r.data_ptr(), out_i.data_ptr(),
                                    t["vox"].data_ptr(), A, S, ch.adc_sample_rate, ch.As_sci, N,
                                    _lib.DTYPE_F32, _lib.MODE_MIXED, None, ws.data_ptr(), need.value,
                                    torch.cuda.current_stream().cuda_stream), "geraf_mf_forward")
    return out_r, out_i


def _noalloc(t, ch):
    lib = _lib.load()
    A, S = t["re"].shape
    N = t["vox"].shape[1]
    out_r = torch.full((N,), float("nan"), device="cuda")
    out_i = torch.full((N,), float("nan"), device="cuda")
    rc = lib.geraf_mf_forward_noalloc(t["re"].data_ptr(), t["im"].data_ptr(), t["tx"].data_ptr(),
                                      t["rx"].data_ptr(), out_r.data_ptr(), out_i.data_ptr(),
                                      t["vox"].data_ptr(), A, S, ch.adc_sample_rate, ch.As_sci, N,
                                      torch.cuda.current_stream().cuda_stream)
    _lib.check(rc, "geraf_mf_forward_noalloc")
    return out_r, out_i


def test_noalloc_matches_regular_entry_point_twice_in_a_row(cuda):
    # Two calls in a row on different problems: the second, smaller one reuses
    # the scratch the first one filled.
    for seed, scan, S, n in ((0, 4, 64, 20), (1, 3, 40, 9)):
        t, ch = _case(seed, scan, S, n)
        ref_r, ref_i = _regular(t, ch)
        got_r, got_i = _noalloc(t, ch)
        torch.cuda.synchronize()
        ref = ref_r.double().cpu().numpy() + 1j * ref_i.double().cpu().numpy()
        got = got_r.double().cpu().numpy() + 1j * got_i.double().cpu().numpy()
        assert np.isfinite(got).all()
        assert rel_l2(got, ref) < TOL, (seed, rel_l2(got, ref))


def test_noalloc_with_fewer_antennas_than_one_stage(cuda):
    """4 antennas fill less than one 8-antenna stage, so the second of the two
    forced partial sums covers no antenna and must contribute exactly zero."""
    t, ch = _case(2, 1, 48, 7, n_tx=1, n_rx=4)
    assert t["re"].shape[0] == 4
    ref_r, ref_i = _regular(t, ch)
    got_r, got_i = _noalloc(t, ch)
    torch.cuda.synchronize()
    ref = ref_r.double().cpu().numpy() + 1j * ref_i.double().cpu().numpy()
    got = got_r.double().cpu().numpy() + 1j * got_i.double().cpu().numpy()
    assert np.isfinite(got).all()
    assert rel_l2(got, ref) < TOL


def test_noalloc_without_antennas_matches_regular_nan(cuda):
    """No antennas: the reference divides a zero sum by zero antennas, so both
    entry points write NaN."""
    t, ch = _case(3, 2, 32, 5)
    t = dict(t, re=t["re"][:0].contiguous(), im=t["im"][:0].contiguous(), tx=t["tx"][:0].contiguous(),
             rx=t["rx"][:0].contiguous())
    ref_r, ref_i = _regular(t, ch)
    got_r, got_i = _noalloc(t, ch)
    torch.cuda.synchronize()
    assert torch.isnan(ref_r).all() and torch.isnan(ref_i).all()
    assert torch.isnan(got_r).all() and torch.isnan(got_i).all()


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    lib = _lib.load()
    rc = lib.geraf_mf_forward_noalloc(None, None, None, None, None, None, None, 8, 8, 5e6, 1e6,
                                      (1 << 20) + 1, None)
    assert rc == _lib.GERAF_ERR_INVALID_ARGUMENT
    assert b"exceeds the fixed scratch" in lib.geraf_rf_last_error()
