"""The matched filter's NUFFT form on the GPU: error against the FP64 oracle per
interpolation width, the adjoint identity (the NUFFT adjoint is the transpose
of the NUFFT forward), element types, odd and edge sizes, launch shapes, the
autograd wrapper and the argument checks."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from benchkit import scenes
from gpu_helpers import cu, mf_backward, mf_forward
from oracle import rf_oracle as orc

pytestmark = pytest.mark.gpu

# FP32 library: the model's truncation error (tests/test_nufft_model.py) plus rounding
TOL = {4: 3e-3, 6: 5e-5, 8: 5e-6, 12: 5e-6}


def scene_case(seed=0, scan=4, S=64, k=8, n=9):
    rng = np.random.default_rng(seed)
    tx, rx = scenes.virtual_array(scan)
    pos, amp = scenes.point_scene(rng, k, size=0.12)
    ch = scenes.chirp(S)
    re, im = scenes.synthesize_if_numpy(tx, rx, pos, amp, ch, snr_db=20.0, rng=rng)
    return dict(re=re, im=im, tx=tx, rx=rx, vox=scenes.voxel_grid(n, size=0.12), ch=ch)


@pytest.fixture(scope="module")
def case():
    return scene_case()


def oracle_fwd(c):
    ch = c["ch"]
    r = orc.mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci)
    return r[0] + 1j * r[1]


@pytest.mark.parametrize("taps", sorted(TOL))
def test_forward_vs_fp64(cuda, case, taps, parity_log):
    c, ch = case, case["ch"]
    ref = oracle_fwd(c)
    yr, yi = mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci,
                        "nufft", tuning={"taps": taps})
    err = rel_l2(yr + 1j * yi, ref)
    parity_log(f"mf_nufft_forward_W{taps}_vs_fp64", rel_l2=err)
    assert err < TOL[taps]


def test_backward_vs_fp64(cuda, case, parity_log):
    c, ch = case, case["ch"]
    A, S = c["re"].shape
    rng = np.random.default_rng(4)
    gr = rng.standard_normal(c["vox"].shape[1]).astype(np.float32)
    gi = rng.standard_normal(c["vox"].shape[1]).astype(np.float32)
    ref = orc.mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, ch.adc_sample_rate, ch.As_sci)
    ref = ref[0] + 1j * ref[1]
    hr, hi = mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, ch.adc_sample_rate, ch.As_sci, "nufft")
    err = rel_l2(hr + 1j * hi, ref)
    parity_log("mf_nufft_adjoint_W8_vs_fp64", rel_l2=err)
    assert err < TOL[8]


@pytest.mark.parametrize("taps", [4, 8])
def test_adjoint_identity(cuda, case, taps):
    """<F s, g> = <s, F^T g> for the NUFFT pair itself, far below its truncation error."""
    c, ch = case, case["ch"]
    A, S = c["re"].shape
    N = c["vox"].shape[1]
    rng = np.random.default_rng(9)
    sr, si = rng.standard_normal((A, S)).astype(np.float32), rng.standard_normal((A, S)).astype(np.float32)
    gr, gi = rng.standard_normal(N).astype(np.float32), rng.standard_normal(N).astype(np.float32)
    t = {"taps": taps}
    yr, yi = mf_forward(sr, si, c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci, "nufft", tuning=t)
    hr, hi = mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, ch.adc_sample_rate, ch.As_sci, "nufft",
                         tuning=t)
    lhs = gr @ yr + gi @ yi
    rhs = np.sum(hr * sr) + np.sum(hi * si)
    scale = np.linalg.norm(yr + 1j * yi) * np.linalg.norm(gr + 1j * gi)
    assert abs(lhs - rhs) < 2e-6 * scale


@pytest.mark.parametrize("S", [1, 2, 37, 101, 128])
def test_odd_and_small_sample_counts(cuda, S):
    c = scene_case(seed=S, scan=2, S=S, k=4, n=5)
    ch = c["ch"]
    ref = oracle_fwd(c)
    yr, yi = mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci, "nufft")
    assert rel_l2(yr + 1j * yi, ref) < TOL[8]
    A = c["re"].shape[0]
    rng = np.random.default_rng(S)
    N = c["vox"].shape[1]
    gr, gi = rng.standard_normal(N).astype(np.float32), rng.standard_normal(N).astype(np.float32)
    ref_b = orc.mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, ch.adc_sample_rate, ch.As_sci)
    hr, hi = mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, ch.adc_sample_rate, ch.As_sci, "nufft")
    assert rel_l2(hr + 1j * hi, ref_b[0] + 1j * ref_b[1]) < TOL[8]


@pytest.mark.parametrize("dtype,tol", [(torch.float64, TOL[8]), (torch.float16, 2e-3)])
def test_element_types(cuda, case, dtype, tol):
    c, ch = case, case["ch"]
    if dtype == torch.float16:
        # checked against the oracle on the half-rounded inputs
        c = {k: (v.astype(np.float16).astype(np.float32) if isinstance(v, np.ndarray) else v)
             for k, v in c.items()}
    ref = oracle_fwd(c)
    yr, yi = mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci,
                        "nufft", dtype=dtype)
    assert rel_l2(yr + 1j * yi, ref) < tol


@pytest.mark.parametrize("tuning", [
    {"threads": 64, "items_per_thread": 1, "stage_rows": 1},
    {"threads": 256, "items_per_thread": 2, "stage_rows": 16, "splits": 3},
    {"threads": 128, "items_per_thread": 4, "stage_rows": 4, "splits": 7},
])
def test_launch_shapes_agree(cuda, case, tuning):
    c, ch = case, case["ch"]
    base = mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci, "nufft")
    alt = mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci, "nufft",
                     tuning=tuning)
    assert rel_l2(alt[0] + 1j * alt[1], base[0] + 1j * base[1]) < 2e-6
    A, S = c["re"].shape
    rng = np.random.default_rng(2)
    N = c["vox"].shape[1]
    gr, gi = rng.standard_normal(N).astype(np.float32), rng.standard_normal(N).astype(np.float32)
    b0 = mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, ch.adc_sample_rate, ch.As_sci, "nufft")
    b1 = mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, ch.adc_sample_rate, ch.As_sci, "nufft",
                     tuning={k: v for k, v in tuning.items() if k != "items_per_thread"})
    assert rel_l2(b1[0] + 1j * b1[1], b0[0] + 1j * b0[1]) < 2e-6


def test_adjoint_band_paths_agree(cuda, case):
    """Scattered voxels far apart in range push every antenna's band past the
    private-window width (the shared-row path); the two paths agree, and no
    device check fired."""
    from geraf_b200 import _lib

    c, ch = case, case["ch"]
    A, S = c["re"].shape
    rng = np.random.default_rng(11)
    wide = np.concatenate([c["vox"], (rng.uniform(-1.0, 1.0, (3, 40)) + np.array([[0.0], [0.0], [3.0]]))],
                          1).astype(np.float32)
    N = wide.shape[1]
    gr, gi = rng.standard_normal(N).astype(np.float32), rng.standard_normal(N).astype(np.float32)
    ref = orc.mf_backward(gr, gi, c["tx"], c["rx"], wide, A, S, ch.adc_sample_rate, ch.As_sci)
    hr, hi = mf_backward(gr, gi, c["tx"], c["rx"], wide, A, S, ch.adc_sample_rate, ch.As_sci, "nufft")
    assert rel_l2(hr + 1j * hi, ref[0] + 1j * ref[1]) < TOL[8]
    assert _lib.device_status() == _lib.GERAF_OK


def test_adjoint_is_deterministic(cuda, case):
    c, ch = case, case["ch"]
    A, S = c["re"].shape
    rng = np.random.default_rng(12)
    N = c["vox"].shape[1]
    gr, gi = rng.standard_normal(N).astype(np.float32), rng.standard_normal(N).astype(np.float32)
    runs = [mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, ch.adc_sample_rate, ch.As_sci, "nufft")
            for _ in range(3)]
    for r in runs[1:]:
        np.testing.assert_array_equal(r[0], runs[0][0])
        np.testing.assert_array_equal(r[1], runs[0][1])


def test_empty_voxels_give_zero_gradient(cuda, case):
    c, ch = case, case["ch"]
    A, S = c["re"].shape
    empty = np.zeros((3, 0), np.float32)
    hr, hi = mf_backward(np.zeros(0, np.float32), np.zeros(0, np.float32), c["tx"], c["rx"], empty, A, S,
                         ch.adc_sample_rate, ch.As_sci, "nufft")
    assert np.all(hr == 0) and np.all(hi == 0)


def test_autograd_uses_the_nufft_adjoint(cuda, case):
    from geraf_b200.ops.RFMatchedFilter import matched_filter_cuda

    c, ch = case, case["ch"]
    A, S = c["re"].shape
    N = c["vox"].shape[1]
    re = cu(c["re"]).requires_grad_(True)
    im = cu(c["im"]).requires_grad_(True)
    vox = cu(c["vox"].T.copy())
    yr, yi = matched_filter_cuda(re, im, cu(c["tx"]), cu(c["rx"]), vox, A, S, ch.adc_sample_rate, ch.As_sci, N,
                                 precision="nufft", tuning={"taps": 6})
    rng = np.random.default_rng(5)
    gr, gi = rng.standard_normal(N).astype(np.float32), rng.standard_normal(N).astype(np.float32)
    (yr * cu(gr) + yi * cu(gi)).sum().backward()
    hr, hi = mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, ch.adc_sample_rate, ch.As_sci, "nufft",
                         tuning={"taps": 6})
    assert rel_l2(re.grad.double().cpu().numpy(), hr) < 1e-5
    assert rel_l2(im.grad.double().cpu().numpy(), hi) < 1e-5


def test_argument_checks(cuda, case):
    from geraf_b200.ops.RFMatchedFilter import _C
    from geraf_b200.ops.RFSignalTracer import _C as _T

    c, ch = case, case["ch"]
    A = 4
    S = 5000  # above the NUFFT limit of 4096 samples
    z = torch.zeros((A, S), device="cuda")
    pos = torch.zeros((A, 3), device="cuda")
    vox = torch.zeros((3, 8), device="cuda")
    out = torch.empty(8, device="cuda")
    with pytest.raises(RuntimeError, match="4096"):
        _C.MatchedFilter_forward(z, z, pos, pos, out, out.clone(), vox, A, S, 5e6, 1e6, 8, precision="nufft")
    xr = torch.empty((A, S), device="cuda")
    with pytest.raises(RuntimeError, match="4096"):
        _T.SignalTracer_forward(torch.zeros((8, 3), device="cuda"), torch.zeros((A, 8), device="cuda"),
                                torch.zeros((8, 3), device="cuda"), pos, pos,
                                torch.ones(8, dtype=torch.bool, device="cuda"), xr, xr.clone(), S, 5e6,
                                770.0, 1e6, A, 8, precision="nufft")
