"""Matched filter on the GPU vs the CPU FP64 oracle: error bounds of both forms,
adjoint identity, launch-shape invariance, element types, edge cases and the
autograd wrappers."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from benchkit import scenes
from gpu_helpers import cu, mf_backward, mf_forward
from oracle import rf_oracle as orc

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-4   # bound stated for the mixed form vs FP64
PLAIN_TOL = 5e-4   # the reference's own FP32 level vs FP64


def scene_case(seed=0, scan=4, S=64, k=8, n=9, snr=20.0):
    rng = np.random.default_rng(seed)
    tx, rx = scenes.virtual_array(scan)
    pos, amp = scenes.point_scene(rng, k, size=0.12)
    ch = scenes.chirp(S)
    re, im = scenes.synthesize_if_numpy(tx, rx, pos, amp, ch, snr_db=snr, rng=rng)
    return dict(re=re, im=im, tx=tx, rx=rx, vox=scenes.voxel_grid(n, size=0.12), ch=ch)


@pytest.fixture(scope="module")
def case():
    return scene_case()


def test_forward_forms_vs_fp64(cuda, case):
    c, ch = case, case["ch"]
    ref = orc.mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci)
    ref = ref[0] + 1j * ref[1]
    mr, mi = mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci, "mixed")
    pr, pi = mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci, "plain")
    err_mixed = rel_l2(mr + 1j * mi, ref)
    err_plain = rel_l2(pr + 1j * pi, ref)
    assert err_mixed < MIXED_TOL
    assert err_plain < PLAIN_TOL
    assert err_mixed < err_plain  # the mixed form is the more accurate one


def test_backward_forms_vs_fp64(cuda, case):
    c, ch = case, case["ch"]
    A, S = c["re"].shape
    rng = np.random.default_rng(4)
    gr = rng.standard_normal(c["vox"].shape[1]).astype(np.float32)
    gi = rng.standard_normal(c["vox"].shape[1]).astype(np.float32)
    ref = orc.mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, ch.adc_sample_rate, ch.As_sci)
    ref = ref[0] + 1j * ref[1]
    for prec, tol in (("mixed", MIXED_TOL), ("plain", PLAIN_TOL)):
        hr, hi = mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, ch.adc_sample_rate, ch.As_sci, prec)
        assert rel_l2(hr + 1j * hi, ref) < tol, prec


@pytest.mark.parametrize("prec", ["mixed", "plain"])
def test_adjoint_identity(cuda, case, prec):
    c, ch = case, case["ch"]
    A, S = c["re"].shape
    N = c["vox"].shape[1]
    rng = np.random.default_rng(9)
    sr, si = rng.standard_normal((A, S)).astype(np.float32), rng.standard_normal((A, S)).astype(np.float32)
    gr, gi = rng.standard_normal(N).astype(np.float32), rng.standard_normal(N).astype(np.float32)
    yr, yi = mf_forward(sr, si, c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci, prec)
    hr, hi = mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, ch.adc_sample_rate, ch.As_sci, prec)
    lhs = gr @ yr + gi @ yi
    rhs = np.sum(hr * sr) + np.sum(hi * si)
    assert abs(lhs - rhs) < 2e-4 * (np.linalg.norm(yr) * np.linalg.norm(gr) + 1e-30) * 4


@pytest.mark.parametrize("tuning", [
    {"threads": 64, "items_per_thread": 1, "stage_rows": 1},
    {"threads": 128, "items_per_thread": 2, "stage_rows": 8},
    {"threads": 256, "items_per_thread": 4, "stage_rows": 16, "splits": 3},
    {"threads": 128, "items_per_thread": 2, "stage_rows": 4, "splits": 7},
])
def test_forward_launch_shapes_agree(cuda, case, tuning):
    c, ch = case, case["ch"]
    base = mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci, "mixed")
    alt = mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci,
                     "mixed", tuning=tuning)
    assert rel_l2(alt[0] + 1j * alt[1], base[0] + 1j * base[1]) < 2e-6
    plain = mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci,
                       "plain", tuning={k: v for k, v in tuning.items() if k != "splits"})
    plain0 = mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci, "plain")
    # the plain form keeps one accumulator per voxel in reference order: shape-independent bits
    np.testing.assert_array_equal(plain[0], plain0[0])
    np.testing.assert_array_equal(plain[1], plain0[1])


@pytest.mark.parametrize("tuning", [
    {"threads": 128, "chunk": 8}, {"threads": 256, "chunk": 32}, {"threads": 64, "chunk": 16, "splits": 5},
])
def test_backward_launch_shapes_agree(cuda, case, tuning):
    c, ch = case, case["ch"]
    A, S = c["re"].shape
    rng = np.random.default_rng(2)
    gr = rng.standard_normal(c["vox"].shape[1]).astype(np.float32)
    gi = rng.standard_normal(c["vox"].shape[1]).astype(np.float32)
    base = mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, ch.adc_sample_rate, ch.As_sci, "mixed")
    alt = mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, ch.adc_sample_rate, ch.As_sci, "mixed",
                      tuning=tuning)
    assert rel_l2(alt[0] + 1j * alt[1], base[0] + 1j * base[1]) < 2e-6


def test_unaligned_inputs_use_copy_path(cuda, case):
    """Row views that break 16-byte alignment go through the cooperative copy path."""
    from geraf_b200.ops.RFMatchedFilter import _C

    c, ch = case, case["ch"]
    A, S = c["re"].shape
    N = c["vox"].shape[1]
    big_r = torch.zeros(A * S + 1, device="cuda")
    big_i = torch.zeros(A * S + 1, device="cuda")
    big_r[1:] = cu(c["re"]).reshape(-1)
    big_i[1:] = cu(c["im"]).reshape(-1)
    re_v, im_v = big_r[1:].view(A, S), big_i[1:].view(A, S)
    assert re_v.data_ptr() % 16 != 0
    for prec in ("mixed", "plain"):
        out_r = torch.empty(N, device="cuda")
        out_i = torch.empty(N, device="cuda")
        _C.MatchedFilter_forward(re_v, im_v, cu(c["tx"]), cu(c["rx"]), out_r, out_i, cu(c["vox"]), A,
                                 S, ch.adc_sample_rate, ch.As_sci, N, precision=prec)
        base = mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci, prec)
        assert rel_l2(out_r.double().cpu().numpy() + 1j * out_i.double().cpu().numpy(),
                      base[0] + 1j * base[1]) < 1e-6


@pytest.mark.parametrize("S", [1, 3, 5, 130])
def test_odd_sample_counts(cuda, S):
    c = scene_case(seed=3, scan=2, S=S, k=3, n=4)
    ch = c["ch"]
    ref = orc.mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci)
    for prec, tol in (("mixed", MIXED_TOL), ("plain", PLAIN_TOL)):
        yr, yi = mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci, prec)
        assert rel_l2(yr + 1j * yi, ref[0] + 1j * ref[1]) < tol, (prec, S)


def test_float64_and_float16_inputs(cuda, case):
    """Other element types: the oracle sees the inputs rounded to that type
    (half-precision voxel coordinates alone move the phase by ~0.5 rad)."""
    c, ch = case, case["ch"]
    for dt, npdt, tol in ((torch.float64, np.float64, MIXED_TOL), (torch.float16, np.float16, 2e-3)):
        r = {k: c[k].astype(npdt).astype(np.float32) for k in ("re", "im", "tx", "rx", "vox")}
        ref = orc.mf_forward(r["re"], r["im"], r["tx"], r["rx"], r["vox"], ch.adc_sample_rate, ch.As_sci)
        yr, yi = mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci,
                            "mixed", dtype=dt)
        # half outputs carry 11-bit rounding (~3e-4 relative L2)
        assert rel_l2(yr + 1j * yi, ref[0] + 1j * ref[1]) < tol, dt


def test_empty_and_degenerate_sizes(cuda):
    from geraf_b200.ops.RFMatchedFilter import _C

    c = scene_case(seed=1, scan=2, S=8, k=2, n=3)
    ch = c["ch"]
    A, S = c["re"].shape
    # N = 0: nothing to do
    e = torch.empty(0, device="cuda")
    _C.MatchedFilter_forward(cu(c["re"]), cu(c["im"]), cu(c["tx"]), cu(c["rx"]), e, e,
                             torch.empty((3, 0), device="cuda"), A, S, ch.adc_sample_rate, ch.As_sci, 0)
    # A = 0: the reference divides 0 by 0 -> NaN, in both forms
    for prec in ("plain", "mixed"):
        out_r = torch.zeros(5, device="cuda")
        out_i = torch.zeros(5, device="cuda")
        _C.MatchedFilter_forward(torch.empty((0, S), device="cuda"), torch.empty((0, S), device="cuda"),
                                 torch.empty((0, 3), device="cuda"), torch.empty((0, 3), device="cuda"),
                                 out_r, out_i, cu(c["vox"][:, :5]), 0, S, ch.adc_sample_rate,
                                 ch.As_sci, 5, precision=prec)
        assert torch.isnan(out_r).all() and torch.isnan(out_i).all()
    # S = 0: zero output
    out_r = torch.full((5,), 7.0, device="cuda")
    out_i = torch.full((5,), 7.0, device="cuda")
    _C.MatchedFilter_forward(torch.empty((A, 0), device="cuda"), torch.empty((A, 0), device="cuda"),
                             cu(c["tx"]), cu(c["rx"]), out_r, out_i, cu(c["vox"][:, :5]), A, 0,
                             ch.adc_sample_rate, ch.As_sci, 5)
    assert (out_r == 0).all() and (out_i == 0).all()
    # backward with N = 0: zero gradients
    g_r = torch.full((A, S), 7.0, device="cuda")
    g_i = torch.full((A, S), 7.0, device="cuda")
    _C.MatchedFilter_backward_realimag(e, e, cu(c["re"]), cu(c["im"]), cu(c["tx"]), cu(c["rx"]), g_r,
                                       g_i, torch.empty((3, 0), device="cuda"), A, S,
                                       ch.adc_sample_rate, ch.As_sci, 0)
    assert (g_r == 0).all() and (g_i == 0).all()


def test_drop_in_errors(cuda, case):
    from geraf_b200.ops.RFMatchedFilter import _C, matched_filter_cuda

    c, ch = case, case["ch"]
    A, S = c["re"].shape
    N = c["vox"].shape[1]
    out = torch.empty(N, device="cuda")
    with pytest.raises(RuntimeError, match="`voxel` must be laid out as"):
        _C.MatchedFilter_forward(cu(c["re"]), cu(c["im"]), cu(c["tx"]), cu(c["rx"]), out, out,
                                 cu(c["vox"].T.copy()), A, S, 5e6, 1.0, N)
    with pytest.raises(RuntimeError, match="`real` must be a CUDA tensor"):
        _C.MatchedFilter_forward(torch.zeros(A, S), cu(c["im"]), cu(c["tx"]), cu(c["rx"]), out, out,
                                 cu(c["vox"]), A, S, 5e6, 1.0, N)
    with pytest.raises(RuntimeError, match="must be contiguous"):
        _C.MatchedFilter_forward(cu(c["re"]).t(), cu(c["im"]), cu(c["tx"]), cu(c["rx"]), out, out,
                                 cu(c["vox"]), A, S, 5e6, 1.0, N)
    with pytest.raises(AssertionError):
        matched_filter_cuda(cu(c["re"]), cu(c["im"]), cu(c["tx"]), cu(c["rx"]), cu(c["vox"]), A, S,
                            5e6, 1.0, N)  # voxel must be [N,3] at this level
    with pytest.raises(AssertionError):
        matched_filter_cuda(torch.zeros(A, S), cu(c["im"]), cu(c["tx"]), cu(c["rx"]),
                            cu(c["vox"].T.copy()), A, S, 5e6, 1.0, N)


def test_autograd_wrapper_and_gating(cuda, case):
    from geraf_b200.ops.RFMatchedFilter import matched_filter_cuda

    c, ch = case, case["ch"]
    A, S = c["re"].shape
    N = c["vox"].shape[1]
    re = cu(c["re"]).requires_grad_(True)
    im = cu(c["im"]).requires_grad_(True)
    vox = cu(c["vox"].T.copy())
    yr, yi = matched_filter_cuda(re, im, cu(c["tx"]), cu(c["rx"]), vox, A, S, ch.adc_sample_rate,
                                 ch.As_sci, N)
    rng = np.random.default_rng(0)
    gr, gi = rng.standard_normal(N).astype(np.float32), rng.standard_normal(N).astype(np.float32)
    (yr * cu(gr)).sum().add((yi * cu(gi)).sum()).backward()
    hr, hi = mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, ch.adc_sample_rate, ch.As_sci, None)
    assert rel_l2(re.grad.double().cpu().numpy() + 1j * im.grad.double().cpu().numpy(), hr + 1j * hi) < 1e-6
    # only one of (real, image) requiring grad -> no gradient computed (reference :175)
    re2 = cu(c["re"]).requires_grad_(True)
    yr, yi = matched_filter_cuda(re2, cu(c["im"]), cu(c["tx"]), cu(c["rx"]), vox, A, S,
                                 ch.adc_sample_rate, ch.As_sci, N)
    (yr.sum() + yi.sum()).backward()
    assert re2.grad is None


def test_faster_matched_filter_split(cuda, case):
    from geraf_b200.ops.RFMatchedFilter import faster_matched_filter_cuda, matched_filter_cuda

    c, ch = case, case["ch"]
    A, S = c["re"].shape
    N = c["vox"].shape[1]
    k = 70
    vox = cu(c["vox"].T.copy())
    re = cu(c["re"])
    im = cu(c["im"])
    tx, rx = cu(c["tx"]), cu(c["rx"])
    full = matched_filter_cuda(re, im, tx, rx, vox, A, S, ch.adc_sample_rate, ch.As_sci, N)
    rs = re[:k].clone().requires_grad_(True)
    is_ = im[:k].clone().requires_grad_(True)
    yr, yi = faster_matched_filter_cuda(rs, is_, re[k:], im[k:], tx[:k], rx[:k], tx[k:], rx[k:], vox, A,
                                        k, S, ch.adc_sample_rate, ch.As_sci, N)
    assert torch.allclose(yr, full[0]) and torch.allclose(yi, full[1])
    gr = torch.randn(N, device="cuda")
    gi = torch.randn(N, device="cuda")
    ((yr * gr).sum() + (yi * gi).sum()).backward()
    hr, hi = mf_backward(gr.cpu().numpy(), gi.cpu().numpy(), c["tx"][:k], c["rx"][:k], c["vox"], k, S,
                         ch.adc_sample_rate, ch.As_sci, None)
    # adjoint over the selected antennas, rescaled from 1/num_sel to 1/total
    assert rel_l2(rs.grad.double().cpu().numpy(), hr * k / A) < 1e-6
    assert rel_l2(is_.grad.double().cpu().numpy(), hi * k / A) < 1e-6


def test_model_utils_adapters(cuda, case):
    from geraf_b200 import model_utils

    c, ch = case, case["ch"]
    N = c["vox"].shape[1]
    cfg = ch.radar_cfg()
    yr, yi = model_utils.base_matched_filter(cu(c["re"]), cu(c["im"]), cu(c["tx"]), cu(c["rx"]),
                                             cu(c["vox"].T.copy()), cfg)
    base = mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci, None)
    assert yr.shape == (N,)
    assert rel_l2(yr.double().cpu().numpy() + 1j * yi.double().cpu().numpy(), base[0] + 1j * base[1]) < 1e-7
    with pytest.raises(ValueError):
        model_utils.base_matched_filter(cu(c["re"]), cu(c["im"]), cu(c["tx"]), cu(c["rx"]),
                                        cu(c["vox"].T.copy()), cfg, backend="torch")


@pytest.mark.parametrize("S", [512, 576, 1024], ids=["8_blocks", "9_blocks", "16_blocks"])
def test_mixed_long_rows_vs_fp64(cuda, S):
    """The forward's rows of up to 8 blocks of 64 samples take the hardware phasor
    for the block rotator z^64, longer rows the accurate one; the adjoint's group
    rotator switches the same way above 8 sample groups (these rows have 16 to 64).
    Both sides of the switch stay two orders of magnitude inside the MIXED bound."""
    c = scene_case(seed=5, scan=2, S=S, k=6, n=7)
    ch = c["ch"]
    A = c["re"].shape[0]
    ref = orc.mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci)
    mr, mi = mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], ch.adc_sample_rate, ch.As_sci, "mixed")
    assert rel_l2(mr + 1j * mi, ref[0] + 1j * ref[1]) < 1e-5
    rng = np.random.default_rng(6)
    gr = rng.standard_normal(c["vox"].shape[1]).astype(np.float32)
    gi = rng.standard_normal(c["vox"].shape[1]).astype(np.float32)
    bref = orc.mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, ch.adc_sample_rate, ch.As_sci)
    for tun in (None, {"threads": 64, "chunk": 32}):
        hr, hi = mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, ch.adc_sample_rate, ch.As_sci, "mixed",
                             tuning=tun)
        assert rel_l2(hr + 1j * hi, bref[0] + 1j * bref[1]) < 1e-5, tun


def test_mixed_near_field_block_lengths_vs_fp64(cuda):
    """Voxels 1 cm to 30 cm in front of the array at the 256-sample chirp: the
    per-sample phase step theta runs from about 0.05 to 0.25 rad, so the forward's
    voxels restart their recurrence every 64 samples (|sin theta| < 0.1, the near
    ones) or every 128 (the rest), both within the same launch and thread."""
    rng = np.random.default_rng(9)
    tx, rx = scenes.virtual_array(2)
    ch = scenes.chirp(256)
    pos = np.stack([rng.uniform(-0.04, 0.04, 12), rng.uniform(-0.04, 0.04, 12), rng.uniform(0.02, 0.28, 12)], 1)
    amp = rng.standard_normal(12) + 1j * rng.standard_normal(12)
    re, im = scenes.synthesize_if_numpy(tx, rx, pos, amp, ch, snr_db=20.0, rng=rng)
    g = np.linspace(-0.05, 0.05, 6)
    z = np.linspace(0.01, 0.30, 24)
    vx, vy, vz = np.meshgrid(g, g, z, indexing="ij")
    vox = np.stack([vx.ravel(), vy.ravel(), vz.ravel()]).astype(np.float32)
    d = (np.linalg.norm(tx[:, None, :] - vox.T[None], axis=2) + np.linalg.norm(rx[:, None, :] - vox.T[None], axis=2))
    k1 = (np.float32(np.pi) / np.pi) * ch.As_sci / (ch.adc_sample_rate * 2.9979)
    sin_theta = np.abs(np.sin(2 * np.pi * (d + 0.15) * k1))
    assert (sin_theta < 0.1).any() and (sin_theta >= 0.1).any()
    ref = orc.mf_forward(re, im, tx, rx, vox, ch.adc_sample_rate, ch.As_sci)
    mr, mi = mf_forward(re, im, tx, rx, vox, ch.adc_sample_rate, ch.As_sci, "mixed")
    assert rel_l2(mr + 1j * mi, ref[0] + 1j * ref[1]) < 1e-5
