"""Parity with the REFERENCE's own CUDA kernels: golden vectors produced by the
unmodified GeRaF extensions (tests/golden/make_golden.py) vs this library's
kernels through the drop-in ``_C`` modules.

Bars: the PLAIN form within relative L2 1e-5 of the reference (it evaluates
the reference's FP32 expressions in the reference's summation order); the
MIXED form within 1e-4 of the FP64 oracle (tests/test_gpu_mf.py) -- against
the reference it can only be as close as the reference is to FP64 (~1e-4)."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from gpu_helpers import cu, golden_cases, load_golden, mf_backward, mf_forward, tracer_backward, tracer_forward
from oracle import rf_oracle as orc

pytestmark = pytest.mark.gpu

PLAIN_TOL = 1e-5


def bitexact(a, b):
    """Fraction of elements equal to the last bit (complex pairs count once)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.mean(a == b))


def _dtype(name):
    return {"f32": torch.float32, "f16": torch.float16, "f64": torch.float64}[name.rsplit("_", 1)[1]]


@pytest.mark.parametrize("name", [c for c in golden_cases("mf_") if "fft" not in c])
def test_mf_plain_matches_reference(cuda, name, parity_log):
    g = load_golden(name)
    dt = _dtype(name)
    yr, yi = mf_forward(g["real"], g["imag"], g["tx"], g["rx"], g["voxel"], g["fs"], g["As"],
                        "plain", dt)
    ref = g["out_real"] + 1j * g["out_imag"]
    tol = PLAIN_TOL if dt != torch.float16 else 2e-3  # f16 outputs are rounded to 11 bits
    A, S = g["real"].shape
    hr, hi = mf_backward(g["grad_output_real"], g["grad_output_imag"], g["tx"], g["rx"], g["voxel"],
                         A, S, g["fs"], g["As"], "plain", dt)
    e_f = rel_l2(yr + 1j * yi, ref)
    e_b = rel_l2(hr + 1j * hi, g["grad_real"] + 1j * g["grad_imag"])
    bx_f = bitexact(np.r_[yr, yi], np.r_[g["out_real"], g["out_imag"]])
    bx_b = bitexact(np.r_[hr.ravel(), hi.ravel()], np.r_[g["grad_real"].ravel(), g["grad_imag"].ravel()])
    parity_log(f"mf_plain_vs_reference[{name}]", forward_rel_l2=e_f, adjoint_rel_l2=e_b,
               forward_bitexact=bx_f, adjoint_bitexact=bx_b)
    assert e_f < tol
    assert e_b < tol
    # same FP32 expressions, same per-output order: every output bit equals the reference's
    assert bx_f == 1.0 and bx_b == 1.0


@pytest.mark.parametrize("name", [c for c in golden_cases("mf_") if "fft" not in c])
def test_mf_mixed_close_to_reference(cuda, name, parity_log):
    """The mixed form differs from the reference by about the reference's own FP32 error."""
    g = load_golden(name)
    dt = _dtype(name)
    yr, yi = mf_forward(g["real"], g["imag"], g["tx"], g["rx"], g["voxel"], g["fs"], g["As"],
                        "mixed", dt)
    e = rel_l2(yr + 1j * yi, g["out_real"] + 1j * g["out_imag"])
    parity_log(f"mf_mixed_vs_reference[{name}]", forward_rel_l2=e)
    assert e < 1e-3


@pytest.mark.parametrize("name", golden_cases("mf_fft"))
def test_mf_fft_matches_reference(cuda, name):
    from geraf_b200.ops.RFMatchedFilter import _C

    g = load_golden(name)
    A, B = g["spec_real"].shape
    N = g["voxel"].shape[1]
    out_r = torch.full((N,), float("nan"), device="cuda")
    out_i = torch.full((N,), float("nan"), device="cuda")
    args = [cu(g["spec_real"]), cu(g["spec_imag"]), cu(g["tx"]), cu(g["rx"])]
    _C.MatchedFilter_fft_forward(*args, out_r, out_i, cu(g["voxel"]), A, B, float(g["spacing"]),
                                 float(g["fs"]), float(g["As"]), N)
    assert rel_l2(out_r.cpu().numpy() + 1j * out_i.cpu().numpy(), g["out_real"] + 1j * g["out_imag"]) < PLAIN_TOL
    g_r = torch.full((A, B), float("nan"), device="cuda")
    g_i = torch.full((A, B), float("nan"), device="cuda")
    _C.MatchedFilter_fft_backward_realimag(cu(g["grad_output_real"]), cu(g["grad_output_imag"]),
                                           *args, g_r, g_i, cu(g["voxel"]), A, B,
                                           float(g["spacing"]), float(g["fs"]), float(g["As"]), N)
    assert rel_l2(g_r.cpu().numpy() + 1j * g_i.cpu().numpy(), g["grad_real"] + 1j * g["grad_imag"]) < PLAIN_TOL


@pytest.mark.parametrize("name", golden_cases("tracer_"))
def test_tracer_plain_matches_reference(cuda, name, parity_log):
    g = load_golden(name)
    dt = _dtype(name)
    S = int(g["S"])
    xr, xi = tracer_forward(g, S, "plain", dt)
    gn, gs, _ = tracer_backward(g, g["grad_output_real"], g["grad_output_imag"], "plain", dt,
                                with_points=False)
    inb = g["inbounds"].astype(bool)
    parity_log(f"tracer_plain_vs_reference[{name}]",
               forward_rel_l2=rel_l2(xr + 1j * xi, g["out_real"] + 1j * g["out_imag"]),
               forward_bitexact=bitexact(np.r_[xr.ravel(), xi.ravel()],
                                         np.r_[g["out_real"].ravel(), g["out_imag"].ravel()]),
               grad_normals_rel_l2=rel_l2(gn[inb], g["grad_normals"][inb]),
               grad_sigmas_rel_l2=rel_l2(gs[:, inb], g["grad_sigmas"][:, inb]),
               grad_bitexact=bitexact(np.r_[gn[inb].ravel(), gs[:, inb].ravel()],
                                      np.r_[g["grad_normals"][inb].ravel(), g["grad_sigmas"][:, inb].ravel()]))
    assert rel_l2(xr + 1j * xi, g["out_real"] + 1j * g["out_imag"]) < PLAIN_TOL
    if dt == torch.float32:
        # FP32 inputs: every output bit equals the reference's
        assert bitexact(np.r_[xr.ravel(), xi.ravel()], np.r_[g["out_real"].ravel(), g["out_imag"].ravel()]) == 1.0
        assert bitexact(np.r_[gn[inb].ravel(), gs[:, inb].ravel()],
                        np.r_[g["grad_normals"][inb].ravel(), g["grad_sigmas"][:, inb].ravel()]) == 1.0
    # the reference leaves out-of-bounds entries unwritten (NaN-prefilled); this library writes 0
    assert np.all(np.isnan(g["grad_normals"][~inb])) and np.all(gn[~inb] == 0)
    assert np.all(gs[:, ~inb] == 0)
    assert rel_l2(gn[inb], g["grad_normals"][inb]) < PLAIN_TOL
    assert rel_l2(gs[:, inb], g["grad_sigmas"][:, inb]) < PLAIN_TOL


@pytest.mark.parametrize("name", golden_cases("tracer_"))
def test_tracer_mixed_close_to_reference(cuda, name):
    g = load_golden(name)
    dt = _dtype(name)
    S = int(g["S"])
    xr, xi = tracer_forward(g, S, "mixed", dt)
    assert rel_l2(xr + 1j * xi, g["out_real"] + 1j * g["out_imag"]) < 1e-3
    gn, gs, _ = tracer_backward(g, g["grad_output_real"], g["grad_output_imag"], "mixed", dt,
                                with_points=False)
    inb = g["inbounds"].astype(bool)
    assert rel_l2(gn[inb], g["grad_normals"][inb]) < 1e-3
    assert rel_l2(gs[:, inb], g["grad_sigmas"][:, inb]) < 1e-3


@pytest.mark.parametrize("name", golden_cases("bilinear_"))
def test_bilinear_matches_reference_bitwise(cuda, name):
    from geraf_b200.ops.RFSignalTracer import _C

    g = load_golden(name)
    A, R, S = g["sigmas"].shape
    T = g["tgt_z_vals"].shape[1]
    on = torch.full((R, T, 3), float("nan"), device="cuda")
    os_ = torch.full((A, R, T), float("nan"), device="cuda")
    ob = torch.zeros((R, T), dtype=torch.bool, device="cuda")
    _C.BilinearRaysample_forward(cu(g["normals"]), cu(g["sigmas"]), cu(g["z_vals"]),
                                 cu(g["tgt_z_vals"]), on, os_, ob, A, R, S, T)
    np.testing.assert_array_equal(ob.cpu().numpy(), g["out_inbounds"])
    np.testing.assert_array_equal(on.cpu().numpy(), g["out_normals"])
    np.testing.assert_array_equal(os_.cpu().numpy(), g["out_sigmas"])
    gn = cu(g["grad_normals_init"]).clone()
    gs = cu(g["grad_sigmas_init"]).clone()
    _C.BilinearRaysample_backward(cu(g["grad_out_normals"]), cu(g["grad_out_sigmas"]),
                                  cu(g["z_vals"]), cu(g["tgt_z_vals"]), gn, gs, A, R, S, T)
    np.testing.assert_array_equal(gn.cpu().numpy(), g["grad_normals"])
    np.testing.assert_array_equal(gs.cpu().numpy(), g["grad_sigmas"])


ORACLE_FP32_LEVEL = 5e-4  # the FP32 oracle has no fused multiply-adds: the reference's FP32 phase level


def _fft_flag_case(consistent):
    """The range-bin kernels with and without the bound made consistent with the
    bin index (an opt-in fix of MatchedFilter_cuda_kernel.cu:143-148) against the
    FP32 oracle with the same bound; returns the adjoint's non-zero count."""
    from geraf_b200.ops.RFMatchedFilter import _C

    g = load_golden("mf_fft_f32")
    A, B = g["spec_real"].shape
    N = g["voxel"].shape[1]
    spacing = 0.0245  # the scene's delays (0.87-1.0 m) straddle the reference's bound 0.98 m
    args = [cu(g[k]) for k in ("spec_real", "spec_imag", "tx", "rx")]
    out_r = torch.full((N,), float("nan"), device="cuda")
    out_i = torch.full((N,), float("nan"), device="cuda")
    _C.MatchedFilter_fft_forward(*args, out_r, out_i, cu(g["voxel"]), A, B, spacing, float(g["fs"]),
                                 float(g["As"]), N, consistent_bins=consistent)
    h_r = torch.full((A, B), float("nan"), device="cuda")
    h_i = torch.full((A, B), float("nan"), device="cuda")
    _C.MatchedFilter_fft_backward_realimag(cu(g["grad_output_real"]), cu(g["grad_output_imag"]), *args, h_r, h_i,
                                           cu(g["voxel"]), A, B, spacing, float(g["fs"]), float(g["As"]), N,
                                           consistent_bins=consistent)
    torch.cuda.synchronize()
    rr, ri = orc.mf_fft_forward(g["spec_real"], g["spec_imag"], g["tx"], g["rx"], g["voxel"], spacing, consistent)
    hr, hi = orc.mf_fft_backward(g["grad_output_real"], g["grad_output_imag"], g["tx"], g["rx"], g["voxel"], A,
                                 B, spacing, consistent)
    got = out_r.cpu().numpy() + 1j * out_i.cpu().numpy()
    assert rel_l2(got, rr + 1j * ri) < ORACLE_FP32_LEVEL
    assert rel_l2(h_r.cpu().numpy() + 1j * h_i.cpu().numpy(), hr + 1j * hi) < ORACLE_FP32_LEVEL
    return np.count_nonzero(h_r.cpu().numpy())


def test_mf_fft_consistent_bins_flag(cuda):
    """The consistent bound keeps the delays between the reference's bound and
    twice it; below it both agree with the oracle."""
    assert _fft_flag_case(True) > _fft_flag_case(False) > 0

