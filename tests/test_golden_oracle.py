"""Pins the CPU oracle to the REFERENCE's own outputs (golden vectors produced by
the unmodified GeRaF CUDA kernels, tests/golden/make_golden.py).  No GPU needed.

The reference computes in FP32 with its carrier phase (~1.5e3 rad) rounded to
FP32, so against the exact-arithmetic oracle it sits ~1e-4 away; the FP32
reference-order oracle (no fused multiply-adds) sits at the same level.  What
is pinned exactly: the arithmetic model (constants, phase formula, geometry,
culling, normalisation) -- a wrong model shows up as O(1) errors."""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_helpers import golden_cases, load_golden
from oracle import rf_oracle as orc

REF_FP32_LEVEL = 5e-4


@pytest.mark.parametrize("name", [c for c in golden_cases("mf_") if "fft" not in c])
def test_mf_oracle_vs_reference(name):
    g = load_golden(name)
    if name.endswith("f16"):
        pytest.skip("half outputs: compared on the GPU only")
    A, S = g["real"].shape
    for form in ("f64", "f32"):
        yr, yi = orc.mf_forward(g["real"], g["imag"], g["tx"], g["rx"], g["voxel"], float(g["fs"]),
                                float(g["As"]), form)
        assert rel_l2(yr + 1j * yi, g["out_real"] + 1j * g["out_imag"]) < REF_FP32_LEVEL, form
        hr, hi = orc.mf_backward(g["grad_output_real"], g["grad_output_imag"], g["tx"], g["rx"],
                                 g["voxel"], A, S, float(g["fs"]), float(g["As"]), form)
        assert rel_l2(hr + 1j * hi, g["grad_real"] + 1j * g["grad_imag"]) < REF_FP32_LEVEL, form


@pytest.mark.parametrize("name", golden_cases("mf_fft"))
def test_mf_fft_oracle_vs_reference(name):
    g = load_golden(name)
    A, B = g["spec_real"].shape
    yr, yi = orc.mf_fft_forward(g["spec_real"], g["spec_imag"], g["tx"], g["rx"], g["voxel"], float(g["spacing"]))
    ref = g["out_real"] + 1j * g["out_imag"]
    assert np.count_nonzero(ref) > 0
    assert rel_l2(yr + 1j * yi, ref) < REF_FP32_LEVEL
    hr, hi = orc.mf_fft_backward(g["grad_output_real"], g["grad_output_imag"], g["tx"], g["rx"], g["voxel"],
                                 A, B, float(g["spacing"]))
    assert rel_l2(hr + 1j * hi, g["grad_real"] + 1j * g["grad_imag"]) < REF_FP32_LEVEL


@pytest.mark.parametrize("name", golden_cases("tracer_"))
def test_tracer_oracle_vs_reference(name):
    g = load_golden(name)
    S = int(g["S"])
    inb = g["inbounds"].astype(bool)
    for form in ("f64", "f32"):
        xr, xi = orc.tracer_forward(g["normals"], g["sigmas"], g["points"], g["tx"], g["rx"], inb, S,
                                    float(g["fs"]), float(g["f0"]), float(g["As"]), form)
        assert rel_l2(xr + 1j * xi, g["out_real"] + 1j * g["out_imag"]) < REF_FP32_LEVEL, form
        gn, gs, _ = orc.tracer_backward(g["grad_output_real"], g["grad_output_imag"], g["normals"],
                                        g["sigmas"], g["points"], g["tx"], g["rx"], inb, float(g["fs"]),
                                        float(g["f0"]), float(g["As"]), form, with_points=False)
        assert rel_l2(gn[inb], g["grad_normals"][inb]) < REF_FP32_LEVEL, form
        assert rel_l2(gs[:, inb], g["grad_sigmas"][:, inb]) < REF_FP32_LEVEL, form
    # the reference leaves out-of-bounds rows unwritten (NaN-prefilled in the fixture)
    assert np.isnan(g["grad_normals"][~inb]).all() and np.isnan(g["grad_sigmas"][:, ~inb]).all()


@pytest.mark.parametrize("name", golden_cases("bilinear_"))
def test_bilinear_oracle_vs_reference(name):
    g = load_golden(name)
    on, os_, ob = orc.bilinear_forward(g["normals"], g["sigmas"], g["z_vals"], g["tgt_z_vals"])
    np.testing.assert_array_equal(ob, g["out_inbounds"])
    np.testing.assert_allclose(on, g["out_normals"], rtol=2e-6, atol=1e-7)
    np.testing.assert_allclose(os_, g["out_sigmas"], rtol=2e-6, atol=1e-7)
    gn, gs = orc.bilinear_backward(g["grad_out_normals"], g["grad_out_sigmas"], g["z_vals"], g["tgt_z_vals"],
                                   g["grad_normals_init"], g["grad_sigmas_init"])
    np.testing.assert_allclose(gn, g["grad_normals"], rtol=2e-6, atol=1e-7)
    np.testing.assert_allclose(gs, g["grad_sigmas"], rtol=2e-6, atol=1e-7)


def test_golden_fixtures_present():
    names = golden_cases("")
    for expected in ("mf_scene_f32", "mf_odd_f32", "mf_scene_f16", "mf_scene_f64", "mf_fft_f32",
                     "tracer_f32", "tracer_f64", "bilinear_f32", "fullsize_mf3072ch_f32"):
        assert expected in names


def test_oracle_matches_reference_kernels_at_full_3072_channel_size():
    """The oracle against the reference's own kernels run on the whole
    3072-channel workload (3072 x 128 x 48^3; inputs regenerated from their seed):
    the FP32 form within the reference's own FP32 phase error, the FP64 form too."""
    from oracle import workload_parity as wp

    g = load_golden("fullsize_mf3072ch_f32")
    w = wp.mf3072_inputs(0)
    sums = np.array([np.abs(w["re"].astype(np.float64)).sum(), np.abs(w["im"].astype(np.float64)).sum()])
    np.testing.assert_allclose(sums, g["input_abs_sums"], rtol=1e-9)
    vi = g["voxel_ids"]
    ref = g["out_real"].astype(np.float64) + 1j * g["out_imag"]
    yr, yi = orc.mf_forward(w["re"], w["im"], w["tx"], w["rx"], w["vox"][:, vi], w["fs"], w["As"], "f32")
    assert rel_l2(yr + 1j * yi, ref) < REF_FP32_LEVEL
    assert rel_l2(wp.mf_forward_ref(w, vi, "f64"), ref) < REF_FP32_LEVEL
