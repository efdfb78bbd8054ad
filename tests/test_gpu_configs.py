"""Parity of the RF operators at the full sizes of the benchmark workloads,
where the carrier phase is largest (~5e3 rad), checked against the FP64 oracle
on subsets it finishes in seconds (oracle/workload_parity.py names them):

* 3072 channels x 128 samples x 48^3 voxels: every voxel and antenna is run on
  the GPU; the forward is checked at 4096 voxels, the adjoint at 96 antenna
  rows.  The PLAIN form is also checked against the reference's own kernels at
  this size (tests/golden/fullsize_mf3072ch_f32.npz).
* 49152 channels x 256 samples x 128^3 voxels: the whole volume and the whole
  adjoint on the GPU; checked at a 16^3 voxel sub-lattice and 16 antenna rows.
* The tracer on 64 antennas x 4096 rays x 128 samples of a random-init SDF
  network: forward at 16 antenna rows, the sigma / normal / position gradients
  at the 32768 points of 256 random rays, and those rays' directional
  derivatives against FP64 central differences.

Bars: MIXED <= 1e-4 relative L2 against FP64; PLAIN <= 5e-4 (the reference's own
FP32 phase error) and <= 1e-5 against the reference's kernels; finite
differences <= 1e-3 per ray and per parameter kind."""
import numpy as np
import pytest

from gpu_helpers import load_golden, mf_backward, mf_forward, tracer_backward, tracer_forward
from oracle import workload_parity as wp

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-4
PLAIN_TOL = 5e-4
PLAIN_REF_TOL = 1e-5
FD_TOL = 1e-3


def _c(pair):
    return pair[0] + 1j * pair[1]


@pytest.fixture(scope="module")
def mf3072():
    return wp.mf3072_inputs(0)


@pytest.fixture(scope="module")
def mf49152(cuda):
    return wp.mf49152_inputs(cuda, 0)


@pytest.fixture(scope="module")
def tracer(cuda):
    return wp.tracer_inputs(cuda, 0)


def _fwd(w, precision, voxels=None):
    vox = w["vox"] if voxels is None else np.ascontiguousarray(w["vox"][:, voxels])
    return _c(mf_forward(w["re"], w["im"], w["tx"], w["rx"], vox, w["fs"], w["As"], precision))


def _adj(w, g, precision):
    A = w["tx"].shape[0]
    return _c(mf_backward(g.real.copy(), g.imag.copy(), w["tx"], w["rx"], w["vox"], A, w["S"], w["fs"], w["As"],
                          precision))


def test_mf3072_forward_vs_fp64(cuda, mf3072, parity_log):
    vi = wp.MF3072_VOXELS
    ref = wp.mf_forward_ref(mf3072, vi, form="f64")
    mixed = _fwd(mf3072, "mixed")[vi]
    plain = _fwd(mf3072, "plain")[vi]
    e_mixed, e_plain = wp.rel(mixed, ref), wp.rel(plain, ref)
    parity_log("mf3072_forward_vs_fp64", mixed=e_mixed, plain=e_plain, voxels=len(vi))
    assert e_mixed < MIXED_TOL
    assert e_plain < PLAIN_TOL
    assert e_mixed < e_plain


def test_mf3072_adjoint_vs_fp64(cuda, mf3072, parity_log):
    N = mf3072["vox"].shape[1]
    g = wp.adjoint_grad(N, 21)
    rows = wp.MF3072_ROWS
    ref = wp.mf_adjoint_ref(g, mf3072, rows)
    e_mixed = wp.rel(_adj(mf3072, g, "mixed")[rows], ref)
    e_plain = wp.rel(_adj(mf3072, g, "plain")[rows], ref)
    parity_log("mf3072_adjoint_vs_fp64", mixed=e_mixed, plain=e_plain, rows=len(rows))
    assert e_mixed < MIXED_TOL
    assert e_plain < PLAIN_TOL


def test_mf3072_plain_matches_reference_kernels(cuda, mf3072, parity_log):
    """PLAIN forward and adjoint against the reference's own CUDA kernels run on
    the same full-size inputs (regenerated here from their seed)."""
    gold = load_golden("fullsize_mf3072ch_f32")
    sums = np.array([np.abs(mf3072["re"].astype(np.float64)).sum(), np.abs(mf3072["im"].astype(np.float64)).sum()])
    np.testing.assert_allclose(sums, gold["input_abs_sums"], rtol=1e-9)
    vi, rows = gold["voxel_ids"], gold["rows"]
    ref_y = gold["out_real"].astype(np.float64) + 1j * gold["out_imag"]
    y = _fwd(mf3072, "plain")[vi]
    g = wp.adjoint_grad(mf3072["vox"].shape[1], int(gold["grad_seed"]))
    ref_h = gold["grad_real"].astype(np.float64) + 1j * gold["grad_imag"]
    h = _adj(mf3072, g, "plain")[rows]
    e_f, e_b = wp.rel(y, ref_y), wp.rel(h, ref_h)
    exact_f = float(np.mean((y.real.astype(np.float32) == gold["out_real"]) &
                            (y.imag.astype(np.float32) == gold["out_imag"])))
    exact_b = float(np.mean((h.real.astype(np.float32) == gold["grad_real"]) &
                            (h.imag.astype(np.float32) == gold["grad_imag"])))
    parity_log("mf3072_plain_vs_reference", forward=e_f, adjoint=e_b, forward_bit_exact_fraction=exact_f,
               adjoint_bit_exact_fraction=exact_b)
    assert e_f < PLAIN_REF_TOL
    assert e_b < PLAIN_REF_TOL


def test_mf49152_forward_vs_fp64(cuda, mf49152, parity_log):
    vi = wp.MF49152_VOXELS
    ref = wp.mf_forward_ref(mf49152, vi)
    e_mixed = wp.rel(_fwd(mf49152, "mixed")[vi], ref)          # the whole 128^3 volume on the GPU
    e_nufft = wp.rel(_fwd(mf49152, "nufft")[vi], ref)
    e_plain = wp.rel(_fwd(mf49152, "plain", vi), ref)          # PLAIN on the subset voxels only
    parity_log("mf49152_forward_vs_fp64", mixed=e_mixed, nufft=e_nufft, plain=e_plain, voxels=len(vi))
    assert e_mixed < MIXED_TOL
    assert e_nufft < MIXED_TOL
    assert e_plain < PLAIN_TOL


def test_mf49152_adjoint_vs_fp64(cuda, mf49152, parity_log):
    N = mf49152["vox"].shape[1]
    g = wp.adjoint_grad(N, 22)
    rows = wp.MF49152_ROWS
    ref = wp.mf_adjoint_ref(g, mf49152, rows)
    e_mixed = wp.rel(_adj(mf49152, g, "mixed")[rows], ref)
    e_nufft = wp.rel(_adj(mf49152, g, "nufft")[rows], ref)
    parity_log("mf49152_adjoint_vs_fp64", mixed=e_mixed, nufft=e_nufft, rows=len(rows))
    assert e_mixed < MIXED_TOL
    assert e_nufft < MIXED_TOL


@pytest.mark.parametrize("prec", ["mixed", "plain"])
def test_tracer_forward_and_adjoint_vs_fp64(cuda, tracer, prec, parity_log):
    A, S = tracer["tx"].shape[0], tracer["S"]
    x = _c(tracer_forward(tracer, S, prec))
    e_fwd = wp.tracer_forward_error(x, tracer, wp.TRACER_ROWS)
    g = wp.residual(A, S, 31)
    gn, gs, gp = tracer_backward(tracer, g.real.copy(), g.imag.copy(), prec)
    pts = wp.ray_points(tracer, wp.fd_rays(tracer))
    e = wp.tracer_adjoint_errors({"normals": gn, "sigmas": gs, "points": gp}, g, tracer, pts)
    parity_log(f"tracer_vs_fp64_{prec}", forward=e_fwd, **{f"grad_{k}": v for k, v in e.items()})
    tol = MIXED_TOL if prec == "mixed" else PLAIN_TOL
    assert e_fwd < tol
    assert e["sigma"] < tol and e["normal"] < tol
    # PLAIN: the delay derivative multiplies the FP32 phase error by ~w0 tau
    assert e["position"] < (tol if prec == "mixed" else 2e-3)


def test_tracer_adjoint_matches_finite_differences_on_256_rays(cuda, tracer, parity_log):
    A, S = tracer["tx"].shape[0], tracer["S"]
    g = wp.residual(A, S, 32)
    gn, gs, gp = tracer_backward(tracer, g.real.copy(), g.imag.copy(), "mixed")
    errs = wp.tracer_fd_errors({"normals": gn, "sigmas": gs, "points": gp}, g, tracer, wp.fd_rays(tracer))
    parity_log("tracer_fd_256_rays", **errs)
    assert errs["sigma"] < FD_TOL
    assert errs["normal"] < FD_TOL
    assert errs["position"] < FD_TOL
    assert errs["dropped_points"] < 0.01 * wp.FD_RAYS * tracer["samples_per_ray"]
