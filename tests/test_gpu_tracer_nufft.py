"""The signal tracer's NUFFT form on the GPU: forward and adjoint (sigma,
normals, positions) against the FP64 oracle per interpolation width, the
adjoint identity in sigma, culled and out-of-bounds points, element types, odd
sample counts, split launch shapes and the autograd wrapper."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from gpu_helpers import cu, tracer_backward, tracer_forward
from oracle import rf_oracle as orc
from test_gpu_tracer import tracer_case

pytestmark = pytest.mark.gpu

# FP32 library: the kernel's truncation error (tests/test_nufft_model.py) plus rounding
TOL = {4: 3e-3, 6: 5e-5, 8: 1e-5}


@pytest.fixture(scope="module")
def case():
    return tracer_case()


def oracle_fwd(c):
    r = orc.tracer_forward(c["normals"], c["sigmas"], c["points"], c["tx"], c["rx"], c["inbounds"], c["S"],
                           float(c["fs"]), float(c["f0"]), float(c["As"]), "f64")
    return r[0] + 1j * r[1]


def residual(c, seed=5):
    A = c["sigmas"].shape[0]
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((A, c["S"])).astype(np.float32),
            rng.standard_normal((A, c["S"])).astype(np.float32))


@pytest.mark.parametrize("taps", sorted(TOL))
def test_forward_vs_fp64(cuda, case, taps, parity_log):
    xr, xi = tracer_forward(case, case["S"], "nufft", tuning={"taps": taps})
    err = rel_l2(xr + 1j * xi, oracle_fwd(case))
    parity_log(f"tracer_nufft_forward_W{taps}_vs_fp64", rel_l2=err)
    assert err < TOL[taps]


@pytest.mark.parametrize("taps", [4, 8])
def test_adjoint_vs_fp64(cuda, case, taps, parity_log):
    gr, gi = residual(case)
    rn, rs, rp = orc.tracer_backward(gr, gi, case["normals"], case["sigmas"], case["points"], case["tx"],
                                     case["rx"], case["inbounds"], float(case["fs"]), float(case["f0"]),
                                     float(case["As"]))
    gn, gs, gp = tracer_backward(case, gr, gi, "nufft", tuning={"taps": taps})
    errs = {"sigmas": rel_l2(gs, rs), "normals": rel_l2(gn, rn), "points": rel_l2(gp, rp)}
    parity_log(f"tracer_nufft_adjoint_W{taps}_vs_fp64", **errs)
    # positions: the delay derivative weights samples by n, so the interpolation error
    # of the n-weighted grid enters at a few times the level of the others
    for k, v in errs.items():
        assert v < (TOL[taps] * (4 if k == "points" else 1)), (k, v)
    inb = case["inbounds"]
    assert np.all(gs[:, ~inb] == 0) and np.all(gn[~inb] == 0) and np.all(gp[~inb] == 0)


def test_adjoint_identity_in_sigma(cuda, case):
    """x is linear in sigma: <x(sigma), g> = <sigma, dL/dsigma> for the NUFFT pair."""
    gr, gi = residual(case, seed=9)
    xr, xi = tracer_forward(case, case["S"], "nufft")
    _, gs, _ = tracer_backward(case, gr, gi, "nufft", with_points=False)
    lhs = float(np.sum(xr * gr) + np.sum(xi * gi))
    rhs = float(np.sum(gs * case["sigmas"].astype(np.float64)))
    scale = np.linalg.norm(xr + 1j * xi) * np.linalg.norm(gr + 1j * gi)
    assert abs(lhs - rhs) < 1e-5 * scale


@pytest.mark.parametrize("S", [1, 37, 128])
def test_odd_sample_counts(cuda, S):
    c = tracer_case(seed=S, A=4, P=500, S=S)
    xr, xi = tracer_forward(c, S, "nufft")
    assert rel_l2(xr + 1j * xi, oracle_fwd(c)) < TOL[8]
    gr, gi = residual(c, seed=S)
    rn, rs, rp = orc.tracer_backward(gr, gi, c["normals"], c["sigmas"], c["points"], c["tx"], c["rx"],
                                     c["inbounds"], float(c["fs"]), float(c["f0"]), float(c["As"]))
    gn, gs, gp = tracer_backward(c, gr, gi, "nufft")
    assert rel_l2(gs, rs) < TOL[8] and rel_l2(gn, rn) < TOL[8] and rel_l2(gp, rp) < 4 * TOL[8]


def test_double_precision_inputs(cuda, case):
    xr, xi = tracer_forward(case, case["S"], "nufft", dtype=torch.float64)
    assert rel_l2(xr + 1j * xi, oracle_fwd(case)) < TOL[8]


@pytest.mark.parametrize("tuning", [{"splits": 1}, {"splits": 3}, {"threads": 64, "stage_rows": 2, "splits": 2}])
def test_launch_shapes_agree(cuda, case, tuning):
    base = tracer_forward(case, case["S"], "nufft")
    alt = tracer_forward(case, case["S"], "nufft", tuning=tuning)
    assert rel_l2(alt[0] + 1j * alt[1], base[0] + 1j * base[1]) < 2e-6
    gr, gi = residual(case, seed=2)
    b0 = tracer_backward(case, gr, gi, "nufft")
    b1 = tracer_backward(case, gr, gi, "nufft", tuning=tuning)
    for x, y in zip(b0, b1):
        assert rel_l2(x, y) < 2e-6


def test_autograd_runs_the_nufft_adjoint(cuda, case):
    from geraf_b200.ops.RFSignalTracer import signal_tracer_cuda

    A, P = case["sigmas"].shape
    dev = {k: cu(case[k]).requires_grad_(k in ("normals", "sigmas", "points"))
           for k in ("normals", "sigmas", "points", "tx", "rx")}
    xr, xi = signal_tracer_cuda(dev["normals"], dev["sigmas"], dev["points"], dev["tx"], dev["rx"],
                                cu(case["inbounds"]), case["S"], float(case["fs"]), float(case["f0"]),
                                float(case["As"]), A, P, precision="nufft", tuning={"taps": 6})
    gr, gi = residual(case, seed=8)
    ((xr * cu(gr)).sum() + (xi * cu(gi)).sum()).backward()
    gn, gs, gp = tracer_backward(case, gr, gi, "nufft", tuning={"taps": 6})
    assert rel_l2(dev["sigmas"].grad.double().cpu().numpy(), gs) < 1e-6
    assert rel_l2(dev["normals"].grad.double().cpu().numpy(), gn) < 1e-6
    assert rel_l2(dev["points"].grad.double().cpu().numpy(), gp) < 1e-6
