"""Signal tracer and resampler on the GPU vs the CPU oracle: FP64 error bounds,
the hand-written adjoint (sigma, normals and positions) vs the FP64 adjoint,
central finite differences and autograd through the pure-torch tracer, launch
shapes, out-of-bounds handling, errors and autograd wrappers."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from benchkit import scenes
from gpu_helpers import cu, tracer_backward, tracer_forward
from oracle import rf_oracle as orc
from oracle import torch_tracer

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-4
PLAIN_TOL = 5e-4
FD_TOL = 1e-3


def tracer_case(seed=0, A=6, P=900, S=32, f0=770.0, inb_frac=0.85):
    rng = np.random.default_rng(seed)
    tx, rx = scenes.virtual_array(2)
    tx = (tx[:A] + rng.normal(0, 0.01, (A, 3))).astype(np.float32)
    rx = (rx[:A] + rng.normal(0, 0.01, (A, 3))).astype(np.float32)
    d = rng.normal(0, 1, (P, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    points = (np.array([0, 0, 0.4]) + 0.08 * d).astype(np.float32)
    nrm = d - rng.uniform(0.5, 1.2, (P, 1)) * np.array([0, 0, 1.0])
    nrm = (nrm / np.linalg.norm(nrm, axis=1, keepdims=True)).astype(np.float32)
    ch = scenes.chirp(S)
    return dict(normals=nrm, sigmas=rng.uniform(0, 1, (A, P)).astype(np.float32), points=points,
                tx=tx, rx=rx, inbounds=rng.uniform(0, 1, P) < inb_frac,
                fs=np.float32(ch.adc_sample_rate), f0=np.float32(f0), As=np.float32(ch.As_sci), S=S)


@pytest.fixture(scope="module")
def case():
    return tracer_case()


def oracle_fwd(c, form="f64"):
    return orc.tracer_forward(c["normals"], c["sigmas"], c["points"], c["tx"], c["rx"], c["inbounds"],
                              c["S"], float(c["fs"]), float(c["f0"]), float(c["As"]), form)


def oracle_bwd(c, gr, gi):
    return orc.tracer_backward(gr, gi, c["normals"], c["sigmas"], c["points"], c["tx"], c["rx"],
                               c["inbounds"], float(c["fs"]), float(c["f0"]), float(c["As"]))


def test_forward_forms_vs_fp64(cuda, case):
    ref = oracle_fwd(case)
    ref = ref[0] + 1j * ref[1]
    mr, mi = tracer_forward(case, case["S"], "mixed")
    pr, pi = tracer_forward(case, case["S"], "plain")
    assert rel_l2(mr + 1j * mi, ref) < MIXED_TOL
    assert rel_l2(pr + 1j * pi, ref) < PLAIN_TOL
    assert rel_l2(mr + 1j * mi, ref) < rel_l2(pr + 1j * pi, ref)


@pytest.mark.parametrize("prec,tol", [("mixed", MIXED_TOL), ("plain", PLAIN_TOL)])
def test_adjoint_vs_fp64(cuda, case, prec, tol):
    A = case["sigmas"].shape[0]
    rng = np.random.default_rng(5)
    gr = rng.standard_normal((A, case["S"])).astype(np.float32)
    gi = rng.standard_normal((A, case["S"])).astype(np.float32)
    rn, rs, rp = oracle_bwd(case, gr, gi)
    gn, gs, gp = tracer_backward(case, gr, gi, prec)
    assert rel_l2(gs, rs) < tol
    assert rel_l2(gn, rn) < tol
    # positions: the delay derivative multiplies the phase error by ~w0 tau; FP32 adds ~1e-4
    assert rel_l2(gp, rp) < (tol if prec == "mixed" else 2e-3)
    inb = case["inbounds"]
    assert np.all(gs[:, ~inb] == 0) and np.all(gn[~inb] == 0) and np.all(gp[~inb] == 0)


def test_adjoint_matches_finite_differences(cuda):
    """The CUDA adjoint vs central differences of the FP64 forward on 256 rays
    (points), along random directions for sigma, normals and positions."""
    c = tracer_case(seed=4, A=4, P=256, S=32)
    A, P = c["sigmas"].shape
    rng = np.random.default_rng(17)
    gr = rng.standard_normal((A, c["S"])).astype(np.float32)
    gi = rng.standard_normal((A, c["S"])).astype(np.float32)
    gn, gs, gp = tracer_backward(c, gr, gi, "mixed")
    t = {k: torch.tensor(c[k], dtype=torch.float64) for k in ("tx", "rx", "points", "normals", "sigmas")}
    inb = torch.tensor(c["inbounds"])

    def loss(normals, sigmas, points):
        r, i = torch_tracer.tracer_forward(normals, sigmas, points, t["tx"], t["rx"], inb, c["S"],
                                           float(c["fs"]), float(c["f0"]), float(c["As"]))
        return float((r * torch.tensor(gr, dtype=torch.float64)).sum()
                     + (i * torch.tensor(gi, dtype=torch.float64)).sum())

    for name, grad, eps in (("sigmas", gs, 1e-4), ("normals", gn, 1e-6), ("points", gp, 1e-7)):
        for trial in range(3):
            v = torch.tensor(rng.standard_normal(grad.shape))
            plus = {k: t[k].clone() for k in ("normals", "sigmas", "points")}
            minus = {k: t[k].clone() for k in ("normals", "sigmas", "points")}
            plus[name] += eps * v
            minus[name] -= eps * v
            fd = (loss(**plus) - loss(**minus)) / (2 * eps)
            an = float(np.sum(grad * v.numpy()))
            assert abs(fd - an) <= FD_TOL * abs(an), (name, trial, fd, an)


def test_autograd_wrapper_matches_torch_autograd(cuda, case):
    from geraf_b200.ops.RFSignalTracer import signal_tracer_cuda

    A, P = case["sigmas"].shape
    dev = {k: cu(case[k]).requires_grad_(k in ("normals", "sigmas", "points"))
           for k in ("normals", "sigmas", "points", "tx", "rx")}
    inb = cu(case["inbounds"])
    xr, xi = signal_tracer_cuda(dev["normals"], dev["sigmas"], dev["points"], dev["tx"], dev["rx"], inb,
                                case["S"], float(case["fs"]), float(case["f0"]), float(case["As"]), A, P)
    rng = np.random.default_rng(8)
    gr = torch.tensor(rng.standard_normal((A, case["S"])), dtype=torch.float32, device="cuda")
    gi = torch.tensor(rng.standard_normal((A, case["S"])), dtype=torch.float32, device="cuda")
    ((xr * gr).sum() + (xi * gi).sum()).backward()
    t = {k: torch.tensor(case[k], dtype=torch.float64).requires_grad_(k in ("normals", "sigmas", "points"))
         for k in ("normals", "sigmas", "points", "tx", "rx")}
    r, i = torch_tracer.tracer_forward(t["normals"], t["sigmas"], t["points"], t["tx"], t["rx"],
                                       torch.tensor(case["inbounds"]), case["S"], float(case["fs"]),
                                       float(case["f0"]), float(case["As"]))
    ((r * gr.double().cpu()).sum() + (i * gi.double().cpu()).sum()).backward()
    for k in ("sigmas", "normals", "points"):
        assert rel_l2(dev[k].grad.double().cpu().numpy(), t[k].grad.numpy()) < 2e-4, k


def test_reference_gradient_set_when_points_do_not_require_grad(cuda, case):
    from geraf_b200.ops.RFSignalTracer import signal_tracer_cuda

    A, P = case["sigmas"].shape
    n = cu(case["normals"]).requires_grad_(True)
    s = cu(case["sigmas"]).requires_grad_(True)
    p = cu(case["points"])
    xr, xi = signal_tracer_cuda(n, s, p, cu(case["tx"]), cu(case["rx"]), cu(case["inbounds"]),
                                case["S"], float(case["fs"]), float(case["f0"]), float(case["As"]), A, P)
    (xr.sum() + xi.sum()).backward()
    assert n.grad is not None and s.grad is not None and p.grad is None


@pytest.mark.parametrize("tuning", [{"threads": 128, "chunk": 8}, {"threads": 256, "chunk": 32},
                                    {"threads": 64, "chunk": 16, "splits": 6}])
def test_forward_launch_shapes_agree(cuda, case, tuning):
    base = tracer_forward(case, case["S"], "mixed")
    alt = tracer_forward(case, case["S"], "mixed", tuning=tuning)
    assert rel_l2(alt[0] + 1j * alt[1], base[0] + 1j * base[1]) < 2e-6


@pytest.mark.parametrize("tuning", [{"threads": 64, "stage_rows": 1}, {"threads": 128, "stage_rows": 4, "splits": 3}])
def test_adjoint_launch_shapes_agree(cuda, case, tuning):
    A = case["sigmas"].shape[0]
    rng = np.random.default_rng(1)
    gr = rng.standard_normal((A, case["S"])).astype(np.float32)
    gi = rng.standard_normal((A, case["S"])).astype(np.float32)
    base = tracer_backward(case, gr, gi, "mixed")
    alt = tracer_backward(case, gr, gi, "mixed", tuning=tuning)
    for a, b in zip(alt, base):
        assert rel_l2(a, b) < 2e-6


def test_float64_inputs_and_odd_sizes(cuda):
    c = tracer_case(seed=9, A=3, P=77, S=13, f0=773.704)
    ref = oracle_fwd(c)
    for prec, tol in (("mixed", MIXED_TOL), ("plain", PLAIN_TOL)):
        xr, xi = tracer_forward(c, c["S"], prec, dtype=torch.float64)
        assert rel_l2(xr + 1j * xi, ref[0] + 1j * ref[1]) < tol


def test_all_points_out_of_bounds_and_empty(cuda):
    from geraf_b200.ops.RFSignalTracer import _C

    c = tracer_case(seed=2, A=2, P=50, S=8, inb_frac=0.0)
    xr, xi = tracer_forward(c, c["S"], "mixed")
    assert np.all(xr == 0) and np.all(xi == 0)
    # P = 0: the reference divides 0 by 0 -> NaN
    out_r = torch.zeros((2, 8), device="cuda")
    out_i = torch.zeros((2, 8), device="cuda")
    z3 = torch.empty((0, 3), device="cuda")
    for prec in ("plain", "mixed"):
        _C.SignalTracer_forward(z3, torch.empty((2, 0), device="cuda"), z3, cu(c["tx"]), cu(c["rx"]),
                                torch.empty(0, dtype=torch.bool, device="cuda"), out_r, out_i, 8,
                                5e6, 770.0, 1e6, 2, 0, precision=prec)
        assert torch.isnan(out_r).all()


def test_drop_in_errors(cuda, case):
    from geraf_b200.ops.RFSignalTracer import _C, signal_tracer_cuda

    A, P = case["sigmas"].shape
    args = [cu(case[k]) for k in ("normals", "sigmas", "points", "tx", "rx")]
    inb = cu(case["inbounds"])
    with pytest.raises(ValueError, match="retains only the differentiable"):
        signal_tracer_cuda(*args, inb, case["S"], 5e6, 770.0, 1e6, A, P, use_diff=False)
    with pytest.raises(ValueError, match="CUDA tensors"):
        signal_tracer_cuda(args[0].cpu(), *args[1:], inb, case["S"], 5e6, 770.0, 1e6, A, P)
    with pytest.raises(ValueError, match="`normals` must have shape"):
        signal_tracer_cuda(args[0][:, :2], *args[1:], inb, case["S"], 5e6, 770.0, 1e6, A, P)
    out = torch.empty((A, case["S"]), device="cuda")
    with pytest.raises(RuntimeError, match="`inbounds` must be bool"):
        _C.SignalTracer_forward(*args, inb.float(), out, out, case["S"], 5e6, 770.0, 1e6, A, P)
    with pytest.raises(RuntimeError, match="not implemented for 'Half'"):
        h = [a.half() for a in args]
        _C.SignalTracer_forward(*h, inb, out.half(), out.half(), case["S"], 5e6, 770.0, 1e6, A, P)


def test_bilinear_wrapper_vs_oracle_and_autograd(cuda):
    from geraf_b200 import model_utils

    rng = np.random.default_rng(3)
    R, S, T, A = 33, 32, 64, 1
    z = np.sort(rng.uniform(0.2, 0.6, (R, S)), axis=1).astype(np.float32)
    tz = rng.uniform(0.18, 0.62, (R, T)).astype(np.float32)
    nrm = rng.standard_normal((R, S, 3)).astype(np.float32)
    sig = rng.uniform(0, 1, (A, R, S)).astype(np.float32)
    n_t = cu(nrm).requires_grad_(True)
    s_t = cu(sig).requires_grad_(True)
    on, os_, ob = model_utils.bilinear_ray_sampler(n_t, s_t, cu(z), cu(tz))
    rn, rs, rb = orc.bilinear_forward(nrm, sig, z, tz)
    np.testing.assert_array_equal(ob.cpu().numpy(), rb)
    np.testing.assert_allclose(on.detach().cpu().numpy(), rn, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(os_.detach().cpu().numpy(), rs, rtol=1e-6, atol=1e-7)
    gon = rng.standard_normal((R, T, 3)).astype(np.float32)
    gos = rng.standard_normal((A, R, T)).astype(np.float32)
    ((on * cu(gon)).sum() + (os_ * cu(gos)).sum()).backward()
    gn, gs = orc.bilinear_backward(gon, gos, z, tz)
    np.testing.assert_allclose(n_t.grad.cpu().numpy(), gn, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(s_t.grad.cpu().numpy(), gs, rtol=1e-5, atol=1e-6)
