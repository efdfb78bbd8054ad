"""The MIXED tracer's per-point pre-cull (csrc/tracer_precull.cu) on the device:
no (point, antenna) pair that the reference keeps is lost, every gradient of a
point left out is written (as zero), and results agree across the launch shapes
that read the point list (splits of the forward's points and of the adjoint's
antennas).  The workload is the SDF scene of the tracer benchmark at 512 rays
(64 antennas x 65536 points), where the pre-cull leaves out most points."""
import numpy as np
import pytest
import torch

from gpu_helpers import tracer_backward, tracer_forward
from oracle import workload_parity as wp

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-4
MARGIN = 1e-5  # pairs this close to a culling threshold (FP64) are not classified


def _clear_masks(w):
    """Pairs [A, P] that the reference geometry clearly keeps / clearly culls,
    from the FP64 geometry of the FP32 inputs."""
    n = w["normals"].astype(np.float64)
    p = w["points"].astype(np.float64)
    inb = w["inbounds"].astype(bool)
    A = w["tx"].shape[0]
    live = np.zeros((A, p.shape[0]), bool)
    dead = np.zeros_like(live)
    for a in range(A):
        i = p - w["tx"][a].astype(np.float64)
        o = w["rx"][a].astype(np.float64) - p
        i /= np.linalg.norm(i, axis=1, keepdims=True) + 1e-7
        o /= np.linalg.norm(o, axis=1, keepdims=True) + 1e-7
        idn = (i * n).sum(1)
        r = i - 2.0 * idn[:, None] * n
        r /= np.linalg.norm(r, axis=1, keepdims=True) + 1e-7
        rho = (o * r).sum(1)
        live[a] = inb & (idn < -MARGIN) & (rho > 1e-6 + MARGIN)
        dead[a] = ~inb | (idn > MARGIN) | (rho < 1e-6 - MARGIN)
    return live, dead


@pytest.fixture(scope="module")
def scene(cuda):
    w = wp.tracer_inputs(cuda, 0, num_rays=512)
    live, dead = _clear_masks(w)
    return w, live, dead


def _c(pair):
    return pair[0] + 1j * pair[1]


def test_precull_keeps_every_live_pair(scene, parity_log):
    w, live, dead = scene
    A, P = w["sigmas"].shape
    # most pairs are culled and most points have no live pair: the pre-cull has work to skip
    assert live.mean() < 0.2 and (~live.any(0)).mean() > 0.5
    g = wp.residual(A, w["S"], 3)
    shapes = [None, {"threads": 128, "stage_rows": 8, "splits": 1}, {"threads": 64, "stage_rows": 4, "splits": 3}]
    results = []
    for tun in shapes:
        gn, gs, gp = tracer_backward(w, g.real.copy(), g.imag.copy(), "mixed", tuning=tun)
        assert np.isfinite(gs).all() and np.isfinite(gn).all() and np.isfinite(gp).all()
        assert (gs[live] != 0).all(), "a live pair lost its sigma gradient"
        assert (gs[dead] == 0).all()
        none_live = dead.all(0)
        assert (gn[none_live] == 0).all() and (gp[none_live] == 0).all()
        results.append((gn, gs, gp))
    for gn, gs, gp in results[1:]:
        for x, y in zip((gn, gs, gp), results[0]):
            assert wp.rel(x, y) < 1e-6
    pts = np.arange(0, P, 16)
    errs = wp.tracer_adjoint_errors({"normals": results[0][0], "sigmas": results[0][1], "points": results[0][2]},
                                    g, w, pts)
    parity_log("tracer_precull_adjoint_512rays", **errs)
    assert max(errs.values()) < MIXED_TOL

    rows = np.arange(0, A, 8)
    outs = [_c(tracer_forward(w, w["S"], "mixed", tuning=t))
            for t in (None, {"threads": 64, "chunk": 8, "splits": 1}, {"threads": 128, "chunk": 16, "splits": 5})]
    for x in outs[1:]:
        assert wp.rel(x, outs[0]) < 1e-6
    err = wp.tracer_forward_error(outs[0], w, rows)
    parity_log("tracer_precull_forward_512rays", forward=err)
    assert err < MIXED_TOL


def test_precull_float64_inputs(scene):
    w, live, dead = scene
    A = w["sigmas"].shape[0]
    g = wp.residual(A, w["S"], 4)
    gn, gs, gp = tracer_backward(w, g.real.copy(), g.imag.copy(), "mixed", dtype=torch.float64)
    assert (gs[live] != 0).all() and (gs[dead] == 0).all()
    x = _c(tracer_forward(w, w["S"], "mixed", dtype=torch.float64))
    assert wp.tracer_forward_error(x, w, np.arange(0, A, 8)) < MIXED_TOL


def test_precull_all_points_back_facing(scene):
    """Normals turned away from the whole array: no point is listed, the IF is
    exactly zero and every gradient is written as zero."""
    w, _, _ = scene
    w = dict(w)
    away = w["points"].astype(np.float64) - w["tx"].astype(np.float64).mean(0)
    w["normals"] = (away / np.linalg.norm(away, axis=1, keepdims=True)).astype(np.float32)
    A = w["sigmas"].shape[0]
    xr, xi = tracer_forward(w, w["S"], "mixed")
    assert (xr == 0).all() and (xi == 0).all()
    g = wp.residual(A, w["S"], 5)
    gn, gs, gp = tracer_backward(w, g.real.copy(), g.imag.copy(), "mixed", tuning={"splits": 2})
    assert (gn == 0).all() and (gs == 0).all() and (gp == 0).all()


def test_precull_out_of_bounds_and_non_finite(scene):
    """Out-of-bounds points are never listed (a NaN normal there changes nothing);
    a NaN normal on an in-bounds point is listed and decided by the exact form,
    which carries the NaN into every antenna's IF, as the reference does."""
    w, _, _ = scene
    w = dict(w)
    A, P = w["sigmas"].shape
    inb = w["inbounds"].copy()
    inb[1::2] = False
    w["inbounds"] = inb
    ref = _c(tracer_forward(w, w["S"], "mixed"))
    assert np.isfinite(ref).all()
    nrm = w["normals"].copy()
    nrm[1] = np.nan  # out of bounds
    w["normals"] = nrm
    x = _c(tracer_forward(w, w["S"], "mixed"))
    assert np.array_equal(x, ref)
    g = wp.residual(A, w["S"], 6)
    gn, gs, gp = tracer_backward(w, g.real.copy(), g.imag.copy(), "mixed")
    assert (gn[1::2] == 0).all() and (gs[:, 1::2] == 0).all() and (gp[1::2] == 0).all()
    nrm[2] = np.nan  # in bounds
    x = _c(tracer_forward(w, w["S"], "mixed"))
    assert np.isnan(x).all()


def test_precull_nufft_form(scene):
    """The NUFFT tracer reads the same point list: live pairs keep their sigma
    gradient, culled pairs and points left out get exact zeros, the results agree
    with the MIXED form to the NUFFT's accuracy, and an empty list gives zeros."""
    w, live, dead = scene
    A = w["sigmas"].shape[0]
    g = wp.residual(A, w["S"], 7)
    gn, gs, gp = tracer_backward(w, g.real.copy(), g.imag.copy(), "nufft", tuning={"splits": 2})
    assert np.isfinite(gs).all() and np.isfinite(gn).all() and np.isfinite(gp).all()
    assert (gs[live] != 0).all() and (gs[dead] == 0).all()
    none_live = dead.all(0)
    assert (gn[none_live] == 0).all() and (gp[none_live] == 0).all()
    mn, ms, mp = tracer_backward(w, g.real.copy(), g.imag.copy(), "mixed")
    assert wp.rel(gs, ms) < 1e-4 and wp.rel(gn, mn) < 1e-4 and wp.rel(gp, mp) < 1e-4
    x = _c(tracer_forward(w, w["S"], "nufft"))
    assert wp.rel(x, _c(tracer_forward(w, w["S"], "mixed"))) < 1e-4

    w = dict(w)
    away = w["points"].astype(np.float64) - w["tx"].astype(np.float64).mean(0)
    w["normals"] = (away / np.linalg.norm(away, axis=1, keepdims=True)).astype(np.float32)
    xr, xi = tracer_forward(w, w["S"], "nufft")
    assert (xr == 0).all() and (xi == 0).all()
    gn, gs, gp = tracer_backward(w, g.real.copy(), g.imag.copy(), "nufft")
    assert (gn == 0).all() and (gs == 0).all() and (gp == 0).all()


def _synthetic(A, P, S, seed, spread=0.01):
    """Random specular points at ~0.4 m in front of an array of A antennas;
    normals mostly face the array."""
    from benchkit import scenes

    rng = np.random.default_rng(seed)
    tx = rng.normal(0, spread, (A, 3)).astype(np.float32)
    rx = (tx + rng.normal(0, spread / 2, (A, 3))).astype(np.float32)
    pts = (np.array([0.0, 0.0, 0.4]) + rng.normal(0, 0.08, (P, 3))).astype(np.float32)
    n = rng.normal(0, 1, (P, 3)) - 1.2 * pts / np.linalg.norm(pts, axis=1, keepdims=True)
    n = (n / np.linalg.norm(n, axis=1, keepdims=True)).astype(np.float32)
    ch = scenes.chirp(S)
    return dict(normals=n, sigmas=rng.uniform(0.1, 1.0, (A, P)).astype(np.float32), points=pts, tx=tx, rx=rx,
                inbounds=rng.uniform(size=P) < 0.9, S=S, fs=ch.adc_sample_rate, f0=770.0, As=ch.As_sci)


@pytest.mark.parametrize("A,P,S", [(2100, 4096, 32), (4, 2_200_000, 16)], ids=["wide_aperture", "many_chunks"])
def test_precull_one_block_kernels(cuda, A, P, S):
    """Past 2048 antennas the aperture is bounded by its own one-block kernel, past
    2048 chunks of 1024 points the chunk counts are scanned by one: the same
    guarantees as the in-block forms (every clearly live pair kept, exact zeros
    elsewhere, the IF within the MIXED bar of FP64)."""
    w = _synthetic(A, P, S, 11)
    live, dead = _clear_masks(w)
    assert live.any() and (~live.any(0)).any()
    g = wp.residual(A, S, 12)
    gn, gs, gp = tracer_backward(w, g.real.copy(), g.imag.copy(), "mixed")
    assert (gs[live] != 0).all() and (gs[dead] == 0).all()
    assert (gn[dead.all(0)] == 0).all()
    rows = np.arange(0, A, max(1, A // 4))
    err = wp.tracer_forward_error(_c(tracer_forward(w, S, "mixed")), w, rows)
    assert err < MIXED_TOL
