"""CPU oracle checks (no GPU): analytic known answers, adjoint identities,
FP32-vs-FP64 agreement, and the FP64 tracer adjoint against autograd through the
pure-torch tracer and against central finite differences."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from benchkit import scenes
from oracle import rf_oracle as orc
from oracle import torch_tracer


def small_mf_case(seed=0, scan=4, S=32, k=6, n=5):
    rng = np.random.default_rng(seed)
    tx, rx = scenes.virtual_array(scan)
    pos, amp = scenes.point_scene(rng, k, size=0.1)
    ch = scenes.chirp(S)
    re, im = scenes.synthesize_if_numpy(tx, rx, pos, amp, ch, snr_db=None)
    vox = scenes.voxel_grid(n, size=0.1)
    return dict(tx=tx, rx=rx, pos=pos, amp=amp, ch=ch, re=re, im=im, vox=vox)


def test_point_scatterer_focuses_to_amplitude_times_samples():
    """One noise-free scatterer at a voxel: y = (1/A) sum_a sum_n a e^{+j phi} e^{-j phi} = S a."""
    tx, rx = scenes.virtual_array(3)
    ch = scenes.chirp(16)
    pos = np.array([[0.01, -0.02, 0.41]], np.float32)
    amp = np.array([0.7 - 0.3j], np.complex64)
    re, im = scenes.synthesize_if_numpy(tx, rx, pos, amp, ch, snr_db=None)
    yr, yi = orc.mf_forward(re, im, tx, rx, pos.T.copy(), ch.adc_sample_rate, ch.As_sci, "f64")
    y = yr[0] + 1j * yi[0]
    expect = ch.num_samples * complex(amp[0])
    # synthesize_if_numpy rounds the IF to FP32 (~1e-7 relative)
    assert abs(y - expect) / abs(expect) < 1e-6


def test_mf_peak_at_scatterer_voxel():
    c = small_mf_case(k=1)
    c["pos"][0] = c["vox"][:, 62]
    re, im = scenes.synthesize_if_numpy(c["tx"], c["rx"], c["pos"], c["amp"], c["ch"], snr_db=None)
    yr, yi = orc.mf_forward(re, im, c["tx"], c["rx"], c["vox"], c["ch"].adc_sample_rate,
                            c["ch"].As_sci, "f64")
    assert int(np.argmax(np.hypot(yr, yi))) == 62


@pytest.mark.parametrize("S", [16, 37, 256])
def test_mf_rotation_form_matches_per_sample_f64(S):
    """The FP64 rotation form used for full-size checks is the same model as the
    per-sample libm form to ~1e-13 (forward and adjoint, S below, at and above
    the 16-sample re-seed, antennas not a multiple of the 4 interleaved)."""
    c = small_mf_case(S=S)
    rng = np.random.default_rng(11)
    A = c["re"].shape[0] - 3
    tx, rx = c["tx"][:A], c["rx"][:A]
    re = rng.standard_normal((A, S)).astype(np.float32)
    im = rng.standard_normal((A, S)).astype(np.float32)
    fs, As = c["ch"].adc_sample_rate, scenes.chirp(256).As_sci
    exact = orc.mf_forward(re, im, tx, rx, c["vox"], fs, As, "f64")
    rot = orc.mf_forward(re, im, tx, rx, c["vox"], fs, As, "f64r")
    assert rel_l2(rot[0] + 1j * rot[1], exact[0] + 1j * exact[1]) < 1e-12
    N = c["vox"].shape[1]
    gr, gi = rng.standard_normal(N).astype(np.float32), rng.standard_normal(N).astype(np.float32)
    exact = orc.mf_backward(gr, gi, tx, rx, c["vox"], A, S, fs, As, "f64")
    rot = orc.mf_backward(gr, gi, tx, rx, c["vox"], A, S, fs, As, "f64r")
    assert rel_l2(rot[0] + 1j * rot[1], exact[0] + 1j * exact[1]) < 1e-12
    with pytest.raises(ValueError):
        orc.mf_forward(re, im, tx, rx, c["vox"], fs, As, "f16")


def test_mf_adjoint_identity_f64():
    """<F s, g> = <s, F^T g> for the real-linear map (re, im) -> (y_re, y_im)."""
    c = small_mf_case()
    rng = np.random.default_rng(3)
    A, S = c["re"].shape
    N = c["vox"].shape[1]
    sr, si = rng.standard_normal((A, S)).astype(np.float32), rng.standard_normal((A, S)).astype(np.float32)
    gr, gi = rng.standard_normal(N).astype(np.float32), rng.standard_normal(N).astype(np.float32)
    yr, yi = orc.mf_forward(sr, si, c["tx"], c["rx"], c["vox"], c["ch"].adc_sample_rate, c["ch"].As_sci)
    hr, hi = orc.mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, c["ch"].adc_sample_rate,
                             c["ch"].As_sci)
    lhs = np.dot(gr.astype(np.float64), yr) + np.dot(gi.astype(np.float64), yi)
    rhs = np.sum(hr * sr) + np.sum(hi * si)
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), 1.0)


def test_mf_f32_tracks_f64():
    """The reference's FP32 arithmetic sits ~1e-4 from FP64: its carrier phase
    (~1.5e3 rad) carries FP32 rounding of ~1e-4 rad.  The bound here is that
    observed level, not the mixed form's target."""
    c = small_mf_case()
    f = orc.mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], c["ch"].adc_sample_rate,
                       c["ch"].As_sci, "f64")
    g = orc.mf_forward(c["re"], c["im"], c["tx"], c["rx"], c["vox"], c["ch"].adc_sample_rate,
                       c["ch"].As_sci, "f32")
    assert rel_l2(g[0] + 1j * g[1], f[0] + 1j * f[1]) < 5e-4
    A, S = c["re"].shape
    rng = np.random.default_rng(1)
    gr = rng.standard_normal(c["vox"].shape[1]).astype(np.float32)
    gi = rng.standard_normal(c["vox"].shape[1]).astype(np.float32)
    b64 = orc.mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, c["ch"].adc_sample_rate, c["ch"].As_sci)
    b32 = orc.mf_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, S, c["ch"].adc_sample_rate,
                          c["ch"].As_sci, "f32")
    assert rel_l2(b32[0] + 1j * b32[1], b64[0] + 1j * b64[1]) < 5e-4


@pytest.mark.parametrize("consistent", [False, True])
def test_mf_fft_adjoint_identity_f32(consistent):
    c = small_mf_case()
    rng = np.random.default_rng(5)
    A, B = c["tx"].shape[0], 40
    N = c["vox"].shape[1]
    sr, si = rng.standard_normal((A, B)).astype(np.float32), rng.standard_normal((A, B)).astype(np.float32)
    gr, gi = rng.standard_normal(N).astype(np.float32), rng.standard_normal(N).astype(np.float32)
    spacing = 0.03
    yr, yi = orc.mf_fft_forward(sr, si, c["tx"], c["rx"], c["vox"], spacing, consistent)
    hr, hi = orc.mf_fft_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, B, spacing, consistent)
    lhs = np.dot(gr.astype(np.float64), yr) + np.dot(gi.astype(np.float64), yi)
    rhs = np.sum(hr.astype(np.float64) * sr) + np.sum(hi.astype(np.float64) * si)
    assert np.count_nonzero(hr) > 0
    assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), 1.0)


def test_mf_fft_consistent_bins_reach_the_upper_half():
    """The reference keeps delays d <= spacing * bins although the bin index
    floor(d / spacing / 2) then reaches only bins [0, bins/2]; with the consistent
    bound the upper bins are filled and the lower ones are unchanged."""
    c = small_mf_case()
    A, N = c["tx"].shape[0], c["vox"].shape[1]
    rng = np.random.default_rng(6)
    gr, gi = rng.standard_normal(N).astype(np.float32), rng.standard_normal(N).astype(np.float32)
    spacing, B = 0.02, 64      # delays ~0.95 m: bins ~24, past the reference's bound 1.28 m / 2
    ref_r, _ = orc.mf_fft_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, B, spacing, False)
    fix_r, _ = orc.mf_fft_backward(gr, gi, c["tx"], c["rx"], c["vox"], A, B, spacing, True)
    assert np.count_nonzero(ref_r[:, B // 2:]) == 0
    assert np.count_nonzero(fix_r) > 0
    both = ref_r != 0
    assert np.array_equal(fix_r[both], ref_r[both])


def tracer_case(seed=0, A=5, P=300, S=24):
    rng = np.random.default_rng(seed)
    tx, rx = scenes.virtual_array(1)
    tx = (tx[:A] + rng.normal(0, 0.01, (A, 3))).astype(np.float32)
    rx = (rx[:A] + rng.normal(0, 0.01, (A, 3))).astype(np.float32)
    d = rng.normal(0, 1, (P, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    points = (np.array([0, 0, 0.4]) + 0.08 * d).astype(np.float32)
    # outward sphere normals tilted towards the radar, so most points are not culled
    normals = d - 0.9 * np.array([0, 0, 1.0])
    normals = (normals / np.linalg.norm(normals, axis=1, keepdims=True)).astype(np.float32)
    sigmas = rng.uniform(0, 1, (A, P)).astype(np.float32)
    inb = rng.uniform(0, 1, P) < 0.85
    ch = scenes.chirp(S)
    return dict(tx=tx, rx=rx, points=points, normals=normals, sigmas=sigmas, inb=inb, ch=ch,
                f0=770.0)


def _torch_inputs(c, dtype=torch.float64):
    t = {k: torch.tensor(c[k], dtype=dtype) for k in ("tx", "rx", "points", "normals", "sigmas")}
    t["inb"] = torch.tensor(c["inb"])
    return t


def test_tracer_oracle_matches_torch_restatement():
    c = tracer_case()
    ch = c["ch"]
    fr, fi = orc.tracer_forward(c["normals"], c["sigmas"], c["points"], c["tx"], c["rx"], c["inb"],
                                ch.num_samples, ch.adc_sample_rate, c["f0"], ch.As_sci)
    t = _torch_inputs(c)
    tr, ti = torch_tracer.tracer_forward(t["normals"], t["sigmas"], t["points"], t["tx"], t["rx"],
                                         t["inb"], ch.num_samples, ch.adc_sample_rate, c["f0"],
                                         ch.As_sci)
    assert rel_l2(fr + 1j * fi, tr.numpy() + 1j * ti.numpy()) < 1e-12
    # the reference's FP32 arithmetic sits ~1e-4 from FP64 (phase rounding), as for the MF
    g32 = orc.tracer_forward(c["normals"], c["sigmas"], c["points"], c["tx"], c["rx"], c["inb"],
                             ch.num_samples, ch.adc_sample_rate, c["f0"], ch.As_sci, "f32")
    assert rel_l2(g32[0] + 1j * g32[1], fr + 1j * fi) < 5e-4


def test_tracer_adjoint_f64_matches_autograd():
    c = tracer_case()
    ch = c["ch"]
    A, P = c["sigmas"].shape
    rng = np.random.default_rng(7)
    gr = rng.standard_normal((A, ch.num_samples)).astype(np.float32)
    gi = rng.standard_normal((A, ch.num_samples)).astype(np.float32)
    gn, gs, gp = orc.tracer_backward(gr, gi, c["normals"], c["sigmas"], c["points"], c["tx"],
                                     c["rx"], c["inb"], ch.adc_sample_rate, c["f0"], ch.As_sci)
    t = _torch_inputs(c)
    for k in ("normals", "sigmas", "points"):
        t[k].requires_grad_(True)
    tr, ti = torch_tracer.tracer_forward(t["normals"], t["sigmas"], t["points"], t["tx"], t["rx"],
                                         t["inb"], ch.num_samples, ch.adc_sample_rate, c["f0"],
                                         ch.As_sci)
    loss = (tr * torch.tensor(gr, dtype=torch.float64)).sum() + (ti * torch.tensor(gi, dtype=torch.float64)).sum()
    loss.backward()
    # autograd differentiates through the 1e-7 normalisation epsilon; the oracle does not
    assert rel_l2(gs, t["sigmas"].grad.numpy()) < 1e-9
    assert rel_l2(gn, t["normals"].grad.numpy()) < 1e-5
    assert rel_l2(gp, t["points"].grad.numpy()) < 1e-5
    assert np.all(gs[:, ~c["inb"]] == 0) and np.all(gn[~c["inb"]] == 0) and np.all(gp[~c["inb"]] == 0)


def test_tracer_adjoint_f64_matches_finite_differences():
    """Directional central differences of the FP64 forward vs the FP64 adjoint."""
    c = tracer_case(seed=2, A=3, P=64, S=16)
    ch = c["ch"]
    A, P = c["sigmas"].shape
    rng = np.random.default_rng(11)
    gr = rng.standard_normal((A, ch.num_samples))
    gi = rng.standard_normal((A, ch.num_samples))
    gn, gs, gp = orc.tracer_backward(gr, gi, c["normals"], c["sigmas"], c["points"], c["tx"],
                                     c["rx"], c["inb"], ch.adc_sample_rate, c["f0"], ch.As_sci)
    t = _torch_inputs(c)

    def loss(normals, sigmas, points):
        r, i = torch_tracer.tracer_forward(normals, sigmas, points, t["tx"], t["rx"], t["inb"],
                                           ch.num_samples, ch.adc_sample_rate, c["f0"], ch.As_sci)
        return float((r * torch.tensor(gr)).sum() + (i * torch.tensor(gi)).sum())

    for name, grad in (("sigmas", gs), ("normals", gn), ("points", gp)):
        v = torch.tensor(rng.standard_normal(grad.shape))
        eps = 1e-6 if name != "points" else 1e-7
        plus = {k: t[k].clone() for k in ("normals", "sigmas", "points")}
        minus = {k: t[k].clone() for k in ("normals", "sigmas", "points")}
        plus[name] += eps * v
        minus[name] -= eps * v
        fd = (loss(**plus) - loss(**minus)) / (2 * eps)
        an = float(np.sum(grad * v.numpy()))
        assert abs(fd - an) <= 1e-3 * max(abs(an), 1e-12), (name, fd, an)


def test_bilinear_oracle_interpolates_and_masks():
    rng = np.random.default_rng(0)
    R, S, T, A = 5, 8, 11, 2
    z = np.sort(rng.uniform(0.2, 0.6, (R, S)), axis=1).astype(np.float32)
    tz = rng.uniform(0.15, 0.65, (R, T)).astype(np.float32)
    normals = rng.standard_normal((R, S, 3)).astype(np.float32)
    sig = rng.uniform(0, 1, (A, R, S)).astype(np.float32)
    on, os_, ob = orc.bilinear_forward(normals, sig, z, tz)
    for r in range(R):
        for t in range(T):
            inside = z[r, 0] <= tz[r, t] <= z[r, -1]
            assert ob[r, t] == inside
            if inside:
                np.testing.assert_allclose(os_[:, r, t], [np.interp(tz[r, t], z[r], sig[a, r]) for a in range(A)],
                                           rtol=1e-5, atol=1e-6)
            else:
                assert np.all(os_[:, r, t] == 0) and np.all(on[r, t] == 0)
    # adjoint identity of the resampler (inbounds mask is constant)
    gon = rng.standard_normal((R, T, 3)).astype(np.float32)
    gos = rng.standard_normal((A, R, T)).astype(np.float32)
    gn, gs = orc.bilinear_backward(gon, gos, z, tz)
    lhs = np.sum(gon.astype(np.float64) * on) + np.sum(gos.astype(np.float64) * os_)
    rhs = np.sum(gn.astype(np.float64) * normals) + np.sum(gs.astype(np.float64) * sig)
    assert abs(lhs - rhs) < 1e-4 * max(1.0, abs(lhs))


def test_fd_check_machinery_against_the_fp64_adjoint():
    """The per-ray finite-difference check used on the full-size tracer workload
    (oracle.workload_parity.tracer_fd_errors), run here with the FP64 oracle's
    own adjoint as the 'analytic' gradient: it must report agreement far below
    the 1e-3 bar, and a planted error in the oracle gradient must show."""
    from oracle import workload_parity as wp

    c = tracer_case(seed=3, A=4, P=8 * 16, S=32)
    ch = c["ch"]
    w = dict(normals=c["normals"], sigmas=c["sigmas"], points=c["points"], tx=c["tx"], rx=c["rx"],
             inbounds=np.ones(c["points"].shape[0], bool), S=ch.num_samples, fs=ch.adc_sample_rate,
             f0=c["f0"], As=ch.As_sci, rays=8, samples_per_ray=16)
    g = wp.residual(4, ch.num_samples, 5)
    gn, gs, gp = orc.tracer_backward(g.real, g.imag, c["normals"], c["sigmas"], c["points"], c["tx"], c["rx"],
                                     w["inbounds"], ch.adc_sample_rate, c["f0"], ch.As_sci)
    grads = {"normals": gn, "sigmas": gs, "points": gp}
    rays = np.arange(8)
    errs = wp.tracer_fd_errors(grads, g, w, rays)
    assert max(errs["sigma"], errs["normal"], errs["position"]) < 1e-6, errs
    bad = dict(grads, points=gp * (1 + 1e-2))
    assert wp.tracer_fd_errors(bad, g, w, rays)["position"] > 1e-3


@pytest.mark.parametrize("mode,align", [("bilinear", True), ("bilinear", False), ("nearest", True)])
def test_volume_sampling_restatement_matches_torch_grid_sample(mode, align):
    """The FP64 restatement of the reference's target-point sampling against the
    call it restates (torch grid_sample on the host, loading.py:20-25): a ragged
    volume, points inside, on the faces and corners, and outside (zero padding)."""
    import torch.nn.functional as F

    from oracle import rf_oracle as o

    rng = np.random.default_rng(2)
    vol = rng.standard_normal((9, 7, 5)).astype(np.float32)
    pts = rng.uniform(-1.3, 1.3, (400, 3)).astype(np.float32)
    pts[:8] = np.array([[sx, sy, sz] for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)], np.float32)
    pts[8:20, 0] = 1.0
    pts[20:24] = [[2.5, 0, 0], [0, -2.5, 0], [0, 0, 3.0], [-2.5, 2.5, 0]]  # wholly outside
    grid = torch.tensor(np.stack([pts[:, 2], pts[:, 1], pts[:, 0]], -1)).view(1, 1, 1, -1, 3)
    ref = F.grid_sample(torch.tensor(vol)[None, None], grid, mode=mode, align_corners=align).reshape(-1)
    got = o.sample_volume(vol, pts, mode, align)
    assert np.max(np.abs(got - ref.double().numpy())) < 1e-6 * np.abs(vol).max()
    assert np.all(got[20:24] == 0.0)
