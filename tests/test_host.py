"""Host-side logic that needs no GPU: arithmetic-form selection, the autotune
cache, synthetic scenes, the SDF input generator's initialisation and the
error behaviour of the drop-in wrappers on CPU tensors."""
import json
import math

import numpy as np
import pytest
import torch

from benchkit import scenes
from geraf_b200 import autotune, runtime


def test_precision_selection(monkeypatch):
    monkeypatch.delenv("GERAF_RF_PRECISION", raising=False)
    assert runtime.default_precision() == "mixed"
    monkeypatch.setenv("GERAF_RF_PRECISION", "plain")
    assert runtime.default_precision() == "plain"
    with runtime.precision("mixed"):
        assert runtime.default_precision() == "mixed"
        assert runtime.mode_code(None) == 1
    assert runtime.mode_code(None) == 0
    with pytest.raises(ValueError):
        with runtime.precision("fast"):
            pass
    monkeypatch.setenv("GERAF_RF_PRECISION", "bogus")
    assert runtime.default_precision() == "mixed"


def test_nufft_form_is_matched_filter_only(monkeypatch):
    monkeypatch.setenv("GERAF_RF_PRECISION", "nufft")
    assert runtime.default_precision() == "nufft"
    assert runtime.mode_code(None, allow_nufft=True) == 2
    assert runtime.mode_code(None) == 1  # ambient nufft: the tracer runs mixed
    with pytest.raises(ValueError, match="matched filter"):
        runtime.mode_code("nufft")
    assert runtime.mode_code("nufft", allow_nufft=True) == 2


def test_dtype_codes_and_errors():
    assert runtime.dtype_code(torch.zeros(1), "op", True) == 0
    assert runtime.dtype_code(torch.zeros(1, dtype=torch.float64), "op", True) == 1
    assert runtime.dtype_code(torch.zeros(1, dtype=torch.float16), "op", True) == 2
    with pytest.raises(RuntimeError, match="not implemented for 'Half'"):
        runtime.dtype_code(torch.zeros(1, dtype=torch.float16), "op", False)
    with pytest.raises(RuntimeError, match="not implemented"):
        runtime.dtype_code(torch.zeros(1, dtype=torch.int32), "op", True)


def test_autotune_cache_roundtrip(tmp_path, monkeypatch):
    path = tmp_path / "tune.json"
    monkeypatch.setenv("GERAF_RF_TUNE_CACHE", str(path))
    autotune.clear()
    assert autotune.lookup("mf_forward", (8, 4, 100), 1) is None
    autotune.record("mf_forward", (8, 4, 100), 1, {"threads": 256, "items_per_thread": 2})
    assert autotune.lookup("mf_forward", (8, 4, 100), 1)["threads"] == 256
    data = json.loads(path.read_text())
    assert any(k.startswith("mf_forward|1|8x4x100|") for k in data)
    autotune.clear()
    monkeypatch.setenv("GERAF_RF_TUNE_CACHE", str(path))
    autotune._loaded_from = None
    assert autotune.lookup("mf_forward", (8, 4, 100), 1)["items_per_thread"] == 2
    # candidate lists are well-formed launch shapes
    for c in autotune.mf_forward_candidates(1) + autotune.sample_major_candidates() + autotune.tracer_backward_candidates():
        assert c["threads"] in (64, 128, 256)


def test_virtual_arrays_and_grids():
    tx, rx = scenes.virtual_array(16)
    assert tx.shape == (3072, 3) and rx.shape == (3072, 3) and tx.dtype == np.float32
    tx, rx = scenes.virtual_array(64)
    assert tx.shape[0] == 49152
    v = scenes.voxel_grid(48)
    assert v.shape == (3, 48 ** 3)
    assert np.isclose(v[2].mean(), 0.4, atol=1e-6) and np.isclose(v[0].max() - v[0].min(), 0.2, atol=1e-6)
    ch = scenes.chirp(128)
    assert math.isclose(ch.slope, 1.5625e14) and math.isclose(ch.As_sci, 1.5625e6)
    assert math.isclose(scenes.chirp(256).As_sci, 7.8125e5)


def test_shell_torus_scene():
    rng = np.random.default_rng(0)
    pos, amp = scenes.shell_torus_scene(rng)
    assert pos.shape == (30000, 3) and amp.shape == (30000,)
    rel = pos - np.array([0, 0, 0.4])
    shell = np.abs(rel[:20000]).max(axis=1)
    assert np.all(shell <= 0.15 + 1e-6) and np.all(shell >= 0.147 - 1e-6)
    torus = rel[20000:]
    ring = np.hypot(np.hypot(torus[:, 0], torus[:, 1]) - 0.08, torus[:, 2])
    assert np.allclose(ring, 0.03, atol=1e-6)


def test_sdf_geometric_init_is_a_sphere():
    from benchkit.sdf import SDFNetwork

    torch.manual_seed(0)
    net = SDFNetwork()
    x = torch.randn(512, 3)
    x = x / x.norm(dim=1, keepdim=True) * torch.rand(512, 1)
    sdf, feat = net(x)
    assert feat.shape == (512, 256)
    # approximately |x| - 0.5 (the init is exact only in the infinite-width limit)
    target = x.norm(dim=1) - 0.5
    dev = (sdf[:, 0] - target).detach()
    assert dev.abs().mean() < 0.15
    assert torch.corrcoef(torch.stack([sdf[:, 0].detach(), target]))[0, 1] > 0.9


def test_wrappers_reject_cpu_tensors_before_any_gpu_call():
    from geraf_b200.ops.RFMatchedFilter import matched_filter_cuda
    from geraf_b200.ops.RFSignalTracer import signal_tracer_cuda

    with pytest.raises(AssertionError, match="CUDA"):
        matched_filter_cuda(torch.zeros(2, 4), torch.zeros(2, 4), torch.zeros(2, 3), torch.zeros(2, 3),
                            torch.zeros(5, 3), 2, 4, 5e6, 1.0, 5)
    with pytest.raises(ValueError, match="CUDA"):
        signal_tracer_cuda(torch.zeros(5, 3), torch.zeros(2, 5), torch.zeros(5, 3), torch.zeros(2, 3),
                           torch.zeros(2, 3), torch.ones(5, dtype=torch.bool), 4, 5e6, 770.0, 1.0, 2, 5)


def test_model_utils_reject_other_backends():
    from geraf_b200 import model_utils

    cfg = scenes.chirp(8).radar_cfg()
    with pytest.raises(ValueError, match="Only 'cuda'"):
        model_utils.base_matched_filter(None, None, torch.zeros(1, 3), None, torch.zeros(1, 3), cfg,
                                        backend="cpu")
    with pytest.raises(ValueError, match="Only 'cuda'"):
        model_utils.lensless_ray_tracer(torch.zeros(2, 3), None, torch.zeros(2, 3), torch.zeros(1, 3),
                                        None, cfg, backend="numpy")
    with pytest.raises(ValueError, match="Unsupported backend"):
        model_utils.bilinear_ray_sampler(torch.zeros(1, 2, 3), torch.zeros(1, 1, 2), None,
                                         torch.zeros(1, 2), backend="torch")


def test_volume_grid_layout_matches_reference_reshape():
    """Flat index = (ix * Ny + iy) * Nz + iz, as np.fromfile(...).reshape(nx, ny, nz) reads it."""
    from geraf_b200 import volume

    bound = [0.5, 0.503, -0.37, -0.368, -0.15, -0.146]
    res = [0.001, 0.001, 0.002]
    assert volume.grid_shape(bound, res) == (4, 3, 3)
    v = volume.grid_voxels(bound, res).numpy()
    nx, ny, nz = volume.grid_shape(bound, res)
    g = v.reshape(nx, ny, nz, 3)
    assert np.allclose(g[2, 1, 0], [0.502, -0.369, -0.15], atol=1e-7)
    assert np.allclose(g[3, 2, 2], [0.503, -0.368, -0.146], atol=1e-7)
    part = volume.grid_voxels(bound, res, start=5, count=7).numpy()
    assert np.array_equal(part, v[5:12])
    with pytest.raises(ValueError):
        volume.grid_num(1.0, 0.0, 0.0)


def test_sarimage_roundtrip_and_sampling(tmp_path):
    from geraf_b200 import volume

    vol = torch.arange(4 * 3 * 5, dtype=torch.float32).reshape(4, 3, 5)
    p = tmp_path / "sarimage.bin"
    volume.write_sarimage(str(p), vol)
    assert np.array_equal(volume.read_sarimage(str(p), (4, 3, 5)), vol.numpy())
    # corners of the normalised cube hit the corner voxels (align_corners=True), in the
    # FP64 restatement of the reference's sampling; the library samples on the GPU only
    from oracle import rf_oracle as orc

    pts = torch.tensor([[-1.0, -1.0, -1.0], [1.0, 1.0, 1.0], [1.0, -1.0, 1.0]])
    got = orc.sample_volume(vol.numpy(), pts.numpy())
    assert np.allclose(got, [vol[0, 0, 0], vol[3, 2, 4], vol[3, 0, 4]])
    with pytest.raises(ValueError, match="CUDA"):
        volume.sample_volume(vol, pts)


def test_stage1_eval_geometry_helpers():
    """Surface samples lie on the analytic cube + torus, the grid zero-crossing
    extractor recovers a sphere, and the Chamfer distance behaves as a metric."""
    from benchkit import stage1_eval as ev

    rng = np.random.default_rng(0)
    pts = ev.analytic_surface_points(4000, rng).astype(np.float64) - np.array([0.0, 0.0, 0.4])
    on_cube = np.isclose(np.abs(pts).max(1), 0.15, atol=1e-6)
    rho = np.hypot(pts[:, 0], pts[:, 1])
    on_torus = np.isclose((rho - 0.08) ** 2 + pts[:, 2] ** 2, 0.03 ** 2, atol=1e-7)
    assert np.all(on_cube | on_torus) and on_cube.any() and on_torus.any()

    center = torch.tensor([0.0, 0.0, 0.4])

    def sphere(x):  # normalised coordinates, radius 0.5 -> 0.1 m at scale 0.2
        return x.norm(dim=-1, keepdim=True) - 0.5, None

    surf = ev.sdf_surface_points(sphere, center, 0.2, res=48)
    radius = (surf - center).norm(dim=-1)
    assert surf.shape[0] > 1000 and torch.allclose(radius, torch.full_like(radius, 0.1), atol=2e-4)
    a = torch.tensor(rng.standard_normal((300, 3)), dtype=torch.float32)
    assert ev.chamfer(a, a) == 0.0
    assert ev.chamfer(a, a + torch.tensor([0.01, 0.0, 0.0])) > 0.0


def test_missing_library_fails_loudly():
    """Without the built CUDA library the loader every operator goes through raises:
    nothing falls back to a CPU path."""
    import os
    import subprocess
    import sys

    code = (
        "import torch\n"
        "from geraf_b200 import _lib\n"
        "_lib.LIB_PATH = '/nonexistent/libgeraf_rf.so'\n"
        "from geraf_b200.ops.RFMatchedFilter import _C\n"
        "try:\n"
        "    _lib.load()\n"
        "except ImportError as e:\n"
        "    print('raised:', e)\n"
    )
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, PYTHONPATH=os.path.join(root, "geraf-sens_b200") + os.pathsep + root)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    assert "raised:" in out.stdout and "not found" in out.stdout


def _surely_culled_f32(tx, rx, n, p):
    """numpy FP32 restatement of surely_culled() in csrc/tracer_geometry.cuh."""
    f = np.float32
    i = (p - tx).astype(f)
    o = (rx - p).astype(f)
    inn = (i * n).sum(-1, dtype=f)
    ii, nn = (i * i).sum(-1, dtype=f), (n * n).sum(-1, dtype=f)
    back = (inn > 0) & (inn * inn > f(1e-8) * (ii * nn))
    r = (i - f(2.0) * inn[:, None] * n).astype(f)
    orr = (o * r).sum(-1, dtype=f)
    m = f(1.0) + f(2.0) * nn
    away = (orr < 0) & (orr * orr > f(1e-8) * ((o * o).sum(-1, dtype=f) * ii * (m * m)))
    return back | away


def _culled_reference_f32(tx, rx, n, p):
    """The reference's FP32 culling (SignalTracer_cuda_kernel.cu:172-197, 417-420)."""
    f = np.float32

    def normalize(v):
        return (v * (f(1.0) / (np.sqrt((v * v).sum(-1, dtype=f)) + f(1e-7)))[:, None]).astype(f)

    inc = normalize((p - tx).astype(f))
    idn = (inc * n).sum(-1, dtype=f)
    refl = normalize((inc - f(2.0) * idn[:, None] * n).astype(f))
    ret = normalize((rx - p).astype(f))
    align = (ret * refl).sum(-1, dtype=f)
    return (align < f(1e-6)) | (idn > 0)


def test_early_cull_is_conservative():
    """Every pair the tracer kernels' early test culls is culled by the reference's
    FP32 geometry, on random and near-boundary pairs with unit and non-unit normals
    (the early test only skips work the exact form would discard)."""
    rng = np.random.default_rng(0)
    f = np.float32
    total = kept_early = 0
    for trial in range(8):
        M = 400_000
        tx = rng.normal(0, 0.05, (M, 3)).astype(f)
        rx = (tx + rng.normal(0, 0.01, (M, 3))).astype(f)
        p = (np.array([0, 0, 0.4]) + rng.normal(0, 0.1, (M, 3))).astype(f)
        n = rng.normal(0, 1, (M, 3))
        n /= np.linalg.norm(n, axis=1, keepdims=True)
        if trial % 2:   # non-unit normals
            n *= rng.uniform(0.1, 3.0, (M, 1))
        i = (p - tx).astype(np.float64)
        if trial in (4, 5):  # push pairs onto the back-facing boundary, i.n = 0
            n -= ((i * n).sum(1) / (i * i).sum(1))[:, None] * i * rng.uniform(0.999, 1.001, (M, 1))
        if trial in (6, 7):  # and onto the alignment boundary, o.r = 0
            r = i - 2.0 * (i * n).sum(1)[:, None] * n / (n * n).sum(1)[:, None]
            o = rng.normal(0, 1, (M, 3))
            o -= ((o * r).sum(1) / (r * r).sum(1))[:, None] * r * rng.uniform(0.999, 1.001, (M, 1))
            rx = (p + 0.3 * o / np.linalg.norm(o, axis=1, keepdims=True)).astype(f)
        n = n.astype(f)
        early = _surely_culled_f32(tx, rx, n, p)
        exact = _culled_reference_f32(tx, rx, n, p)
        assert not np.any(early & ~exact)
        total += M
        kept_early += int(early.sum())
    assert kept_early > total // 4  # the early test does take most culled pairs


def _aperture_f64(tx, rx):
    """numpy restatement of aperture_kernel() in csrc/tracer_precull.cu."""
    t, r = tx.astype(np.float64), rx.astype(np.float64)
    ct, cr = t.mean(0), r.mean(0)
    rt = np.sqrt(((t - ct) ** 2).sum(1)).max()
    rr = np.sqrt(((r - cr) ** 2).sum(1)).max()
    rt += 1e-12 * (rt + np.abs(ct).sum())
    rr += 1e-12 * (rr + np.abs(cr).sum())
    return ct, rt, cr, rr


def _culled_for_all_f64(ap, n, p):
    """numpy restatement of culled_for_all() in csrc/tracer_precull.cu."""
    ct, rt, cr, rr = ap
    n = n.astype(np.float64)
    ic = p.astype(np.float64) - ct
    oc = cr - p.astype(np.float64)
    nn = (n * n).sum(1)
    nrm = np.sqrt(nn)
    m = 1.0 + 2.0 * nn
    icn = (ic * n).sum(1)
    ni = np.sqrt((ic * ic).sum(1))
    no = np.sqrt((oc * oc).sum(1))
    back = icn - rt * nrm > 1e-4 * (ni + rt) * nrm
    hi = ic - 2.0 * icn[:, None] * n
    ho = oc - 2.0 * (oc * n).sum(1)[:, None] * n
    bound = (oc * hi).sum(1) + rr * np.sqrt((hi * hi).sum(1)) + rt * np.sqrt((ho * ho).sum(1)) + m * rr * rt
    away = bound < -1e-4 * (no + rr) * (ni + rt) * m
    return back | away


def test_point_precull_is_conservative():
    """Every point the tracer's per-point pre-cull leaves out is culled for every
    antenna of the call by the reference's FP32 geometry: compact and wide
    apertures, unit and non-unit normals, and points pushed onto the boundary of
    the back-facing bound (the pre-cull only skips work the exact form discards)."""
    rng = np.random.default_rng(1)
    f = np.float32
    skipped = total = 0
    for trial in range(8):
        A, M = 48, 60_000
        spread = (0.002, 0.02, 0.1, 0.3)[trial % 4]
        tx = (np.array([0.0, 0.0, 0.0]) + rng.normal(0, spread, (A, 3))).astype(f)
        rx = (tx + rng.normal(0, spread / 2, (A, 3))).astype(f)
        p = (np.array([0, 0, 0.4]) + rng.normal(0, 0.15, (M, 3))).astype(f)
        n = rng.normal(0, 1, (M, 3))
        n /= np.linalg.norm(n, axis=1, keepdims=True)
        if trial >= 4:
            n *= rng.uniform(0.1, 3.0, (M, 1))
        ap = _aperture_f64(tx, rx)
        if trial in (2, 6):
            # normals tilted so that i_c.n - R_t|n| sits just above the margin
            ct, rt = ap[0], ap[1]
            ic = p.astype(np.float64) - ct
            d = np.linalg.norm(ic, axis=1)
            u = ic / d[:, None]
            cos_a = np.minimum((rt + 1e-4 * (d + rt)) / d * (1 + rng.uniform(1e-9, 1e-6, M)), 1.0)
            w = rng.normal(0, 1, (M, 3))
            w -= (w * u).sum(1)[:, None] * u
            w /= np.linalg.norm(w, axis=1, keepdims=True)
            scale = np.linalg.norm(n, axis=1)[:, None]
            n = (cos_a[:, None] * u + np.sqrt(1 - cos_a ** 2)[:, None] * w) * scale
        n = n.astype(f)
        skip = _culled_for_all_f64(ap, n, p)
        for a in range(A):
            exact = _culled_reference_f32(np.broadcast_to(tx[a], p.shape), np.broadcast_to(rx[a], p.shape), n, p)
            assert not np.any(skip & ~exact), (trial, a)
        skipped += int(skip.sum())
        total += M
    assert skipped > total // 4  # most points facing away are left out
