"""Training steps built from the operators, captured in CUDA graphs: a replayed
step reproduces the eager step exactly (the kernels are deterministic), and the
stage-1 step trains (finite, moving loss) in both arithmetic forms."""
import numpy as np
import pytest
import torch

from benchkit import scenes

pytestmark = pytest.mark.gpu


def ragged_inputs(seed=0, A=6, S=64, N=512):
    rng = np.random.default_rng(seed)
    tx, rx = scenes.virtual_array(2)
    tx, rx = tx[:A].copy(), rx[:A].copy()
    counts = rng.integers(200, 2500, A)
    P = int(counts.sum())
    d = rng.normal(0, 1, (P, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pts = (np.array([0, 0, 0.4]) + 0.08 * d).astype(np.float32)
    nrm = d - 0.9 * np.array([0, 0, 1.0])
    nrm = (nrm / np.linalg.norm(nrm, axis=1, keepdims=True)).astype(np.float32)
    vox = scenes.voxel_grid(8, size=0.16).T.copy()
    cu = lambda x: torch.tensor(x, device="cuda")  # noqa: E731
    ch = scenes.chirp(S)
    return dict(normals=cu(nrm), sigmas=cu(rng.uniform(0, 1, P).astype(np.float32)), points=cu(pts),
                point_offsets=cu(np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)), tx=cu(tx),
                rx=cu(rx), voxels=cu(vox), target_mag=cu(rng.uniform(0, 1e-3, vox.shape[0]).astype(np.float32)),
                radar_cfg=ch.radar_cfg(fc_start=770.0))


def test_ragged_step_graph_replay_equals_eager(cuda):
    from geraf_b200.step import RaggedRFStep

    inp = ragged_inputs()
    eager = RaggedRFStep(**inp)
    loss_e = eager.run().item()
    grads_e = [t.grad.clone() for t in (eager.normals, eager.sigmas, eager.points)]
    graphed = RaggedRFStep(**inp)
    graphed.capture()
    for _ in range(2):
        loss_g = graphed.run().item()
        torch.cuda.synchronize()
        assert loss_g == loss_e
        for a, b in zip(grads_e, (graphed.normals.grad, graphed.sigmas.grad, graphed.points.grad)):
            assert torch.equal(a, b)
    assert all(torch.isfinite(g).all() for g in grads_e)


@pytest.mark.parametrize("precision", ["mixed", "plain"])
def test_stage1_step_graph_matches_eager_and_trains(cuda, precision):
    from benchkit.stage1 import Stage1RFStep

    kw = dict(num_antennas=8, num_rays=128, samples_per_ray=32, num_adc=32, precision=precision, seed=3)
    eager = Stage1RFStep(**kw)
    losses = [eager.run().item() for _ in range(3)]
    graphed = Stage1RFStep(**kw)
    graphed.capture()          # runs two eager warm-up steps, then records the third
    loss3 = graphed.run().item()
    torch.cuda.synchronize()
    assert np.isfinite(losses).all()
    assert loss3 == pytest.approx(losses[2], rel=1e-5)
    more = [graphed.run().item() for _ in range(5)]
    assert np.isfinite(more).all() and more[-1] != more[0]


def test_stage1_antenna_bank_matches_full_step_and_replays(cuda):
    """With the network unchanged, the banked step's first loss equals the full
    step's (the bank holds every chunk rendered by the same network); the banked
    step rotates through its chunks identically eager and graph-replayed."""
    from benchkit.stage1 import Stage1RFStep

    kw = dict(num_antennas=8, num_rays=128, samples_per_ray=32, num_adc=32, precision="mixed", seed=5)
    full = Stage1RFStep(**kw).run().item()
    banked = Stage1RFStep(bank_size=4, **kw)
    assert banked.run().item() == pytest.approx(full, rel=1e-5)

    eager = Stage1RFStep(bank_size=2, **kw)
    losses = [eager.run().item() for _ in range(4)]
    graphed = Stage1RFStep(bank_size=2, **kw)
    graphed.capture()          # two eager warm-up steps (chunks 0, 1), then records a step
    more = [graphed.run().item() for _ in range(2)]   # replays on chunks 0, 1
    torch.cuda.synchronize()
    assert np.isfinite(losses).all() and np.isfinite(more).all()
    assert more[0] == pytest.approx(losses[2], rel=1e-5)
    assert more[1] == pytest.approx(losses[3], rel=1e-5)
