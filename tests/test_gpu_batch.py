"""Batched independent scenes: every scene of the packed systems must evolve as
if it were solved alone.  Gauss-Seidel cloths are colored per scene, so each
cloth matches its solo run exactly; piles (Jacobi, float-atomic order) match to
1e-4 m over a few frames, and their candidate pairs match the solo pairs."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from xpbd_b200.batch import BatchedScenes, SceneSpec, batch_specs  # noqa: E402


def _small_specs():
    return [SceneSpec("cloth", 6, 0), SceneSpec("pile", 8, 1), SceneSpec("cloth", 9, 2),
            SceneSpec("pile", 27, 3), SceneSpec("cloth", 12, 4), SceneSpec("pile", 1, 5),
            SceneSpec("pile", 40, 6)]


@pytest.mark.parametrize("mode", ["gs", "jacobi"])
def test_batched_scenes_match_solo(mode):
    b = BatchedScenes(_small_specs(), cloth_mode=mode, substeps=10, iterations=2)
    solos = {i: b.solo(i) for i in range(len(b.specs))}
    frames = 8
    for _ in range(frames):
        b.step()
        for s in solos.values():
            s.step()
    torch.cuda.synchronize()
    res = b.residuals()
    for i, s in solos.items():
        x = b.scene_positions(i)
        d = np.abs(x - s.positions()).max()
        if b.specs[i].kind == "cloth":
            assert d <= (0.0 if mode == "gs" else 1e-4), (i, d)
            assert abs(res[i] - s.residual()[0]) <= (0.0 if mode == "gs" else 1e-4)
        else:
            assert d <= 1e-4, (i, d)
            assert abs(res[i] - s.residual()[0]) <= 1e-4
    assert b.piles.status() == 0


def test_batched_pairs_equal_solo_pairs():
    b = BatchedScenes(_small_specs(), substeps=10, iterations=2)
    b.piles.sync_pairs = True
    solos = {i: b.solo(i) for i, sp in enumerate(b.specs) if sp.kind == "pile"}
    for s in solos.values():
        s.sync_pairs = True
    for _ in range(6):
        b.piles.step()
        for s in solos.values():
            s.step()
    allp = b.piles.pairs()
    for k, i in enumerate(b.pile_ids):
        b0, b1 = b.pile_bodies[k]
        mine = allp[(allp[:, 0] >= b0) & (allp[:, 0] < b1)] - b0
        np.testing.assert_array_equal(mine, solos[i].pairs())
        assert np.all(allp[(allp[:, 0] >= b0) & (allp[:, 0] < b1)][:, 1] < b1)


def test_batch_specs_distribution():
    sp = batch_specs(256, seed=0)
    cl = [s.size for s in sp if s.kind == "cloth"]
    pi = [s.size for s in sp if s.kind == "pile"]
    assert len(cl) == len(pi) == 128
    assert min(cl) >= 16 and max(cl) <= 128 and min(pi) >= 64 and max(pi) <= 1024


def test_sharded_batch_holds_only_its_scenes():
    """A rank's share of a sharded batch (scene_ids): only those scenes are
    built, each still evolves exactly as when solved alone, and the residuals of
    the scenes held elsewhere are NaN (the all-gather fills them in)."""
    specs = _small_specs()
    mine = [1, 2, 4, 6]
    b = BatchedScenes(specs, substeps=10, iterations=2, scene_ids=mine)
    assert b.scene_ids == mine
    assert sorted(b.cloth_ids + b.pile_ids) == mine
    assert b.cloth.num_bodies == sum(specs[i].size ** 2 for i in mine if specs[i].kind == "cloth")
    assert b.piles.num_bodies == sum(specs[i].size for i in mine if specs[i].kind == "pile")
    solos = {i: b.solo(i) for i in mine}
    b.reset_projection_count()
    for _ in range(4):
        b.step()
        for s in solos.values():
            s.step()
    torch.cuda.synchronize()
    res = b.residuals()
    for i in range(len(specs)):
        if i not in mine:
            assert np.isnan(res[i])
            continue
        d = np.abs(b.scene_positions(i) - solos[i].positions()).max()
        assert d <= (0.0 if specs[i].kind == "cloth" else 1e-4), (i, d)
    # projections: cloth rows x S x I per frame plus the pile substeps' counted points
    assert b.projections(4) > 4 * 10 * 2 * b.cloth.num_constraints
