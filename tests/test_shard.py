"""Host logic of the multi-GPU batch path, on CPU: LPT partition of scenes and
the all-gather of per-scene metrics over a world-size-2 gloo process group."""

import os
import socket

import numpy as np
import pytest

from xpbd_b200.shard import gather_scene_metrics, lpt_partition, scene_cost


class _Spec:
    def __init__(self, kind, size):
        self.kind, self.size = kind, size


def test_lpt_partition_covers_and_balances():
    rng = np.random.default_rng(0)
    costs = rng.integers(1, 1000, 257).astype(float)
    for n in (1, 2, 3, 8):
        parts = lpt_partition(costs, n)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [costs[p].sum() for p in parts]
        # LPT bound: max load <= (4/3 - 1/(3n)) OPT <= that times the average
        assert max(loads) <= (4 / 3) * max(np.mean(loads), costs.max()) + 1e-9
        assert parts == lpt_partition(costs, n)  # deterministic


def test_lpt_partition_edge_cases():
    assert lpt_partition([], 4) == [[], [], [], []]
    assert lpt_partition([5.0], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        lpt_partition([1.0], 0)


def test_scene_cost_matches_row_counts():
    # 32 x 32 cloth: 1984 structural + 1922 shear + 1920 bend + 1024 floor rows
    assert scene_cost(_Spec("cloth", 32)) == 1984 + 1922 + 1920 + 1024
    assert scene_cost(_Spec("pile", 100)) == 1000


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n_total, costs, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = lpt_partition(costs, world)[rank]
        vals = [1000.0 * rank + i for i in mine]  # a metric that records who computed it
        out = gather_scene_metrics(mine, vals, n_total)
        q.put((rank, out.tolist()))
    finally:
        dist.destroy_process_group()


def test_gather_scene_metrics_gloo_world2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    costs = list(np.random.default_rng(1).integers(1, 100, 11).astype(float))
    procs = [ctx.Process(target=_worker, args=(r, 2, port, len(costs), costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    parts = lpt_partition(costs, 2)
    expect = np.zeros(len(costs))
    for r, ids in enumerate(parts):
        for i in ids:
            expect[i] = 1000.0 * r + i
    for r in range(2):
        np.testing.assert_array_equal(np.asarray(res[r]), expect)


def test_gather_without_process_group_is_local():
    out = gather_scene_metrics([1, 3], [0.5, 0.25], 4)
    assert out[1] == 0.5 and out[3] == 0.25 and np.isnan(out[0]) and np.isnan(out[2])


def _scene_residuals(specs, ids, frames=2):
    """Each scene of `ids` stepped alone on the CPU oracle (the stepping path a
    rank runs for its share, with the oracle standing in for the device)."""
    from oracle import oracle as O
    from xpbd_b200.batch import CLOTH_KW, PILE_KW, build_cloth_scene, build_pile_k
    out = []
    for i in ids:
        sp = specs[i]
        if sp.kind == "cloth":
            s = O.OracleSolver(solve_mode="gs", **CLOTH_KW)
            build_cloth_scene(s, sp.size)
        else:
            s = O.OracleSolver6DOF(**PILE_KW)
            build_pile_k(s, sp.size, sp.seed)
        for _ in range(frames):
            s.step()
        out.append(float(s.residual()))
    return out


def _batch_worker(rank, world, port, q):
    import torch.distributed as dist

    from oracle import oracle as O
    from xpbd_b200.batch import CLOTH_KW, PILE_KW, batch_specs, build_batch, rank_scene_ids
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        specs = batch_specs(10, seed=3, cloth_range=(4, 8), pile_range=(4, 12))
        ids = rank_scene_ids(specs, rank, world)
        # the rank's packed systems hold exactly its scenes
        lay = build_batch(specs, ids, O.OracleSolver(solve_mode="gs", **CLOTH_KW), O.OracleSolver6DOF(**PILE_KW))
        res = _scene_residuals(specs, ids)
        out = gather_scene_metrics(ids, res, len(specs))
        q.put((rank, ids, lay.cloth_ids, lay.pile_ids, lay.cloth_bodies, lay.cloth_rows, lay.pile_bodies,
               out.tolist()))
    finally:
        dist.destroy_process_group()


def test_sharded_batch_gloo_world2():
    """Two gloo ranks split a batch of ten small scenes by LPT: each rank builds
    exactly its scenes (body and row ranges as the specs give them), steps them,
    and the all-gathered per-scene residuals cover every scene once and equal a
    single-process run of all scenes."""
    import torch.multiprocessing as mp

    from xpbd_b200.batch import batch_specs, rank_scene_ids
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_batch_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(2):
        item = q.get(timeout=300)
        got[item[0]] = item[1:]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    specs = batch_specs(10, seed=3, cloth_range=(4, 8), pile_range=(4, 12))
    ids0, ids1 = got[0][0], got[1][0]
    assert sorted(ids0 + ids1) == list(range(len(specs))) and not set(ids0) & set(ids1)
    assert ids0 == rank_scene_ids(specs, 0, 2) and ids1 == rank_scene_ids(specs, 1, 2)
    for r in (0, 1):
        ids, cloth_ids, pile_ids, cloth_bodies, cloth_rows, pile_bodies, _ = got[r]
        assert sorted(cloth_ids + pile_ids) == ids
        assert all(specs[i].kind == "cloth" for i in cloth_ids) and all(specs[i].kind == "pile" for i in pile_ids)
        b = 0
        for i, (b0, b1) in zip(cloth_ids, cloth_bodies):
            assert (b0, b1) == (b, b + specs[i].size ** 2)
            b = b1
        r0 = 0
        for i, (a0, a1) in zip(cloth_ids, cloth_rows):
            assert (a0, a1) == (r0, r0 + int(scene_cost(specs[i])))
            r0 = a1
        b = 0
        for i, (b0, b1) in zip(pile_ids, pile_bodies):
            assert (b0, b1) == (b, b + specs[i].size)
            b = b1
    expect = np.asarray(_scene_residuals(specs, list(range(len(specs)))))
    for r in (0, 1):
        np.testing.assert_array_equal(np.asarray(got[r][-1]), expect)
