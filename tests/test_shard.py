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
