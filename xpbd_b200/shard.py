"""Sharding independent scenes across GPUs (one process per GPU).

A single scene does not shard (every Jacobi/Gauss-Seidel iteration needs every
correction of the previous one), so one scene runs as replicas.  A batch of
independent scenes does shard: scenes are assigned to ranks by LPT (longest
processing time first) bin packing on their projection count, each rank steps
its scenes with no communication, and at the end one all-gather collects the
per-scene metrics (residual, projections) on every rank.
"""

from __future__ import annotations

import heapq

import numpy as np


def scene_cost(spec) -> float:
    """Projections per substep-iteration of one scene (the work estimate):
    cloth n x n: 7 n^2 rows (structural, shear, bend, floor); pile of k boxes:
    8 floor slots per box plus about two manifold points per box."""
    if spec.kind == "cloth":
        n = spec.size
        return float(2 * n * (n - 1) + 2 * (n - 1) ** 2 + 2 * n * max(n - 2, 0) + n * n)
    return float(10 * spec.size)


def lpt_partition(costs, n_ranks: int):
    """Assign items to ranks, heaviest first, each to the least-loaded rank
    (ties: lowest rank).  Returns one ascending index list per rank."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(n_ranks)]
    heapq.heapify(heap)
    parts = [[] for _ in range(n_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def gather_scene_metrics(local_ids, local_values, n_total, group=None):
    """All-gather per-scene float metrics from every rank into one array of
    length n_total (index = scene id).  Works with any torch.distributed backend
    (NCCL on GPUs, gloo on CPU); with no process group it returns the local part."""
    import torch
    import torch.distributed as dist

    out = np.full(n_total, np.nan, np.float64)
    if not (dist.is_available() and dist.is_initialized()):
        out[np.asarray(local_ids, int)] = np.asarray(local_values, np.float64)
        return out
    world = dist.get_world_size(group)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    n_max = int(np.ceil(n_total / 1.0))
    buf = torch.full((2, n_max), -1.0, dtype=torch.float64, device=dev)
    k = len(local_ids)
    buf[0, :k] = torch.as_tensor(np.asarray(local_ids, np.float64), device=dev)
    buf[1, :k] = torch.as_tensor(np.asarray(local_values, np.float64), device=dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    for p in parts:
        p = p.cpu().numpy()
        ids = p[0]
        live = ids >= 0
        out[ids[live].astype(int)] = p[1][live]
    return out
