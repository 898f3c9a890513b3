"""Batched scenes across GPUs: one process per GPU, each advancing its own
share of the scenes in one batch context, no collective inside a step.

A single scene does not shard (every neighbour pass would need a halo of
ghost cells and the sort is global), so multi-GPU runs split *scenes*: the
partition is a greedy longest-processing-time assignment of scenes, by
particle count, to the least-loaded rank, identical on every rank because it
depends only on the counts.  After the run the per-scene stats are gathered
to every rank (one all_gather of a small float64 tensor per call); that is
the only communication.
"""
from __future__ import annotations

import heapq

import numpy as np

from . import _abi

STAT_FIELDS = ("max_speed", "avg_density_error_f64", "avg_divergence_error_f64",
               "density_residual", "divergence_residual", "dt", "density_iterations",
               "divergence_iterations", "substeps", "flags")


def lpt_partition(work, n_ranks: int) -> list:
    """Scenes per rank: scenes in decreasing work (ties by index) each go to
    the rank with the least work so far (ties by rank).  Deterministic."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(work)), key=lambda k: (-work[k], k))
    heap = [(0, r) for r in range(n_ranks)]
    out = [[] for _ in range(n_ranks)]
    for k in order:
        load, r = heapq.heappop(heap)
        out[r].append(k)
        heapq.heappush(heap, (load + work[k], r))
    return [sorted(v) for v in out]


def imbalance(work, parts) -> float:
    """max rank load over mean rank load (1.0 = perfect)."""
    loads = [sum(work[k] for k in p) for p in parts]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean else 1.0


def stats_row(st: _abi.FeStats) -> np.ndarray:
    return np.array([float(getattr(st, f)) for f in STAT_FIELDS], dtype=np.float64)


def gather_scene_stats(local_scenes, local_rows, n_scenes: int, group=None, device=None):
    """All-gathers per-scene stats rows: returns float64[n_scenes][len(STAT_FIELDS)]
    on every rank, row k for scene k.  local_rows[i] belongs to
    local_scenes[i].  Uses torch.distributed (NCCL on GPUs, gloo on CPU);
    with no process group it returns the local rows in place."""
    import torch
    import torch.distributed as dist

    width = len(STAT_FIELDS) + 1
    buf = np.full((n_scenes, width), np.nan)
    mine = np.zeros((n_scenes, width))
    for k, row in zip(local_scenes, local_rows):
        mine[k, :-1] = row
        mine[k, -1] = 1.0                     # owner mark
    if not (dist.is_available() and dist.is_initialized()):
        return mine[:, :-1]
    t = torch.from_numpy(mine)
    if device is not None:
        t = t.to(device)
    parts = [torch.zeros_like(t) for _ in range(dist.get_world_size(group))]
    dist.all_gather(parts, t, group=group)
    for p in parts:
        p = p.cpu().numpy()
        own = p[:, -1] == 1.0
        buf[own] = p[own]
    if np.isnan(buf[:, -1]).any():
        raise RuntimeError("a scene has no owner rank")
    return buf[:, :-1]


def _dist_ready() -> bool:
    import torch.distributed as dist
    return dist.is_available() and dist.is_initialized()


def max_over_ranks(value: float, device=None, group=None) -> float:
    """The largest `value` over the ranks of the process group (the value
    itself without one)."""
    if not _dist_ready():
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64)
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def run_scene_shard(work, rank: int, world: int, open_shard, steps: int, warmup: int,
                    device=None, group=None) -> dict:
    """One rank's part of a scene-sharded run.

    The rank takes its LPT share of the scenes (`work` = particles per scene),
    opens one batch over them with open_shard(scene_indices), runs `warmup`
    untimed steps, then `steps` timed ones (shard.timed_steps(k) returns the
    seconds its own clock measured), and closes it.  The time is the maximum
    over ranks; the per-scene stats rows are all-gathered into the table of
    every scene.  Every rank makes the same collective calls in the same
    order: a barrier before the timed steps, the max, the gather.

    The shard object provides step(), timed_steps(k) -> seconds,
    scene_stats(i) -> FeStats of its i-th scene, close()."""
    parts = lpt_partition(work, world)
    mine = parts[rank]
    shard = open_shard(mine)
    try:
        for _ in range(warmup):
            shard.step()
        if _dist_ready():
            import torch.distributed as dist
            dist.barrier(group=group)
        seconds = shard.timed_steps(steps)
        rows = [stats_row(shard.scene_stats(i)) for i in range(len(mine))]
    finally:
        shard.close()
    seconds = max_over_ranks(seconds, device=device, group=group)
    table = gather_scene_stats(mine, rows, len(work), group=group, device=device)
    return {"parts": parts, "mine": mine, "seconds": seconds, "table": table,
            "imbalance": imbalance(work, parts)}
