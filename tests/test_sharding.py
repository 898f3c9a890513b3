"""Scene sharding across ranks (no GPU): the LPT partition and the per-scene
stats gather, the latter with two gloo ranks on CPU."""
import os
import socket

import numpy as np
import pytest

from fluid_step import scene
from fluid_step.sharding import STAT_FIELDS, gather_scene_stats, imbalance, lpt_partition


def test_partition_covers_every_scene_once():
    w = scene.batch_workload()
    for ranks in (1, 2, 3, 4, 8):
        parts = lpt_partition(w.counts, ranks)
        assert len(parts) == ranks
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(w.counts)))
        assert parts == lpt_partition(w.counts, ranks)           # deterministic


def test_partition_balance_meets_the_lpt_bound():
    w = scene.batch_workload()
    for m in (2, 4, 8):
        parts = lpt_partition(w.counts, m)
        loads = [sum(w.counts[k] for k in p) for p in parts]
        lower = max(sum(w.counts) / m, max(w.counts))             # any partition's makespan
        assert max(loads) <= (4 / 3 - 1 / (3 * m)) * lower + 1e-9
        assert imbalance(w.counts, parts) < 1.1


def test_partition_edge_cases():
    assert lpt_partition([], 3) == [[], [], []]
    assert lpt_partition([5], 2) == [[0], []]
    assert lpt_partition([3, 3, 3, 3], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        lpt_partition([1], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, counts, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mine = lpt_partition(counts, world)[rank]
        rows = [np.arange(len(STAT_FIELDS), dtype=np.float64) + 100.0 * k for k in mine]
        table = gather_scene_stats(mine, rows, len(counts))
        q.put((rank, mine, table))
    finally:
        dist.destroy_process_group()


def test_gather_scene_stats_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    counts = scene.batch_workload(n_scenes=11).counts
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, counts, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = np.stack([np.arange(len(STAT_FIELDS), dtype=np.float64) + 100.0 * k
                       for k in range(len(counts))])
    owned = []
    for rank, mine, table in results:
        assert np.array_equal(table, expect), rank
        owned += mine
    assert sorted(owned) == list(range(len(counts)))


def test_gather_without_process_group_returns_local_rows():
    rows = [np.ones(len(STAT_FIELDS)), 2 * np.ones(len(STAT_FIELDS))]
    t = gather_scene_stats([0, 2], rows, 3)
    assert np.array_equal(t[0], rows[0]) and np.array_equal(t[2], rows[1])
    assert np.all(t[1] == 0)


class _StandInShard:
    """A CPU stand-in for one rank's batch context: each step advances every
    scene of the share; a scene's stats name the scene and its step count,
    so the gathered table shows which rank ran which scene how often."""

    def __init__(self, mine, counts):
        self.mine, self.counts, self.steps = list(mine), counts, 0

    def step(self):
        self.steps += 1

    def timed_steps(self, k):
        import time
        t0 = time.perf_counter()
        for _ in range(k):
            self.step()
        # make the ranks' times differ, so that the max over ranks shows
        return time.perf_counter() - t0 + 1e-6 * sum(self.counts[s] for s in self.mine)

    def scene_stats(self, i):
        from fluid_step import _abi
        st = _abi.FeStats()
        k = self.mine[i]
        st.max_speed = float(k)
        st.dt = 1e-3 * (k + 1)
        st.substeps = self.steps
        st.density_iterations = self.counts[k] % 97
        return st

    def close(self):
        pass


def _shard_rank_main(rank, world, port, counts, q):
    import datetime

    import torch.distributed as dist

    from fluid_step.sharding import run_scene_shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        res = run_scene_shard(counts, rank, world, lambda mine: _StandInShard(mine, counts),
                              steps=5, warmup=3)
        own = 1e-6 * sum(counts[s] for s in res["mine"])
        q.put((rank, res["mine"], res["seconds"], own, res["table"]))
    finally:
        dist.destroy_process_group()


def test_sharded_batch_run_two_gloo_ranks():
    """The scene-sharded run path end to end on two gloo ranks: the LPT
    partition, a per-rank stand-in for the batch step (warm-up, timed steps),
    the time as the max over ranks and the gathered per-scene table."""
    import torch.multiprocessing as mp

    from fluid_step.sharding import STAT_FIELDS
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    counts = scene.batch_workload(n_scenes=11).counts
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank_main, args=(r, 2, port, counts, q))
             for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    parts = lpt_partition(counts, 2)
    assert [r[1] for r in results] == parts
    # the time every rank reports is the larger of the two ranks' own
    assert results[0][2] == results[1][2] >= max(r[3] for r in results)
    col = {f: i for i, f in enumerate(STAT_FIELDS)}
    for rank, mine, _, _, table in results:
        assert table.shape == (len(counts), len(STAT_FIELDS))
        assert np.array_equal(table[:, col["max_speed"]], np.arange(len(counts)))
        assert np.all(table[:, col["substeps"]] == 3 + 5)   # warm-up + timed, every scene
        assert np.array_equal(table[:, col["density_iterations"]], np.array(counts) % 97)
