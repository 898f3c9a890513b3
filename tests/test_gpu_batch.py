"""Batched scenes (fe_batch_create): each scene of a batch gets the result it
gets in a context of its own, bit for bit, and therefore the oracle's.

Keys, indices and bucket starts of a batch are offset by the scene's table
base and first particle; they are compared after removing the offset.
"""
import numpy as np
import pytest

from fluid_step import _abi, scene
from fluid_step.pipelines import BatchSimulation, Simulation

pytestmark = pytest.mark.gpu

PARTICLE_FIELDS = [_abi.FE_FIELD_POSITION_A, _abi.FE_FIELD_POSITION_B, _abi.FE_FIELD_VELOCITY_A,
                   _abi.FE_FIELD_VELOCITY_B, _abi.FE_FIELD_DENSITY, _abi.FE_FIELD_FACTOR,
                   _abi.FE_FIELD_SOURCE_TERM, _abi.FE_FIELD_PRESSURE,
                   _abi.FE_FIELD_PRESSURE_ACCEL]
STAT_NAMES = ("max_speed_bits", "density_error_fp", "divergence_error_fp", "density_iterations",
              "divergence_iterations", "avg_density_error_f64", "avg_divergence_error_f64",
              "density_residual", "divergence_residual", "dt", "substeps",
              "total_density_iterations", "total_divergence_iterations")


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def assert_same(a, b, what):
    a, b = bits(a), bits(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    bad = np.nonzero(a.reshape(-1) != b.reshape(-1))[0]
    assert bad.size == 0, f"{what}: {bad.size} of {a.size} differ, first at {bad[0]}"


def small_batch(counts=(1, 256, 257, 3001, 1700), seed=3):
    rng = np.random.Generator(np.random.PCG64(seed))
    boxes = []
    for n in counts:
        edge = float((n * 0.05 ** 3 / 0.25) ** (1 / 3))
        boxes.append(((0.0, 0.0, 0.0), (max(edge, 0.3),) * 3))
    return scene.BatchWorkload("small", list(counts), boxes,
                               list(rng.uniform(0.005, 0.05, len(counts))), 3, seed)


def compare_with_singles(batch: BatchSimulation, singles, label):
    d = batch.data
    base = 0
    for s, single in enumerate(singles):
        n = int(d.scene_count[s])
        t = 1 << max(0, (n - 1).bit_length())
        for f in PARTICLE_FIELDS:
            assert_same(d.scene(d.download(f), s), single.data.download(f),
                        f"{label} scene {s} field {f}")
        first = int(d.scene_first[s])
        hsh = d.scene(d.download(_abi.FE_FIELD_ENTRY_HASH), s).astype(np.int64) - base
        idx = d.scene(d.download(_abi.FE_FIELD_ENTRY_INDEX), s).astype(np.int64) - first
        assert_same(hsh.astype(np.uint32),
                    single.data.download(_abi.FE_FIELD_ENTRY_HASH)[:n], f"{label} {s} hash")
        assert_same(idx.astype(np.uint32),
                    single.data.download(_abi.FE_FIELD_ENTRY_INDEX)[:n], f"{label} {s} index")
        gs = d.download(_abi.FE_FIELD_GRID_START)[base:base + t].astype(np.int64)
        gs = np.where(gs == 0xFFFFFFFF, gs, gs - first).astype(np.uint32)
        assert_same(gs, single.data.download(_abi.FE_FIELD_GRID_START), f"{label} {s} grid_start")
        a, b = d.read_scene_stats(s), single.data.read_stats()
        for name in STAT_NAMES:
            assert getattr(a, name) == getattr(b, name), (label, s, name, getattr(a, name),
                                                          getattr(b, name))
        base += t


def run_both(w, params, frames, substeps=1):
    pos = w.positions()
    batch = BatchSimulation(pos, params)
    singles = [Simulation(p, q) for p, q in zip(pos, params)]
    for _ in range(frames):
        batch.step(substeps)
        for sim in singles:
            sim.step(substeps)
    return batch, singles


def close_all(batch, singles):
    batch.close()
    for s in singles:
        s.close()


def test_batch_reference_mode_equals_single_scenes():
    w = small_batch()
    batch, singles = run_both(w, w.params(), frames=3)
    assert batch.data.n_scenes == 5
    assert list(batch.data.scene_count) == w.counts
    compare_with_singles(batch, singles, "reference k4")
    close_all(batch, singles)


def test_batch_per_scene_solver_and_cfl():
    """Scenes differ in solver, tolerance and time-step control: scene 1 runs
    fixed iterations, the others the tolerance solver with adaptive CFL from
    different initial dt, so every scene takes its own iteration counts and
    dt sequence inside the same launches."""
    w = small_batch(counts=(2000, 700, 4100, 33), seed=5)
    params = w.params()
    for k, p in enumerate(params):
        p.mode = _abi.FE_MODE_FIXED
        if k != 1:
            p.solver = _abi.FE_SOLVER_TOLERANCE
            p.use_cfl = 1
            p.dt = 0.002 + 0.001 * k
            p.density_tolerance = 0.001 * (k + 1)
    batch, singles = run_both(w, params, frames=4, substeps=2)
    compare_with_singles(batch, singles, "mixed solvers")
    dts = [batch.data.read_scene_stats(s).dt for s in range(4)]
    assert len(set(dts)) > 1
    close_all(batch, singles)


def test_batch_matches_oracle(oracle_mod):
    w = small_batch(counts=(900, 2500, 64), seed=7)
    pos, params = w.positions(), w.params()
    batch = BatchSimulation(pos, params)
    orcs = [oracle_mod.Oracle(q, p) for p, q in zip(pos, params)]
    for _ in range(2):
        batch.step(1)
        for o in orcs:
            o.step(1)
    d = batch.data
    for s, o in enumerate(orcs):
        for f in PARTICLE_FIELDS:
            assert_same(d.scene(d.download(f), s), o.field(f), f"oracle scene {s} field {f}")
    batch.close()


def test_set_scene_params_touches_one_scene():
    w = small_batch(counts=(1500, 1500, 1500), seed=9)
    params = w.params()
    batch = BatchSimulation(w.positions(), params)
    q = _abi.copy_params(params[1])
    q.viscosity = 0.3
    q.gravity[:] = [0.0, -3.0, 0.0]
    batch.data.set_scene_params(1, q)
    assert batch.data.scene_params(1).viscosity == pytest.approx(0.3)
    assert batch.data.scene_params(0).viscosity == pytest.approx(params[0].viscosity)
    params = [params[0], q, params[2]]
    singles = [Simulation(p, pp) for p, pp in zip(w.positions(), params)]
    for _ in range(2):
        batch.step(1)
        for sim in singles:
            sim.step(1)
    compare_with_singles(batch, singles, "set_scene_params")
    close_all(batch, singles)


def test_full_size_batch_advances():
    """The 64-scene batch (4.2M particles): a few frames, every scene's stats
    finite and its own."""
    w = scene.batch_workload()
    sim = BatchSimulation(w.positions(), w.params())
    for _ in range(3):
        st = sim.step(1)
    assert not (st.flags & _abi.FE_STATS_NON_FINITE)
    for s in (0, 17, 63):
        ss = sim.data.read_scene_stats(s)
        assert ss.substeps == 1 and np.isfinite(ss.avg_density_error_f64)
        assert ss.density_iterations == 4 and ss.divergence_iterations == 4
    sim.close()
