"""Checkpoint / resume (fe_state_export / fe_state_import): a context restored
from a snapshot continues bit for bit as the original does, in both modes,
with adaptive CFL, with the learned warm start's carried state and for a
batch; damaged or mismatched snapshots are refused and leave the context as
it was."""
import ctypes
import struct

import numpy as np
import pytest

from fluid_step import _abi, scene
from fluid_step.learned import Model
from fluid_step.pipelines import BatchSimulation, Simulation

pytestmark = pytest.mark.gpu

FIELDS = [_abi.FE_FIELD_POSITION_A, _abi.FE_FIELD_POSITION_B, _abi.FE_FIELD_VELOCITY_A,
          _abi.FE_FIELD_VELOCITY_B, _abi.FE_FIELD_DENSITY, _abi.FE_FIELD_FACTOR,
          _abi.FE_FIELD_SOURCE_TERM, _abi.FE_FIELD_PRESSURE, _abi.FE_FIELD_PRESSURE_ACCEL,
          _abi.FE_FIELD_ENTRY_HASH, _abi.FE_FIELD_ENTRY_INDEX, _abi.FE_FIELD_GRID_START]
STATS = ["max_speed_bits", "density_error_fp", "divergence_error_fp", "substeps", "dt",
         "avg_density_error_f64", "avg_divergence_error_f64", "density_residual",
         "divergence_residual", "density_iterations", "divergence_iterations",
         "total_density_iterations", "total_divergence_iterations", "flags",
         "density_residual_max", "divergence_residual_max"]


def snapshot_of(sim):
    return {f: sim.data.download(f).copy() for f in FIELDS}


def assert_same_state(a, b, label):
    for f in FIELDS:
        assert np.array_equal(a[f].view(np.uint32), b[f].view(np.uint32)), (label, f)


def assert_same_stats(a, b, label):
    for name in STATS:
        assert getattr(a, name) == getattr(b, name), (label, name, getattr(a, name),
                                                      getattr(b, name))


def small_params(mode, solver, cfl):
    w = scene.workload("dam_break_16k")
    p = _abi.copy_params(w.params)
    p.mode = mode
    p.solver = solver
    p.use_cfl = 1 if cfl else 0
    p.sort_algorithm = _abi.FE_SORT_RADIX
    return w.positions(), p


def run(sim, frames, substeps):
    st = None
    for _ in range(frames):
        st = sim.step(substeps)
    return st


@pytest.mark.parametrize("mode,solver,cfl,substeps", [
    (_abi.FE_MODE_REFERENCE, _abi.FE_SOLVER_FIXED_ITERS, False, 2),
    (_abi.FE_MODE_FIXED, _abi.FE_SOLVER_TOLERANCE, True, 1),
])
def test_resume_continues_bit_for_bit(mode, solver, cfl, substeps):
    pos, p = small_params(mode, solver, cfl)
    a = Simulation(pos, p)
    run(a, 6, substeps)
    snap = a.data.export_state()
    hdr = struct.unpack_from("<8sII", snap)
    assert hdr[0] == b"FESTATE\x00" and hdr[1] == _abi.FE_STATE_VERSION
    assert hdr[2] == _abi.ABI_VERSION
    st_a = run(a, 5, substeps)
    want = snapshot_of(a)
    # a fresh context of the same shape, started elsewhere, takes the snapshot
    b = Simulation(pos[::-1].copy(), p)
    run(b, 2, substeps)
    b.data.import_state(snap)
    st_b = run(b, 5, substeps)
    assert_same_state(want, snapshot_of(b), "fresh context")
    assert_same_stats(st_a, st_b, "fresh context")
    if cfl:
        assert st_a.dt != p.dt   # adaptive CFL moved dt away from its start
    # rewinding the original context replays the same frames
    a.data.import_state(snap)
    st_r = run(a, 5, substeps)
    assert_same_state(want, snapshot_of(a), "rewind")
    assert_same_stats(st_a, st_r, "rewind")
    a.close()
    b.close()


def attach(sim, model):
    lib = sim.data._lib
    _abi.check(lib, lib.fe_set_model(sim.data.handle, model.handle), "fe_set_model")


def test_resume_with_learned_carry():
    """The learned warm start carries each particle's last solved pressures
    from frame to frame; the snapshot holds them."""
    pos, p = small_params(_abi.FE_MODE_FIXED, _abi.FE_SOLVER_TOLERANCE, False)
    p.warm_start = _abi.FE_WARM_LEARNED
    model = Model(seed=3)
    model.set_normalization(np.zeros(12), np.ones(12), np.zeros(2), np.full(2, 100.0))
    a = Simulation(pos, p)
    attach(a, model)
    run(a, 4, 1)
    snap = a.data.export_state()
    st_a = run(a, 4, 1)
    want = snapshot_of(a)
    b = Simulation(pos, p)
    attach(b, model)
    b.data.import_state(snap)
    st_b = run(b, 4, 1)
    assert_same_state(want, snapshot_of(b), "learned")
    assert_same_stats(st_a, st_b, "learned")
    # importing before the model is attached restores the carried state too
    q = _abi.copy_params(p)
    q.warm_start = _abi.FE_WARM_REFERENCE
    c = Simulation(pos, q)
    c.data.import_state(snap)
    attach(c, model)
    st_c = run(c, 4, 1)
    assert_same_state(want, snapshot_of(c), "import then attach")
    assert_same_stats(st_a, st_c, "import then attach")
    a.close()
    b.close()
    c.close()
    model.close()


def test_batch_resume():
    counts = (700, 2100, 33)
    boxes = [((0.0, 0.0, 0.0), (max(float((n * 0.05 ** 3 / 0.25) ** (1 / 3)), 0.3),) * 3)
             for n in counts]
    w = scene.BatchWorkload("ckpt", list(counts), boxes, [0.01, 0.02, 0.03], 3, 5)
    pos, params = w.positions(), w.params()
    a = BatchSimulation(pos, params)
    for _ in range(3):
        a.step(1)
    snap = a.data.export_state()
    for _ in range(3):
        a.step(1)
    want = snapshot_of(a)
    b = BatchSimulation(pos, params)
    b.data.import_state(snap)
    for _ in range(3):
        b.step(1)
    assert_same_state(want, snapshot_of(b), "batch")
    for s in range(len(counts)):
        assert_same_stats(a.data.read_scene_stats(s), b.data.read_scene_stats(s), f"scene {s}")
    a.close()
    b.close()


def test_damaged_or_foreign_snapshots_are_refused():
    pos, p = small_params(_abi.FE_MODE_REFERENCE, _abi.FE_SOLVER_FIXED_ITERS, False)
    a = Simulation(pos, p)
    run(a, 3, 1)
    snap = a.data.export_state()
    before = snapshot_of(a)
    lib, h = a.data._lib, a.data.handle

    def rc(buf, n=None):
        b = ctypes.create_string_buffer(bytes(buf), len(buf))
        return lib.fe_state_import(h, b, len(buf) if n is None else n)

    bad = bytearray(snap)
    bad[0:1] = b"X"
    assert rc(bad) == _abi.FE_ERR_INVALID_ARGUMENT
    assert rc(snap[:-4]) == _abi.FE_ERR_INVALID_ARGUMENT
    assert rc(snap[:16]) == _abi.FE_ERR_INVALID_ARGUMENT
    other = Simulation(pos[:1000].copy(), p)
    assert rc(other.data.export_state()) == _abi.FE_ERR_INVALID_ARGUMENT
    # a too-small export buffer is refused too
    size = ctypes.c_size_t()
    assert lib.fe_state_size(h, ctypes.byref(size)) == _abi.FE_OK and size.value == len(snap)
    small = ctypes.create_string_buffer(16)
    assert lib.fe_state_export(h, small, 16) == _abi.FE_ERR_INVALID_ARGUMENT
    assert_same_state(before, snapshot_of(a), "after refused imports")
    other.close()
    a.close()
