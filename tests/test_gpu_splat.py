"""The density splat (splat_density.comp) as a headless grid: bit-exact with
the oracle's loop-by-loop restatement, and exactly additive over particle
sets at sizes the oracle cannot run quickly."""
import ctypes

import numpy as np
import pytest

from fluid_step import _abi, scene
from fluid_step.pipelines import BatchSimulation, Simulation

pytestmark = pytest.mark.gpu


def _params(res):
    w = scene.workload("dam_break_16k")
    p = _abi.copy_params(w.params)
    p.grid_res[:] = list(res)
    return w, p


@pytest.mark.parametrize("res", [(64, 64, 64), (40, 24, 56), (128, 128, 128)])
def test_splat_matches_oracle(oracle_mod, res):
    w, p = _params(res)
    sim = Simulation(w.positions(), p)
    orc = oracle_mod.Oracle(p, w.positions())
    for frames in (0, 3):
        for _ in range(frames):
            sim.step(1)
            orc.step(1)
        got = sim.data.splat_density()
        ref = oracle_mod.splat_density(orc.field(_abi.FE_FIELD_POSITION_A), p)
        assert got.shape == (res[2], res[1], res[0])
        assert np.array_equal(got, ref), (frames, int(np.abs(got.astype(np.int64) - ref).max()))
        assert got.sum() > 0
    sim.close()


def test_splat_boundaries(oracle_mod):
    """Particles on box_min, on box_max (centre voxel = grid_res, outside the
    grid, its neighbours inside), just outside the box, and a clump."""
    _, p = _params((32, 16, 24))
    lo, hi = np.asarray(p.box_min, np.float32), np.asarray(p.box_max, np.float32)
    pts = [lo, hi, (lo + hi) / 2, hi + np.float32(1e-3), lo - np.float32(1e-3),
           np.array([hi[0], lo[1], (lo[2] + hi[2]) / 2], np.float32)]
    pts += [(lo + hi) / 3 + np.float32(0.001) * k for k in range(50)]
    pos = np.stack(pts).astype(np.float32)
    sim = Simulation(pos, p)
    got = sim.data.splat_density()
    pos4 = np.concatenate([pos, np.ones((pos.shape[0], 1), np.float32)], 1)
    ref = oracle_mod.splat_density(pos4, p)
    assert np.array_equal(got, ref)
    sim.close()


def test_splat_is_additive_at_262k():
    w = scene.workload("dam_break_256k")
    p = _abi.copy_params(w.params)
    p.grid_res[:] = [128, 128, 128]
    pos = w.positions()
    half = pos.shape[0] // 2
    grids = []
    for part in (pos, pos[:half], pos[half:]):
        sim = Simulation(part, p)
        grids.append(sim.data.splat_density().astype(np.uint64))
        sim.close()
    assert np.array_equal(grids[0], grids[1] + grids[2])
    # and repeatable: a second splat of the same state is identical
    sim = Simulation(pos, p)
    a = sim.data.splat_density()
    b = sim.data.splat_density()
    assert np.array_equal(a, b) and np.array_equal(a.astype(np.uint64), grids[0])
    sim.close()


def test_splat_errors():
    w, p = _params((16, 16, 16))
    sim = Simulation(w.positions()[:500], p)
    lib = sim.data._lib
    out = np.empty(16 ** 3, np.uint32)
    # no grid before the first splat
    assert lib.fe_download(sim.data.handle, _abi.FE_FIELD_DENSITY_GRID,
                           out.ctypes.data_as(ctypes.c_void_p), out.nbytes) \
        == _abi.FE_ERR_INVALID_ARGUMENT
    q = _abi.copy_params(p)
    q.grid_res[:] = [0, 16, 16]
    sim.data.sync_with_scene(q)
    assert lib.fe_density_splat(sim.data.handle) == _abi.FE_ERR_INVALID_ARGUMENT
    sim.close()
    b = scene.batch_workload(n_scenes=2, lo=500, hi=900)
    bs = BatchSimulation(b.positions(), b.params())
    assert bs.data._lib.fe_density_splat(bs.data.handle) == _abi.FE_ERR_UNSUPPORTED
    bs.close()
