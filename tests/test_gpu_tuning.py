"""The autotuner's candidates change speed, never results: every radix shape
gives the stable sort, frames are bit-identical under every shape, and the
tuner's choice is one of the candidates."""
import ctypes

import numpy as np
import pytest
import torch

from fluid_step import _abi, learned, scene
from fluid_step.pipelines import Simulation

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("digit_bits,items", _abi.RADIX_CANDIDATES)
@pytest.mark.parametrize("n,key_bits", [(2, 32), (255, 8), (1025, 20), (4097, 32),
                                        (65537, 20), (1 << 20, 32), (3 << 19, 23)])
def test_every_radix_shape_is_the_stable_sort(digit_bits, items, n, key_bits):
    lib = _abi.load_library()
    rng = np.random.default_rng(n + 7 * digit_bits + items)
    keys = rng.integers(0, 1 << key_bits, n, dtype=np.uint64).astype(np.uint32)
    if n > 16:
        keys[: n // 3] = keys[n // 2]                 # long runs of equal keys
    vals = np.arange(n, dtype=np.uint32)
    k, v = dev(keys.view(np.int32)), dev(vals.view(np.int32))
    rc = lib.fe_sort_pairs_config(ptr(k), ptr(v), n, key_bits, digit_bits, items, None)
    _abi.check(lib, rc, "fe_sort_pairs_config")
    torch.cuda.synchronize()
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k.cpu().numpy().view(np.uint32), keys[order])
    assert np.array_equal(v.cpu().numpy().view(np.uint32), vals[order])


def _frames(tuning=None, frames=3, autotune=False):
    w = scene.workload("dam_break_16k")
    p = _abi.copy_params(w.params)
    p.solver = _abi.FE_SOLVER_TOLERANCE
    p.mode = _abi.FE_MODE_FIXED
    sim = Simulation(w.positions(), p)
    report = None
    if autotune:
        report = sim.data.autotune()
    if tuning is not None:
        sim.data.set_tuning(tuning)
    for _ in range(frames):
        st = sim.step(1)
    out = {f: sim.data.download(f).copy() for f in (_abi.FE_FIELD_POSITION_A,
                                                    _abi.FE_FIELD_VELOCITY_A,
                                                    _abi.FE_FIELD_PRESSURE,
                                                    _abi.FE_FIELD_ENTRY_INDEX)}
    t = sim.data.tuning()
    sim.close()
    return out, st, t, report


def _same(a, b):
    for f in a:
        assert np.array_equal(a[f].view(np.uint32), b[f].view(np.uint32)), f


@pytest.mark.parametrize("digit_bits,items", _abi.RADIX_CANDIDATES)
def test_frames_identical_under_every_shape(digit_bits, items):
    ref, st_ref, _, _ = _frames()
    got, st, t, _ = _frames(_abi.FeTuning(digit_bits, items, 3, 0))
    assert (t.radix_digit_bits, t.radix_items, t.mlp_ctas_per_sm) == (digit_bits, items, 3)
    _same(ref, got)
    assert st.total_density_iterations == st_ref.total_density_iterations


def test_autotune_picks_a_candidate_and_keeps_results():
    ref, _, _, _ = _frames()
    got, _, t, report = _frames(autotune=True)
    _same(ref, got)
    assert (t.radix_digit_bits, t.radix_items) in _abi.RADIX_CANDIDATES
    assert report.radix_candidates == len(_abi.RADIX_CANDIDATES)
    assert all(report.radix_ms[k] > 0 for k in range(report.radix_candidates))
    best = min(range(report.radix_candidates), key=lambda k: report.radix_ms[k])
    assert (report.radix_digit_bits[best], report.radix_items[best]) == \
        (t.radix_digit_bits, t.radix_items)
    assert report.mlp_candidates == 0


def test_set_tuning_rejects_non_candidates():
    w = scene.workload("dam_break_16k")
    sim = Simulation(w.positions()[:2000], w.params)
    lib = sim.data._lib
    for bad in (_abi.FeTuning(9, 8, 3, 0), _abi.FeTuning(8, 5, 3, 0), _abi.FeTuning(8, 8, 0, 0),
                _abi.FeTuning(8, 8, 7, 0)):
        assert lib.fe_set_tuning(sim.data.handle, ctypes.byref(bad)) == \
            _abi.FE_ERR_INVALID_ARGUMENT
    sim.close()


def test_autotune_with_model_tunes_the_network_grid():
    x, y = learned.capture(workload_names=("dam_break_16k",), frames=(20,), strides=(8,))
    m = learned.train(x, y, epochs=3).model
    w = scene.workload("dam_break_16k")
    p = _abi.copy_params(w.params)
    p.solver, p.mode, p.warm_start = (_abi.FE_SOLVER_TOLERANCE, _abi.FE_MODE_FIXED,
                                      _abi.FE_WARM_LEARNED)
    runs = []
    for ctas in (None, 2, 6):
        sim = Simulation(w.positions(), p)
        _abi.check(sim.data._lib, sim.data._lib.fe_set_model(sim.data.handle, m.handle), "")
        if ctas is None:
            r = sim.data.autotune()
            assert r.mlp_candidates == 4 and all(r.mlp_ms[k] > 0 for k in range(4))
        else:
            sim.data.set_tuning(_abi.FeTuning(8, 16, ctas, 0))
        for _ in range(3):
            sim.step(1)
        runs.append(sim.data.download(_abi.FE_FIELD_POSITION_A).copy())
        sim.close()
    for r in runs[1:]:
        assert np.array_equal(runs[0].view(np.uint32), r.view(np.uint32))
    m.close()


def test_autotune_sort_applies_to_fe_sort_pairs():
    lib = _abi.load_library()
    n = 1 << 18
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    k, v = dev(keys.view(np.int32)), dev(vals.view(np.int32))
    r = _abi.FeTuneReport()
    assert lib.fe_autotune_sort(ptr(k), ptr(v), n, 32, ctypes.byref(r)) == 0
    assert (r.chosen.radix_digit_bits, r.chosen.radix_items) in _abi.RADIX_CANDIDATES
    # the tuning run left the inputs alone
    assert np.array_equal(k.cpu().numpy().view(np.uint32), keys)
    assert lib.fe_sort_pairs(ptr(k), ptr(v), n, 32, _abi.FE_SORT_RADIX, None) == 0
    torch.cuda.synchronize()
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k.cpu().numpy().view(np.uint32), keys[order])
    assert np.array_equal(v.cpu().numpy().view(np.uint32), vals[order])


# --------------------------------------------------------------------------
# Neighbour-kernel shapes: threads per block and persistent grids over the
# chunk (scene-offset) table
# --------------------------------------------------------------------------
NBR_SHAPES = [(128, 0), (256, 0), (512, 0), (128, 1), (256, 1), (512, 1)]


def _nbr_tuning(threads, persistent):
    """Every neighbour group at (threads, persistent), as far as the group
    takes that block size (density_alpha 128/256, pressure_update 256)."""
    t = _abi.FeTuning(8, 16, 3, 0)
    for g in range(_abi.FE_NBR_GROUPS):
        tg = threads
        if g == _abi.FE_NBR_DENSITY_ALPHA:
            tg = min(threads, 256)
        if g == _abi.FE_NBR_PRESSURE_UPDATE:
            tg = 256
        t.nbr_threads[g] = tg
        t.nbr_persistent[g] = persistent
    return t


@pytest.mark.parametrize("threads,persistent", NBR_SHAPES)
def test_frames_identical_under_every_neighbour_shape(threads, persistent):
    ref, st_ref, _, _ = _frames()
    got, st, t, _ = _frames(_nbr_tuning(threads, persistent))
    assert list(t.nbr_persistent) == [persistent] * 4
    _same(ref, got)
    assert st.total_density_iterations == st_ref.total_density_iterations
    assert st.density_residual == st_ref.density_residual


@pytest.mark.parametrize("threads,persistent", [(128, 1), (512, 0), (512, 1)])
def test_learned_frames_identical_under_neighbour_shapes(threads, persistent):
    """The source passes that also emit the warm start's features."""
    m = learned.Model(seed=5)
    w = scene.workload("dam_break_16k")
    p = _abi.copy_params(w.params)
    p.solver, p.mode, p.warm_start = (_abi.FE_SOLVER_TOLERANCE, _abi.FE_MODE_FIXED,
                                      _abi.FE_WARM_LEARNED)
    runs = []
    for tuning in (None, _nbr_tuning(threads, persistent)):
        sim = Simulation(w.positions(), p)
        _abi.check(sim.data._lib, sim.data._lib.fe_set_model(sim.data.handle, m.handle), "")
        if tuning is not None:
            sim.data.set_tuning(tuning)
        for _ in range(3):
            sim.step(1)
        runs.append({f: sim.data.download(f).copy() for f in (_abi.FE_FIELD_POSITION_A,
                                                              _abi.FE_FIELD_PRESSURE)})
        sim.close()
    _same(runs[0], runs[1])
    m.close()


def test_persistent_batch_matches_one_block_per_chunk():
    """A persistent grid strides over the chunks of all scenes of a batch;
    every scene's result is the same as with one block per chunk."""
    from fluid_step.pipelines import BatchSimulation
    w = scene.workload("dam_break_16k")
    base = w.positions()
    pos = [base[:3000].copy(), base[:16384].copy(), base[:777].copy()]
    pars = []
    for k in range(3):
        p = _abi.copy_params(w.params)
        p.mode = _abi.FE_MODE_FIXED
        p.solver = _abi.FE_SOLVER_TOLERANCE if k != 1 else _abi.FE_SOLVER_FIXED_ITERS
        pars.append(p)
    runs = []
    for tuning in (None, _nbr_tuning(512, 1), _nbr_tuning(128, 1)):
        sim = BatchSimulation(pos, pars)
        if tuning is not None:
            sim.data.set_tuning(tuning)
        for _ in range(3):
            sim.step(1)
        runs.append(sim.data.download(_abi.FE_FIELD_POSITION_A).copy())
        sim.close()
    for r in runs[1:]:
        assert np.array_equal(runs[0].view(np.uint32), r.view(np.uint32))


def test_autotune_times_neighbour_shapes_and_restores_the_state():
    """After a frame the tuner also times every neighbour shape on the
    current state; the state afterwards is bit for bit what it was, and the
    run continues exactly as an untuned one."""
    w = scene.workload("dam_break_16k")
    p = _abi.copy_params(w.params)
    p.solver, p.mode = _abi.FE_SOLVER_TOLERANCE, _abi.FE_MODE_FIXED
    ref = Simulation(w.positions(), p)
    sim = Simulation(w.positions(), p)
    ref.step(1)
    sim.step(1)
    before = {f: sim.data.download(f).copy() for f in
              (_abi.FE_FIELD_POSITION_A, _abi.FE_FIELD_PRESSURE, _abi.FE_FIELD_DENSITY,
               _abi.FE_FIELD_SOURCE_TERM, _abi.FE_FIELD_VELOCITY_A)}
    r = sim.data.autotune()
    after = {f: sim.data.download(f).copy() for f in before}
    _same(before, after)
    assert r.nbr_candidates == len(NBR_SHAPES)
    t = sim.data.tuning()
    for g in range(_abi.FE_NBR_GROUPS):
        timed = [k for k in range(r.nbr_candidates) if r.nbr_ms[g][k] >= 0]
        assert timed and all(r.nbr_ms[g][k] > 0 for k in timed)
        best = min(timed, key=lambda k: r.nbr_ms[g][k])
        assert (r.nbr_threads[best], r.nbr_persistent[best]) == \
            (t.nbr_threads[g], t.nbr_persistent[g])
    assert all(r.nbr_threads[k] == 256 for k in range(r.nbr_candidates)
               if r.nbr_ms[_abi.FE_NBR_PRESSURE_UPDATE][k] >= 0)
    for _ in range(3):
        ref.step(1)
        sim.step(1)
    for f in before:
        assert np.array_equal(ref.data.download(f).view(np.uint32),
                              sim.data.download(f).view(np.uint32)), f
    ref.close()
    sim.close()


def test_set_tuning_rejects_neighbour_shapes_outside_the_candidates():
    w = scene.workload("dam_break_16k")
    sim = Simulation(w.positions()[:2000], w.params)
    lib = sim.data._lib
    bad = []
    for g, threads, pers in ((_abi.FE_NBR_DENSITY_ALPHA, 512, 0),
                             (_abi.FE_NBR_PRESSURE_UPDATE, 128, 0),
                             (_abi.FE_NBR_LIST_PASSES, 384, 0),
                             (_abi.FE_NBR_PRESSURE_FORCE, 256, 2)):
        t = _abi.FeTuning(8, 16, 3, 0)
        t.nbr_threads[g] = threads
        t.nbr_persistent[g] = pers
        bad.append(t)
    for t in bad:
        assert lib.fe_set_tuning(sim.data.handle, ctypes.byref(t)) == _abi.FE_ERR_INVALID_ARGUMENT
    sim.close()
