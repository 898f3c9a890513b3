"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Bit-exact for every field: the kernels round exactly like the oracle
(IEEE single precision, no contraction, same summation order), so sorts,
permutations, hash tables and all physics fields must be identical, not
merely close.  Sizes are chosen so the oracle finishes in seconds.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN
from fluid_step import _abi, scene
from fluid_step.pipelines import (CommandBufferBuilder, ComputePipelines, GpuPhysicsData,
                                  Simulation, sort_pairs_host)

pytestmark = pytest.mark.gpu

FIELDS = [_abi.FE_FIELD_POSITION_A, _abi.FE_FIELD_POSITION_B, _abi.FE_FIELD_VELOCITY_A,
          _abi.FE_FIELD_VELOCITY_B, _abi.FE_FIELD_DENSITY, _abi.FE_FIELD_FACTOR,
          _abi.FE_FIELD_SOURCE_TERM, _abi.FE_FIELD_PRESSURE, _abi.FE_FIELD_PRESSURE_ACCEL,
          _abi.FE_FIELD_ENTRY_HASH, _abi.FE_FIELD_ENTRY_INDEX, _abi.FE_FIELD_GRID_START,
          _abi.FE_FIELD_STATS]


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def assert_same(gpu, ref, what):
    g, r = bits(gpu), bits(ref)
    assert g.shape == r.shape, (what, g.shape, r.shape)
    bad = np.nonzero(g.reshape(-1) != r.reshape(-1))[0]
    if bad.size:
        i = bad[0]
        raise AssertionError(f"{what}: {bad.size} of {g.size} differ; first at {i}: "
                             f"gpu={gpu.reshape(-1)[i]!r} oracle={ref.reshape(-1)[i]!r}")


def compare_all(data, orc, label, fields=FIELDS):
    for f in fields:
        assert_same(data.download(f), orc.field(f), f"{label}: field {f}")


# --------------------------------------------------------------------------
# Sorting
# --------------------------------------------------------------------------
@pytest.mark.parametrize("n", [1, 2, 7, 255, 4096, 4097, 65537, 1 << 20])
@pytest.mark.parametrize("key_bits", [32, 20, 8])
def test_radix_sort_is_the_stable_sort(n, key_bits):
    rng = np.random.default_rng(n * 31 + key_bits)
    hi = 1 << key_bits
    keys = rng.integers(0, hi, n, dtype=np.uint64).astype(np.uint32)
    if n > 16:
        keys[: n // 4] = keys[0]                              # heavy duplicates
    vals = np.arange(n, dtype=np.uint32)
    k, v = sort_pairs_host(keys, vals, key_bits=key_bits)
    order = np.argsort(keys, kind="stable")
    assert_same(k, keys[order], "keys")
    assert_same(v, vals[order], "values")


def test_radix_sort_matches_reference_mirror(oracle_mod):
    rng = np.random.default_rng(5)
    keys = rng.integers(0, 2**32, 70_000, dtype=np.uint64).astype(np.uint32)
    vals = rng.integers(0, 2**32, 70_000, dtype=np.uint64).astype(np.uint32)
    k, v = sort_pairs_host(keys, vals)
    rk, rv = oracle_mod.sort_radix_mirror(keys, vals)
    assert_same(k, rk, "keys")
    assert_same(v, rv, "values")


@pytest.mark.parametrize("n", [2, 1024, 2048, 4096, 1 << 16, 1 << 18])
def test_bitonic_sort_is_the_reference_network(oracle_mod, n):
    rng = np.random.default_rng(n)
    keys = rng.integers(0, max(2, n // 8), n, dtype=np.uint32)  # many ties
    vals = np.arange(n, dtype=np.uint32)
    k, v = sort_pairs_host(keys, vals, algorithm=_abi.FE_SORT_BITONIC)
    rk, rv = oracle_mod.sort_bitonic(keys, vals)
    assert_same(k, rk, "keys")
    assert_same(v, rv, "values (tie order of the network)")


def test_sort_known_answers():
    from test_oracle_golden import kat_inputs, padded
    for name, h in kat_inputs().items():
        k, v = padded(h)
        for algo in (_abi.FE_SORT_RADIX, _abi.FE_SORT_BITONIC):
            ks, vs = sort_pairs_host(k, v, algorithm=algo)
            assert np.array_equal(ks, np.sort(k)), name
            if name == "sentinels_land_at_end":
                assert int(np.searchsorted(ks, 0xFFFFFFFF)) == 100


def test_sort_errors():
    lib = _abi.load_library()
    k = np.zeros(6, np.uint32)
    st = lib.fe_sort_pairs_host(k.ctypes.data_as(ctypes.c_void_p), k.ctypes.data_as(ctypes.c_void_p),
                                6, 32, _abi.FE_SORT_BITONIC)
    assert st == _abi.FE_ERR_INVALID_ARGUMENT                     # not a power of two
    assert lib.fe_sort_pairs_host(None, None, 5, 32, 1) == _abi.FE_ERR_INVALID_ARGUMENT


# --------------------------------------------------------------------------
# Passes
# --------------------------------------------------------------------------
def _scene(n_drop=0, mode=_abi.FE_MODE_REFERENCE, sort=_abi.FE_SORT_RADIX):
    w = scene.workload("dam_break_16k")
    p = _abi.copy_params(w.params)
    p.mode = mode
    p.sort_algorithm = sort
    pos = w.positions()
    if n_drop:
        pos = pos[: pos.shape[0] - n_drop]
    return p, pos


@pytest.mark.parametrize("sort", [_abi.FE_SORT_RADIX, _abi.FE_SORT_BITONIC])
@pytest.mark.parametrize("n_drop", [0, 37])
def test_neighbor_search_bit_exact(oracle_mod, sort, n_drop):
    p, pos = _scene(n_drop, sort=sort)
    data = GpuPhysicsData(pos, p)
    pipes = ComputePipelines()
    pipes.prepare_all(data)
    orc = oracle_mod.Oracle(p, pos)
    b = CommandBufferBuilder(data)
    pipes.neighbor_search.execute(b)
    b.execute_and_wait()
    orc.run("neighbor_search")
    compare_all(data, orc, "neighbor_search",
                [_abi.FE_FIELD_ENTRY_HASH, _abi.FE_FIELD_ENTRY_INDEX, _abi.FE_FIELD_GRID_START,
                 _abi.FE_FIELD_POSITION_B, _abi.FE_FIELD_VELOCITY_B])


@pytest.mark.parametrize("mode", [_abi.FE_MODE_REFERENCE, _abi.FE_MODE_FIXED])
def test_every_pass_bit_exact(oracle_mod, mode):
    """submit_substeps (convergence_benchmark.rs:108-163) pass by pass,
    comparing every field after every pass."""
    p, pos = _scene(n_drop=11, mode=mode)
    data = GpuPhysicsData(pos, p)
    pipes = ComputePipelines()
    pipes.prepare_all(data)
    orc = oracle_mod.Oracle(p, pos)
    b = CommandBufferBuilder(data)
    seq = ["neighbor_search", "density_alpha"]
    for _ in range(2):
        seq += ["viscosity", "density_source"]
        seq += ["pressure_force", "pressure_update"] * 3
        seq += ["pressure_integration", "neighbor_search", "density_alpha", "divergence_source"]
        seq += ["pressure_force", "pressure_update"] * 2
        seq += ["divergence_integration", "stats_pass"]
    attr = {"density_source": "density_source_term", "divergence_source": "divergence_source_term",
            "stats_pass": "stats"}
    for k, name in enumerate(seq):
        getattr(pipes, attr.get(name, name)).execute(b)
        b.execute_and_wait()
        orc.run(name)
        compare_all(data, orc, f"pass {k} {name}")


def _run_frames(oracle_mod, p, pos, frames, substeps=1, flags=0, vel=None):
    sim = Simulation(pos, p, velocities=vel)
    orc = oracle_mod.Oracle(p, pos, vel)
    for f in range(frames):
        st = sim.step(substeps, flags)
        rs = orc.step(substeps, flags & _abi.FE_STEP_INIT_NS)
        for name in ("max_speed_bits", "density_error_fp", "divergence_error_fp",
                     "density_iterations", "divergence_iterations",
                     "avg_density_error_f64", "avg_divergence_error_f64",
                     "density_residual", "divergence_residual", "dt",
                     "density_residual_max", "divergence_residual_max"):
            assert getattr(st, name) == getattr(rs, name), (f, name, getattr(st, name),
                                                           getattr(rs, name))
    compare_all(sim.data, orc, f"after {frames} frames")
    return sim, orc, st


CASES = {
    "reference_k4": dict(),
    "fixed_mode": dict(mode=_abi.FE_MODE_FIXED),
    "tolerance": dict(mode=_abi.FE_MODE_FIXED, solver=_abi.FE_SOLVER_TOLERANCE),
    "tolerance_cfl": dict(mode=_abi.FE_MODE_FIXED, solver=_abi.FE_SOLVER_TOLERANCE, use_cfl=1,
                          dt=0.004),
    "early_exit": dict(use_solver_error_threshold=1, density_error_pct=5.0,
                       divergence_error_pct=5.0),
    "bitonic": dict(sort_algorithm=_abi.FE_SORT_BITONIC),
    "cfl_reference": dict(use_cfl=1, dt=0.005),
    # another smoothing radius: the r / h reciprocal step is checked for it
    # anew, and more particles overflow the 64-entry list into the walk
    "radius_0p12": dict(smoothing_radius=0.12),
}


@pytest.mark.parametrize("case", list(CASES))
def test_frames_bit_exact(oracle_mod, case):
    p, pos = _scene(n_drop=5)
    for k, v in CASES[case].items():
        setattr(p, k, v)
    sim, orc, st = _run_frames(oracle_mod, p, pos, frames=4, substeps=1)
    if case.startswith("tolerance"):
        assert st.density_iterations >= p.min_iterations
        assert st.density_residual <= p.density_tolerance or st.density_iterations == p.max_iterations


def test_multi_substep_and_init_flag(oracle_mod):
    p, pos = _scene()
    _run_frames(oracle_mod, p, pos, frames=2, substeps=3, flags=_abi.FE_STEP_INIT_NS)


def test_graph_and_eager_agree():
    p, pos = _scene(mode=_abi.FE_MODE_FIXED)
    p.solver = _abi.FE_SOLVER_TOLERANCE
    a = Simulation(pos, p)
    b = Simulation(pos, p)
    for _ in range(3):
        sa = a.step(1)
        sb = b.step(1, _abi.FE_STEP_NO_GRAPH)
        assert sa.density_iterations == sb.density_iterations
    for f in FIELDS:
        assert_same(a.data.download(f), b.data.download(f), f"field {f}")


def test_nonzero_initial_velocity(oracle_mod):
    p, pos = _scene(n_drop=3)
    vel = np.random.default_rng(2).normal(0, 0.3, pos.shape).astype(np.float32)
    _run_frames(oracle_mod, p, pos, frames=2, vel=vel)


# --------------------------------------------------------------------------
# Golden vector and edge cases
# --------------------------------------------------------------------------
def test_rest_density_golden_on_gpu(oracle_mod):
    p, pos = scene.rest_density_scene()
    data = GpuPhysicsData(pos, p)
    pipes = ComputePipelines()
    pipes.prepare_all(data)
    b = CommandBufferBuilder(data)
    pipes.neighbor_search.execute(b)
    pipes.density_alpha.execute(b)
    b.execute_and_wait()
    rho = data.download(_abi.FE_FIELD_DENSITY)
    ref = np.load(os.path.join(GOLDEN, "rest_density.npy"))
    rel = np.abs(np.sort(rho) - np.sort(ref)) / np.sort(ref)
    assert rel.max() < 2e-6
    orc = oracle_mod.Oracle(p, pos)
    orc.run("neighbor_search")
    orc.run("density_alpha")
    assert_same(rho, orc.field(_abi.FE_FIELD_DENSITY), "rest density")


@pytest.mark.parametrize("n", [1, 2, 7, 255, 2049])
def test_small_and_ragged_counts(oracle_mod, n):
    p, pos = _scene()
    pos = pos[:n].copy()
    _run_frames(oracle_mod, p, pos, frames=2)


def test_neighbour_list_overflow_falls_back_to_walk(oracle_mod):
    """A clump denser than the list capacity (64): those particles walk the
    buckets in every pass; results stay bit-exact."""
    p, pos = _scene()
    rng = np.random.default_rng(9)
    clump = (np.array([1.0, 0.5, 1.0], np.float32)
             + rng.uniform(-0.03, 0.03, (300, 3)).astype(np.float32))
    pos = np.concatenate([pos[:4000], clump]).astype(np.float32)
    sim, orc, st = _run_frames(oracle_mod, p, pos, frames=2)
    assert st.flags & _abi.FE_STATS_NEIGHBOR_OVERFLOW


def test_particles_outside_the_box(oracle_mod):
    p, pos = _scene()
    pos = pos[:3000].copy()
    pos[:50] += np.float32(5.0)     # outside box_max: clamped by the collisions
    pos[50:100] -= np.float32(3.0)  # negative cells
    _run_frames(oracle_mod, p, pos, frames=2)


def test_execute_before_prepare_raises():
    p, pos = _scene()
    data = GpuPhysicsData(pos[:100], p)
    lib = data._lib
    assert lib.fe_density_alpha(data.handle) == _abi.FE_ERR_NOT_PREPARED
    assert b"prepare" in lib.fe_last_error()
    with pytest.raises(RuntimeError, match="call prepare"):
        ComputePipelines().density_alpha.execute(CommandBufferBuilder(data))


def test_upload_download_size_checks():
    p, pos = _scene()
    data = GpuPhysicsData(pos[:100], p)
    lib = data._lib
    buf = np.zeros(10, np.float32)
    assert lib.fe_download(data.handle, _abi.FE_FIELD_DENSITY, buf.ctypes.data_as(ctypes.c_void_p),
                           buf.nbytes) == _abi.FE_ERR_INVALID_ARGUMENT
    rho = np.full(100, 1000.0, np.float32)
    data.upload(_abi.FE_FIELD_DENSITY, rho)
    assert np.array_equal(data.download(_abi.FE_FIELD_DENSITY), rho)


def test_nan_state_reports_non_finite():
    p, pos = _scene()
    sim = Simulation(pos[:500], p)
    v = np.zeros((500, 4), np.float32)
    v[7, 0] = np.nan
    sim.step(1)
    sim.data.upload(_abi.FE_FIELD_VELOCITY_A, v)
    sim.data.upload(_abi.FE_FIELD_VELOCITY_B, v)
    with pytest.raises(_abi.FluidStepError) as e:
        sim.step(1)
    assert e.value.status == _abi.FE_ERR_NON_FINITE


# --------------------------------------------------------------------------
# Benchmarked sizes: the 2^20-slot hash table, bucket collisions (Q3) and
# neighbour-list overflow at scale
# --------------------------------------------------------------------------
def test_frames_bit_exact_1m_tolerance(oracle_mod):
    """The benchmarked 1M dam break (FIXED mode, Jacobi to 0.1 % density
    and divergence error) with a seeded velocity field, so that the solves
    iterate: 2 frames, every field and every stats word."""
    w = scene.workload("dam_break_1m")
    pos = w.positions()
    vel = np.random.default_rng(3).normal(0, 0.3, pos.shape).astype(np.float32)
    sim, orc, st = _run_frames(oracle_mod, w.params, pos, frames=2, vel=vel)
    assert sim.data.table_size == 1 << 20
    assert st.density_iterations >= 1 and st.divergence_iterations >= 1


def test_frames_bit_exact_4m_tolerance(oracle_mod):
    """The benchmarked 4M dam break (256x64x256 lattice, FIXED mode, the
    tolerance solver): the 2^22-slot hash table, a 22-bit radix key and the
    FP64 residual sums over 16384 chunks; 2 frames from rest, every field and
    every stats word.  The first frames from rest need 19 + 14 iterations,
    which would take the oracle minutes at this size, so the iteration cap is
    4: both solves stop at the cap above the 0.1 % tolerance."""
    w = scene.workload("dam_break_4m")
    p = _abi.copy_params(w.params)
    p.max_iterations = 4
    pos = w.positions()
    sim, orc, st = _run_frames(oracle_mod, p, pos, frames=2)
    assert pos.shape[0] == 1 << 22
    assert sim.data.table_size == 1 << 22
    assert st.density_iterations == 4 and st.divergence_iterations == 4
    assert st.density_residual > p.density_tolerance
    sim.close()


def test_frames_bit_exact_262k_adaptive_cfl(oracle_mod):
    """The 262k dam break with adaptive CFL and the tolerance solver: 3
    frames (dt changes every frame on the device)."""
    w = scene.workload("dam_break_256k")
    _run_frames(oracle_mod, w.params, w.positions(), frames=3)
