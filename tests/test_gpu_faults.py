"""Failure paths driven from the host, without faulting the GPU: injected
device-allocation failures, poisoned allocations (a read of memory no pass
wrote would surface as NaN or a wrong index), and a bounded device wait that
runs out."""
import ctypes
import time

import numpy as np
import pytest

from test_gpu_parity import CASES, _run_frames, _scene
from fluid_step import _abi, scene
from fluid_step.pipelines import Simulation

pytestmark = pytest.mark.gpu


@pytest.fixture
def lib():
    L = _abi.load_library()
    yield L
    L.fe_debug_fail_allocation(0)
    L.fe_debug_poison_allocations(0)


def _create(L, p, pos):
    flat = np.ascontiguousarray(pos, np.float32)
    h = ctypes.c_void_p()
    rc = L.fe_create(ctypes.byref(p), flat.shape[0], flat.ctypes.data_as(ctypes.c_void_p), None, 0,
                     ctypes.byref(h))
    return rc, h


def test_every_creation_allocation_failure_is_reported_and_released(lib):
    import torch
    p, pos = _scene(n_drop=7)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    failures = 0
    for k in range(1, 200):
        lib.fe_debug_fail_allocation(k)
        rc, h = _create(lib, p, pos)
        if rc == _abi.FE_OK:
            lib.fe_debug_fail_allocation(0)
            assert lib.fe_destroy(h) == _abi.FE_OK
            break
        assert rc == _abi.FE_ERR_OUT_OF_MEMORY, (k, rc)
        assert b"injected" in lib.fe_last_error()
        assert not h.value
        failures += 1
    else:
        pytest.fail("creation never succeeded")
    assert failures >= 10          # every buffer of the context was tried
    torch.cuda.synchronize()
    # nothing is left allocated by the failed creations (driver granularity slack)
    assert free0 - torch.cuda.mem_get_info()[0] < 8 << 20


def test_later_allocation_failure_leaves_the_context_usable(lib):
    p, pos = _scene(n_drop=7)
    sim = Simulation(pos, p)
    sim.step(1)
    lib.fe_debug_fail_allocation(1)
    assert lib.fe_density_splat(sim.data.handle) == _abi.FE_ERR_OUT_OF_MEMORY
    lib.fe_debug_fail_allocation(0)
    grid = sim.data.splat_density()      # the retry allocates and splats
    assert grid.sum() > 0
    sim.step(1)
    sim.close()


@pytest.mark.parametrize("case", ["reference_k4", "tolerance_cfl", "bitonic"])
def test_poisoned_allocations_keep_parity(lib, oracle_mod, case):
    lib.fe_debug_poison_allocations(1)
    p, pos = _scene(n_drop=5)
    for k, v in CASES[case].items():
        setattr(p, k, v)
    sim, orc, st = _run_frames(oracle_mod, p, pos, frames=3, substeps=2)
    assert st.flags & _abi.FE_STATS_NON_FINITE == 0
    grid = sim.data.splat_density()
    assert np.array_equal(grid, oracle_mod.splat_density(sim.data.download(_abi.FE_FIELD_POSITION_A),
                                                         sim.data.current_params()))
    sim.close()


def test_bounded_wait_runs_out_and_the_device_stays_usable(lib):
    flags = ctypes.c_uint32(7)
    t0 = time.perf_counter()
    rc = lib.fe_debug_bounded_wait(0, 2000, ctypes.byref(flags))
    assert time.perf_counter() - t0 < 5.0
    assert rc == _abi.FE_ERR_TIMEOUT
    assert flags.value & _abi.FE_STATS_LOOKBACK_TIMEOUT
    assert b"timed out" in lib.fe_last_error()
    # the device still sorts
    keys = np.random.default_rng(4).integers(0, 1 << 32, 5000, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(5000, dtype=np.uint32)
    k, v = keys.copy(), vals.copy()
    assert lib.fe_sort_pairs_host(k.ctypes.data_as(ctypes.c_void_p), v.ctypes.data_as(ctypes.c_void_p),
                                  5000, 32, _abi.FE_SORT_RADIX) == _abi.FE_OK
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k, keys[order]) and np.array_equal(v, vals[order])
