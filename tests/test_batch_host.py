"""Host side of batched scenes, without a GPU: argument validation of
fe_batch_create (it runs before any device call) and the batched dam-break
generator."""
import ctypes

import numpy as np
import pytest

from fluid_step import _abi, scene


def _create(lib, params, counts, pos=None):
    ns = len(counts)
    P = (_abi.FeParams * max(ns, 1))(*params)
    C = (ctypes.c_uint32 * max(ns, 1))(*counts)
    if pos is None:
        pos = np.zeros((max(int(sum(counts)), 1), 3), np.float32)
    h = ctypes.c_void_p()
    return lib.fe_batch_create(P, C, ns, pos.ctypes.data_as(ctypes.c_void_p), None, 0,
                               ctypes.byref(h))


@pytest.fixture
def lib():
    return _abi.load_library()


def _params(**kw):
    p = scene.dam_break_params((0, 0, 0), (1, 1, 1))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def test_rejects_empty_and_zero_counts(lib):
    assert _create(lib, [], []) == _abi.FE_ERR_INVALID_ARGUMENT
    assert _create(lib, [_params(), _params()], [10, 0]) == _abi.FE_ERR_INVALID_ARGUMENT


def test_rejects_mixed_mode_and_warm_start(lib):
    a, b = _params(), _params(mode=_abi.FE_MODE_FIXED)
    assert _create(lib, [a, b], [10, 10]) == _abi.FE_ERR_INVALID_ARGUMENT
    c = _params(warm_start=_abi.FE_WARM_LEARNED)
    assert _create(lib, [a, c], [10, 10]) == _abi.FE_ERR_INVALID_ARGUMENT


def test_rejects_bitonic_batches(lib):
    a = _params(sort_algorithm=_abi.FE_SORT_BITONIC)
    assert _create(lib, [a, a], [10, 10]) == _abi.FE_ERR_UNSUPPORTED


def test_rejects_too_many_particles(lib):
    big = _abi.FE_MAX_PARTICLES // 2 + 1
    # counts are checked before positions are read: a 1-particle array is enough
    assert _create(lib, [_params(), _params()], [big, big],
                   pos=np.zeros((1, 3), np.float32)) == _abi.FE_ERR_CAPACITY


def test_rejects_invalid_scene_params(lib):
    bad = _params(smoothing_radius=-1.0)
    assert _create(lib, [_params(), bad], [10, 10]) == _abi.FE_ERR_INVALID_ARGUMENT


def test_rejects_non_finite_positions(lib):
    pos = np.zeros((20, 3), np.float32)
    pos[13, 1] = np.nan
    assert _create(lib, [_params(), _params()], [10, 10], pos=pos) == _abi.FE_ERR_NON_FINITE


def test_batch_workload_is_the_specified_distribution():
    w = scene.batch_workload()
    assert len(w.counts) == 64
    assert all(4096 <= n <= 262144 for n in w.counts)
    logs = np.log(w.counts)
    # log-uniform: the mean of log N sits near the middle of the range
    assert abs(logs.mean() - (np.log(4096) + np.log(262144)) / 2) < 0.5
    assert all(0.005 <= v <= 0.05 for v in w.viscosities)
    for n, (bmin, bmax) in zip(w.counts, w.boxes):
        vol = np.prod(np.subtract(bmax, bmin))
        assert n * 0.05 ** 3 / vol == pytest.approx(0.25, rel=1e-9)
    again = scene.batch_workload()
    assert again.counts == w.counts and again.viscosities == w.viscosities
    assert scene.batch_workload(seed=2).counts != w.counts


def test_batch_positions_fit_their_boxes():
    w = scene.batch_workload(n_scenes=6)
    for pos, n, (bmin, bmax) in zip(w.positions(), w.counts, w.boxes):
        assert pos.shape == (n, 3)
        assert np.all(pos > np.asarray(bmin)) and np.all(pos < np.asarray(bmax))
    params = w.params()
    assert [p.viscosity for p in params] == pytest.approx(w.viscosities)
