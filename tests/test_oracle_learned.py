"""The oracle's learned warm start on the CPU (no GPU): its plumbing, checked
through properties that need no network.

With the standardisation y mean 0 / std 1 and network outputs of exactly 0,
the warm start applies p = base + 0 * scale = base: 0 before the density
solve and the carried density kappa before the divergence solve.  In FIXED
mode that is exactly where the plain solver starts (the pressures travel
with the re-sort), so the two oracles must agree bit for bit, frame after
frame; a carry that missed a permutation, or a clamp that moved a start,
would show.  Outputs of 1e30 instead hit the upper clamp, max(d_i, kappa).
"""
import numpy as np
import pytest

from fluid_step import _abi, scene

FIELDS = [_abi.FE_FIELD_POSITION_A, _abi.FE_FIELD_VELOCITY_A, _abi.FE_FIELD_VELOCITY_B,
          _abi.FE_FIELD_DENSITY, _abi.FE_FIELD_PRESSURE, _abi.FE_FIELD_SOURCE_TERM,
          _abi.FE_FIELD_ENTRY_INDEX]


def _norm():
    n = np.zeros(28, np.float32)
    n[12:24] = 1.0
    n[26:28] = 1.0
    return n


def _scene(n_keep=3000):
    w = scene.workload("dam_break_16k")
    p = _abi.copy_params(w.params)
    p.mode = _abi.FE_MODE_FIXED
    p.solver = _abi.FE_SOLVER_TOLERANCE
    pos = w.positions()[:n_keep].copy()
    vel = np.random.default_rng(5).normal(0, 0.3, pos.shape).astype(np.float32)
    return p, pos, vel


def test_zero_outputs_give_the_plain_solver_bit_for_bit(oracle_mod):
    p, pos, vel = _scene()
    plain = oracle_mod.Oracle(p, pos, vel)
    lrn = oracle_mod.Oracle(p, pos, vel)
    lrn.set_learned(_norm())
    for f in range(4):
        lrn.set_network_outputs(np.zeros((4, pos.shape[0], 2), np.float32))
        a = plain.step(2)
        b = lrn.step(2)
        assert not lrn.missing_network_outputs()
        assert a.density_iterations == b.density_iterations
        assert a.divergence_residual == b.divergence_residual
        for fld in FIELDS:
            assert np.array_equal(plain.field(fld), lrn.field(fld)), (f, fld)
        for slot in range(4):
            rows = lrn.feature_rows(slot)
            assert np.all(rows[:, 12:] == 0)
            assert np.any(rows[:, :12] != 0)


def test_large_outputs_are_clamped_to_the_bound(oracle_mod):
    """Outputs far above any solution start every solve at its upper bound,
    a finite pressure; the run stays finite."""
    p, pos, vel = _scene()
    lrn = oracle_mod.Oracle(p, pos, vel)
    lrn.set_learned(_norm())
    for _ in range(3):
        lrn.set_network_outputs(np.full((2, pos.shape[0], 2), 1e30, np.float32))
        st = lrn.step(1)
        assert np.all(np.isfinite(lrn.field(_abi.FE_FIELD_PRESSURE)))
        assert np.isfinite(st.max_speed)


def test_missing_outputs_are_reported(oracle_mod):
    p, pos, vel = _scene(500)
    lrn = oracle_mod.Oracle(p, pos, vel)
    lrn.set_learned(_norm())
    lrn.set_network_outputs(np.zeros((1, pos.shape[0], 2), np.float32))  # density solve only
    lrn.step(1)
    assert lrn.missing_network_outputs()


def test_bf16_rounding_of_feature_rows_is_nearest_even(oracle_mod):
    """Feature 3 is min(neighbour count, 64) / 32: with a zero mean and unit
    standard deviation its BF16 value is exact, so the row holds the count."""
    p, pos, vel = _scene(2000)
    lrn = oracle_mod.Oracle(p, pos, vel)
    lrn.set_learned(_norm())
    lrn.set_network_outputs(np.zeros((2, pos.shape[0], 2), np.float32))
    lrn.step(1)
    rows = lrn.feature_rows(0)
    f3 = (rows[:, 3].astype(np.uint32) << 16).view(np.float32)
    cnt = np.round(f3 * 32)
    assert np.array_equal(f3, (cnt / 32).astype(np.float32))
    assert cnt.max() <= 64 and cnt.mean() > 10
