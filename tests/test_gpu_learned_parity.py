"""Parity of the learned warm start with the oracle, bit for bit.

The oracle restates the warm start around the network: the 12 features the
source passes emit (their BF16 rows), the clamp and gate of the applied
start, the after-solve bookkeeping and the carry of the last pressures
through every re-sort.  The network itself runs on the tensor cores, whose
accumulation order has no host restatement, so its per-particle outputs are
read back from the GPU (test hook fe_debug_trace_learned) and given to the
oracle for the same solve.  Every feature row, every physics field and the
solver's iteration counts and residuals must then be identical.
"""
import numpy as np
import pytest

from fluid_step import _abi, learned, scene
from fluid_step.pipelines import Simulation
from test_gpu_parity import assert_same, compare_all

pytestmark = pytest.mark.gpu

STATS = ("max_speed_bits", "density_error_fp", "divergence_error_fp", "density_iterations",
         "divergence_iterations", "avg_density_error_f64", "avg_divergence_error_f64",
         "density_residual", "divergence_residual", "dt", "density_residual_max",
         "divergence_residual_max")


@pytest.fixture(scope="module")
def small_model():
    """A network trained briefly on captures of the 16k dam break: its
    outputs fall inside and outside the clamp, like a real model's."""
    x, y = learned.capture(workload_names=("dam_break_16k",), frames=(40,), strides=(4,),
                           capacity=60_000)
    r = learned.train(x, y, epochs=4)
    yield r.model
    r.model.close()


@pytest.fixture(scope="module")
def random_model():
    m = learned.Model(seed=7)
    yield m
    m.close()


def _learned_frames(oracle_mod, model, name, frames, substeps=1, mode=_abi.FE_MODE_FIXED,
                    solver=None, n_keep=None, vel_sigma=0.0):
    w = scene.workload(name)
    p = _abi.copy_params(w.params)
    p.mode = mode
    if solver is not None:
        p.solver = solver
    p.warm_start = _abi.FE_WARM_LEARNED
    pos = w.positions()
    if n_keep:
        pos = pos[:n_keep].copy()
    vel = None
    if vel_sigma:
        vel = np.random.default_rng(4).normal(0, vel_sigma, pos.shape).astype(np.float32)
    sim = Simulation(pos, p, velocities=vel)
    lib = sim.data._lib
    _abi.check(lib, lib.fe_set_model(sim.data.handle, model.handle), "fe_set_model")
    slots = 2 * substeps
    sim.data.trace_learned(slots)
    orc = oracle_mod.Oracle(p, pos, vel)
    orc.set_learned(model.normalization())
    for f in range(frames):
        st = sim.step(substeps)
        trace = [sim.data.read_trace(k) for k in range(slots)]
        orc.set_network_outputs(np.stack([t[1] for t in trace]))
        rs = orc.step(substeps)
        assert not orc.missing_network_outputs()
        for k in range(slots):
            assert_same(trace[k][0], orc.feature_rows(k),
                        f"frame {f}, solve slot {k}: network input rows")
        for s_ in STATS:
            assert getattr(st, s_) == getattr(rs, s_), (f, s_, getattr(st, s_), getattr(rs, s_))
    compare_all(sim.data, orc, f"{name}: after {frames} learned frames")
    return sim, orc, trace


def test_learned_frames_bit_exact_16k(oracle_mod, small_model):
    """The bench's configuration (FIXED mode, tolerance 0.1 %) on the 16k
    dam break with a small initial velocity field so that every solve has
    work: 4 frames."""
    sim, orc, trace = _learned_frames(oracle_mod, small_model, "dam_break_16k", frames=4,
                                      solver=_abi.FE_SOLVER_TOLERANCE, vel_sigma=0.3)
    rows = trace[0][0]
    assert np.any(rows[:, :12] != 0)          # the features are not trivially zero
    assert np.all(rows[:, 12:] == 0)          # padding columns


def test_learned_frames_bit_exact_reference_mode_two_substeps(oracle_mod, random_model):
    """REFERENCE mode, fixed iterations, two substeps per frame (solve slots
    0..3), ragged particle count, an untrained network (outputs hit the clamp
    on both sides)."""
    _learned_frames(oracle_mod, random_model, "dam_break_16k", frames=3, substeps=2,
                    mode=_abi.FE_MODE_REFERENCE, n_keep=16_384 - 77, vel_sigma=0.2)


def test_learned_frames_bit_exact_262k_cfl(oracle_mod, small_model):
    """The 262k dam break with adaptive CFL (dt grows from frame to frame)."""
    _learned_frames(oracle_mod, small_model, "dam_break_256k", frames=3)


def test_learned_frames_bit_exact_1m(oracle_mod, small_model):
    """The benchmarked 1M dam break (2^20 particles, table of 2^20 slots),
    FIXED mode, tolerance 0.1 %, with an initial velocity field: 2 frames."""
    _learned_frames(oracle_mod, small_model, "dam_break_1m", frames=2, vel_sigma=0.3)

