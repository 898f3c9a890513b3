"""The learned warm start end to end: capture from the plain solver, train
on the GPU, then solve to the same tolerance with fewer Jacobi iterations.

The network only chooses where the iterations start; the plain solver always
runs to the tolerance afterwards, so both arms must meet it on every frame.
"""
import ctypes

import numpy as np
import pytest

from fluid_step import _abi, learned, scene
from fluid_step.pipelines import Simulation

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained():
    # 100 frames of the 16k dam break and 300 of the 262k adaptive-CFL one
    x, y = learned.capture()
    assert x.shape[0] > 150_000 and x.shape[1] == 12
    # each sample trains exactly one output (the other target is NaN)
    assert np.all(np.isfinite(y).sum(1) == 1)
    r = learned.train(x, y, epochs=20)
    assert r.train_loss[-1] < 0.5 * r.train_loss[0]
    yield r
    r.model.close()


def test_validation_error(trained):
    assert trained.val_loss < 0.3


def test_fewer_iterations_same_tolerance(trained):
    res = learned.compare_iterations(trained.model, "dam_break_16k", frames=15, warmup=3)
    plain = res["plain"]["density_iterations"] + res["plain"]["divergence_iterations"]
    lrn = res["learned"]["density_iterations"] + res["learned"]["divergence_iterations"]
    assert lrn <= plain
    for arm in ("plain", "learned"):
        assert res[arm]["max_density_residual"] <= 1e-3
        assert res[arm]["max_divergence_residual"] <= 1e-3
        assert res[arm]["cap_hits"] == 0


def test_cfl_scene_fewer_iterations_and_stable(trained):
    """On the 262k adaptive-CFL dam break, where the plain solver needs many
    iterations, the warm start must cut them while the flow stays the same
    flow: same tolerance every frame, no blown-up particles (the largest
    speed stays near the plain arm's) and about the same simulated time."""
    res = learned.compare_iterations(trained.model, "dam_break_256k", frames=120, warmup=2)
    plain, lrn = res["plain"], res["learned"]
    it_p = plain["density_iterations"] + plain["divergence_iterations"]
    it_l = lrn["density_iterations"] + lrn["divergence_iterations"]
    assert it_l <= 0.6 * it_p, (it_l, it_p)
    for arm in (plain, lrn):
        assert arm["max_density_residual"] <= 1e-3 + 1e-9
        assert arm["max_divergence_residual"] <= 1e-3 + 1e-9
        assert arm["cap_hits"] == 0 and arm["non_finite"] == 0
    assert lrn["max_speed"] <= 1.5 * plain["max_speed"] + 1.0, (lrn["max_speed"],
                                                                 plain["max_speed"])
    assert abs(lrn["simulated_seconds"] - plain["simulated_seconds"]) \
        <= 0.2 * plain["simulated_seconds"]


def test_learned_frames_are_deterministic(trained):
    w = scene.workload("dam_break_16k")
    p = _abi.copy_params(w.params)
    p.warm_start = _abi.FE_WARM_LEARNED
    out = []
    for _ in range(2):
        sim = Simulation(w.positions(), p)
        _abi.check(sim.data._lib, sim.data._lib.fe_set_model(sim.data.handle, trained.model.handle),
                   "fe_set_model")
        for _ in range(3):
            sim.step(1)
        out.append(sim.data.download(_abi.FE_FIELD_POSITION_A).copy())
        sim.close()
    assert np.array_equal(out[0], out[1])


def test_learned_without_model_is_refused():
    w = scene.workload("dam_break_16k")
    p = _abi.copy_params(w.params)
    p.warm_start = _abi.FE_WARM_LEARNED
    sim = Simulation(w.positions()[:1000], p)
    st = sim.data._lib.fe_step(sim.data.handle, 1, 0, None)
    assert st == _abi.FE_ERR_UNSUPPORTED
    sim.close()


def test_model_save_and_load(trained, tmp_path):
    path = str(tmp_path / "m.npz")
    trained.model.save(path)
    m2 = learned.Model.load(path)
    x = np.random.default_rng(0).normal(0, 1, (500, 12)).astype(np.float32)
    assert np.array_equal(learned.predict(trained.model, x), learned.predict(m2, x))
    m2.close()


def test_long_cfl_run_stays_stable(trained):
    """All 1000 frames of the 262k dam break with adaptive CFL (CFL number
    0.3): the warm-started flow keeps the plain flow's largest speed (no
    particle thrown out late in the run) and still needs far fewer
    iterations to the same tolerance."""
    res = learned.compare_iterations(trained.model, "dam_break_256k_cfl03", frames=998, warmup=2)
    plain, lrn = res["plain"], res["learned"]
    assert lrn["max_speed"] <= 1.5 * plain["max_speed"] + 1.0, (lrn["max_speed"],
                                                                plain["max_speed"])
    it_p = plain["density_iterations"] + plain["divergence_iterations"]
    it_l = lrn["density_iterations"] + lrn["divergence_iterations"]
    assert it_l <= it_p / 1.5, (it_l, it_p)
    for arm in (plain, lrn):
        assert arm["cap_hits"] == 0 and arm["non_finite"] == 0
        assert arm["max_density_residual"] <= 1e-3 + 1e-9
