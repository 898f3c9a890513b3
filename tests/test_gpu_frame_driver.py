"""The application frame loop (Renderer::step) with the moving wall, CFL and
early exit decided on the host: bit-exact with the oracle driven by the same
parameter uploads and substep counts."""
import numpy as np
import pytest

from fluid_step import _abi, scene
from fluid_step.frame import CollisionBox, FrameDriver
from fluid_step.pipelines import Simulation

pytestmark = pytest.mark.gpu

FIELDS = [_abi.FE_FIELD_POSITION_A, _abi.FE_FIELD_VELOCITY_A, _abi.FE_FIELD_DENSITY,
          _abi.FE_FIELD_PRESSURE]


@pytest.mark.parametrize("cfl,thr", [(False, False), (True, True)])
def test_app_frames_match_oracle(oracle_mod, cfl, thr):
    p, pos, (amp, freq) = scene.app_scene()
    p.sort_algorithm = _abi.FE_SORT_RADIX
    sim = Simulation(pos, p)
    orc = oracle_mod.Oracle(p, pos)
    box = CollisionBox(p.box_min, p.box_max, amp, freq)
    drv = FrameDriver(sim.data, p, box, use_cfl=cfl, use_solver_error_threshold=thr,
                      density_error_pct=5.0, divergence_error_pct=5.0)
    # the oracle follows the same host decisions
    shadow = FrameDriver(sim.data, p, CollisionBox(p.box_min, p.box_max, amp, freq),
                         use_cfl=cfl, use_solver_error_threshold=thr,
                         density_error_pct=5.0, divergence_error_pct=5.0)
    xs = []
    for f in range(8):
        up, k, _ = shadow.frame_params(1 / 60)
        st = drv.step(1 / 60)
        assert drv.last["substeps"] == k and up.dt == drv.last["dt"]
        orc.set_params(up)
        rs = orc.step(k, _abi.FE_STEP_INIT_NS)
        shadow.stats = rs
        for name in ("max_speed_bits", "density_error_fp", "divergence_error_fp", "substeps"):
            assert getattr(st, name) == getattr(rs, name), (f, name)
        xs.append(drv.last["box_min_x"])
    for fld in FIELDS:
        a, b = sim.data.download(fld), orc.field(fld)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), fld
    # the wall moved (min.x lags the wave by one frame: frame 0 sees the base)
    assert xs[0] == pytest.approx(-1.5) and xs[-1] > -1.5 + 0.01
    sim.close()
