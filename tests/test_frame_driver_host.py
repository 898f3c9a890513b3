"""The frame driver's host arithmetic (no GPU): the f32 substep loop, the CFL
rule and the wall's wave."""
import math

import numpy as np

from fluid_step.frame import CollisionBox, cfl_dt, substep_count


def test_substep_count_follows_the_f32_loop():
    assert substep_count(1 / 60, 0.005) == 4          # 0.005 .. 0.020 >= 0.01667
    assert substep_count(0.01, 0.005) == 2
    assert substep_count(0.005, 0.005) == 1
    # f32 accumulation: 10 x 0.001 in f32 is just below 0.01, so 11 substeps
    s, n = np.float32(0), 0
    while s < np.float32(0.01):
        s = np.float32(s + np.float32(0.001))
        n += 1
    assert substep_count(0.01, 0.001) == n


def test_cfl_rule():
    # clamp to [1 ms, 50 ms] and growth limit 1.1 dt
    assert cfl_dt(100.0, 0.08, 0.005) == np.float32(0.001)
    assert cfl_dt(0.02, 0.08, 0.005) == np.float32(np.float32(0.005) * np.float32(1.1))
    assert abs(cfl_dt(2.0, 0.08, 0.05) - 0.016) < 1e-7


def test_wave_moves_min_x_only():
    b = CollisionBox((-1.5, 0.0, -1.0), (0.8, 4.0, 1.0), 0.3, 0.5)
    xs = []
    for _ in range(120):
        b.update(1 / 60)
        xs.append(float(b.min[0]))
    t = np.arange(1, 121) / 60
    expect = -1.5 + 0.3 * np.sin(t * 0.5 * 2 * math.pi)
    assert np.max(np.abs(np.array(xs) - expect)) < 1e-5
    assert tuple(b.min[1:]) == (0.0, -1.0) and tuple(b.max) == (np.float32(0.8), 4.0, 1.0)
