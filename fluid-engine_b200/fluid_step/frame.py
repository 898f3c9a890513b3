"""The application's frame driver, `Renderer::step` (renderer/mod.rs:227-342),
and the moving-wall wave of `CollisionBox` (collision.rs:31-35), on this
library.

Per frame, as the reference does it on the host:
  1. from the previous frame's stats: the adaptive CFL time step
     dt <- min(clamp(0.4 h / v_max, 1 ms, 50 ms), 1.1 dt) when v_max > 0.01,
     and the early-exit iteration counts (2 density / 1 divergence iterations
     when the previous errors are below the thresholds);
  2. the boundary the UI copied into the parameters (box_min/box_max, with
     the wave's current offset) and the parameter upload (sync_with_scene);
  3. the wave advances by the frame length (after the upload: the physics
     sees the previous position);
  4. one neighbour search + density/alpha, then substeps while the f32
     accumulator `step += dt` is below max_dt, then stats — one fe_step with
     FE_STEP_INIT_NS and the substep count.
The device prologue's own CFL and early exit are switched off in the uploaded
parameters, since the host has made those choices for this frame.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _abi
from ._abi import check

F = np.float32
TAU = F(2.0 * math.pi)


class CollisionBox:
    """collision.rs:11-35: box whose min.x oscillates with amplitude A and
    frequency f: min.x = base + A sin(t f 2 pi), t the accumulated time."""

    def __init__(self, box_min, box_max, wave_amplitude=0.0, wave_frequency=1.0):
        self.min = np.asarray(box_min, F).copy()
        self.max = np.asarray(box_max, F).copy()
        self.wave_amplitude = F(wave_amplitude)
        self.wave_frequency = F(wave_frequency)
        self.time = F(0.0)
        self.base_min_x = F(self.min[0])

    def update(self, dt) -> None:
        self.time = F(self.time + F(dt))
        phase = F(F(self.time * self.wave_frequency) * TAU)
        offset = F(self.wave_amplitude * F(np.sin(phase)))
        self.min[0] = F(self.base_min_x + offset)


def substep_count(max_dt, dt) -> int:
    """`let mut step = 0.0; while step < max_dt { ...; step += dt }` in f32."""
    step, n = F(0.0), 0
    max_dt, dt = F(max_dt), F(dt)
    if not dt > 0:
        raise ValueError("dt must be > 0")
    while step < max_dt:
        step = F(step + dt)
        n += 1
    return n


def cfl_dt(max_speed, h, dt) -> float:
    """renderer/mod.rs:238-245 in f32."""
    c = F(F(F(0.4) * F(h)) / F(max_speed))
    c = min(max(c, F(0.001)), F(0.05))
    return float(min(c, F(F(dt) * F(1.1))))


class FrameDriver:
    """Drives a GpuPhysicsData (or its Simulation) frame by frame like the app.

    use_cfl, use_solver_error_threshold, density_error_pct and
    divergence_error_pct are the AppUI settings (ui.rs:31-49)."""

    def __init__(self, data, params: _abi.FeParams, boundary: CollisionBox | None = None, *,
                 use_cfl: bool = False, use_solver_error_threshold: bool = False,
                 density_error_pct: float = 1.0, divergence_error_pct: float = 1.0):
        self.data = data
        self.params = _abi.copy_params(params)
        self.boundary = boundary or CollisionBox(params.box_min, params.box_max)
        self.use_cfl = use_cfl
        self.use_thr = use_solver_error_threshold
        self.density_error_pct = F(density_error_pct)
        self.divergence_error_pct = F(divergence_error_pct)
        self.stats = _abi.FeStats()          # zeroed, like the first read of stats_buffer
        self.frame = 0
        self.last = {}

    def frame_params(self, max_dt):
        """Steps 1-3 of a frame: the parameter block to upload and the
        substep count (advances the wave)."""
        p = self.params
        n = F(self.data.count)
        max_speed = F(np.frombuffer(np.uint32(self.stats.max_speed_bits).tobytes(), F)[0])
        avg_de = F(F(self.stats.density_error_fp) / F(F(1.0) * n))
        avg_ve = F(F(self.stats.divergence_error_fp) / F(F(10.0) * n))
        if self.use_cfl and max_speed > F(0.01):
            p.dt = cfl_dt(max_speed, p.smoothing_radius, p.dt)
        rho0 = F(p.target_density)
        thr_d = F(F(self.density_error_pct / F(100.0)) * rho0)
        thr_v = F(F(self.divergence_error_pct / F(100.0)) * rho0)
        d_it = 2 if (self.use_thr and avg_de < thr_d) else p.density_solver_iterations
        v_it = 1 if (self.use_thr and avg_ve < thr_v) else p.divergence_solver_iterations
        p.box_min[:] = [float(v) for v in self.boundary.min]
        p.box_max[:] = [float(v) for v in self.boundary.max]
        up = _abi.copy_params(p)
        up.use_cfl = 0
        up.use_solver_error_threshold = 0
        up.density_solver_iterations = d_it
        up.divergence_solver_iterations = v_it
        self.boundary.update(max_dt)
        return up, substep_count(max_dt, p.dt), (d_it, v_it)

    def step(self, max_dt: float = 1.0 / 60.0) -> _abi.FeStats:
        up, k, iters = self.frame_params(max_dt)
        lib, h = self.data._lib, self.data.handle
        check(lib, lib.fe_set_params(h, ctypes.byref(up)), "fe_set_params")
        st = _abi.FeStats()
        check(lib, lib.fe_step(h, k, _abi.FE_STEP_INIT_NS, ctypes.byref(st)), "fe_step")
        self.stats = st
        self.frame += 1
        self.last = {"substeps": k, "iterations": iters, "dt": up.dt,
                     "box_min_x": up.box_min[0]}
        return st
