"""Scene generation: `ParticleGenerator::generate_volume` and the workloads.

`generate_volume` follows src/entities/particle.rs:371-407 in float32:
    offset = origin + radius
    for x, for y, for z (z fastest):
        j = (rand() - 0.5) * jitter          # ONE scalar for all three axes
        p = (offset + index * spacing) + j
    mass = density * spacing^3
The reference draws `rand::random::<f32>()` unseeded; here the draw comes from
a seeded numpy PCG64 stream so that runs repeat.

Dam-break workloads (particle-steps/s benchmarks and parity cases):
  dam_break_16k   16x32x32 lattice, s=0.05, box [0,2]^3, jitter 0.01,
                  rho0 1000, m 0.125, h 0.1, nu 0.01, dt 1 ms, K 4+4, radix
  dam_break_256k  64^3 lattice in [0,4]^3, adaptive CFL, tolerance 0.1 %
  dam_break_256k_cfl03  the same with CFL number 0.3 instead of 0.4: with the
                  reference's 0.4 h / v_max the plain solver's flow clumps
                  and blows up near frame 630 of the 1000
  dam_break_1m    128x64x128 lattice in [0,8]x[0,4]x[0,8], tolerance 0.1 %
  dam_break_1m_cfl  the same scene with the adaptive CFL step of the 262k one
  dam_break_4m    256x64x256 lattice in [0,16]x[0,4]x[0,16] (the 1M scene
                  widened in x and z at the same fill), tolerance 0.1 %
All start at rest; the lattice origin is box_min, shifted by the particle
radius as in generate_volume.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi


def generate_volume(origin, width, height, depth, radius, density, spacing,
                    jitter, seed: int = 0):
    """particle.rs:371-407 with a seeded jitter stream.

    Returns (positions float32[N, 3], mass float32).
    """
    f = np.float32
    spacing = f(spacing)
    nx = int(math.floor(f(width) / spacing))
    ny = int(math.floor(f(height) / spacing))
    nz = int(math.floor(f(depth) / spacing))
    return lattice(origin, (nx, ny, nz), radius, density, spacing, jitter, seed)


def lattice(origin, counts, radius, density, spacing, jitter, seed: int = 0):
    """The loop body of generate_volume for given per-axis counts."""
    f = np.float32
    nx, ny, nz = (int(c) for c in counts)
    spacing = f(spacing)
    off = np.asarray(origin, dtype=np.float32) + f(radius)
    rng = np.random.Generator(np.random.PCG64(seed))
    n = nx * ny * nz
    u = rng.random(n, dtype=np.float32)
    j = (u - f(0.5)) * f(jitter)
    ix, iy, iz = np.meshgrid(np.arange(nx, dtype=np.float32),
                             np.arange(ny, dtype=np.float32),
                             np.arange(nz, dtype=np.float32), indexing="ij")
    pos = np.empty((n, 3), dtype=np.float32)
    pos[:, 0] = (off[0] + ix.reshape(-1) * spacing) + j
    pos[:, 1] = (off[1] + iy.reshape(-1) * spacing) + j
    pos[:, 2] = (off[2] + iz.reshape(-1) * spacing) + j
    mass = f(density) * (spacing * spacing * spacing)
    return pos, mass


@dataclass
class Workload:
    name: str
    counts: tuple
    box_min: tuple
    box_max: tuple
    steps: int
    params: _abi.FeParams = field(repr=False, default=None)
    seed: int = 1
    jitter: float = 0.01

    @property
    def n(self) -> int:
        return self.counts[0] * self.counts[1] * self.counts[2]

    def positions(self) -> np.ndarray:
        pos, _ = lattice(self.box_min, self.counts, self.params.particle_radius,
                         self.params.target_density, 0.05, self.jitter, self.seed)
        return pos


def dam_break_params(box_min, box_max, *, solver=_abi.FE_SOLVER_FIXED_ITERS,
                     use_cfl=False, mode=_abi.FE_MODE_REFERENCE,
                     sort=_abi.FE_SORT_RADIX, viscosity=0.01) -> _abi.FeParams:
    """Physics shared by the dam-break workloads (spacing 0.05, h = 2 s)."""
    p = _abi.default_params()
    s = np.float32(0.05)
    p.particle_radius = 0.025            # spacing / 2 (scene.rs:16,32)
    p.particle_mass = float(np.float32(1000.0) * (s * s * s))
    p.smoothing_radius = 0.1
    p.target_density = 1000.0
    p.viscosity = viscosity
    p.relax_factor = 0.5                 # scene.rs:55
    p.dt = 0.001
    p.density_solver_iterations = 4
    p.divergence_solver_iterations = 4
    p.gravity[:] = [0.0, -9.81, 0.0]
    p.box_min[:] = list(box_min)
    p.box_max[:] = list(box_max)
    p.sort_algorithm = sort
    p.use_cfl = 1 if use_cfl else 0
    p.mode = mode
    p.solver = solver
    p.density_tolerance = 0.001
    p.divergence_tolerance = 0.001
    p.min_iterations = 1
    return p


def workload(name: str) -> Workload:
    if name == "dam_break_16k":
        w = Workload(name, (16, 32, 32), (0.0, 0.0, 0.0), (2.0, 2.0, 2.0), 100)
        w.params = dam_break_params(w.box_min, w.box_max)
    elif name == "dam_break_256k":
        w = Workload(name, (64, 64, 64), (0.0, 0.0, 0.0), (4.0, 4.0, 4.0), 1000)
        w.params = dam_break_params(w.box_min, w.box_max, use_cfl=True,
                                    solver=_abi.FE_SOLVER_TOLERANCE,
                                    mode=_abi.FE_MODE_FIXED)
    elif name == "dam_break_256k_cfl03":
        w = Workload(name, (64, 64, 64), (0.0, 0.0, 0.0), (4.0, 4.0, 4.0), 1000)
        w.params = dam_break_params(w.box_min, w.box_max, use_cfl=True,
                                    solver=_abi.FE_SOLVER_TOLERANCE,
                                    mode=_abi.FE_MODE_FIXED)
        w.params.cfl_lambda = 0.3
    elif name == "dam_break_1m":
        w = Workload(name, (128, 64, 128), (0.0, 0.0, 0.0), (8.0, 4.0, 8.0), 200)
        w.params = dam_break_params(w.box_min, w.box_max,
                                    solver=_abi.FE_SOLVER_TOLERANCE,
                                    mode=_abi.FE_MODE_FIXED)
    elif name == "dam_break_1m_cfl":
        w = Workload(name, (128, 64, 128), (0.0, 0.0, 0.0), (8.0, 4.0, 8.0), 200)
        w.params = dam_break_params(w.box_min, w.box_max, use_cfl=True,
                                    solver=_abi.FE_SOLVER_TOLERANCE,
                                    mode=_abi.FE_MODE_FIXED)
    elif name == "dam_break_1m_cfl03":
        # the 1M dam break where the solver has work: adaptive CFL (CFL
        # number 0.3 on h, as the 262k whole run uses), tolerance 0.1 %
        w = Workload(name, (128, 64, 128), (0.0, 0.0, 0.0), (8.0, 4.0, 8.0), 200)
        w.params = dam_break_params(w.box_min, w.box_max, use_cfl=True,
                                    solver=_abi.FE_SOLVER_TOLERANCE,
                                    mode=_abi.FE_MODE_FIXED)
        w.params.cfl_lambda = 0.3
    elif name == "dam_break_1m_k4":
        w = Workload(name, (128, 64, 128), (0.0, 0.0, 0.0), (8.0, 4.0, 8.0), 200)
        w.params = dam_break_params(w.box_min, w.box_max)
    elif name == "dam_break_4m":
        w = Workload(name, (256, 64, 256), (0.0, 0.0, 0.0), (16.0, 4.0, 16.0), 200)
        w.params = dam_break_params(w.box_min, w.box_max,
                                    solver=_abi.FE_SOLVER_TOLERANCE,
                                    mode=_abi.FE_MODE_FIXED)
    else:
        raise KeyError(name)
    return w


@dataclass
class BatchWorkload:
    """Independent dam-break scenes advanced together (fe_batch_create)."""
    name: str
    counts: list
    boxes: list          # (box_min, box_max) per scene
    viscosities: list
    steps: int
    seed: int = 1

    def positions(self) -> list:
        out = []
        sp = np.float32(0.05)
        for k, (n, (bmin, _)) in enumerate(zip(self.counts, self.boxes)):
            nx = int(math.ceil((n / 4.0) ** (1.0 / 3.0) - 1e-9))
            pos, _ = lattice(bmin, (nx, 2 * nx, 2 * nx), 0.025, 1000.0, sp, 0.01,
                             seed=self.seed * 1000 + k)
            out.append(pos[:n])
        return out

    def params(self) -> list:
        return [dam_break_params(bmin, bmax, viscosity=float(nu))
                for (bmin, bmax), nu in zip(self.boxes, self.viscosities)]


def batch_workload(n_scenes: int = 64, seed: int = 1, lo: int = 4096, hi: int = 262144,
                   fill: float = 0.25, steps: int = 500) -> BatchWorkload:
    """The batched dam breaks: n_scenes scenes with particle counts drawn
    log-uniform in [lo, hi] and XSPH coefficients uniform in [0.005, 0.05]
    (one seeded stream), each a column of the 16k dam break's 1:2:2 shape
    (nx x 2nx x 2nx lattice at spacing 0.05, cut to the drawn count) in a
    cubic box whose volume is count * spacing^3 / fill.  Physics otherwise as
    the 16k dam break (dt 1 ms, 4 + 4 Jacobi iterations, radix sort)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    counts = np.exp(rng.uniform(math.log(lo), math.log(hi), n_scenes)).astype(np.int64)
    counts = np.clip(counts, lo, hi)
    nus = rng.uniform(0.005, 0.05, n_scenes)
    boxes = []
    for n in counts:
        edge = float((float(n) * 0.05 ** 3 / fill) ** (1.0 / 3.0))
        boxes.append(((0.0, 0.0, 0.0), (edge, edge, edge)))
    return BatchWorkload(f"dam_break_batch{n_scenes}", [int(c) for c in counts], boxes,
                         [float(v) for v in nus], steps, seed)


def app_scene(seed: int = 0):
    """Scene::new (core/scene.rs:14-86): a 1.0 x 2.0 x 0.8 block at spacing
    0.04 from (-1, 1, -0.8) with jitter 0.01 in the box (-1.5, 0, -1) ..
    (0.8, 4, 1), whose min.x wall moves with amplitude 0.3 at 0.5 Hz.
    Returns (params, positions, (wave_amplitude, wave_frequency))."""
    p = _abi.default_params()
    pos, mass = generate_volume((-1.0, 1.0, -0.8), 1.0, 2.0, 0.8, 0.02, 1000.0,
                                np.float32(0.02) * np.float32(2.0), 0.01, seed)
    p.particle_mass = float(mass)
    return p, pos, (0.3, 0.5)


def rest_density_scene():
    """rest_density_diagnostic (convergence_benchmark.rs:420-542): no jitter,
    20x20x12 lattice, r 0.02, s 0.04, h 0.08, bitonic sort (the
    NeighborSearch default, neighbor_search.rs:99)."""
    p = _abi.default_params()
    p.sort_algorithm = _abi.FE_SORT_BITONIC
    p.viscosity = 0.15
    p.dt = 0.005
    pos, mass = generate_volume((-0.8, 0.5, -0.4), 0.8, 0.8, 0.5, 0.02, 1000.0,
                                np.float32(0.02) * np.float32(2.0), 0.0)
    p.particle_mass = float(mass)
    return p, pos


def convergence_scene(seed: int = 0):
    """solver_convergence_benchmark scene (convergence_benchmark.rs:212-235):
    4800 particles with jitter 0.01, dt 5 ms, nu 0.15."""
    p = _abi.default_params()
    p.sort_algorithm = _abi.FE_SORT_BITONIC
    pos, mass = generate_volume((-0.8, 0.5, -0.4), 0.8, 0.8, 0.5, 0.02, 1000.0,
                                np.float32(0.02) * np.float32(2.0), 0.01, seed)
    p.particle_mass = float(mass)
    return p, pos
