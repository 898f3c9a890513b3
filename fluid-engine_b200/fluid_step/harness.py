"""The reference's headless benchmark harnesses on this library, writing
their CSV files with the same columns and number formats, so the
reference's scripts/plot_*.py read them unchanged.

    python -m fluid_step.harness convergence   [--out scripts/convergence.csv]
    python -m fluid_step.harness rest_density  [--out scripts/rest_density.csv]
    python -m fluid_step.harness cfl_comparison [--out scripts/cfl_comparison.csv]
    python -m fluid_step.harness sort_benchmark [--out scripts/sort_benchmark.csv]

Each function follows the procedure of the reference test of the same name
(convergence_benchmark.rs, sorter.rs); the reference's jitter is unseeded,
here it is seeded.
"""
from __future__ import annotations

import argparse
import ctypes
import os
import statistics
import time

import numpy as np

from . import _abi, scene
from ._abi import check, load_library
from .pipelines import Simulation

# convergence_benchmark.rs:46-63, sorter.rs:696-710
ITER_VALUES = (1, 2, 3, 4, 5, 6, 8, 10, 12, 16, 20)
WARMUP_SUBSTEPS = 50
MEASUREMENT_SUBSTEPS = 40
CFL_FRAMES = 500
CFL_STATIC_ITERS = 4
CFL_MAX_ITERS = 100
STATIC_DT = 0.005
SORT_N_VALUES = (1024, 4096, 16384, 65536, 131072, 262144, 524288, 1048576, 2097152, 4194304)
SORT_WARMUP_RUNS = 3
SORT_TIMED_RUNS = 15


def _mkdir(path: str) -> None:
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)


def _f32_mean(xs) -> float:
    """xs.iter().sum::<f32>() / len as f32: sequential single-precision sum."""
    acc = np.float32(0.0)
    for x in xs:
        acc = np.float32(acc + np.float32(x))
    return float(np.float32(acc / np.float32(len(xs)))) if len(xs) else 0.0


def write_convergence_csv(path: str, rows) -> None:
    """write_csv (convergence_benchmark.rs:181-191)."""
    _mkdir(path)
    with open(path, "w") as f:
        f.write("iters,density_error,divergence_error\n")
        for n, de, ve in rows:
            f.write(f"{n},{de:.6f},{ve:.6f}\n")


def write_rest_density_csv(path: str, densities) -> None:
    """convergence_benchmark.rs:535-540."""
    _mkdir(path)
    with open(path, "w") as f:
        f.write("density\n")
        for d in densities:
            f.write(f"{float(d):.6f}\n")


def write_cfl_csv(path: str, rows) -> None:
    """write_cfl_csv (convergence_benchmark.rs:741-749)."""
    _mkdir(path)
    with open(path, "w") as f:
        f.write("frame,mode,dt,max_speed,iters\n")
        for frame, mode, dt, vmax, iters in rows:
            f.write(f"{frame},{mode},{dt:.6f},{vmax:.4f},{iters}\n")


def write_sort_csv(path: str, rows) -> None:
    """sorter.rs:889-918."""
    _mkdir(path)
    with open(path, "w") as f:
        f.write("n,algorithm,time_ms\n")
        for n, algo, ms in rows:
            f.write(f"{n},{algo},{ms:.4f}\n")


def _errors(st: _abi.FeStats, n: int):
    """read_stats (convergence_benchmark.rs:164-170): fixed point / (scale n)."""
    nf = np.float32(n)
    de = np.float32(np.float32(st.density_error_fp) / np.float32(np.float32(1.0) * nf))
    ve = np.float32(np.float32(st.divergence_error_fp) / np.float32(np.float32(10.0) * nf))
    return float(de), float(ve)


def convergence(path: str | None = "scripts/convergence.csv", iter_values=ITER_VALUES,
                warmup: int = WARMUP_SUBSTEPS, measure: int = MEASUREMENT_SUBSTEPS,
                seed: int = 0, device: int = 0):
    """solver_convergence_benchmark (convergence_benchmark.rs:197-330): per
    iteration count a fresh state, one submit of `warmup` substeps, then
    `measure` single-substep submits with the stats read after each."""
    rows = []
    for k in iter_values:
        p, pos = scene.convergence_scene(seed)
        p.density_solver_iterations = k
        p.divergence_solver_iterations = k
        sim = Simulation(pos, p, device=device)
        n = pos.shape[0]
        sim.step(warmup, _abi.FE_STEP_INIT_NS)
        de, ve = [], []
        for _ in range(measure):
            st = sim.step(1)
            a, b = _errors(st, n)
            de.append(a)
            ve.append(b)
        sim.close()
        rows.append((k, _f32_mean(de), _f32_mean(ve)))
    if path:
        write_convergence_csv(path, rows)
    return rows


def rest_density(path: str | None = "scripts/rest_density.csv", device: int = 0):
    """rest_density_diagnostic (convergence_benchmark.rs:420-542): one
    neighbour search and density_alpha of the zero-jitter scene, densities in
    sorted order."""
    p, pos = scene.rest_density_scene()
    sim = Simulation(pos, p, device=device)
    lib, h = sim.data._lib, sim.data.handle
    check(lib, lib.fe_neighbor_search(h), "fe_neighbor_search")
    check(lib, lib.fe_density_alpha(h), "fe_density_alpha")
    check(lib, lib.fe_synchronize(h), "fe_synchronize")
    d = sim.data.download(_abi.FE_FIELD_DENSITY).copy()
    sim.close()
    if path:
        write_rest_density_csv(path, d)
    return d


def cfl_scene(seed: int = 0):
    """cfl_comparison's scene (convergence_benchmark.rs:766-777): the
    convergence scene's block, nu 0.15, relax 0.5."""
    p, pos = scene.convergence_scene(seed)
    return p, pos


def cfl_comparison(path: str | None = "scripts/cfl_comparison.csv", frames: int = CFL_FRAMES,
                   seed: int = 0, device: int = 0):
    """cfl_comparison (convergence_benchmark.rs:757-852): static dt 5 ms with
    4 iterations, then adaptive CFL (dt <- min(clamp(0.4 h / v_max, 1 ms,
    50 ms), 1.1 dt) from the previous frame's v_max, skipped on frame 0) with
    100 iterations; one substep per frame; rows (frame, mode, dt, v_max after
    the frame, iterations)."""
    rows = []
    for use_cfl in (False, True):
        mode = "adaptive" if use_cfl else "static"
        iters = CFL_MAX_ITERS if use_cfl else CFL_STATIC_ITERS
        p, pos = cfl_scene(seed)
        p.dt = STATIC_DT
        p.density_solver_iterations = iters
        p.divergence_solver_iterations = iters
        p.use_cfl = 1 if use_cfl else 0
        p.cfl_lambda, p.cfl_min_dt, p.cfl_max_dt, p.cfl_growth = 0.4, 0.001, 0.05, 1.1
        sim = Simulation(pos, p, device=device)
        for frame in range(frames):
            st = sim.step(1, _abi.FE_STEP_INIT_NS if frame == 0 else 0)
            rows.append((frame, mode, st.dt, st.max_speed, iters))
        sim.close()
    if path:
        write_cfl_csv(path, rows)
    return rows


def sort_benchmark(path: str | None = "scripts/sort_benchmark.csv", n_values=SORT_N_VALUES,
                   warmup: int = SORT_WARMUP_RUNS, timed: int = SORT_TIMED_RUNS):
    """sort_benchmark (sorter.rs:694-920): per N, random u32 hashes with the
    index as payload (fresh keys every run), bitonic then radix, host time of
    submit + wait, median of `timed` runs after `warmup`."""
    import torch
    lib = load_library()
    rows = []
    for n in n_values:
        for algo, name in ((_abi.FE_SORT_BITONIC, "Bitonic"), (_abi.FE_SORT_RADIX, "Radix")):
            samples = []
            for run in range(warmup + timed):
                rng = np.random.default_rng(run)
                k = torch.from_numpy(rng.integers(0, 1 << 32, n, dtype=np.uint64)
                                     .astype(np.uint32).view(np.int32)).cuda()
                v = torch.arange(n, dtype=torch.int32, device="cuda")
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                check(lib, lib.fe_sort_pairs(ctypes.c_void_p(k.data_ptr()),
                                             ctypes.c_void_p(v.data_ptr()), n, 32, algo, None),
                      "fe_sort_pairs")
                torch.cuda.synchronize()
                if run >= warmup:
                    samples.append((time.perf_counter() - t0) * 1e3)
            samples.sort()
            rows.append((n, name, samples[len(samples) // 2]))
    if path:
        write_sort_csv(path, rows)
    return rows


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("harness", choices=["convergence", "rest_density", "cfl_comparison",
                                        "sort_benchmark"])
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    out = a.out or f"scripts/{a.harness}.csv"
    globals()[a.harness](out)
    print(f"wrote {out}")


if __name__ == "__main__":
    main()
