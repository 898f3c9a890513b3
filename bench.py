"""Benchmark of the DFSPH step: particle-steps/s on one or more B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
    python bench.py --impl reference ...   # the reference algorithm on CPU

A step is one frame of the physics half of `Renderer::step` with one substep
(renderer/mod.rs:227-342): viscosity, density solve, integration, neighbour
search, density/alpha, divergence solve, divergence integration, stats.  The
default workload is the 1M-particle dam break (128x64x128 lattice, Jacobi to
0.1 % density and divergence error).  Multi-GPU runs are independent replicas
of the workload (one scene per GPU, no exchange): weak scaling.

value: particles x steps / device time of K graph-replayed frames (CUDA
events, max over ranks).  e2e: the same through the C ABI as a host
application drives it, with the per-frame host<->device traffic inside the
timed region.  roofline: the dominant kernel's algorithmic bytes per launch
over its CUDA-event launch time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "fluid-engine_b200"))

import numpy as np  # noqa: E402

# Algorithmic bytes per particle per pass (compulsory traffic: SOA xyz 12 B,
# scalars 4 B, keys/values 4 B, each array read once and written once).
PASS_BYTES = {
    "viscosity": 40, "density_source": 36, "pressure_force": 32, "pressure_update": 44,
    "pressure_integration": 60, "density_alpha": 20, "divergence_source": 28,
    "divergence_integration": 36, "stats": 20,
}


def ns_bytes(passes: int) -> int:
    # hash 20 + sort (4 + 16 P) + offsets 12 + reorder 52
    return 20 + 4 + 16 * passes + 12 + 52


def step_bytes(iters: float, passes: int) -> float:
    b = (PASS_BYTES["viscosity"] + PASS_BYTES["density_source"] + PASS_BYTES["pressure_integration"]
         + PASS_BYTES["density_alpha"] + PASS_BYTES["divergence_source"]
         + PASS_BYTES["divergence_integration"] + PASS_BYTES["stats"] + ns_bytes(passes))
    return b + iters * (PASS_BYTES["pressure_force"] + PASS_BYTES["pressure_update"])


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def reduce_max(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def launches_per_frame(stats, passes: int, fixed_mode: bool) -> int:
    # prologue + substep fixed kernels + NS + solves + stats
    ns = 1 + 1 + 1 + passes + 1 + 1 + 1 + (1 if fixed_mode else 0)  # hash fill hist P cells offs reorder
    per_substep = (1 + 1 + 1 + 1 + 1 + ns + 1 + 1 + 1 + 1 + 1 + 1
                   + 2 * (stats.density_iterations + stats.divergence_iterations))
    return 1 + per_substep + 1


# ---------------------------------------------------------------------------
def run_gpu(args) -> None:
    import torch

    from fluid_step import _abi, scene
    from fluid_step.pipelines import Simulation

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    w = scene.workload(args.workload)
    pos = w.positions()
    n = pos.shape[0]
    sim = Simulation(pos, w.params, device=local)
    lib = sim.data._lib
    h = sim.data.handle
    stream = torch.cuda.ExternalStream(lib.fe_get_stream(h), device=local)

    # --eager launches each frame's kernels directly (FE_STEP_NO_GRAPH); the
    # kernels and their work are the same as in the graph replay.
    step_flags = _abi.FE_STEP_NO_GRAPH if args.eager else 0
    for _ in range(args.warmup):
        st = sim.step(1, step_flags)
    barrier(world)
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    it0 = (st.total_density_iterations, st.total_divergence_iterations)
    launches = 0
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            rc = lib.fe_step(h, 1, step_flags, None)
            if rc:
                raise RuntimeError(f"fe_step failed: {rc}")
        end.record(stream)
        end.synchronize()
    dev_ms = start.elapsed_time(end)
    st = sim.data.read_stats()
    if st.flags & (_abi.FE_STATS_NON_FINITE | _abi.FE_STATS_LOOKBACK_TIMEOUT):
        raise RuntimeError(f"step reported flags {st.flags:#x}")
    iters_d = (st.total_density_iterations - it0[0]) / args.steps
    iters_v = (st.total_divergence_iterations - it0[1]) / args.steps
    passes = int(np.ceil(np.log2(sim.data.table_size) / 8)) or 1
    fixed_mode = w.params.mode == _abi.FE_MODE_FIXED
    avg_stats = type("S", (), {"density_iterations": iters_d, "divergence_iterations": iters_v})
    launches = int(round(args.steps * launches_per_frame(avg_stats, passes, fixed_mode)))
    dev_ms_max = reduce_max(dev_ms, world)
    value = n * args.steps * world / (dev_ms_max / 1e3)

    # ---- e2e through the C ABI: params in, stats + positions out, per frame
    p = _abi.copy_params(sim.data.current_params())
    pos_host = np.empty((n, 4), np.float32)
    stats_host = _abi.FeStats()
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        lib.fe_set_params(h, ctypes.byref(p))
        lib.fe_step(h, 1, step_flags, None)
        lib.fe_read_stats(h, ctypes.byref(stats_host))
        lib.fe_download(h, _abi.FE_FIELD_POSITION_A, pos_host.ctypes.data_as(ctypes.c_void_p),
                        pos_host.nbytes)
        p.dt = stats_host.dt
    e2e_s = reduce_max(time.perf_counter() - t0, world)
    e2e = n * args.steps * world / e2e_s

    # ---- per-kernel CUDA-event timing of the dominant passes (same stream)
    kern = {}
    reps = 20
    for name, fn in [("pressure_force", lib.fe_pressure_force),
                     ("pressure_update", lib.fe_pressure_update),
                     ("density_alpha", lib.fe_density_alpha),
                     ("neighbor_search", lib.fe_neighbor_search)]:
        if name == "neighbor_search":
            fn(h)
        fn(h)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn(h)
        b.record(stream)
        b.synchronize()
        kern[name] = a.elapsed_time(b) / reps
        if name == "neighbor_search":
            lib.fe_density_alpha(h)
    lib.fe_synchronize(h)

    # share of the frame: pressure solve passes dominate
    total_iters = iters_d + iters_v
    share = {
        "pressure_force": kern["pressure_force"] * total_iters,
        "pressure_update": kern["pressure_update"] * total_iters,
        "density_alpha": kern["density_alpha"],
        "neighbor_search": kern["neighbor_search"],
    }
    dom = max(("pressure_force", "pressure_update"), key=lambda k: share[k])
    peak, peak_kind = load_peaks()
    alg = PASS_BYTES[dom] * n
    achieved = alg / (kern[dom] / 1e3) / 1e9
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            tj = json.load(f)
        if dom in tj and tj[dom].get("workload") == args.workload:
            traffic = tj[dom]["dram_bytes_per_launch"]
    except Exception:
        pass

    # ---- isolated radix sort, 2^22 random u32 keys + u32 payload
    sort_n = 1 << 22
    rng = np.random.default_rng(0)
    kd = torch.from_numpy(rng.integers(0, 2**32, sort_n, dtype=np.uint64).astype(np.uint32)
                          .view(np.int32)).cuda()
    vd = torch.arange(sort_n, dtype=torch.int32, device="cuda")
    k2, v2 = kd.clone(), vd.clone()
    cs = torch.cuda.current_stream()
    for _ in range(3):
        k2.copy_(kd)
        v2.copy_(vd)
        lib.fe_sort_pairs(ctypes.c_void_p(k2.data_ptr()), ctypes.c_void_p(v2.data_ptr()), sort_n, 32,
                          _abi.FE_SORT_RADIX, ctypes.c_void_p(cs.cuda_stream))
    times = []
    for _ in range(15):
        k2.copy_(kd)
        v2.copy_(vd)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(cs)
        lib.fe_sort_pairs(ctypes.c_void_p(k2.data_ptr()), ctypes.c_void_p(v2.data_ptr()), sort_n, 32,
                          _abi.FE_SORT_RADIX, ctypes.c_void_p(cs.cuda_stream))
        b.record(cs)
        b.synchronize()
        times.append(a.elapsed_time(b))
    sort_ms = statistics.median(times)

    out = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(args.workload, w)
        out = {
            "metric": "DFSPH particle-steps/s (plain Jacobi to 0.1% density/divergence error)",
            "value": value,
            "unit": "particle-steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": dev_ms_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic: seeded dam-break lattice, random jitter +-0.005",
            "config": {"workload": args.workload, "particles_per_gpu": n,
                       "mode": "FIXED", "solver": "tolerance 0.1%/0.1%, FP64 residuals",
                       "avg_jacobi_iterations": {"density": iters_d, "divergence": iters_v},
                       "l2": "working set > L2 (no flush needed)",
                       "timing": "CUDA events on the context stream, "
                                 + ("eager launches" if args.eager else "graph replay per frame")},
            "e2e": {"value": e2e, "unit": "particle-steps/s",
                    "h2d_bytes_per_step": ctypes.sizeof(_abi.FeParams),
                    "d2h_bytes_per_step": n * 16 + 192,
                    "path": "fe_set_params + fe_step + fe_read_stats + fe_download(position_a)"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": alg,
                         "launch_ms": kern[dom]},
            "kernel_ms": kern,
            "step_roofline": {"algorithmic_bytes_per_step": step_bytes(total_iters, passes) * n,
                              "frac": step_bytes(total_iters, passes) * n
                              / (dev_ms_max / args.steps / 1e3) / 1e9 / peak},
            "sort": {"n": sort_n, "ms": sort_ms, "keys_per_s": sort_n / (sort_ms / 1e3),
                     "roofline_frac": 68 * sort_n / (sort_ms / 1e3) / 1e9 / peak},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(out))
    sim.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def cpu_baseline(workload: str, w=None, frames: int = 1):
    """The oracle (FP32 shader-order C++ port, OpenMP) on the same workload:
    `frames` frames from rest, timed with the host clock."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    from fluid_step import scene
    w = w or scene.workload(workload)
    pos = w.positions()
    o = oracle.Oracle(w.params, pos)
    t0 = time.perf_counter()
    for _ in range(frames):
        o.step(1)
    dt = time.perf_counter() - t0
    return {"value": pos.shape[0] * frames / dt, "unit": "particle-steps/s",
            "cores": oracle.get_threads(), "kind": "port",
            "sample": f"{frames} frame(s) of {workload} ({pos.shape[0]} particles) from rest"}


def run_profile_passes(args) -> None:
    """A short, profiler-friendly run: a few frames launched eagerly
    (FE_STEP_NO_GRAPH), then one launch of each hot pass on the same state."""
    from fluid_step import _abi, scene
    from fluid_step.pipelines import Simulation
    w = scene.workload(args.workload)
    sim = Simulation(w.positions(), w.params)
    for _ in range(3):
        st = sim.step(1, _abi.FE_STEP_NO_GRAPH)
    lib, h = sim.data._lib, sim.data.handle
    for name in ("fe_pressure_force", "fe_pressure_update", "fe_neighbor_search",
                 "fe_density_alpha", "fe_viscosity", "fe_density_source"):
        rc = getattr(lib, name)(h)
        if rc:
            raise RuntimeError(f"{name}: {rc}")
    lib.fe_synchronize(h)
    print(json.dumps({"profile_passes": args.workload,
                      "iterations": [st.density_iterations, st.divergence_iterations]}))
    sim.close()


def run_reference(args) -> None:
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from fluid_step import scene
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    w = scene.workload(args.workload)
    pos = w.positions()
    o = oracle.Oracle(w.params, pos)
    for _ in range(min(args.warmup, 1)):
        o.step(1)
    t0 = time.perf_counter()
    steps = max(1, min(args.steps, args.reference_steps))
    for _ in range(steps):
        o.step(1)
    dt = time.perf_counter() - t0
    v = pos.shape[0] * steps / dt
    out = {"impl": "reference",
           "metric": "DFSPH particle-steps/s (plain Jacobi to 0.1% density/divergence error)",
           "value": v, "unit": "particle-steps/s", "n_gpus": world, "steps": steps,
           "warmup": min(args.warmup, 1), "ms_per_step": dt * 1e3 / steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic: seeded dam-break lattice, random jitter +-0.005",
           "config": {"workload": args.workload, "particles_per_gpu": pos.shape[0]},
           "cpu_baseline": {"value": v, "unit": "particle-steps/s", "cores": oracle.get_threads(),
                            "kind": "port",
                            "sample": f"{steps} frame(s) of {args.workload} after "
                                      f"{min(args.warmup, 1)} warm-up frame"},
           "e2e": {"value": v, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="dam_break_1m")
    ap.add_argument("--impl", default="own", choices=["own", "reference"])
    ap.add_argument("--reference-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-passes", action="store_true",
                    help="eager frames, then one launch of each hot pass (for ncu -k)")
    ap.add_argument("--eager", action="store_true",
                    help="launch frames without CUDA graphs (for profilers)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.profile_passes:
        run_profile_passes(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
