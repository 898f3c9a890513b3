"""Learned warm start: training-data capture, training and evaluation.

The network (12 -> 64 -> 64 -> 2, SiLU, BF16 tensor cores; see fe_mlp.cu)
predicts the initial pressure of the density and divergence solves from 12
per-particle features (fe_features.cuh), which the two source-term passes
emit as they walk each particle's neighbours.  It is trained on pairs that the plain
Jacobi solver produces: with capture on, each substep records a hashed sample
of particles' features and, after both solves, their converged pressures in
normalised units.  Training runs on the GPU with the library's own forward,
backward and Adam kernels.  The plain solver always runs afterwards to the
same tolerance, so the network only changes where the iterations start.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _abi, scene
from ._abi import check, load_library
from .pipelines import Simulation


class Model:
    """fe_model: parameters, standardisation, forward and training steps."""

    def __init__(self, seed: int = 1, device: int = 0):
        self.lib = load_library()
        self.handle = ctypes.c_void_p()
        check(self.lib, self.lib.fe_model_create(seed, device, ctypes.byref(self.handle)),
              "fe_model_create")

    def close(self):
        if self.handle:
            self.lib.fe_model_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- parameters ----------------------------------------------------------
    def parameters(self) -> np.ndarray:
        p = np.empty(_abi.FE_MODEL_PARAMS, np.float32)
        check(self.lib, self.lib.fe_model_get_parameters(
            self.handle, p.ctypes.data_as(ctypes.c_void_p), p.size), "get_parameters")
        return p

    def set_parameters(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        check(self.lib, self.lib.fe_model_set_parameters(
            self.handle, p.ctypes.data_as(ctypes.c_void_p), p.size), "set_parameters")

    def normalization(self) -> np.ndarray:
        out = np.empty(32, np.float32)
        check(self.lib, self.lib.fe_model_get_normalization(
            self.handle, out.ctypes.data_as(ctypes.c_void_p)), "get_normalization")
        return out

    def set_normalization(self, x_mean, x_std, y_mean, y_std) -> None:
        arrs = [np.ascontiguousarray(a, np.float32) for a in (x_mean, x_std, y_mean, y_std)]
        check(self.lib, self.lib.fe_model_set_normalization(
            self.handle, *[a.ctypes.data_as(ctypes.c_void_p) for a in arrs]), "set_normalization")
        self._keep = arrs

    def save(self, path: str) -> None:
        np.savez(path, params=self.parameters(), norm=self.normalization())

    @classmethod
    def load(cls, path: str, device: int = 0) -> "Model":
        d = np.load(path)
        m = cls(device=device)
        m.set_parameters(d["params"])
        n = d["norm"]
        m.set_normalization(n[:12], n[12:24], n[24:26], n[26:28])
        return m


@dataclass
class TrainResult:
    model: Model
    train_loss: list
    val_loss: float
    samples: int


def capture(workload_names=("dam_break_16k", "dam_break_256k"), frames=(100, 300),
            strides=(32, 1536), capacity=120_000, warmup=2, device=0, seed=1, model=None):
    """Runs the tolerance solver and returns captured (x[n][12], y[n][2]).

    The defaults sample the 16,384-particle dam break (fixed dt 1 ms) over 100
    frames and the 262,144-particle one (adaptive CFL) over 300 frames, about
    100k solve snapshots each: a sample is taken for a (particle, substep,
    solve) triple whose hash is 0 modulo the stride.  Without `model` the
    plain solver runs; with it, the solves start from that network's warm
    start (the features then carry the pressures of learned-started solves,
    and the divergence target is relative to the density solve's pressure as
    the warm start sees it)."""
    lib = load_library()
    xs, ys = [], []
    for name, nf, stride in zip(workload_names, frames, strides):
        w = scene.workload(name)
        p = _abi.copy_params(w.params)
        p.solver = _abi.FE_SOLVER_TOLERANCE
        p.mode = _abi.FE_MODE_FIXED
        if model is not None:
            p.warm_start = _abi.FE_WARM_LEARNED
        w.seed = seed
        sim = Simulation(w.positions(), p, device=device)
        h = sim.data.handle
        if model is not None:
            check(lib, lib.fe_set_model(h, model.handle), "fe_set_model")
        for _ in range(warmup):
            sim.step(1)
        check(lib, lib.fe_capture_begin(h, capacity, stride), "fe_capture_begin")
        for _ in range(nf):
            sim.step(1)
        cnt = ctypes.c_uint32()
        x = np.empty((capacity, 12), np.float32)
        y = np.empty((capacity, 2), np.float32)
        check(lib, lib.fe_capture_read(h, x.ctypes.data_as(ctypes.c_void_p),
                                       y.ctypes.data_as(ctypes.c_void_p), capacity,
                                       ctypes.byref(cnt)), "fe_capture_read")
        lib.fe_capture_end(h)
        k = cnt.value
        xs.append(x[:k])
        ys.append(y[:k])
        sim.close()
    x, y = np.concatenate(xs), np.concatenate(ys)
    # Which samples are taken is fixed by a hash of (particle, substep,
    # solve), but their slots come from a device atomic counter, so the row
    # order varies from run to run.  A canonical order (lexicographic over
    # the row's values) makes training, and everything after it, repeatable.
    order = np.lexsort(np.concatenate([x, y], axis=1).T[::-1])
    return x[order], y[order]


def train(x: np.ndarray, y: np.ndarray, *, epochs: int = 30, batch: int = 4096,
          lr: float = 2e-3, seed: int = 1, val_fraction: float = 0.1, device: int = 0,
          log=None) -> TrainResult:
    """Standardises, shuffles and trains with Adam on the GPU."""
    import torch

    rng = np.random.default_rng(seed)
    # A sample trains the output of the solve it was captured before; the
    # other target is NaN (masked in the loss).
    keep = np.all(np.isfinite(x), 1) & np.any(np.isfinite(y), 1)
    x, y = x[keep], y[keep]
    order = rng.permutation(x.shape[0])
    x, y = x[order], y[order]
    n_val = max(1, int(val_fraction * x.shape[0]))
    xv, yv, xt, yt = x[:n_val], y[:n_val], x[n_val:], y[n_val:]
    x_mean, x_std = xt.mean(0), xt.std(0)
    x_std = np.where(x_std > 1e-6, x_std, 1.0)
    y_mean, y_std = np.nanmean(yt, 0), np.nanstd(yt, 0)
    y_std = np.where(y_std > 1e-6, y_std, 1.0)
    model = Model(seed=seed, device=device)
    model.set_normalization(x_mean, x_std, y_mean, y_std)
    dev = f"cuda:{device}"
    xt_d = torch.from_numpy(np.ascontiguousarray(xt)).to(dev)
    yt_d = torch.from_numpy(np.ascontiguousarray(yt)).to(dev)
    lib = model.lib
    losses = []
    nt = xt.shape[0]
    for ep in range(epochs):
        perm = torch.randperm(nt, device=dev, generator=torch.Generator(device=dev).manual_seed(ep))
        xs, ys_ = xt_d[perm].contiguous(), yt_d[perm].contiguous()
        ep_loss = []
        lr_ep = lr * 0.5 * (1 + np.cos(np.pi * ep / epochs))
        for i0 in range(0, nt - batch + 1, batch):
            loss = ctypes.c_float()
            check(lib, lib.fe_model_train_step(
                model.handle, ctypes.c_void_p(xs.data_ptr() + i0 * 48),
                ctypes.c_void_p(ys_.data_ptr() + i0 * 8), batch, float(lr_ep), 1e-5, None,
                ctypes.byref(loss)), "fe_model_train_step")
            ep_loss.append(loss.value)
        losses.append(float(np.mean(ep_loss)) if ep_loss else float("nan"))
        if log:
            log(f"epoch {ep}: loss {losses[-1]:.4f}")
    val = evaluate(model, xv, yv)
    return TrainResult(model, losses, val, int(x.shape[0]))


def train_on_own_starts(epochs: int = 30, device: int = 0, log=None) -> TrainResult:
    """Two rounds of capture and training.  The first network learns from the
    plain solver.  Its divergence output, though, corrects the density
    solve's pressure, and under the warm start that pressure comes from a
    learned-started density solve, not a plain one.  So the same scenes are
    captured again with the first network's warm start, and the final
    network is trained on both captures (the capture order is canonical, so
    the result is repeatable)."""
    x1, y1 = capture(device=device)
    first = train(x1, y1, epochs=epochs, device=device, log=log)
    x2, y2 = capture(device=device, model=first.model)
    first.model.close()
    x = np.concatenate([x1, x2])
    y = np.concatenate([y1, y2])
    return train(x, y, epochs=epochs, device=device, log=log)


def predict(model: Model, x: np.ndarray) -> np.ndarray:
    import torch
    xd = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    yd = torch.empty((x.shape[0], 2), dtype=torch.float32, device="cuda")
    check(model.lib, model.lib.fe_model_forward(model.handle, ctypes.c_void_p(xd.data_ptr()),
                                                ctypes.c_void_p(yd.data_ptr()), x.shape[0], None),
          "fe_model_forward")
    torch.cuda.synchronize()
    return yd.cpu().numpy()


def evaluate(model: Model, x: np.ndarray, y: np.ndarray) -> float:
    """Mean squared error in standardised target units over the present
    (non-NaN) targets."""
    pred = predict(model, x)
    n = model.normalization()
    err = ((pred - y) / n[26:28]) ** 2
    return float(np.nanmean(err))


def compare_iterations(model: Model, workload: str = "dam_break_16k", frames: int = 20,
                       warmup: int = 5, min_iterations: int = 1, device: int = 0):
    """Plain versus learned warm start on the same scene and tolerance:
    average Jacobi iterations per frame (density, divergence), the largest
    residual metrics and speed seen, and the simulated time covered."""
    lib = load_library()
    out = {}
    for arm in ("plain", "learned"):
        w = scene.workload(workload)
        p = _abi.copy_params(w.params)
        p.solver = _abi.FE_SOLVER_TOLERANCE
        p.mode = _abi.FE_MODE_FIXED
        p.min_iterations = min_iterations
        if arm == "learned":
            p.warm_start = _abi.FE_WARM_LEARNED
        sim = Simulation(w.positions(), p, device=device)
        if arm == "learned":
            check(lib, lib.fe_set_model(sim.data.handle, model.handle), "fe_set_model")
        for _ in range(warmup):
            sim.step(1)
        st0 = sim.data.read_stats()
        res = []
        sim_time = 0.0
        for _ in range(frames):
            st = sim.step(1)
            res.append((st.density_residual, st.divergence_residual, st.max_speed))
            sim_time += st.dt
        st = sim.data.read_stats()
        out[arm] = {
            "density_iterations": (st.total_density_iterations - st0.total_density_iterations) / frames,
            "divergence_iterations": (st.total_divergence_iterations
                                      - st0.total_divergence_iterations) / frames,
            "max_density_residual": float(max(r[0] for r in res)),
            "max_divergence_residual": float(max(r[1] for r in res)),
            "max_speed": float(max(r[2] for r in res)),
            "simulated_seconds": sim_time,
            "cap_hits": int(st.flags & _abi.FE_STATS_ITERATION_CAP_HIT),
            "non_finite": int(st.flags & _abi.FE_STATS_NON_FINITE),
        }
        sim.close()
    return out
