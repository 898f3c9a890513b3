"""ctypes wrapper of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product path never imports
it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys
from ctypes import POINTER, c_double, c_int, c_size_t, c_uint32, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "fluid-engine_b200"))

from fluid_step import _abi  # noqa: E402  (struct layouts only)

LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = POINTER(_abi.FeParams)
        S = POINTER(_abi.FeStats)
        sig = {
            "fo_create": (c_void_p, [P, c_uint32, c_void_p, c_void_p, c_int]),
            "fo_destroy": (None, [c_void_p]),
            "fo_set_params": (c_int, [c_void_p, P]),
            "fo_get_params": (c_int, [c_void_p, P]),
            "fo_table_size": (c_uint32, [c_void_p]),
            "fo_step": (c_int, [c_void_p, c_uint32, c_uint32, S]),
            "fo_read_stats": (c_int, [c_void_p, S]),
            "fo_download": (c_int, [c_void_p, c_int, c_void_p, c_size_t]),
            "fo_download_f64": (c_int, [c_void_p, c_int, c_void_p, c_size_t]),
            "fo_upload": (c_int, [c_void_p, c_int, c_void_p, c_size_t]),
            "fo_sort_radix_mirror": (None, [c_void_p, c_void_p, c_uint32]),
            "fo_sort_radix_parallel": (None, [c_void_p, c_void_p, c_uint32, c_uint32]),
            "fo_sort_bitonic": (c_int, [c_void_p, c_void_p, c_uint32]),
            "fo_det_sum": (c_double, [c_void_p, c_size_t]),
            "fo_splat_density": (None, [c_void_p, c_uint32, P, c_void_p]),
            "fo_raymarch": (None, [c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_int,
                                   c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int,
                                   c_void_p]),
            "fo_set_learned": (c_int, [c_void_p, c_void_p]),
            "fo_set_network_outputs": (c_int, [c_void_p, c_uint32, c_void_p]),
            "fo_get_feature_rows": (c_int, [c_void_p, c_uint32, c_void_p]),
            "fo_learned_missing_outputs": (c_int, [c_void_p]),
            "fo_set_threads": (c_int, [c_int]),
            "fo_get_threads": (c_int, []),
        }
        for name in ["fo_neighbor_search", "fo_density_alpha", "fo_viscosity",
                     "fo_density_source", "fo_pressure_force", "fo_pressure_update",
                     "fo_pressure_integration", "fo_divergence_source",
                     "fo_divergence_integration", "fo_stats_pass"]:
            sig[name] = (c_int, [c_void_p])
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(c_void_p)


class Oracle:
    """One host simulation context (FP32 shader order, or the FP64 twin)."""

    STAGES = ["neighbor_search", "density_alpha", "viscosity", "density_source",
              "pressure_force", "pressure_update", "pressure_integration",
              "divergence_source", "divergence_integration", "stats_pass"]

    def __init__(self, params, positions, velocities=None, fp64=False):
        L = lib()
        pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
        vel = None if velocities is None else np.ascontiguousarray(
            velocities, dtype=np.float32).reshape(-1, 3)
        self.n = pos.shape[0]
        self.params = _abi.copy_params(params)
        self.h = L.fo_create(ctypes.byref(self.params), self.n, _ptr(pos),
                             None if vel is None else _ptr(vel), 1 if fp64 else 0)
        if not self.h:
            raise ValueError("fo_create rejected its arguments")
        self.T = L.fo_table_size(self.h)
        self.fp64 = fp64

    def close(self):
        if self.h:
            lib().fo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params):
        self.params = _abi.copy_params(params)
        lib().fo_set_params(self.h, ctypes.byref(self.params))

    def get_params(self):
        p = _abi.FeParams()
        lib().fo_get_params(self.h, ctypes.byref(p))
        return p

    def run(self, stage: str):
        rc = getattr(lib(), "fo_" + stage)(self.h)
        if rc:
            raise RuntimeError(f"oracle {stage}: {rc}")

    def step(self, n_substeps=1, flags=0):
        st = _abi.FeStats()
        rc = lib().fo_step(self.h, n_substeps, flags, ctypes.byref(st))
        if rc:
            raise RuntimeError(f"oracle step: {rc}")
        return st

    def stats(self):
        st = _abi.FeStats()
        lib().fo_read_stats(self.h, ctypes.byref(st))
        return st

    def field(self, field: int, f64=False) -> np.ndarray:
        count = self.T if field in _abi.TABLE_FIELDS else (3 if field == _abi.FE_FIELD_STATS else self.n)
        width = 4 if field in _abi.VEC4_FIELDS else 1
        if f64:
            out = np.empty(count * width, dtype=np.float64)
            rc = lib().fo_download_f64(self.h, field, _ptr(out), out.size)
        else:
            dt = np.uint32 if field in _abi.UINT_FIELDS else np.float32
            out = np.empty(count * width, dtype=dt)
            rc = lib().fo_download(self.h, field, _ptr(out), out.nbytes)
        if rc:
            raise RuntimeError(f"oracle download {field}: {rc}")
        return out.reshape(count, width) if width == 4 else out

    # -- learned warm start (the network's outputs are given, not computed) --
    def set_learned(self, norm) -> None:
        """Turns the warm start on with the model's standardisation (28
        floats: x mean[12], x std[12], y mean[2], y std[2]); None: off."""
        if norm is None:
            self._norm = None
            rc = lib().fo_set_learned(self.h, None)
        else:
            self._norm = np.ascontiguousarray(norm[:28], dtype=np.float32)
            rc = lib().fo_set_learned(self.h, _ptr(self._norm))
        if rc:
            raise RuntimeError(f"oracle set_learned: {rc}")

    def set_network_outputs(self, outs) -> None:
        """outs[slot][n][2]: the network's standardised outputs for the
        next frame's solves (slot 2k density, 2k + 1 divergence)."""
        a = np.ascontiguousarray(outs, dtype=np.float32).reshape(-1, self.n, 2)
        self._outs = a
        rc = lib().fo_set_network_outputs(self.h, a.shape[0], _ptr(a))
        if rc:
            raise RuntimeError(f"oracle set_network_outputs: {rc}")

    def feature_rows(self, slot: int) -> np.ndarray:
        """uint16[n][16]: the BF16 network inputs of a solve of the last frame."""
        out = np.empty((self.n, 16), np.uint16)
        rc = lib().fo_get_feature_rows(self.h, slot, _ptr(out))
        if rc:
            raise RuntimeError(f"oracle feature_rows({slot}): {rc}")
        return out

    def missing_network_outputs(self) -> bool:
        return bool(lib().fo_learned_missing_outputs(self.h))

    def upload(self, field: int, data: np.ndarray):
        dt = np.uint32 if field in _abi.UINT_FIELDS else np.float32
        a = np.ascontiguousarray(data, dtype=dt)
        rc = lib().fo_upload(self.h, field, _ptr(a), a.nbytes)
        if rc:
            raise RuntimeError(f"oracle upload {field}: {rc}")


def sort_radix_mirror(keys, values):
    k = np.ascontiguousarray(keys, dtype=np.uint32).copy()
    v = np.ascontiguousarray(values, dtype=np.uint32).copy()
    lib().fo_sort_radix_mirror(_ptr(k), _ptr(v), k.size)
    return k, v


def sort_radix_parallel(keys, values, key_bits=32):
    k = np.ascontiguousarray(keys, dtype=np.uint32).copy()
    v = np.ascontiguousarray(values, dtype=np.uint32).copy()
    lib().fo_sort_radix_parallel(_ptr(k), _ptr(v), k.size, key_bits)
    return k, v


def sort_bitonic(keys, values):
    k = np.ascontiguousarray(keys, dtype=np.uint32).copy()
    v = np.ascontiguousarray(values, dtype=np.uint32).copy()
    if lib().fo_sort_bitonic(_ptr(k), _ptr(v), k.size):
        raise ValueError("bitonic sort needs a power-of-two length")
    return k, v


def splat_density(positions4, params) -> np.ndarray:
    """splat_density.comp on float4 positions: uint32[res_z][res_y][res_x]."""
    pos = np.ascontiguousarray(positions4, dtype=np.float32).reshape(-1, 4)
    rx, ry, rz = (int(v) for v in params.grid_res)
    out = np.empty((rz, ry, rx), dtype=np.uint32)
    p = _abi.copy_params(params)
    lib().fo_splat_density(_ptr(pos), pos.shape[0], ctypes.byref(p), _ptr(out))
    return out


def raymarch(grid, sky, camera, box_min, box_max) -> np.ndarray:
    """raymarch.frag for one ray per pixel: float32[height][width][4]."""
    g = np.ascontiguousarray(grid, dtype=np.uint32)
    rz, ry, rx = g.shape
    sk = np.ascontiguousarray(sky, dtype=np.float32)
    sh, sw = sk.shape[:2]
    ivp = np.ascontiguousarray(np.frombuffer(bytes(camera.inv_view_proj), np.float32))
    cam = np.ascontiguousarray(np.frombuffer(bytes(camera.camera_pos), np.float32))
    bmin = np.ascontiguousarray(box_min, np.float32)
    bmax = np.ascontiguousarray(box_max, np.float32)
    out = np.empty((camera.height, camera.width, 4), np.float32)
    lib().fo_raymarch(_ptr(g), rx, ry, rz, _ptr(sk), sw, sh, _ptr(ivp), _ptr(cam), _ptr(bmin),
                      _ptr(bmax), camera.width, camera.height, _ptr(out))
    return out


def det_sum(values) -> float:
    a = np.ascontiguousarray(values, dtype=np.float64)
    return lib().fo_det_sum(_ptr(a), a.size)


def set_threads(t: int) -> int:
    return lib().fo_set_threads(t)


def get_threads() -> int:
    return lib().fo_get_threads()
