"""ctypes mirror of include/fluid_step.h.

Struct layouts, enum values and status codes are declared once here and used
by the host-side mirror of the reference's ComputeStep API (pipelines.py),
by the tests and by bench.py.  The shared library is the product; this module
only loads it and declares its signatures.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_double, c_float, c_int,
                    c_int32, c_size_t, c_uint32, c_uint64, c_void_p)

ABI_VERSION = 2
FE_STATE_VERSION = 3

# fe_status
FE_OK = 0
FE_ERR_INVALID_ARGUMENT = 1
FE_ERR_NOT_PREPARED = 2
FE_ERR_CUDA = 3
FE_ERR_OUT_OF_MEMORY = 4
FE_ERR_NON_FINITE = 5
FE_ERR_ITERATION_CAP = 6
FE_ERR_TIMEOUT = 7
FE_ERR_NO_DEVICE = 8
FE_ERR_CAPACITY = 9
FE_ERR_UNSUPPORTED = 10

STATUS_NAMES = {
    0: "FE_OK", 1: "FE_ERR_INVALID_ARGUMENT", 2: "FE_ERR_NOT_PREPARED",
    3: "FE_ERR_CUDA", 4: "FE_ERR_OUT_OF_MEMORY", 5: "FE_ERR_NON_FINITE",
    6: "FE_ERR_ITERATION_CAP", 7: "FE_ERR_TIMEOUT", 8: "FE_ERR_NO_DEVICE",
    9: "FE_ERR_CAPACITY", 10: "FE_ERR_UNSUPPORTED",
}

# fe_sort_algorithm (sorter.rs:19-23: Bitonic, Radix)
FE_SORT_BITONIC = 0
FE_SORT_RADIX = 1
# fe_mode
FE_MODE_REFERENCE = 0
FE_MODE_FIXED = 1
# fe_solver
FE_SOLVER_FIXED_ITERS = 0
FE_SOLVER_TOLERANCE = 1
# fe_warm_start
FE_WARM_REFERENCE = 0
FE_WARM_LEARNED = 1

# fe_field
FE_FIELD_POSITION_A = 0
FE_FIELD_POSITION_B = 1
FE_FIELD_VELOCITY_A = 2
FE_FIELD_VELOCITY_B = 3
FE_FIELD_DENSITY = 4
FE_FIELD_FACTOR = 5
FE_FIELD_SOURCE_TERM = 6
FE_FIELD_PRESSURE = 7
FE_FIELD_PRESSURE_ACCEL = 8
FE_FIELD_ENTRY_HASH = 9
FE_FIELD_ENTRY_INDEX = 10
FE_FIELD_GRID_START = 11
FE_FIELD_STATS = 12
FE_FIELD_DENSITY_GRID = 13
FE_FIELD_IMAGE = 14

VEC4_FIELDS = {FE_FIELD_POSITION_A, FE_FIELD_POSITION_B, FE_FIELD_VELOCITY_A,
               FE_FIELD_VELOCITY_B, FE_FIELD_PRESSURE_ACCEL}
UINT_FIELDS = {FE_FIELD_ENTRY_HASH, FE_FIELD_ENTRY_INDEX, FE_FIELD_GRID_START,
               FE_FIELD_STATS, FE_FIELD_DENSITY_GRID}
TABLE_FIELDS = {FE_FIELD_ENTRY_HASH, FE_FIELD_ENTRY_INDEX, FE_FIELD_GRID_START}

FE_STEP_INIT_NS = 0x1
FE_STEP_NO_GRAPH = 0x2

FE_STATS_ITERATION_CAP_HIT = 0x1
FE_STATS_NEIGHBOR_OVERFLOW = 0x2
FE_STATS_LOOKBACK_TIMEOUT = 0x4
FE_STATS_NON_FINITE = 0x8

FE_MAX_PARTICLES = 1 << 26
FE_MAX_SCENES = 65536


class FeParams(Structure):
    """fe_params: SimulationParams (particle.rs:310-331) + AppUI knobs."""
    _fields_ = [
        ("particle_radius", c_float),
        ("particle_mass", c_float),
        ("smoothing_radius", c_float),
        ("target_density", c_float),
        ("viscosity", c_float),
        ("relax_factor", c_float),
        ("dt", c_float),
        ("density_solver_iterations", c_uint32),
        ("divergence_solver_iterations", c_uint32),
        ("gravity", c_float * 3),
        ("box_min", c_float * 3),
        ("box_max", c_float * 3),
        ("grid_res", c_int32 * 3),
        ("sort_algorithm", c_uint32),
        ("use_cfl", c_uint32),
        ("use_solver_error_threshold", c_uint32),
        ("density_error_pct", c_float),
        ("divergence_error_pct", c_float),
        ("cfl_lambda", c_float),
        ("cfl_min_dt", c_float),
        ("cfl_max_dt", c_float),
        ("cfl_growth", c_float),
        ("mode", c_uint32),
        ("solver", c_uint32),
        ("density_tolerance", c_float),
        ("divergence_tolerance", c_float),
        ("min_iterations", c_uint32),
        ("max_iterations", c_uint32),
        ("warm_start", c_uint32),
        ("reserved", c_uint32 * 7),
    ]


class FeStats(Structure):
    """fe_stats: stats_buffer (stats.comp:8) + decoded and FP64 extras."""
    _fields_ = [
        ("max_speed_bits", c_uint32),
        ("density_error_fp", c_uint32),
        ("divergence_error_fp", c_uint32),
        ("substeps", c_uint32),
        ("max_speed", c_float),
        ("avg_density_error", c_float),
        ("avg_divergence_error", c_float),
        ("dt", c_float),
        ("avg_density_error_f64", c_double),
        ("avg_divergence_error_f64", c_double),
        ("density_residual", c_double),
        ("divergence_residual", c_double),
        ("density_iterations", c_uint32),
        ("divergence_iterations", c_uint32),
        ("total_density_iterations", c_uint64),
        ("total_divergence_iterations", c_uint64),
        ("flags", c_uint32),
        ("reserved", c_uint32),
        ("density_residual_max", c_double),
        ("divergence_residual_max", c_double),
    ]

    def as_dict(self) -> dict:
        return {name: (list(getattr(self, name)) if name == "reserved" else getattr(self, name))
                for name, _ in self._fields_ if name != "reserved"}


class FeCamera(Structure):
    """fe_camera: column-major inverse view-projection, camera position,
    image size."""
    _fields_ = [("inv_view_proj", c_float * 16), ("camera_pos", c_float * 3),
                ("width", c_uint32), ("height", c_uint32), ("reserved", c_uint32 * 3)]


FE_NBR_DENSITY_ALPHA = 0
FE_NBR_LIST_PASSES = 1
FE_NBR_PRESSURE_FORCE = 2
FE_NBR_PRESSURE_UPDATE = 3
FE_NBR_GROUPS = 4
NBR_GROUP_NAMES = ("density_alpha", "list_passes", "pressure_force", "pressure_update")


class FeTuning(Structure):
    """fe_tuning: the tunable shapes (none changes a result)."""
    _fields_ = [("radix_digit_bits", c_uint32), ("radix_items", c_uint32),
                ("mlp_ctas_per_sm", c_uint32), ("reserved", c_uint32),
                ("nbr_threads", c_uint32 * FE_NBR_GROUPS),
                ("nbr_persistent", c_uint32 * FE_NBR_GROUPS)]

    def as_dict(self) -> dict:
        return {"radix_digit_bits": self.radix_digit_bits, "radix_items": self.radix_items,
                "mlp_ctas_per_sm": self.mlp_ctas_per_sm,
                "nbr_threads": list(self.nbr_threads),
                "nbr_persistent": list(self.nbr_persistent)}

    @classmethod
    def from_dict(cls, d: dict) -> "FeTuning":
        t = cls(int(d["radix_digit_bits"]), int(d["radix_items"]), int(d["mlp_ctas_per_sm"]), 0)
        for g in range(FE_NBR_GROUPS):
            t.nbr_threads[g] = int(d.get("nbr_threads", [256] * FE_NBR_GROUPS)[g])
            t.nbr_persistent[g] = int(d.get("nbr_persistent", [0] * FE_NBR_GROUPS)[g])
        return t


FE_TUNE_MAX_CANDIDATES = 8


class FeTuneReport(Structure):
    """fe_tune_report: median time of every candidate and the choice."""
    _fields_ = [("radix_candidates", c_uint32),
                ("radix_digit_bits", c_uint32 * FE_TUNE_MAX_CANDIDATES),
                ("radix_items", c_uint32 * FE_TUNE_MAX_CANDIDATES),
                ("radix_ms", c_float * FE_TUNE_MAX_CANDIDATES),
                ("mlp_candidates", c_uint32),
                ("mlp_ctas_per_sm", c_uint32 * FE_TUNE_MAX_CANDIDATES),
                ("mlp_ms", c_float * FE_TUNE_MAX_CANDIDATES),
                ("nbr_candidates", c_uint32),
                ("nbr_threads", c_uint32 * FE_TUNE_MAX_CANDIDATES),
                ("nbr_persistent", c_uint32 * FE_TUNE_MAX_CANDIDATES),
                ("nbr_ms", (c_float * FE_TUNE_MAX_CANDIDATES) * FE_NBR_GROUPS),
                ("chosen", FeTuning)]

    def as_dict(self) -> dict:
        r = {"radix": [{"digit_bits": self.radix_digit_bits[k], "items": self.radix_items[k],
                        "ms": self.radix_ms[k]} for k in range(self.radix_candidates)],
             "mlp": [{"ctas_per_sm": self.mlp_ctas_per_sm[k], "ms": self.mlp_ms[k]}
                     for k in range(self.mlp_candidates)],
             "neighbour": {NBR_GROUP_NAMES[g]: [
                 {"threads": self.nbr_threads[k], "persistent": self.nbr_persistent[k],
                  "ms": self.nbr_ms[g][k]}
                 for k in range(self.nbr_candidates) if self.nbr_ms[g][k] >= 0]
                 for g in range(FE_NBR_GROUPS)},
             "chosen": self.chosen.as_dict()}
        return r


RADIX_CANDIDATES = [(8, 4), (8, 8), (8, 16), (10, 8), (10, 16)]


def default_params() -> FeParams:
    """Defaults of Scene::new() (scene.rs:14-86) and AppUI::new() (ui.rs:31-49).

    Pure-Python twin of fe_default_params(), usable without the library.
    """
    import numpy as np
    p = FeParams()
    radius = np.float32(0.02)
    spacing = np.float32(radius * np.float32(2.0))
    p.particle_radius = float(radius)
    p.particle_mass = float(np.float32(1000.0) * (spacing * spacing * spacing))
    p.smoothing_radius = float(radius * np.float32(4.0))
    p.target_density = 1000.0
    p.viscosity = 0.15
    p.relax_factor = 0.5
    p.dt = 0.005
    p.density_solver_iterations = 4
    p.divergence_solver_iterations = 4
    p.gravity[:] = [0.0, -9.81, 0.0]
    p.box_min[:] = [-1.5, 0.0, -1.0]
    p.box_max[:] = [0.8, 4.0, 1.0]
    p.grid_res[:] = [128, 128, 128]
    p.sort_algorithm = FE_SORT_RADIX
    p.use_cfl = 0
    p.use_solver_error_threshold = 0
    p.density_error_pct = 0.1
    p.divergence_error_pct = 0.5
    p.cfl_lambda = 0.4
    p.cfl_min_dt = 0.001
    p.cfl_max_dt = 0.05
    p.cfl_growth = 1.1
    p.mode = FE_MODE_REFERENCE
    p.solver = FE_SOLVER_FIXED_ITERS
    p.density_tolerance = 0.001
    p.divergence_tolerance = 0.001
    p.min_iterations = 2
    p.max_iterations = 100
    p.warm_start = FE_WARM_REFERENCE
    return p


def copy_params(p: FeParams) -> FeParams:
    q = FeParams()
    ctypes.pointer(q)[0] = p
    return q


PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PACKAGE_DIR, "libfluidstep.so")
# The same C ABI with the physics kernels compiled with fused multiply-add
# contraction: within a relative tolerance of the FP64 step, not bit-exact.
CONTRACT_LIB_PATH = os.path.join(PACKAGE_DIR, "libfluidstep_contract.so")
BUILDS = {"parity": LIB_PATH, "contract": CONTRACT_LIB_PATH}

_lib = None
_libs: dict = {}


class LibraryMissing(RuntimeError):
    pass


def load_library(path: str | None = None, *, build: str = "parity"):
    """Loads libfluidstep.so from the package directory (build="contract":
    libfluidstep_contract.so, the fused multiply-add build).

    Raises LibraryMissing when the library was not built: there is no other
    implementation to fall back to.
    """
    global _lib
    if path is None and build != "parity":
        if build not in BUILDS:
            raise ValueError(f"unknown build {build!r} (expected one of {sorted(BUILDS)})")
        if build not in _libs:
            _libs[build] = load_library(BUILDS[build])
        return _libs[build]
    if _lib is not None and path is None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise LibraryMissing(
            f"{path} not found: build it with `python fluid-engine_b200/build.py` "
            "(or __graft_entry__.build()); the DFSPH step has no CPU fallback")
    lib = ctypes.CDLL(path)
    _declare(lib)
    if lib.fe_abi_version() != ABI_VERSION:
        raise RuntimeError(f"ABI mismatch: library {lib.fe_abi_version()} != {ABI_VERSION}")
    if path == LIB_PATH:
        _lib = lib
    return lib


CTX = c_void_p

# name -> (restype, argtypes); mirrors every declaration of fluid_step.h.
SIGNATURES = {
    "fe_abi_version": (c_uint32, []),
    "fe_status_string": (c_char_p, [c_int]),
    "fe_last_error": (c_char_p, []),
    "fe_default_params": (None, [POINTER(FeParams)]),
    "fe_validate_params": (c_int, [POINTER(FeParams)]),
    "fe_create": (c_int, [POINTER(FeParams), c_uint32, c_void_p, c_void_p, c_int,
                          POINTER(CTX)]),
    "fe_destroy": (c_int, [CTX]),
    "fe_batch_create": (c_int, [POINTER(FeParams), POINTER(c_uint32), c_uint32, c_void_p,
                                c_void_p, c_int, POINTER(CTX)]),
    "fe_scene_count": (c_int, [CTX, POINTER(c_uint32)]),
    "fe_scene_table": (c_int, [CTX, POINTER(c_uint32), POINTER(c_uint32), c_uint32]),
    "fe_set_scene_params": (c_int, [CTX, c_uint32, POINTER(FeParams)]),
    "fe_get_scene_params": (c_int, [CTX, c_uint32, POINTER(FeParams)]),
    "fe_read_scene_stats": (c_int, [CTX, c_uint32, POINTER(FeStats)]),
    "fe_autotune": (c_int, [CTX, POINTER(FeTuneReport)]),
    "fe_get_tuning": (c_int, [CTX, POINTER(FeTuning)]),
    "fe_set_tuning": (c_int, [CTX, POINTER(FeTuning)]),
    "fe_autotune_sort": (c_int, [c_void_p, c_void_p, c_uint32, c_uint32, POINTER(FeTuneReport)]),
    "fe_sort_pairs_config": (c_int, [c_void_p, c_void_p, c_uint32, c_uint32, c_uint32, c_uint32,
                                     c_void_p]),
    "fe_density_splat": (c_int, [CTX]),
    "fe_set_skybox": (c_int, [CTX, c_void_p, c_uint32, c_uint32]),
    "fe_raymarch": (c_int, [CTX, POINTER(FeCamera)]),
    "fe_set_params": (c_int, [CTX, POINTER(FeParams)]),
    "fe_get_params": (c_int, [CTX, POINTER(FeParams)]),
    "fe_prepare": (c_int, [CTX]),
    "fe_get_size": (c_int, [CTX, POINTER(c_uint32), POINTER(c_uint32)]),
    "fe_get_stream": (c_void_p, [CTX]),
    "fe_synchronize": (c_int, [CTX]),
    "fe_upload": (c_int, [CTX, c_int, c_void_p, c_size_t]),
    "fe_download": (c_int, [CTX, c_int, c_void_p, c_size_t]),
    "fe_download_async": (c_int, [CTX, c_int, c_void_p, c_size_t, POINTER(ctypes.c_uint64)]),
    "fe_download_wait": (c_int, [CTX, ctypes.c_uint64]),
    "fe_read_stats_async": (c_int, [CTX, POINTER(ctypes.c_uint64)]),
    "fe_stats_wait": (c_int, [CTX, ctypes.c_uint64, POINTER(FeStats)]),
    "fe_neighbor_search": (c_int, [CTX]),
    "fe_density_alpha": (c_int, [CTX]),
    "fe_viscosity": (c_int, [CTX]),
    "fe_density_source": (c_int, [CTX]),
    "fe_pressure_force": (c_int, [CTX]),
    "fe_pressure_update": (c_int, [CTX]),
    "fe_pressure_integration": (c_int, [CTX]),
    "fe_divergence_source": (c_int, [CTX]),
    "fe_divergence_integration": (c_int, [CTX]),
    "fe_stats_pass": (c_int, [CTX]),
    "fe_read_stats": (c_int, [CTX, POINTER(FeStats)]),
    "fe_debug_fail_allocation": (None, [c_uint32]),
    "fe_debug_poison_allocations": (None, [c_int]),
    "fe_debug_bounded_wait": (c_int, [c_int, c_uint32, POINTER(c_uint32)]),
    "fe_state_size": (c_int, [CTX, POINTER(c_size_t)]),
    "fe_state_export": (c_int, [CTX, c_void_p, c_size_t]),
    "fe_state_import": (c_int, [CTX, c_void_p, c_size_t]),
    "fe_step": (c_int, [CTX, c_uint32, c_uint32, POINTER(FeStats)]),
    "fe_sort_pairs": (c_int, [c_void_p, c_void_p, c_uint32, c_uint32, c_int, c_void_p]),
    "fe_sort_pairs_host": (c_int, [c_void_p, c_void_p, c_uint32, c_uint32, c_int]),
    "fe_sort_pairs_noalloc": (c_int, [c_void_p, c_void_p, c_uint32, c_uint32, c_void_p]),
    "fe_sort_noalloc_flags": (c_int, [c_void_p, c_void_p]),
    "fe_sort_flags": (c_int, [c_void_p, c_void_p]),
    "fe_debug_noalloc_wait_timeout": (c_int, [c_uint32, c_void_p]),
    "fe_debug_trace_learned": (c_int, [c_void_p, c_uint32]),
    "fe_debug_read_trace": (c_int, [c_void_p, c_uint32, c_void_p, c_void_p]),
    "fe_model_create": (c_int, [c_uint32, c_int, POINTER(c_void_p)]),
    "fe_model_destroy": (c_int, [c_void_p]),
    "fe_model_set_parameters": (c_int, [c_void_p, c_void_p, c_size_t]),
    "fe_model_get_parameters": (c_int, [c_void_p, c_void_p, c_size_t]),
    "fe_model_set_normalization": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "fe_model_get_normalization": (c_int, [c_void_p, c_void_p]),
    "fe_model_forward": (c_int, [c_void_p, c_void_p, c_void_p, c_uint32, c_void_p]),
    "fe_model_gradients": (c_int, [c_void_p, c_void_p, c_void_p, c_uint32, c_void_p, c_void_p]),
    "fe_model_train_step": (c_int, [c_void_p, c_void_p, c_void_p, c_uint32, c_float, c_float,
                                    c_void_p, c_void_p]),
    "fe_model_read_flags": (c_int, [c_void_p, POINTER(c_uint32)]),
    "fe_set_model": (c_int, [CTX, c_void_p]),
    "fe_capture_begin": (c_int, [CTX, c_uint32, c_uint32]),
    "fe_capture_read": (c_int, [CTX, c_void_p, c_void_p, c_uint32, POINTER(c_uint32)]),
    "fe_capture_end": (c_int, [CTX]),
}

FE_MODEL_PARAMS = 5378
FE_MODEL_FEATURES = 12

FE_SORT_NOALLOC_MAX_PAIRS = 1 << 20


def _declare(lib) -> None:
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


class FluidStepError(RuntimeError):
    """A non-zero fe_status, with the library's last error message."""

    def __init__(self, status: int, where: str, message: str = ""):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}"
                         + (f" ({message})" if message else ""))


def check(lib, status: int, where: str) -> None:
    if status != FE_OK:
        msg = lib.fe_last_error()
        raise FluidStepError(status, where, msg.decode() if msg else "")
