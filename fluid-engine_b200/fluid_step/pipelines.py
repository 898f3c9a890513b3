"""Host-side mirror of the reference's compute-step plugin API.

Reference (Rust, src/renderer/pipelines/mod.rs:52-124):

    trait ComputeStep { fn new(device); fn prepare(&mut self, allocator,
                        physics_data: &GpuPhysicsData, sim_params); fn execute(&self, builder) }
    struct ComputePipelines { neighbor_search, density_alpha, viscosity,
                        density_source_term, pressure_force, pressure_update,
                        pressure_integration, divergence_source_term,
                        divergence_integration, density_texture, stats }

Here every pass forwards to the C ABI of libfluidstep.so.  `execute(builder)`
enqueues the pass on the context's CUDA stream in call order (the recorded
command buffer of the reference); `builder.execute_and_wait()` is the
submit + fence wait.  Executing before `prepare` raises, with the reference's
panic message ("call prepare() before execute()").
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import check, load_library

SortAlgorithm = type("SortAlgorithm", (), {"Bitonic": _abi.FE_SORT_BITONIC,
                                           "Radix": _abi.FE_SORT_RADIX})


class GpuPhysicsData:
    """`GpuPhysicsData::new` (particle.rs:164-299): device buffers of N
    particles and a hash table of next_pow2(N) entries."""

    def __init__(self, initial_positions, sim_params: _abi.FeParams, *, velocities=None,
                 device: int = 0, build: str = "parity"):
        self._lib = load_library(build=build)
        pos = np.ascontiguousarray(initial_positions, dtype=np.float32).reshape(-1, 3)
        vel = None if velocities is None else np.ascontiguousarray(
            velocities, dtype=np.float32).reshape(-1, 3)
        self.count = int(pos.shape[0])
        self.params = _abi.copy_params(sim_params)
        h = ctypes.c_void_p()
        st = self._lib.fe_create(ctypes.byref(self.params), self.count,
                                 pos.ctypes.data_as(ctypes.c_void_p),
                                 None if vel is None else vel.ctypes.data_as(ctypes.c_void_p),
                                 device, ctypes.byref(h))
        check(self._lib, st, "fe_create")
        self.handle = h
        n = ctypes.c_uint32()
        t = ctypes.c_uint32()
        check(self._lib, self._lib.fe_get_size(h, ctypes.byref(n), ctypes.byref(t)), "fe_get_size")
        self.table_size = int(t.value)

    # -- resources.rs:85-92 -------------------------------------------------
    def sync_with_scene(self, sim_params: _abi.FeParams) -> None:
        self.params = _abi.copy_params(sim_params)
        check(self._lib, self._lib.fe_set_params(self.handle, ctypes.byref(self.params)),
              "fe_set_params")

    def current_params(self) -> _abi.FeParams:
        p = _abi.FeParams()
        check(self._lib, self._lib.fe_get_params(self.handle, ctypes.byref(p)), "fe_get_params")
        return p

    def download(self, field: int) -> np.ndarray:
        count = (self.table_size if field in _abi.TABLE_FIELDS
                 else 3 if field == _abi.FE_FIELD_STATS else self.count)
        width = 4 if field in _abi.VEC4_FIELDS else 1
        dt = np.uint32 if field in _abi.UINT_FIELDS else np.float32
        out = np.empty(count * width, dtype=dt)
        check(self._lib, self._lib.fe_download(self.handle, field,
                                               out.ctypes.data_as(ctypes.c_void_p), out.nbytes),
              "fe_download")
        return out.reshape(count, 4) if width == 4 else out

    def download_async(self, field: int, out: np.ndarray) -> int:
        """Starts copying `field` into `out` (a C-contiguous array of the
        field's size, ideally in page-locked memory) without waiting; returns
        the ticket for download_wait.  `out` must stay alive until then."""
        t = ctypes.c_uint64()
        check(self._lib, self._lib.fe_download_async(
            self.handle, field, out.ctypes.data_as(ctypes.c_void_p), out.nbytes,
            ctypes.byref(t)), "fe_download_async")
        return int(t.value)

    def read_stats_async(self) -> int:
        """Captures the last stats pass's stats without waiting; the ticket
        goes to stats_wait."""
        t = ctypes.c_uint64()
        check(self._lib, self._lib.fe_read_stats_async(self.handle, ctypes.byref(t)),
              "fe_read_stats_async")
        return int(t.value)

    def stats_wait(self, ticket: int) -> _abi.FeStats:
        st = _abi.FeStats()
        check(self._lib, self._lib.fe_stats_wait(self.handle, ticket, ctypes.byref(st)),
              "fe_stats_wait")
        return st

    def download_wait(self, ticket: int) -> None:
        check(self._lib, self._lib.fe_download_wait(self.handle, ticket), "fe_download_wait")

    def upload(self, field: int, data) -> None:
        dt = np.uint32 if field in _abi.UINT_FIELDS else np.float32
        a = np.ascontiguousarray(data, dtype=dt)
        check(self._lib, self._lib.fe_upload(self.handle, field,
                                             a.ctypes.data_as(ctypes.c_void_p), a.nbytes),
              "fe_upload")

    def read_stats(self) -> _abi.FeStats:
        st = _abi.FeStats()
        check(self._lib, self._lib.fe_read_stats(self.handle, ctypes.byref(st)), "fe_read_stats")
        return st

    # -- checkpoint / resume (fe_state_export / fe_state_import) --------------
    def export_state(self) -> bytes:
        """A snapshot of everything a later step reads (versioned binary)."""
        size = ctypes.c_size_t()
        check(self._lib, self._lib.fe_state_size(self.handle, ctypes.byref(size)), "fe_state_size")
        buf = ctypes.create_string_buffer(size.value)
        check(self._lib, self._lib.fe_state_export(self.handle, buf, size.value), "fe_state_export")
        return buf.raw

    def import_state(self, snapshot: bytes) -> None:
        """Restores a snapshot of a context with the same sizes and scene layout."""
        buf = ctypes.create_string_buffer(bytes(snapshot), len(snapshot))
        check(self._lib, self._lib.fe_state_import(self.handle, buf, len(snapshot)),
              "fe_state_import")

    # -- density_texture.rs / splat_density.comp -----------------------------
    def splat_density(self) -> np.ndarray:
        """Clears and splats the headless density grid (fe_density_splat);
        returns uint32[res_z][res_y][res_x]."""
        check(self._lib, self._lib.fe_density_splat(self.handle), "fe_density_splat")
        p = self.current_params()
        rx, ry, rz = (int(v) for v in p.grid_res)
        out = np.empty((rz, ry, rx), dtype=np.uint32)
        check(self._lib, self._lib.fe_download(self.handle, _abi.FE_FIELD_DENSITY_GRID,
                                               out.ctypes.data_as(ctypes.c_void_p), out.nbytes),
              "fe_download(density grid)")
        return out

    # -- water pass (raymarch.frag) into a headless image ---------------------
    def set_skybox(self, rgba) -> None:
        """Equirectangular sky, float32[height][width][4]."""
        a = np.ascontiguousarray(rgba, dtype=np.float32)
        check(self._lib, self._lib.fe_set_skybox(self.handle, a.ctypes.data_as(ctypes.c_void_p),
                                                 a.shape[1], a.shape[0]), "fe_set_skybox")

    def raymarch(self, camera: _abi.FeCamera) -> np.ndarray:
        """Renders the last splat grid; returns float32[height][width][4]."""
        check(self._lib, self._lib.fe_raymarch(self.handle, ctypes.byref(camera)), "fe_raymarch")
        out = np.empty((camera.height, camera.width, 4), dtype=np.float32)
        check(self._lib, self._lib.fe_download(self.handle, _abi.FE_FIELD_IMAGE,
                                               out.ctypes.data_as(ctypes.c_void_p), out.nbytes),
              "fe_download(image)")
        return out

    # -- autotuning (fe_autotune) -------------------------------------------
    # -- test hooks of the learned warm start --------------------------------
    def trace_learned(self, slots: int) -> None:
        """Record the network's input rows and outputs of the first `slots`
        solves of every later frame (0: off)."""
        check(self._lib, self._lib.fe_debug_trace_learned(self.handle, slots),
              "fe_debug_trace_learned")

    def read_trace(self, slot: int):
        """(rows uint16[n][16], out float32[n][2]) of a solve of the last frame."""
        rows = np.empty((self.count, 16), np.uint16)
        out = np.empty((self.count, 2), np.float32)
        check(self._lib, self._lib.fe_debug_read_trace(
            self.handle, slot, rows.ctypes.data_as(ctypes.c_void_p),
            out.ctypes.data_as(ctypes.c_void_p)), "fe_debug_read_trace")
        return rows, out

    def autotune(self) -> _abi.FeTuneReport:
        r = _abi.FeTuneReport()
        check(self._lib, self._lib.fe_autotune(self.handle, ctypes.byref(r)), "fe_autotune")
        return r

    def tuning(self) -> _abi.FeTuning:
        t = _abi.FeTuning()
        check(self._lib, self._lib.fe_get_tuning(self.handle, ctypes.byref(t)), "fe_get_tuning")
        return t

    def set_tuning(self, t: _abi.FeTuning) -> None:
        check(self._lib, self._lib.fe_set_tuning(self.handle, ctypes.byref(t)), "fe_set_tuning")

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.fe_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CommandBufferBuilder:
    """Stands in for vulkano's AutoCommandBufferBuilder: passes enqueue on
    the context stream as they are 'recorded'."""

    def __init__(self, physics_data: GpuPhysicsData):
        self.data = physics_data

    def execute_and_wait(self) -> None:
        lib = self.data._lib
        check(lib, lib.fe_synchronize(self.data.handle), "fe_synchronize")


class ComputeStep:
    """trait ComputeStep (pipelines/mod.rs:52-76)."""
    _fn = None
    _label = "ComputeStep"

    def __init__(self):
        self._data = None

    def prepare(self, physics_data: GpuPhysicsData, sim_params: _abi.FeParams | None = None):
        self._data = physics_data
        if sim_params is not None:
            physics_data.sync_with_scene(sim_params)
        lib = physics_data._lib
        check(lib, lib.fe_prepare(physics_data.handle), "fe_prepare")

    def execute(self, builder: CommandBufferBuilder) -> None:
        if self._data is None:
            raise RuntimeError(f"{self._label}: call prepare() before execute()")
        lib = self._data._lib
        check(lib, getattr(lib, self._fn)(self._data.handle), self._fn)


def _step(name, fn):
    return type(name, (ComputeStep,), {"_fn": fn, "_label": name})


DensityAlphaPipeline = _step("DensityAlphaPipeline", "fe_density_alpha")
ViscosityPipeline = _step("ViscosityPipeline", "fe_viscosity")
DensitySourceTermPipeline = _step("DensitySourceTermPipeline", "fe_density_source")
PressureForcePipeline = _step("PressureForcePipeline", "fe_pressure_force")
PressureUpdatePipeline = _step("PressureUpdatePipeline", "fe_pressure_update")
PressureIntegrationPipeline = _step("PressureIntegrationPipeline", "fe_pressure_integration")
DivergenceSourceTermPipeline = _step("DivergenceSourceTermPipeline", "fe_divergence_source")
DivergenceIntegrationPipeline = _step("DivergenceIntegrationPipeline",
                                      "fe_divergence_integration")
StatsPipeline = _step("StatsPipeline", "fe_stats_pass")


class NeighborSearch(ComputeStep):
    """neighbor_search.rs:31-231; `sort_algorithm` as the reference field."""
    _fn = "fe_neighbor_search"
    _label = "NeighborSearch"

    def __init__(self):
        super().__init__()
        self.sort_algorithm = _abi.FE_SORT_BITONIC      # neighbor_search.rs:99

    def execute(self, builder: CommandBufferBuilder) -> None:
        if self._data is None:
            raise RuntimeError("NeighborSearch: call prepare() before execute()")
        if self._data.params.sort_algorithm != self.sort_algorithm:
            p = _abi.copy_params(self._data.params)
            p.sort_algorithm = self.sort_algorithm
            self._data.sync_with_scene(p)
        super().execute(builder)


class ComputePipelines:
    """pipelines/mod.rs:78-124 (density_texture is render-side, not built)."""

    def __init__(self):
        self.neighbor_search = NeighborSearch()
        self.density_alpha = DensityAlphaPipeline()
        self.viscosity = ViscosityPipeline()
        self.density_source_term = DensitySourceTermPipeline()
        self.pressure_force = PressureForcePipeline()
        self.pressure_update = PressureUpdatePipeline()
        self.pressure_integration = PressureIntegrationPipeline()
        self.divergence_source_term = DivergenceSourceTermPipeline()
        self.divergence_integration = DivergenceIntegrationPipeline()
        self.stats = StatsPipeline()

    def passes(self):
        return [self.neighbor_search, self.density_alpha, self.viscosity,
                self.density_source_term, self.pressure_force, self.pressure_update,
                self.pressure_integration, self.divergence_source_term,
                self.divergence_integration, self.stats]

    def prepare_all(self, physics_data: GpuPhysicsData, sim_params=None) -> None:
        """prepare_all_pipelines (convergence_benchmark.rs:85-99)."""
        for p in self.passes():
            p.prepare(physics_data, sim_params)
        self.neighbor_search.sort_algorithm = physics_data.params.sort_algorithm

    def submit_substeps(self, builder, iter_count: int, n_substeps: int, is_first_call: bool):
        """submit_substeps (convergence_benchmark.rs:108-163), pass by pass."""
        if is_first_call:
            self.neighbor_search.execute(builder)
            self.density_alpha.execute(builder)
        for _ in range(n_substeps):
            self.viscosity.execute(builder)
            self.density_source_term.execute(builder)
            for _ in range(iter_count):
                self.pressure_force.execute(builder)
                self.pressure_update.execute(builder)
            self.pressure_integration.execute(builder)
            self.neighbor_search.execute(builder)
            self.density_alpha.execute(builder)
            self.divergence_source_term.execute(builder)
            for _ in range(iter_count):
                self.pressure_force.execute(builder)
                self.pressure_update.execute(builder)
            self.divergence_integration.execute(builder)
        self.stats.execute(builder)
        builder.execute_and_wait()


class Simulation:
    """The whole frame through fe_step (graph-replayed on the device)."""

    def __init__(self, initial_positions, sim_params, *, velocities=None, device=0,
                 build="parity"):
        self.data = GpuPhysicsData(initial_positions, sim_params, velocities=velocities,
                                   device=device, build=build)
        lib = self.data._lib
        check(lib, lib.fe_prepare(self.data.handle), "fe_prepare")

    def step(self, n_substeps: int = 1, flags: int = 0, want_stats: bool = True):
        lib = self.data._lib
        st = _abi.FeStats() if want_stats else None
        rc = lib.fe_step(self.data.handle, n_substeps, flags,
                         ctypes.byref(st) if want_stats else None)
        check(lib, rc, "fe_step")
        return st

    def close(self):
        self.data.close()


class BatchPhysicsData(GpuPhysicsData):
    """Many independent scenes in one context (fe_batch_create): the
    per-scene GpuPhysicsData of the reference, laid out back to back.
    Fields download and upload as one array over all scenes; `scene(a, s)`
    is scene s's slice of such an array."""

    def __init__(self, scene_positions, scene_params, *, scene_velocities=None, device: int = 0):
        self._lib = load_library()
        pos = [np.ascontiguousarray(p, dtype=np.float32).reshape(-1, 3) for p in scene_positions]
        if len(pos) != len(scene_params) or not pos:
            raise ValueError("one parameter block per scene, at least one scene")
        counts = (ctypes.c_uint32 * len(pos))(*[p.shape[0] for p in pos])
        params = (_abi.FeParams * len(pos))(*[_abi.copy_params(q) for q in scene_params])
        allpos = np.ascontiguousarray(np.concatenate(pos))
        vel = None
        if scene_velocities is not None:
            vel = np.ascontiguousarray(np.concatenate(
                [np.asarray(v, dtype=np.float32).reshape(-1, 3) for v in scene_velocities]))
        self.count = int(allpos.shape[0])
        self.params = _abi.copy_params(scene_params[0])
        h = ctypes.c_void_p()
        st = self._lib.fe_batch_create(params, counts, len(pos),
                                       allpos.ctypes.data_as(ctypes.c_void_p),
                                       None if vel is None else vel.ctypes.data_as(ctypes.c_void_p),
                                       device, ctypes.byref(h))
        check(self._lib, st, "fe_batch_create")
        self.handle = h
        n, t = ctypes.c_uint32(), ctypes.c_uint32()
        check(self._lib, self._lib.fe_get_size(h, ctypes.byref(n), ctypes.byref(t)), "fe_get_size")
        self.table_size = int(t.value)
        ns = len(pos)
        first, cnt = (ctypes.c_uint32 * ns)(), (ctypes.c_uint32 * ns)()
        check(self._lib, self._lib.fe_scene_table(h, first, cnt, ns), "fe_scene_table")
        self.scene_first = np.array(first[:], dtype=np.int64)
        self.scene_count = np.array(cnt[:], dtype=np.int64)

    @property
    def n_scenes(self) -> int:
        return len(self.scene_count)

    def scene(self, array: np.ndarray, s: int) -> np.ndarray:
        a = int(self.scene_first[s])
        return array[a:a + int(self.scene_count[s])]

    def read_scene_stats(self, s: int) -> _abi.FeStats:
        st = _abi.FeStats()
        check(self._lib, self._lib.fe_read_scene_stats(self.handle, s, ctypes.byref(st)),
              "fe_read_scene_stats")
        return st

    def set_scene_params(self, s: int, sim_params: _abi.FeParams) -> None:
        p = _abi.copy_params(sim_params)
        check(self._lib, self._lib.fe_set_scene_params(self.handle, s, ctypes.byref(p)),
              "fe_set_scene_params")

    def scene_params(self, s: int) -> _abi.FeParams:
        p = _abi.FeParams()
        check(self._lib, self._lib.fe_get_scene_params(self.handle, s, ctypes.byref(p)),
              "fe_get_scene_params")
        return p


class BatchSimulation(Simulation):
    """fe_step over a batch: every scene advances one frame per call."""

    def __init__(self, scene_positions, scene_params, *, scene_velocities=None, device=0):
        self.data = BatchPhysicsData(scene_positions, scene_params,
                                     scene_velocities=scene_velocities, device=device)
        lib = self.data._lib
        check(lib, lib.fe_prepare(self.data.handle), "fe_prepare")


def sort_pairs_host(keys, values, key_bits: int = 32, algorithm: int = _abi.FE_SORT_RADIX):
    """fe_sort_pairs_host on copies of the arrays."""
    lib = load_library()
    k = np.ascontiguousarray(keys, dtype=np.uint32).copy()
    v = np.ascontiguousarray(values, dtype=np.uint32).copy()
    check(lib, lib.fe_sort_pairs_host(k.ctypes.data_as(ctypes.c_void_p),
                                      v.ctypes.data_as(ctypes.c_void_p), k.size, key_bits,
                                      algorithm), "fe_sort_pairs_host")
    return k, v
