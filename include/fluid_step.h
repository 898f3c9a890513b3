/*
 * fluid_step.h — C ABI of the B200-native DFSPH physics step.
 *
 * This header is the drop-in boundary for the compute half of a Fluid-Engine
 * frame.  The reference drives its physics through the Rust trait
 * `ComputeStep { load_shader_module, from_pipeline, new, prepare, execute }`
 * (src/renderer/pipelines/mod.rs:52-76) and the `ComputePipelines` registry
 * (src/renderer/pipelines/mod.rs:78-124); buffers live in `GpuPhysicsData`
 * (src/entities/particle.rs:137-308) and parameters in the std140 UBO
 * `SimulationParams` (src/entities/particle.rs:310-331).  Every entry point
 * below names the reference item it replaces.
 *
 * Conventions
 *   - Plain C: pointers, sizes and POD structs only.  No C++ or torch types.
 *   - Every call returns an fe_status and never aborts the process; the
 *     reference panics instead (e.g. "call prepare() before execute()",
 *     density_alpha.rs:57), which maps to FE_ERR_NOT_PREPARED here.
 *   - The library owns all device memory of a context.  Host arrays passed in
 *     are copied; host arrays passed out are written by the call.
 *   - Calls on a context enqueue work on that context's CUDA stream, in call
 *     order, exactly like recording into the reference's command buffer.
 *     fe_synchronize() waits for it (the reference's fence wait).
 *   - One context per host thread.  Contexts are independent.
 */
#ifndef FLUID_STEP_H
#define FLUID_STEP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define FE_API __attribute__((visibility("default")))
#else
#define FE_API
#endif

#define FE_ABI_VERSION 2u

/* ------------------------------------------------------------------------- */
/* Status codes                                                              */
/* ------------------------------------------------------------------------- */
typedef enum fe_status {
    FE_OK = 0,
    FE_ERR_INVALID_ARGUMENT = 1, /* bad pointer, size, enum or parameter   */
    FE_ERR_NOT_PREPARED = 2,     /* execute before prepare                 */
    FE_ERR_CUDA = 3,             /* a CUDA runtime call failed             */
    FE_ERR_OUT_OF_MEMORY = 4,    /* device allocation failed               */
    FE_ERR_NON_FINITE = 5,       /* NaN/Inf found in an input or the state */
    FE_ERR_ITERATION_CAP = 6,    /* a tolerance solve hit max_iterations   */
    FE_ERR_TIMEOUT = 7,          /* a bounded device-side wait gave up     */
    FE_ERR_NO_DEVICE = 8,        /* no CUDA device / wrong architecture    */
    FE_ERR_CAPACITY = 9,         /* a size exceeds a documented maximum    */
    FE_ERR_UNSUPPORTED = 10      /* combination of options not supported   */
} fe_status;

/* Sort choice; same order as `enum SortAlgorithm { Bitonic, Radix }`
 * (src/renderer/pipelines/sorter.rs:19-23). */
typedef enum fe_sort_algorithm {
    FE_SORT_BITONIC = 0,
    FE_SORT_RADIX = 1
} fe_sort_algorithm;

/* Buffer pairing of the substep.
 * FE_MODE_REFERENCE reproduces the reference's bindings exactly, including
 * divergence_source_term / divergence_integration reading `velocity_a` in
 * the previous sort order (divergence_source_term.rs:47,
 * divergence_integration.rs:49-50).
 * FE_MODE_FIXED pairs every velocity with its own particle: the divergence
 * pass reads and corrects `velocity_b` (the re-sorted copy), and pressures
 * are carried through the re-sort. */
typedef enum fe_mode {
    FE_MODE_REFERENCE = 0,
    FE_MODE_FIXED = 1
} fe_mode;

/* Jacobi iteration control.
 * FE_SOLVER_FIXED_ITERS runs density/divergence_solver_iterations (or the
 * early-exit choice of renderer/mod.rs:247-265 when
 * use_solver_error_threshold is set), as the reference does.
 * FE_SOLVER_TOLERANCE iterates on the GPU until the FP64 average predicted
 * density error (resp. divergence error) is within tolerance, with
 * min_iterations..max_iterations bounds.  No reference counterpart. */
typedef enum fe_solver {
    FE_SOLVER_FIXED_ITERS = 0,
    FE_SOLVER_TOLERANCE = 1
} fe_solver;

/* Initial pressure of each solve. */
typedef enum fe_warm_start {
    FE_WARM_REFERENCE = 0, /* density solve from 0, divergence solve from the
                              density solve's pressures (as the reference) */
    FE_WARM_LEARNED = 1    /* both solves start from the learned MLP κ    */
} fe_warm_start;

/* ------------------------------------------------------------------------- */
/* Parameters                                                                */
/* ------------------------------------------------------------------------- */
/* The first block mirrors `SimulationParams` field for field
 * (src/entities/particle.rs:310-331, shaders/include/common.glsl:11-28);
 * the padding and the w lanes of the vec4s are dropped.  The second block
 * mirrors the frame-driver knobs of `AppUI` (src/renderer/ui.rs:12-49) and
 * the CFL constants of renderer/mod.rs:238-245.  The third block holds this
 * library's extensions. */
typedef struct fe_params {
    /* SimulationParams */
    float particle_radius;
    float particle_mass;
    float smoothing_radius;
    float target_density;
    float viscosity;
    float relax_factor;
    float dt;
    uint32_t density_solver_iterations;
    uint32_t divergence_solver_iterations;
    float gravity[3];
    float box_min[3];
    float box_max[3];
    int32_t grid_res[3];
    /* AppUI / frame driver */
    uint32_t sort_algorithm;             /* fe_sort_algorithm                  */
    uint32_t use_cfl;                    /* adaptive dt from previous v_max     */
    uint32_t use_solver_error_threshold; /* early exit: 2 / 1 iterations        */
    float density_error_pct;             /* η  in % of ρ0 (ui.rs:41, 0.1)       */
    float divergence_error_pct;          /* ηv in % of ρ0 (ui.rs:42, 0.5)       */
    float cfl_lambda;                    /* 0.4   (mod.rs:240)                  */
    float cfl_min_dt;                    /* 0.001 (mod.rs:240)                  */
    float cfl_max_dt;                    /* 0.05  (mod.rs:240)                  */
    float cfl_growth;                    /* 1.1   (mod.rs:242)                  */
    /* extensions */
    uint32_t mode;                       /* fe_mode                             */
    uint32_t solver;                     /* fe_solver                           */
    float density_tolerance;             /* fraction of ρ0, e.g. 0.001 = 0.1 %  */
    float divergence_tolerance;          /* fraction of ρ0 per dt               */
    uint32_t min_iterations;             /* tolerance solver lower bound (2)    */
    uint32_t max_iterations;             /* tolerance solver cap (100)          */
    uint32_t warm_start;                 /* fe_warm_start                       */
    uint32_t reserved[7];                /* must be zero                        */
} fe_params;

/* Per-frame statistics.  The first three words are the reference's
 * fixed-point `stats_buffer` (stats.comp:8,14-29); the decoded floats follow
 * renderer/mod.rs:231-236; the FP64 means and solver counters are
 * extensions. */
typedef struct fe_stats {
    uint32_t max_speed_bits;        /* atomicMax of floatBitsToUint(|v|)    */
    uint32_t density_error_fp;      /* Σ min(uint(|ρ-ρ0|·1), 10000)         */
    uint32_t divergence_error_fp;   /* Σ min(uint(|s|·10), 10000)           */
    uint32_t substeps;              /* substeps run by the last fe_step      */
    float max_speed;                /* from max_speed_bits                   */
    float avg_density_error;        /* density_error_fp / (1 · N)            */
    float avg_divergence_error;     /* divergence_error_fp / (10 · N)        */
    float dt;                       /* dt used by the last substep           */
    double avg_density_error_f64;   /* mean |ρ-ρ0| in FP64                   */
    double avg_divergence_error_f64;/* mean |s| in FP64                      */
    double density_residual;        /* tolerance metric at exit, last solve  */
    double divergence_residual;     /* (fraction of ρ0)                      */
    uint32_t density_iterations;    /* Jacobi iterations of the last substep */
    uint32_t divergence_iterations;
    uint64_t total_density_iterations;
    uint64_t total_divergence_iterations;
    uint32_t flags;                 /* FE_STATS_* bits                        */
    uint32_t reserved;
    double density_residual_max;    /* largest per-particle error at exit,   */
    double divergence_residual_max; /* same units as the residuals above      */
} fe_stats;

#define FE_STATS_ITERATION_CAP_HIT   0x1u /* a tolerance solve hit the cap   */
#define FE_STATS_NEIGHBOR_OVERFLOW   0x2u /* some particle exceeded the list */
#define FE_STATS_LOOKBACK_TIMEOUT    0x4u /* a bounded device wait gave up   */
#define FE_STATS_NON_FINITE          0x8u /* NaN/Inf seen by the stats pass  */

/* Fields addressable by fe_upload / fe_download.  Names follow
 * `GpuPhysicsData` (particle.rs:137-161).  Vector fields travel as 4 floats
 * per particle (x, y, z, w) like the reference's vec4 buffers. */
typedef enum fe_field {
    FE_FIELD_POSITION_A = 0,    /* float4[N]                                 */
    FE_FIELD_POSITION_B = 1,    /* float4[N] (sorted copy; w reads as 1)     */
    FE_FIELD_VELOCITY_A = 2,    /* float4[N]                                 */
    FE_FIELD_VELOCITY_B = 3,    /* float4[N]                                 */
    FE_FIELD_DENSITY = 4,       /* float[N]                                  */
    FE_FIELD_FACTOR = 5,        /* float[N]  (α)                             */
    FE_FIELD_SOURCE_TERM = 6,   /* float[N]                                  */
    FE_FIELD_PRESSURE = 7,      /* float[N]  (κ)                             */
    FE_FIELD_PRESSURE_ACCEL = 8,/* float4[N]                                 */
    FE_FIELD_ENTRY_HASH = 9,    /* uint32[T] grid_entries[].hash             */
    FE_FIELD_ENTRY_INDEX = 10,  /* uint32[T] grid_entries[].index            */
    FE_FIELD_GRID_START = 11,   /* uint32[T]                                 */
    FE_FIELD_STATS = 12,        /* uint32[3] stats_buffer                    */
    FE_FIELD_DENSITY_GRID = 13, /* uint32[res_z][res_y][res_x] of the last
                                   fe_density_splat (download only)          */
    FE_FIELD_IMAGE = 14,        /* float4[height][width] RGBA of the last
                                   fe_raymarch (download only)               */
    FE_FIELD_COUNT = 15
} fe_field;

/* Step flags for fe_step. */
#define FE_STEP_INIT_NS      0x1u /* neighbour search + density/α first
                                     (convergence_benchmark.rs:121-124)     */
#define FE_STEP_NO_GRAPH     0x2u /* launch eagerly instead of via a graph  */

typedef struct fe_ctx fe_ctx;

/* ------------------------------------------------------------------------- */
/* Library                                                                   */
/* ------------------------------------------------------------------------- */
/* ABI version of the loaded library (FE_ABI_VERSION). */
FE_API uint32_t fe_abi_version(void);

/* Text of a status code.  Static storage. */
FE_API const char* fe_status_string(fe_status status);

/* Last error message recorded on this host thread (empty if none). */
FE_API const char* fe_last_error(void);

/* Defaults of `Scene::new()` (src/core/scene.rs:14-86) and `AppUI::new()`
 * (src/renderer/ui.rs:31-49), plus the extension defaults. */
FE_API void fe_default_params(fe_params* out);

/* Validates a parameter block (finite values, h > 0, mass > 0, box_min <
 * box_max, iteration bounds, enums).  The reference has no validation. */
FE_API fe_status fe_validate_params(const fe_params* params);

/* ------------------------------------------------------------------------- */
/* Context = GpuPhysicsData + ComputePipelines                               */
/* ------------------------------------------------------------------------- */
/* Creates the device buffers of `GpuPhysicsData::new` (particle.rs:164-299)
 * for n particles on CUDA device `device`: positions from pos_xyz (3 floats
 * per particle, w set to 1), velocities from vel_xyz (may be NULL: zero, as
 * particle.rs:193-204), hash table of T = next_pow2(n) (particle.rs:255).
 * n must be in 1..FE_MAX_PARTICLES. */
#define FE_MAX_PARTICLES (1u << 26)
FE_API fe_status fe_create(const fe_params* params, uint32_t n, const float* pos_xyz,
                    const float* vel_xyz, int device, fe_ctx** out);

/* Batched scenes: one context over n_scenes independent scenes of uneven
 * particle counts, advanced together by every stage launch and every
 * fe_step (one CUDA graph for all of them).  The reference runs one scene
 * per `GpuPhysicsData` (particle.rs:137-308); this replaces n_scenes of
 * them.  params[n_scenes] and counts[n_scenes] are per scene; pos_xyz and
 * vel_xyz hold the scenes back to back (scene s starts at particle
 * first_s = counts[0] + ... + counts[s-1]), and every field of
 * fe_upload/fe_download uses the same layout.  Scenes are independent: each
 * gets the result it would get in a context of its own, bit for bit.  All
 * scenes must share sort_algorithm (FE_SORT_RADIX when n_scenes > 1), mode
 * and warm_start; physics, dt, adaptive CFL, solver and tolerances are per
 * scene.  Sum of counts <= FE_MAX_PARTICLES. */
#define FE_MAX_SCENES 65536u
FE_API fe_status fe_batch_create(const fe_params* params, const uint32_t* counts,
                                 uint32_t n_scenes, const float* pos_xyz,
                                 const float* vel_xyz, int device, fe_ctx** out);
/* Number of scenes (1 for fe_create), and each scene's first particle and
 * particle count (arrays of at least `capacity` entries). */
FE_API fe_status fe_scene_count(const fe_ctx* ctx, uint32_t* out);
FE_API fe_status fe_scene_table(const fe_ctx* ctx, uint32_t* first, uint32_t* count,
                                uint32_t capacity);

/* Frees everything owned by ctx.  NULL is accepted. */
FE_API fe_status fe_destroy(fe_ctx* ctx);

/* `Resources::sync_with_scene` (src/renderer/resources.rs:85-92): replaces
 * the parameter block used by later calls. */
FE_API fe_status fe_set_params(fe_ctx* ctx, const fe_params* params);
FE_API fe_status fe_get_params(const fe_ctx* ctx, fe_params* out);
/* The same for one scene of a batch (fe_set_params sets every scene;
 * fe_get_params reads scene 0). */
FE_API fe_status fe_set_scene_params(fe_ctx* ctx, uint32_t scene, const fe_params* params);
FE_API fe_status fe_get_scene_params(const fe_ctx* ctx, uint32_t scene, fe_params* out);

/* `ComputeStep::prepare` for all passes (renderer/mod.rs:137-192): binds
 * buffers and sizes launches.  Must precede the stage calls and fe_step. */
FE_API fe_status fe_prepare(fe_ctx* ctx);

/* Particle count N and table size T of the context. */
FE_API fe_status fe_get_size(const fe_ctx* ctx, uint32_t* n, uint32_t* table_size);

/* CUDA stream of the context (cudaStream_t as void*). */
FE_API void* fe_get_stream(fe_ctx* ctx);

/* Waits for all work enqueued on the context (the reference's fence wait,
 * convergence_benchmark.rs:156-162). */
FE_API fe_status fe_synchronize(fe_ctx* ctx);

/* Copies a field between host memory and the context (bytes = element count
 * of the field × element size, see fe_field).  Enqueued on the context's
 * stream; download completes before returning. */
FE_API fe_status fe_upload(fe_ctx* ctx, fe_field field, const void* src, size_t bytes);
FE_API fe_status fe_download(fe_ctx* ctx, fe_field field, void* dst, size_t bytes);
/* Download without waiting (the render copy of `Renderer::step`,
 * renderer/mod.rs:347-355, moved off the frame's critical path).  The field
 * is snapshotted on the device in the context's stream order, so fe_step
 * calls made right after see no change, and copied to `dst` on a second
 * stream while later work runs; *ticket identifies the copy.  `dst` must stay
 * valid, and should be page-locked (cudaHostAlloc, cudaHostRegister) for the
 * copy to overlap; it holds the field, with the reference's w as fe_download
 * gives it, once fe_download_wait(ticket) returns.  Two snapshots rotate:
 * a third fe_download_async waits, on the device, for the copy of the first.
 * The first call on a context allocates its two device snapshots and a copy
 * stream (and a larger field later reallocates them): make it at start-up. */
FE_API fe_status fe_download_async(fe_ctx* ctx, fe_field field, void* dst, size_t bytes,
                                   uint64_t* ticket);
FE_API fe_status fe_download_wait(fe_ctx* ctx, uint64_t ticket);

/* ------------------------------------------------------------------------- */
/* Stage entry points: one per `ComputeStep::execute`                         */
/* ------------------------------------------------------------------------- */
/* NeighborSearch::execute (neighbor_search.rs:176-231): spatial_hash.comp,
 * sort (radix or bitonic per params.sort_algorithm), fill(grid_start,
 * 0xFFFFFFFF), grid_offsets.comp, reorder.comp. */
FE_API fe_status fe_neighbor_search(fe_ctx* ctx);
/* DensityAlphaPipeline::execute (density_alpha.rs:56-63; density_and_alpha.comp) */
FE_API fe_status fe_density_alpha(fe_ctx* ctx);
/* ViscosityPipeline::execute (viscosity.rs:56-64; viscosity.comp) */
FE_API fe_status fe_viscosity(fe_ctx* ctx);
/* DensitySourceTermPipeline::execute (density_source_term.rs:53-62) */
FE_API fe_status fe_density_source(fe_ctx* ctx);
/* PressureForcePipeline::execute (pressure_force_pipeline.rs:56-64) */
FE_API fe_status fe_pressure_force(fe_ctx* ctx);
/* PressureUpdatePipeline::execute (pressure_update_pipeline.rs:60-69) */
FE_API fe_status fe_pressure_update(fe_ctx* ctx);
/* PressureIntegrationPipeline::execute (pressure_integration_pipeline.rs:56-65) */
FE_API fe_status fe_pressure_integration(fe_ctx* ctx);
/* DivergenceSourceTermPipeline::execute (divergence_source_term.rs:51-60) */
FE_API fe_status fe_divergence_source(fe_ctx* ctx);
/* DivergenceIntegrationPipeline::execute (divergence_integration.rs:56-64) */
FE_API fe_status fe_divergence_integration(fe_ctx* ctx);
/* StatsPipeline::execute (stats_pipeline.rs:54-66): fill(0) + stats.comp. */
FE_API fe_status fe_stats_pass(fe_ctx* ctx);

/* DensityTexturePipeline::execute after its clear_color_image
 * (renderer/mod.rs:385-390; density_texture.rs:29-77; splat_density.comp):
 * clears the context's headless uint32 voxel grid of params.grid_res and
 * splats position_a into it, exactly (integer weights, order-independent
 * sums).  The reference's R32_UINT 3D image becomes a device buffer read with
 * fe_download(FE_FIELD_DENSITY_GRID).  Enqueued on the context's stream;
 * single-scene contexts only; grid_res in 1..1024 per axis. */
FE_API fe_status fe_density_splat(fe_ctx* ctx);

/* The water pass (water_pipeline.rs, entities/water.rs:136-152,
 * raymarch.vert/.frag) without a graphics API: one ray per pixel through the
 * last fe_density_splat grid, into the context's RGBA32F image (read with
 * fe_download(FE_FIELD_IMAGE)).  Pixels the shader discards get alpha 0.
 * The box is params.box_min/box_max (the water model's bounds); the sky is an
 * equirectangular RGBA32F image [height][width] (row 0 at v = 0), sampled
 * bilinearly with clamp-to-edge like the skybox sampler (water.rs:78-84).
 * inv_view_proj is column-major (GLSL mat4 layout) and maps Vulkan NDC
 * (y down, depth 0..1) to world space; a pixel's ray runs from camera_pos
 * through the far-plane point of its centre. */
typedef struct fe_camera {
    float inv_view_proj[16];
    float camera_pos[3];
    uint32_t width;
    uint32_t height;
    uint32_t reserved[3];
} fe_camera;
FE_API fe_status fe_set_skybox(fe_ctx* ctx, const float* rgba, uint32_t width, uint32_t height);
FE_API fe_status fe_raymarch(fe_ctx* ctx, const fe_camera* camera);

/* Reads the stats of the last stats pass (host read of `stats_buffer`,
 * renderer/mod.rs:231-236).  Synchronises the context's stream. */
FE_API fe_status fe_read_stats(fe_ctx* ctx, fe_stats* out);
/* The same read without waiting.  The stats of the last stats pass (scene 0)
 * are captured on the device in the context's stream order, into
 * page-locked host memory the library owns, so fe_step calls made right
 * after run at once; fe_stats_wait(ticket) waits for the capture and fills
 * `out` (with the same FE_ERR_TIMEOUT / FE_ERR_NON_FINITE results as
 * fe_step).  A host loop can so read frame k's stats while frame k+1 runs
 * (the device keeps dt itself under adaptive CFL).  Two captures rotate: a
 * ticket can be waited for until the capture two after it starts.  The first
 * call on a context allocates the page-locked capture memory. */
FE_API fe_status fe_read_stats_async(fe_ctx* ctx, uint64_t* ticket);
FE_API fe_status fe_stats_wait(fe_ctx* ctx, uint64_t ticket, fe_stats* out);
/* The stats of one scene of a batch (fe_read_stats reads scene 0).  The
 * FE_STATS_ITERATION_CAP_HIT and look-back flags are shared by all scenes. */
FE_API fe_status fe_read_scene_stats(fe_ctx* ctx, uint32_t scene, fe_stats* out);

/* ------------------------------------------------------------------------- */
/* Checkpoint / resume                                                       */
/* ------------------------------------------------------------------------- */
/* The reference keeps its state in GpuPhysicsData's buffers
 * (particle.rs:137-308) and has no checkpoint; these entry points snapshot
 * everything a later fe_step reads, so that a context restored from a
 * snapshot continues bit for bit as the original would have:
 *   a versioned header (magic "FESTATE", FE_STATE_VERSION, ABI version,
 *   particle and table sizes, scene count, struct sizes), the parameter
 *   block of every scene, the device-side scene parameters (dt as adaptive
 *   CFL last set it) and solver state (stats, iteration totals, last
 *   residuals), and the per-particle arrays: position_a/b, velocity_a/b,
 *   pressure acceleration, density, factor, source term, pressure, the grid
 *   entries and cell starts, and the learned warm start's carried
 *   pressures when the context has them.
 * The snapshot is host memory in native byte order.  The neighbour list is
 * not part of it: the import rebuilds it with the density pass that built it
 * last, on the restored positions and cell table.
 * fe_state_size: bytes of a snapshot of this context.
 * fe_state_export: writes it; `bytes` must be at least fe_state_size.
 * fe_state_import: restores one into a context with the same particle count,
 *   table size and scene layout (FE_ERR_INVALID_ARGUMENT otherwise, and for a
 *   damaged header or a short buffer; the context is then unchanged).
 *   Recorded frame graphs are dropped.  An attached model stays attached. */
#define FE_STATE_VERSION 3u
FE_API fe_status fe_state_size(const fe_ctx* ctx, size_t* bytes);
FE_API fe_status fe_state_export(fe_ctx* ctx, void* dst, size_t bytes);
FE_API fe_status fe_state_import(fe_ctx* ctx, const void* src, size_t bytes);

/* ------------------------------------------------------------------------- */
/* Test hooks                                                                */
/* ------------------------------------------------------------------------- */
/* The reference has no failure handling (it panics, density_alpha.rs:57,
 * sorter.rs:57-60); these hooks let tests drive this library's error paths
 * without faulting a GPU.  They are process-wide and not thread-safe with
 * respect to concurrent context creation.
 * fe_debug_fail_allocation(k): the k-th device allocation of a context
 *   (fe_create, fe_batch_create and the buffers contexts add later) from now
 *   on fails with FE_ERR_OUT_OF_MEMORY; 0 turns the hook off.
 * fe_debug_poison_allocations(on): new context allocations are filled with
 *   0xFF bytes (NaN as floats, 0xFFFFFFFF as indices), so that a read of
 *   memory no pass has written shows up in the results.
 * fe_debug_bounded_wait(device, limit, flags): runs one look-back wait of
 *   the radix pass on a status word that is never published, giving up
 *   after `limit` polls; returns FE_ERR_TIMEOUT with FE_STATS_LOOKBACK_TIMEOUT
 *   in *flags, and the device stays usable. */
FE_API void fe_debug_fail_allocation(uint32_t k);
FE_API void fe_debug_poison_allocations(int on);
FE_API fe_status fe_debug_bounded_wait(int device, uint32_t limit, uint32_t* flags);

/* ------------------------------------------------------------------------- */
/* Whole step                                                                */
/* ------------------------------------------------------------------------- */
/* One frame of the physics half of `Renderer::step` (renderer/mod.rs:
 * 227-342) in the headless form of `submit_substeps`
 * (convergence_benchmark.rs:108-163):
 *   [prologue] adaptive CFL dt and early-exit iteration choice from the
 *              previous frame's stats (mod.rs:231-265), on the device;
 *   [init]     neighbour search + density/α if FE_STEP_INIT_NS or first call;
 *   n_substeps × { viscosity, density source, density solve,
 *                  pressure integration, neighbour search, density/α,
 *                  divergence source, divergence solve,
 *                  divergence integration };
 *   stats.
 * The frame is replayed from a CUDA graph (conditional WHILE nodes for the
 * tolerance solver) unless FE_STEP_NO_GRAPH.  `out` may be NULL; when given,
 * the call synchronises and fills it. */
FE_API fe_status fe_step(fe_ctx* ctx, uint32_t n_substeps, uint32_t flags, fe_stats* out);

/* ------------------------------------------------------------------------- */
/* Sorting                                                                   */
/* ------------------------------------------------------------------------- */
/* Sorts (key, value) pairs by key in device memory, on `stream`
 * (cudaStream_t as void*, NULL = legacy default stream).  Replaces
 * `RadixSorter::execute` / `GpuSorter::execute` on an Entry buffer
 * (sorter.rs:73-115, 325-454).
 *   FE_SORT_RADIX: stable LSD radix sort, the permutation of
 *     `cpu_radix_sort` (sorter.rs:465-559).  `key_bits` (1..32) bounds the
 *     key range: keys must be < 2^key_bits; 32 sorts any keys.  Digit width
 *     and keys per thread are those fe_autotune_sort chose for this device
 *     and size class, else 8-bit digits and 16 keys per thread; the result
 *     does not depend on them.
 *   FE_SORT_BITONIC: the compare-exchange network of bitonic_sort.comp;
 *     n must be a power of two; not stable (same network, same result as
 *     the reference for the same input).
 * Scratch is allocated on first use per (device, size class) and kept. */
FE_API fe_status fe_sort_pairs(uint32_t* d_keys, uint32_t* d_values, uint32_t n,
                        uint32_t key_bits, int algorithm, void* stream);
/* Error word (FE_STATS_* bits) of the last radix fe_sort_pairs on the
 * current device, copied to *flags_out (host or device memory) in the order
 * of `stream`, after that sort: the value is there once `stream` has reached
 * this point (for host memory, synchronise the stream first).
 * FE_STATS_LOOKBACK_TIMEOUT means a bounded look-back wait of that sort gave
 * up and its output is not valid.  Each radix call clears the word first.
 * No counterpart in the reference (its sort has no failure path). */
FE_API fe_status fe_sort_flags(uint32_t* flags_out, void* stream);

/* ------------------------------------------------------------------------- */
/* Autotuning (no reference counterpart: the reference fixes its workgroup   */
/* sizes and 8-bit digits in the shaders)                                     */
/* ------------------------------------------------------------------------- */
/* Groups of neighbour-loop kernels that share a launch shape. */
#define FE_NBR_DENSITY_ALPHA 0   /* density_alpha: bucket walk, neighbour list */
#define FE_NBR_LIST_PASSES 1     /* viscosity and the density/divergence sources */
#define FE_NBR_PRESSURE_FORCE 2  /* pressure_force (Jacobi A p, first half) */
#define FE_NBR_PRESSURE_UPDATE 3 /* pressure_update (second half, residual sums) */
#define FE_NBR_GROUPS 4

/* Tunable shapes; none of them changes a result.
 *   radix_digit_bits, radix_items: onesweep digit width (8 or 10) and keys
 *     per thread (4, 8, 16; the pairs (8,4) (8,8) (8,16) (10,8) (10,16)).
 *   mlp_ctas_per_sm: blocks per SM of the learned warm start's inference
 *     grid (1..6; at most 4 fit on an SM, larger values act as 4).
 *   nbr_threads[g]: threads per block of neighbour group g, 128, 256 or 512
 *     (a block covers half a 256-particle chunk per pass, one chunk, or two
 *     chunks at a time; particles per thread = 256 / threads per chunk);
 *     FE_NBR_DENSITY_ALPHA 128 or 256 (its per-warp shared scratch),
 *     FE_NBR_PRESSURE_UPDATE 256 only, its FP64 sums being per chunk.  0
 *     means 256.
 *   nbr_persistent[g]: 1 = persistent grid (as many blocks as fit on the
 *     GPU at once, each striding over the chunk table of all scenes); 0 =
 *     one block per chunk (or chunk pair). */
typedef struct fe_tuning {
    uint32_t radix_digit_bits;
    uint32_t radix_items;
    uint32_t mlp_ctas_per_sm;
    uint32_t reserved;
    uint32_t nbr_threads[FE_NBR_GROUPS];
    uint32_t nbr_persistent[FE_NBR_GROUPS];
} fe_tuning;

#define FE_TUNE_MAX_CANDIDATES 8
/* Median CUDA-event time of every candidate (7 timed runs after one
 * untimed), and the choice. */
typedef struct fe_tune_report {
    uint32_t radix_candidates;
    uint32_t radix_digit_bits[FE_TUNE_MAX_CANDIDATES];
    uint32_t radix_items[FE_TUNE_MAX_CANDIDATES];
    float radix_ms[FE_TUNE_MAX_CANDIDATES];
    uint32_t mlp_candidates;                 /* 0: no model attached */
    uint32_t mlp_ctas_per_sm[FE_TUNE_MAX_CANDIDATES];
    float mlp_ms[FE_TUNE_MAX_CANDIDATES];
    /* neighbour kernels (0 candidates before the first neighbour search):
     * the shared candidate list, and per group the median time of each
     * candidate, negative where it is not a candidate of that group */
    uint32_t nbr_candidates;
    uint32_t nbr_threads[FE_TUNE_MAX_CANDIDATES];
    uint32_t nbr_persistent[FE_TUNE_MAX_CANDIDATES];
    float nbr_ms[FE_NBR_GROUPS][FE_TUNE_MAX_CANDIDATES];
    fe_tuning chosen;
} fe_tune_report;

/* Times the candidate shapes on this context's device and data (the sort on
 * the hashes of the current positions; the network on the current feature
 * rows when a model is attached; each neighbour group's kernels on the
 * current state, which is saved to host memory first and restored bit for
 * bit afterwards), applies the fastest and drops the recorded frame graphs.
 * Synchronises the context; allocates temporary device memory.  `report`
 * may be NULL. */
FE_API fe_status fe_autotune(fe_ctx* ctx, fe_tune_report* report);
/* The context's current shapes, and setting them (e.g. from a cache of
 * earlier tuning runs).  FE_ERR_INVALID_ARGUMENT for a shape outside the
 * candidates. */
FE_API fe_status fe_get_tuning(const fe_ctx* ctx, fe_tuning* out);
FE_API fe_status fe_set_tuning(fe_ctx* ctx, const fe_tuning* tuning);
/* Tunes fe_sort_pairs for the current device and the size class of n
 * (ceil(log2 n), key_bits) on the given device arrays, which are not
 * modified; later fe_sort_pairs calls of that class use the choice. */
FE_API fe_status fe_autotune_sort(const uint32_t* d_keys, const uint32_t* d_values, uint32_t n,
                                  uint32_t key_bits, fe_tune_report* report);
/* fe_sort_pairs (radix) with an explicit shape. */
FE_API fe_status fe_sort_pairs_config(uint32_t* d_keys, uint32_t* d_values, uint32_t n,
                                      uint32_t key_bits, uint32_t digit_bits, uint32_t items,
                                      void* stream);

/* Same as fe_sort_pairs with host arrays: copies in, sorts, copies out
 * (in place).  FE_ERR_TIMEOUT when the radix sort's bounded look-back wait
 * gave up (the arrays then hold no valid result). */
FE_API fe_status fe_sort_pairs_host(uint32_t* keys, uint32_t* values, uint32_t n,
                             uint32_t key_bits, int algorithm);

/* ------------------------------------------------------------------------- */
/* Learned warm start (no reference counterpart)                             */
/* ------------------------------------------------------------------------- */
/* A per-particle MLP 12 -> 64 -> 64 -> 2 (SiLU; BF16 weights, FP32
 * accumulation on the tensor cores) maps neighbourhood features to the
 * initial pressure of the density and divergence solves.  Parameter vector
 * (FE_MODEL_PARAMS floats): w1[64][16] (input columns 12..15 unused),
 * w2[64][64], w3[2][64], b1[64], b2[64], b3[2].  Features and targets are
 * standardised with the model's normalisation before the network. */
#define FE_MODEL_PARAMS 5378u
#define FE_MODEL_FEATURES 12u
typedef struct fe_model fe_model;

/* Random initialisation (seeded) on `device`. */
FE_API fe_status fe_model_create(uint32_t seed, int device, fe_model** out);
FE_API fe_status fe_model_destroy(fe_model* model);
FE_API fe_status fe_model_set_parameters(fe_model* model, const float* params, size_t count);
FE_API fe_status fe_model_get_parameters(const fe_model* model, float* params, size_t count);
/* x_mean/x_std: 12 floats; y_mean/y_std: 2 floats. */
FE_API fe_status fe_model_set_normalization(fe_model* model, const float* x_mean,
                                            const float* x_std, const float* y_mean,
                                            const float* y_std);
/* 32 floats: x mean[12], x std[12], y mean[2], y std[2], 4 unused. */
FE_API fe_status fe_model_get_normalization(const fe_model* model, float* out32);
/* d_y[n][2] = model(d_x[n][12]) in target units (device pointers). */
FE_API fe_status fe_model_forward(fe_model* model, const float* d_x, float* d_y, uint32_t n,
                                  void* stream);
/* Gradients of the mean squared error (standardised targets) over the n
 * samples, copied to h_grads (FE_MODEL_PARAMS floats) and the summed squared
 * error to h_loss (either may be NULL).  Synchronous; no update. */
FE_API fe_status fe_model_gradients(fe_model* model, const float* d_x, const float* d_y,
                                    uint32_t n, float* h_grads, float* h_loss);
/* One Adam step (beta 0.9 / 0.999) on the minibatch d_x[n][12], d_y[n][2].
 * When h_loss is given, waits and stores the mean squared error per sample. */
FE_API fe_status fe_model_train_step(fe_model* model, const float* d_x, const float* d_y,
                                     uint32_t n, float lr, float weight_decay, void* stream,
                                     float* h_loss);
/* Device error word of the model's kernels (FE_STATS_* bits). */
FE_API fe_status fe_model_read_flags(fe_model* model, uint32_t* flags);

/* Attaches a model to a context (not owned; NULL detaches).  With
 * params.warm_start = FE_WARM_LEARNED every substep computes the features
 * after density_source, runs the network on the tensor cores, starts the
 * density solve from its first output and the divergence solve from its
 * second; the Jacobi iterations then run as configured. */
FE_API fe_status fe_set_model(fe_ctx* ctx, fe_model* model);

/* Training-data capture from the running solver: each substep, one particle
 * in `stride` (hashed) with a valid Jacobi diagonal records its 12 features
 * and, after both solves, the two converged pressures in normalised units,
 * until `capacity` samples are held. */
FE_API fe_status fe_capture_begin(fe_ctx* ctx, uint32_t capacity, uint32_t stride);
/* Copies up to `rows` samples: x[rows][12], y[rows][2]; *count = samples held. */
FE_API fe_status fe_capture_read(fe_ctx* ctx, float* x, float* y, uint32_t rows, uint32_t* count);
FE_API fe_status fe_capture_end(fe_ctx* ctx);

/* Test hook (no reference counterpart): with slots > 0, every later fe_step
 * of a learned context records, for the first `slots` solves of the frame
 * (slot 2k = the density solve of substep k, 2k + 1 = its divergence solve),
 * the network's input rows as the source passes wrote them and its output
 * as the warm start read it.  0 turns the record off.  Frame graphs are
 * recorded again.  Lets a test check the features against an independent
 * restatement and feed the same network outputs to it. */
FE_API fe_status fe_debug_trace_learned(fe_ctx* ctx, uint32_t slots);
/* Slot `slot` of the last fe_step: rows[n][16] BF16 bit patterns (features
 * 0..11 standardised, 12..15 zero), out[n][2] the network's standardised
 * outputs.  Either may be NULL.  Synchronous. */
FE_API fe_status fe_debug_read_trace(fe_ctx* ctx, uint32_t slot, uint16_t* rows, float* out);

/* Radix sort that allocates nothing.  No counterpart in the reference: it is
 * for callers that cannot let a library allocate device memory — a frame
 * loop that must not stall (cudaMalloc/cudaFree synchronise the device), or
 * a host that budgets all device memory itself.
 * Same result as fe_sort_pairs with FE_SORT_RADIX.  Its scratch is a static
 * device array of about 9 MiB that every GPU loading the library holds until
 * the process exits; n above FE_SORT_NOALLOC_MAX_PAIRS returns
 * FE_ERR_CAPACITY.  The first call in a device's CUDA context looks up the
 * array's device address (make that first call before any stream capture;
 * after a device reset the next call looks it up again).  All calls share
 * the array, so calls that overlap on the GPU (concurrent streams, devices
 * excepted) race.  Unlike fe_sort_pairs, which orders its callers through an
 * event, this entry point does no ordering across streams: serialise calls
 * on one stream, or order calls on different streams yourself (for example
 * with cudaEventRecord / cudaStreamWaitEvent).  keys and values are device
 * pointers of the current device; work is enqueued on `stream`. */
#define FE_SORT_NOALLOC_MAX_PAIRS (1u << 20)
FE_API fe_status fe_sort_pairs_noalloc(uint32_t* d_keys, uint32_t* d_values, uint32_t n,
                                       uint32_t key_bits, void* stream);
/* Error word (FE_STATS_* bits) of the last fe_sort_pairs_noalloc call on the
 * current device, copied from the static array to *flags_out (host or device
 * memory) in the order of `stream`; for host memory, synchronise the stream
 * before reading it.  FE_STATS_LOOKBACK_TIMEOUT means that call's bounded
 * look-back wait gave up and its output is not valid.  Each call clears the
 * word first; allocates nothing.  No counterpart in the reference. */
FE_API fe_status fe_sort_noalloc_flags(uint32_t* flags_out, void* stream);
/* Test hook: runs the radix pass's bounded look-back wait, on `stream`, on a
 * word of the static array that nothing publishes, so that it gives up after
 * `limit` polls and raises FE_STATS_LOOKBACK_TIMEOUT in the error word that
 * fe_sort_noalloc_flags reports.  No GPU fault is involved. */
FE_API fe_status fe_debug_noalloc_wait_timeout(uint32_t limit, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FLUID_STEP_H */
