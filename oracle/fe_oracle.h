/*
 * fe_oracle.h — CPU oracle of the DFSPH step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: the parity tests,
 * the smoke check and the CPU-baseline leg of the benchmark call it.  The
 * product (libfluidstep.so) never links, loads or calls it.
 *
 * It restates, line by line, the reference's GLSL compute shaders
 * (the shaders/compute .comp files, shaders/include/common.glsl) and the sequencing
 * of src/renderer/mod.rs:227-342 and
 * src/renderer/pipelines/convergence_benchmark.rs:108-163, on the host:
 *   - FP32 mode: float arithmetic in the shaders' source order, compiled with
 *     -ffp-contract=off (no fused multiply-add), IEEE division and sqrt;
 *   - FP64 mode: the same sequence in double, used to state the true error.
 * Per-particle loops run under OpenMP; they are independent per particle,
 * so the thread count does not change any result.
 */
#ifndef FE_ORACLE_H
#define FE_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/fluid_step.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fo_ctx fo_ctx;

/* GpuPhysicsData::new (particle.rs:164-299) on the host. fp64 != 0 selects
 * the double-precision twin. Returns NULL on bad arguments. */
fo_ctx* fo_create(const fe_params* params, uint32_t n, const float* pos_xyz,
                  const float* vel_xyz, int fp64);
void fo_destroy(fo_ctx* ctx);
int fo_set_params(fo_ctx* ctx, const fe_params* params);
int fo_get_params(const fo_ctx* ctx, fe_params* out);
uint32_t fo_table_size(const fo_ctx* ctx);

/* One call per reference pass (same names as the C ABI). */
int fo_neighbor_search(fo_ctx* ctx);
int fo_density_alpha(fo_ctx* ctx);
int fo_viscosity(fo_ctx* ctx);
int fo_density_source(fo_ctx* ctx);
int fo_pressure_force(fo_ctx* ctx);
int fo_pressure_update(fo_ctx* ctx);
int fo_pressure_integration(fo_ctx* ctx);
int fo_divergence_source(fo_ctx* ctx);
int fo_divergence_integration(fo_ctx* ctx);
int fo_stats_pass(fo_ctx* ctx);
int fo_read_stats(const fo_ctx* ctx, fe_stats* out);

/* One frame; same semantics as fe_step. */
int fo_step(fo_ctx* ctx, uint32_t n_substeps, uint32_t flags, fe_stats* out);

/* Field transfer.  fo_download converts to float for FP64 contexts;
 * fo_download_f64 returns the double values (float fields only). */
int fo_download(const fo_ctx* ctx, int field, void* dst, size_t bytes);
int fo_download_f64(const fo_ctx* ctx, int field, double* dst, size_t count);
int fo_upload(fo_ctx* ctx, int field, const void* src, size_t bytes);

/* Sorts on host arrays.
 * fo_sort_radix_mirror: the reference's own CPU mirror `cpu_radix_sort`
 *   (sorter.rs:465-559): 4 passes of count / 3-phase scan / scatter over
 *   work groups of 256×8 entries.
 * fo_sort_radix_parallel: stable LSD radix, 8-bit digits, ceil(key_bits/8)
 *   passes, OpenMP count and scatter (the timed CPU baseline).
 * fo_sort_bitonic: the bitonic_sort.comp network (sorter.rs:73-115);
 *   n must be a power of two. */
void fo_sort_radix_mirror(uint32_t* keys, uint32_t* values, uint32_t n);
void fo_sort_radix_parallel(uint32_t* keys, uint32_t* values, uint32_t n,
                            uint32_t key_bits);
int fo_sort_bitonic(uint32_t* keys, uint32_t* values, uint32_t n);

/* The fixed-order FP64 reduction the GPU uses for the solver residuals and
 * the FP64 stats: chunks of 256, warp-halving trees, sequential strided
 * partial sums over chunks (see fe_oracle.cpp). */
double fo_det_sum(const double* values, size_t n);

/* splat_density.comp:11-51 on float4 positions pos4[n] into
 * out[grid_res z][y][x] (cleared first). */
void fo_splat_density(const float* pos4, uint32_t n, const fe_params* params, uint32_t* out);

/* raymarch.frag:1-215 for one ray per pixel: the ray from cam_pos through
 * the far-plane point of the pixel centre under the column-major
 * inv_view_proj (Vulkan NDC); grid[rz][ry][rx] the splat; sky4[h][w] RGBA,
 * bilinear clamp-to-edge; out[height][width] RGBA, alpha 0 where the shader
 * discards. */
void fo_raymarch(const uint32_t* grid, int rx, int ry, int rz, const float* sky4, int sky_w,
                 int sky_h, const float* inv_view_proj, const float* cam_pos,
                 const float* box_min, const float* box_max, int width, int height, float* out);

/* Learned warm start (restates the CUDA library's fe_features.cuh and
 * fe_learned.cu; no reference counterpart).  fo_set_learned(norm28) turns
 * it on with the model's standardisation (x mean[12], x std[12], y mean[2],
 * y std[2]); NULL turns it off.  The network is not restated: before each
 * fo_step, fo_set_network_outputs gives its standardised outputs out[slot]
 * [n][2] for the frame's first `slots` solves (slot 2k = density solve of
 * substep k, 2k + 1 = divergence solve); after it, fo_get_feature_rows
 * returns the BF16 rows rows[n][16] the source passes computed for a slot.
 * fo_learned_missing_outputs: the last fo_step reached a solve without
 * given outputs (its start was left as without the network). */
int fo_set_learned(fo_ctx* ctx, const float* norm28);
int fo_set_network_outputs(fo_ctx* ctx, uint32_t slots, const float* out);
int fo_get_feature_rows(const fo_ctx* ctx, uint32_t slot, uint16_t* rows);
int fo_learned_missing_outputs(const fo_ctx* ctx);

int fo_set_threads(int threads);
int fo_get_threads(void);

#ifdef __cplusplus
}
#endif

#endif /* FE_ORACLE_H */
