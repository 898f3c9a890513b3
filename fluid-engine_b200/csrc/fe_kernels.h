// fe_kernels.h — declarations of the DFSPH kernels (fe_kernels.cu) and the
// sort (fe_sort.cu) for the host driver.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "fe_device.h"

namespace fe {

// The neighbour kernels are templates over their block size (128, 256 or
// 512 threads) and persistence (a grid of resident blocks striding over the
// chunks, or one block per chunk step; see for_each_particle in
// fe_neighbors.cuh), instantiated for those shapes in fe_kernels.cu.
__global__ void k_fill_u32(uint32_t* p, uint32_t v, size_t count);
__global__ void k_fill_cells(uint2* p, size_t count);
__global__ void k_hash(Bufs B);
__global__ void k_offsets(Bufs B);
__global__ void k_reorder(Bufs B, int carry_pressure);
__global__ void k_reorder_carry(Bufs B, int carry_pressure, LearnArgs L);
__global__ void k_take_pressure(Bufs B);
__global__ void k_take_pressure_carry(Bufs B, LearnArgs L);
__global__ void k_refresh_pr(Bufs B);
template <int kThreads, bool kPersist>
__global__ void k_density_alpha(Bufs B);
template <int kThreads, bool kPersist>
__global__ void k_density_alpha_div(Bufs B, int fixed);
template <int kThreads, bool kPersist>
__global__ void k_density_alpha_div_learn(Bufs B, int fixed, LearnArgs L);
template <int kThreads, bool kPersist>
__global__ void k_viscosity(Bufs B);
// Per-scene finishes of a multi-scene context, one block per scene.
__global__ void k_solve_finish(Bufs B, int which, cudaGraphConditionalHandle handle,
                               int use_handle);
__global__ void k_stats_finish(Bufs B, uint4* upart);
template <int kThreads, bool kPersist>
__global__ void k_density_source(Bufs B);
template <int kThreads, bool kPersist>
__global__ void k_divergence_source(Bufs B, int fixed);
template <int kThreads, bool kPersist>
__global__ void k_pressure_force(Bufs B, int which);
__global__ void k_pressure_update(Bufs B, int which, cudaGraphConditionalHandle handle,
                                  int use_handle);
__global__ void k_solve_begin(Bufs B, int which, cudaGraphConditionalHandle handle,
                              int use_handle);
__global__ void k_solve_end(Bufs B, int which);
__global__ void k_loop_guard(Bufs B, int which, cudaGraphConditionalHandle handle);
__global__ void k_pressure_integration(Bufs B);
__global__ void k_pressure_integration_learn(Bufs B, LearnArgs L);
__global__ void k_divergence_integration(Bufs B, int fixed);
__global__ void k_divergence_integration_learn(Bufs B, int fixed, LearnArgs L);
__global__ void k_stats(Bufs B, int fixed, uint4* upart);
// The last substep's divergence integration with the frame's stats fused in.
__global__ void k_divergence_integration_stats(Bufs B, int fixed, uint4* upart);
__global__ void k_divergence_integration_stats_learn(Bufs B, int fixed, LearnArgs L,
                                                     uint4* upart);
__global__ void k_frame_prologue(Bufs B);
__global__ void k_count_substep(Bufs B);
template <int kThreads, bool kPersist>
__global__ void k_density_source_learn(Bufs B, LearnArgs L);
__global__ void k_carry_take(Bufs B, LearnArgs L);
__global__ void k_stats_snapshot(Bufs B, StatsSnapshot* dst, uint32_t scene);
__global__ void k_snapshot4(float4* dst, const float4* src, uint32_t stride, uint32_t n,
                            int fix_w, float w);

}  // namespace fe
