// fe_splat.h — density splat into a headless voxel grid (fe_splat.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace fe {

constexpr int kSplatRadius = 8;
constexpr int kSplatSide = 2 * kSplatRadius + 1;  // 17 offsets per axis

// The integer weight of every voxel offset, [kSplatSide^3] with x fastest.
cudaError_t splat_weights(uint32_t* d_weights, cudaStream_t stream);

// Adds every particle's splat into grid[res_z][res_y][res_x] (cleared by the
// caller).  taps[n_taps] = {dx, dy, dz, weight} with weight > 0, x fastest.
cudaError_t splat(const float4* pos, uint32_t n, float3 box_min, float3 box_max, int3 res,
                  const int4* taps, uint32_t n_taps, uint32_t* grid, cudaStream_t stream,
                  int num_sms);

}  // namespace fe
