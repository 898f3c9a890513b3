// fe_splat.h — density splat into a headless voxel grid (fe_splat.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace fe {

constexpr int kSplatRadius = 8;
constexpr int kSplatSide = 2 * kSplatRadius + 1;  // 17 offsets per axis
constexpr int kSplatTile = 8;                     // output tile edge (voxels)

// The integer weight of every voxel offset, [kSplatSide^3] with x fastest.
cudaError_t splat_weights(uint32_t* d_weights, cudaStream_t stream);

// The splat as a convolution: hist[(rz+1)][(ry+1)][(rx+1)] counts the
// particles per centre voxel (centres run 0..res inclusive; cleared by the
// caller), then every grid voxel v gets sum_t weight_t * hist[v - offset_t]
// (exact in integers).  One block per 8^3 output tile reads a 24^3 window of
// the counts into shared memory; windows without particles are skipped (the
// caller cleared the grid).
cudaError_t splat_histogram(const float4* pos, uint32_t n, float3 box_min, float3 box_max,
                            int3 res, uint32_t* hist, cudaStream_t stream);
cudaError_t splat_convolve(const uint32_t* hist, int3 res, const int4* taps, uint32_t n_taps,
                           uint32_t* grid, cudaStream_t stream);

}  // namespace fe
