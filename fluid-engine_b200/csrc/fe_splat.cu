// fe_splat.cu — splat_density.comp:11-51 as a headless voxel grid.
//
// Each particle inside the box adds uint(200 (1 - (d/8)^2)^3) to every voxel
// at integer offset (x, y, z), d = |(x, y, z)| < 8, from its centre voxel
// ivec3(uvw * grid_res), uvw = (p - box_min) / (box_max - box_min).  The
// weight depends only on the offset, so it is evaluated once per offset (in
// the shader's FP32 operation order) into a table of the non-zero taps;
// integer sums do not depend on the order of the additions, so the grid is
// bit-identical to the shader's whatever order the reductions land in.
//
// One warp per particle: lanes take consecutive taps (x fastest, so a warp's
// 32 reductions fall on a few consecutive runs of voxels) and issue
// fire-and-forget red.global.add.u32; the grid (8 MB at 128^3) stays in L2.
#include "fe_splat.h"

#include "fe_common.cuh"

namespace fe {

namespace {

// GLSL uint(x) for the splat's weights, which lie in [0, 200]: truncation.
__device__ __forceinline__ uint32_t glsl_uint(float x) { return __float2uint_rz(x); }
// GLSL int(x) with the conversion convention of the rest of the step:
// truncation, saturating, NaN -> 0 (cvt.rzi).
__device__ __forceinline__ int glsl_int(float x) { return __float2int_rz(x); }

__global__ void k_splat_weights(uint32_t* __restrict__ w) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= kSplatSide * kSplatSide * kSplatSide) return;
    const int x = t % kSplatSide - kSplatRadius;
    const int y = (t / kSplatSide) % kSplatSide - kSplatRadius;
    const int z = t / (kSplatSide * kSplatSide) - kSplatRadius;
    const float r = (float)kSplatRadius;
    const float fx = (float)x, fy = (float)y, fz = (float)z;
    const float dist = sqrtf((fx * fx + fy * fy) + fz * fz);   // length(vec3(x, y, z))
    uint32_t c = 0;
    if (dist < r) {
        const float x_norm = dist / r;
        float weight = 1.0f - x_norm * x_norm;
        weight = (weight * weight) * weight;
        c = glsl_uint(weight * 200.0f);
    }
    w[t] = c;
}

__device__ __forceinline__ void red_add(uint32_t* p, uint32_t v) {
    asm volatile("red.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__global__ void __launch_bounds__(256) k_splat(const float4* __restrict__ pos, uint32_t n,
                                               float3 bmin, float3 bmax, int3 res,
                                               const int4* __restrict__ taps, uint32_t n_taps,
                                               uint32_t* __restrict__ grid) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
        const float4 p = __ldg(pos + i);
        const float sx = bmax.x - bmin.x, sy = bmax.y - bmin.y, sz = bmax.z - bmin.z;
        const float u = (p.x - bmin.x) / sx, v = (p.y - bmin.y) / sy, w = (p.z - bmin.z) / sz;
        // any(lessThan(uvw, 0)) || any(greaterThan(uvw, 1)): NaN passes, as in GLSL
        if (u < 0.0f || v < 0.0f || w < 0.0f || u > 1.0f || v > 1.0f || w > 1.0f) continue;
        const int cx = glsl_int(u * (float)res.x), cy = glsl_int(v * (float)res.y),
                  cz = glsl_int(w * (float)res.z);
        for (uint32_t t = lane; t < n_taps; t += 32) {
            const int4 k = __ldg(taps + t);
            const int x = cx + k.x, y = cy + k.y, z = cz + k.z;
            if (x < 0 || y < 0 || z < 0 || x >= res.x || y >= res.y || z >= res.z) continue;
            red_add(grid + ((size_t)z * res.y + y) * res.x + x, (uint32_t)k.w);
        }
    }
}

}  // namespace

cudaError_t splat_weights(uint32_t* d_weights, cudaStream_t stream) {
    const int total = kSplatSide * kSplatSide * kSplatSide;
    k_splat_weights<<<(total + 255) / 256, 256, 0, stream>>>(d_weights);
    return cudaGetLastError();
}

cudaError_t splat(const float4* pos, uint32_t n, float3 box_min, float3 box_max, int3 res,
                  const int4* taps, uint32_t n_taps, uint32_t* grid, cudaStream_t stream,
                  int num_sms) {
    if (n == 0 || n_taps == 0) return cudaSuccess;
    const uint32_t blocks_needed = (n + 7) / 8;               // 8 warps per block
    const uint32_t cap = (uint32_t)num_sms * 8u;
    const uint32_t blocks = blocks_needed < cap ? blocks_needed : cap;
    k_splat<<<blocks, 256, 0, stream>>>(pos, n, box_min, box_max, res, taps, n_taps, grid);
    return cudaGetLastError();
}

}  // namespace fe
