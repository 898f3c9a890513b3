// fe_splat.cu — splat_density.comp:11-51 as a headless voxel grid.
//
// Each particle inside the box adds uint(200 (1 - (d/8)^2)^3) to every voxel
// at integer offset (x, y, z), d = |(x, y, z)| < 8, from its centre voxel
// ivec3(uvw * grid_res), uvw = (p - box_min) / (box_max - box_min).  The
// weight depends only on the offset, so it is evaluated once per offset (in
// the shader's FP32 operation order) into a table of the 1,647 non-zero taps,
// and the grid is the convolution of the per-centre-voxel particle counts with
// that table: grid[v] = sum_t w_t * count[v - d_t].  Integer sums do not
// depend on order, so the grid is bit-identical to the shader's scatter of
// atomic adds.  One block per 8^3 output tile holds a 24^3 window of the
// counts in shared memory; windows with no particle are skipped.  (Scattering
// per particle with global reductions, or accumulating per tile with
// shared-memory atomics, did the same sums 2.4x and 2.7x slower at 1M
// particles on 128^3.)
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

// The centre voxel of a particle, or false outside the box (the shader's
// early return).
__device__ __forceinline__ bool centre_voxel(float4 p, float3 bmin, float3 bmax, int3 res,
                                             int* cx, int* cy, int* cz) {
    const float sx = bmax.x - bmin.x, sy = bmax.y - bmin.y, sz = bmax.z - bmin.z;
    const float u = (p.x - bmin.x) / sx, v = (p.y - bmin.y) / sy, w = (p.z - bmin.z) / sz;
    if (u < 0.0f || v < 0.0f || w < 0.0f || u > 1.0f || v > 1.0f || w > 1.0f) return false;
    *cx = glsl_int(u * (float)res.x);
    *cy = glsl_int(v * (float)res.y);
    *cz = glsl_int(w * (float)res.z);
    return true;
}

constexpr int kWin = kSplatTile + 2 * kSplatRadius;  // 24 voxels per axis
constexpr int kWinVox = kWin * kWin * kWin;          // 13824

__global__ void __launch_bounds__(256) k_splat_hist(const float4* __restrict__ pos, uint32_t n,
                                                    float3 bmin, float3 bmax, int3 res,
                                                    uint32_t* __restrict__ hist) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int cx, cy, cz;
    if (!centre_voxel(__ldg(pos + i), bmin, bmax, res, &cx, &cy, &cz)) return;
    cx = min(max(cx, 0), res.x);
    cy = min(max(cy, 0), res.y);
    cz = min(max(cz, 0), res.z);
    atomicAdd(hist + ((size_t)cz * (res.y + 1) + cy) * (res.x + 1) + cx, 1u);
}

// grid[v] = sum_t w_t * hist[v - d_t] over the taps (offset d_t from a centre
// to a voxel).  Block: 8^3 output voxels, 256 threads, two voxels each (z and
// z + 4); the window holds hist for centres v - d, d in [-8, 8]^3.
__global__ void __launch_bounds__(256) k_splat_conv(const uint32_t* __restrict__ hist, int3 res,
                                                    const int4* __restrict__ taps,
                                                    uint32_t n_taps,
                                                    uint32_t* __restrict__ grid) {
    extern __shared__ uint32_t win[];  // [kWin][kWin][kWin], origin = tile origin - radius
    const int tdx = (res.x + kSplatTile - 1) / kSplatTile, tdy = (res.y + kSplatTile - 1) / kSplatTile;
    const int tx = blockIdx.x % tdx, ty = (blockIdx.x / tdx) % tdy, tz = blockIdx.x / (tdx * tdy);
    const int ox = tx * kSplatTile - kSplatRadius, oy = ty * kSplatTile - kSplatRadius,
              oz = tz * kSplatTile - kSplatRadius;
    const int hx = res.x + 1, hy = res.y + 1, hz = res.z + 1;   // hist extent
    int any = 0;
    for (int v = threadIdx.x; v < kWinVox; v += blockDim.x) {
        const int x = ox + v % kWin, y = oy + (v / kWin) % kWin, z = oz + v / (kWin * kWin);
        uint32_t c = 0u;
        if (x >= 0 && y >= 0 && z >= 0 && x < hx && y < hy && z < hz)
            c = __ldg(hist + ((size_t)z * hy + y) * hx + x);
        win[v] = c;
        any |= c != 0u;
    }
    if (!__syncthreads_or(any)) return;  // no particle within reach: the grid stays 0
    const int lx = threadIdx.x & 7, ly = (threadIdx.x >> 3) & 7, lz = threadIdx.x >> 6;  // lz 0..3
    uint32_t a0 = 0u, a1 = 0u;
    for (uint32_t t = 0; t < n_taps; ++t) {
        const int4 k = __ldg(taps + t);
        // centre = voxel - offset, in window coordinates (+ radius)
        const int wx = lx + kSplatRadius - k.x, wy = ly + kSplatRadius - k.y,
                  wz = lz + kSplatRadius - k.z;
        const uint32_t w = (uint32_t)k.w;
        a0 += w * win[(wz * kWin + wy) * kWin + wx];
        a1 += w * win[((wz + 4) * kWin + wy) * kWin + wx];
    }
    const int x = tx * kSplatTile + lx, y = ty * kSplatTile + ly, z0 = tz * kSplatTile + lz;
    if (x < res.x && y < res.y) {
        if (z0 < res.z) grid[((size_t)z0 * res.y + y) * res.x + x] = a0;
        if (z0 + 4 < res.z) grid[((size_t)(z0 + 4) * res.y + y) * res.x + x] = a1;
    }
}

}  // namespace

cudaError_t splat_histogram(const float4* pos, uint32_t n, float3 box_min, float3 box_max,
                            int3 res, uint32_t* hist, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    k_splat_hist<<<(n + 255) / 256, 256, 0, stream>>>(pos, n, box_min, box_max, res, hist);
    return cudaGetLastError();
}

cudaError_t splat_convolve(const uint32_t* hist, int3 res, const int4* taps, uint32_t n_taps,
                           uint32_t* grid, cudaStream_t stream) {
    const int tdx = (res.x + kSplatTile - 1) / kSplatTile, tdy = (res.y + kSplatTile - 1) / kSplatTile,
              tdz = (res.z + kSplatTile - 1) / kSplatTile;
    const size_t smem = (size_t)kWinVox * 4;
    cudaError_t e = cudaFuncSetAttribute(k_splat_conv, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    k_splat_conv<<<tdx * tdy * tdz, 256, smem, stream>>>(hist, res, taps, n_taps, grid);
    return cudaGetLastError();
}

cudaError_t splat_weights(uint32_t* d_weights, cudaStream_t stream) {
    const int total = kSplatSide * kSplatSide * kSplatSide;
    k_splat_weights<<<(total + 255) / 256, 256, 0, stream>>>(d_weights);
    return cudaGetLastError();
}

}  // namespace fe
