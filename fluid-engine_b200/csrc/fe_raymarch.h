// fe_raymarch.h — raymarch.frag's shading into a headless RGBA image.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace fe {

struct RaymarchArgs {
    const uint32_t* grid;      // density grid [rz][ry][rx] (fe_density_splat)
    int3 res;
    const float4* sky;         // equirectangular sky [sky_h][sky_w] RGBA
    int sky_w, sky_h;
    float inv_view_proj[16];   // column-major (GLSL mat4 layout)
    float3 cam;
    float3 box_min, box_max;   // sim box (the water model's bounds)
    int width, height;
    float4* out;               // [height][width] RGBA, alpha 0 where the shader discards
};

cudaError_t raymarch(const RaymarchArgs& a, cudaStream_t stream);

}  // namespace fe
