// fe_raymarch.cu — raymarch.frag (shaders/raymarch.frag:1-215) as one thread
// per pixel into a headless RGBA32F image.
//
// The fragment's ray, normalize(inWorldPos - inCameraPos), is the ray from
// the camera through the pixel centre: the point (x_ndc, y_ndc, 1, 1) mapped
// by inv_view_proj (Vulkan NDC, y down).  The box comes from the water
// model matrix of water.rs:136-152 (scale = box size, translation = its
// centre) exactly as the shader rebuilds it (centre -/+ length(column) / 2).
// Densities are nearest texel fetches of the splat grid with the shader's
// manual trilinear blend; the sky is bilinear with clamp-to-edge (the
// skybox sampler of water.rs:78-84).  discard -> alpha 0.
#include "fe_raymarch.h"

namespace fe {

namespace {

struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator/(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
__device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ float dot3(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ float len3(V3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ V3 normalize3(V3 a) {
    const float l = len3(a);
    return {a.x / l, a.y / l, a.z / l};
}
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ V3 mix3(V3 a, V3 b, float t) {
    return {mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t)};
}
__device__ __forceinline__ float clampf(float x, float lo, float hi) {
    return fminf(fmaxf(x, lo), hi);
}
__device__ __forceinline__ float smoothstepf(float e0, float e1, float x) {
    const float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}

constexpr float kThreshold = 0.01f, kOffset = 300.0f, kMultiplier = 1.0f;
constexpr int kMaxSteps = 96;
constexpr float kStepSize = 0.007f;
constexpr float kIorWater = 1.333f, kIorAir = 1.0f;

struct Scene {
    const uint32_t* grid;
    int3 res;
    V3 bmin, bmax;
};

__device__ __forceinline__ float texel(const Scene& S, int x, int y, int z) {
    x = min(max(x, 0), S.res.x - 1);
    y = min(max(y, 0), S.res.y - 1);
    z = min(max(z, 0), S.res.z - 1);
    return (float)__ldg(S.grid + ((size_t)z * S.res.y + y) * S.res.x + x);
}

// getDensity (raymarch.frag:54-74).
__device__ float get_density(const Scene& S, V3 p) {
    const V3 uvw = (p - S.bmin) / (S.bmax - S.bmin);
    if (uvw.x < 0.0f || uvw.y < 0.0f || uvw.z < 0.0f || uvw.x > 1.0f || uvw.y > 1.0f ||
        uvw.z > 1.0f)
        return 0.0f;
    const V3 g = v3(uvw.x * (float)S.res.x - 0.5f, uvw.y * (float)S.res.y - 0.5f,
                    uvw.z * (float)S.res.z - 0.5f);
    const float fx = floorf(g.x), fy = floorf(g.y), fz = floorf(g.z);
    const int ix = __float2int_rz(fx), iy = __float2int_rz(fy), iz = __float2int_rz(fz);
    const float tx = g.x - fx, ty = g.y - fy, tz = g.z - fz;
    const float v000 = texel(S, ix, iy, iz), v100 = texel(S, ix + 1, iy, iz);
    const float v010 = texel(S, ix, iy + 1, iz), v110 = texel(S, ix + 1, iy + 1, iz);
    const float v001 = texel(S, ix, iy, iz + 1), v101 = texel(S, ix + 1, iy, iz + 1);
    const float v011 = texel(S, ix, iy + 1, iz + 1), v111 = texel(S, ix + 1, iy + 1, iz + 1);
    const float v0 = mixf(mixf(v000, v100, tx), mixf(v010, v110, tx), ty);
    const float v1 = mixf(mixf(v001, v101, tx), mixf(v011, v111, tx), ty);
    return fmaxf(0.0f, (mixf(v0, v1, tz) - kOffset) * kMultiplier);
}

__device__ V3 calc_normal(const Scene& S, V3 p) {
    const float e = 0.018f;
    return normalize3(v3(get_density(S, p + v3(e, 0, 0)) - get_density(S, p - v3(e, 0, 0)),
                         get_density(S, p + v3(0, e, 0)) - get_density(S, p - v3(0, e, 0)),
                         get_density(S, p + v3(0, 0, e)) - get_density(S, p - v3(0, 0, e))));
}

__device__ float fresnel(float cos_theta, float f0) {
    return f0 + (1.0f - f0) * powf(clampf(1.0f - cos_theta, 0.0f, 1.0f), 5.0f);
}

__device__ V3 sample_sky(const float4* sky, int w, int h, V3 dir) {
    dir = normalize3(dir);
    const float u = atan2f(dir.z, dir.x) * 0.15915f + 0.5f;
    const float v = asinf(clampf(dir.y, -1.0f, 1.0f)) * 0.31831f + 0.5f;
    // bilinear, clamp to edge, texel centres at (i + 0.5) / size
    const float x = u * (float)w - 0.5f, y = v * (float)h - 0.5f;
    const float x0f = floorf(x), y0f = floorf(y);
    const float ax = x - x0f, ay = y - y0f;
    const int x0 = __float2int_rz(x0f), y0 = __float2int_rz(y0f);
    auto at = [&](int xi, int yi) {
        xi = min(max(xi, 0), w - 1);
        yi = min(max(yi, 0), h - 1);
        const float4 c = __ldg(sky + (size_t)yi * w + xi);
        return v3(c.x, c.y, c.z);
    };
    const V3 c0 = mix3(at(x0, y0), at(x0 + 1, y0), ax);
    const V3 c1 = mix3(at(x0, y0 + 1), at(x0 + 1, y0 + 1), ax);
    return mix3(c0, c1, ay);
}

__device__ float calc_thickness(const Scene& S, V3 p, V3 dir, float t_max) {
    float thickness = 0.0f;
    const float d_step = 0.015f;
    float t = 0.0f;
    for (int i = 0; i < 64 && t < t_max; i++, t += d_step)
        if (get_density(S, p + dir * t) > kThreshold) thickness += d_step;
    return thickness;
}

__device__ float ggx_d(float n_dot_h, float roughness) {
    const float a = roughness * roughness;
    const float a2 = a * a;
    const float d = n_dot_h * n_dot_h * (a2 - 1.0f) + 1.0f;
    return a2 / (3.14159f * d * d);
}

__global__ void __launch_bounds__(128) k_raymarch(RaymarchArgs A) {
    const int px = blockIdx.x * 16 + (threadIdx.x & 15), py = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (px >= A.width || py >= A.height) return;
    float4* out = A.out + (size_t)py * A.width + px;
    // pixel centre on the far plane, back to world space
    const float nx = ((float)px + 0.5f) / (float)A.width * 2.0f - 1.0f;
    const float ny = ((float)py + 0.5f) / (float)A.height * 2.0f - 1.0f;
    const float* M = A.inv_view_proj;
    float w4[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) w4[r] = ((M[r] * nx + M[4 + r] * ny) + M[8 + r] * 1.0f) + M[12 + r] * 1.0f;
    const V3 world = v3(w4[0] / w4[3], w4[1] / w4[3], w4[2] / w4[3]);
    const V3 cam = v3(A.cam.x, A.cam.y, A.cam.z);
    const V3 ray_dir = normalize3(world - cam);
    const V3 ray_org = cam;

    // the water model: scale = size, translation = centre (water.rs:136-146)
    const V3 size = v3(A.box_max.x - A.box_min.x, A.box_max.y - A.box_min.y, A.box_max.z - A.box_min.z);
    const V3 center = v3(A.box_min.x + size.x * 0.5f, A.box_min.y + size.y * 0.5f,
                         A.box_min.z + size.z * 0.5f);
    const V3 scale = v3(sqrtf(size.x * size.x), sqrtf(size.y * size.y), sqrtf(size.z * size.z));
    Scene S{A.grid, A.res, center - scale * 0.5f, center + scale * 0.5f};

    // intersectAABB (raymarch.frag:47-52)
    const V3 t1 = (S.bmin - ray_org) / ray_dir, t2 = (S.bmax - ray_org) / ray_dir;
    const float t_near = fmaxf(fmaxf(fminf(t1.x, t2.x), fminf(t1.y, t2.y)), fminf(t1.z, t2.z));
    const float t_far = fminf(fminf(fmaxf(t1.x, t2.x), fmaxf(t1.y, t2.y)), fmaxf(t1.z, t2.z));
    if (t_near > t_far || t_far < 0.0f) {
        *out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    const float step_world = kStepSize * fmaxf(fmaxf(scale.x, scale.y), scale.z);
    float t_cur = fmaxf(t_near, 0.0f);
    bool hit = false;
    for (int i = 0; i < kMaxSteps; i++) {
        if (t_cur > t_far) break;
        if (get_density(S, ray_org + ray_dir * t_cur) > kThreshold) {
            hit = true;
            break;
        }
        t_cur += step_world;
    }
    if (!hit) {
        *out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    float ta = t_cur - step_world, tb = t_cur;
    for (int i = 0; i < 8; i++) {
        const float m = (ta + tb) * 0.5f;
        if (get_density(S, ray_org + ray_dir * m) > kThreshold)
            tb = m;
        else
            ta = m;
    }
    const V3 surf = ray_org + ray_dir * tb;
    V3 N = -calc_normal(S, surf);
    N = normalize3(N);
    if (dot3(N, N) < 0.5f) N = v3(0.0f, 1.0f, 0.0f);

    const V3 V = -ray_dir;
    const V3 L = normalize3(v3(0.4f, 1.0f, 0.3f));
    const V3 H = normalize3(L + V);
    const float n_dot_v = fmaxf(dot3(N, V), 0.0f);
    const float n_dot_l = fmaxf(dot3(N, L), 0.0f);
    const float n_dot_h = fmaxf(dot3(N, H), 0.0f);
    const float f0 = powf((kIorAir - kIorWater) / (kIorAir + kIorWater), 2.0f);
    const float F = clampf(fresnel(n_dot_v, f0), 0.0f, 1.0f);

    const V3 sun = v3(1.0f, 0.95f, 0.85f);
    const V3 refl_dir = ray_dir - N * (2.0f * dot3(N, ray_dir));      // reflect
    V3 reflection = sample_sky(A.sky, A.sky_w, A.sky_h, refl_dir);
    const float spec = ggx_d(n_dot_h, 0.04f) * n_dot_l;
    reflection = reflection + sun * clampf(spec * 0.15f, 0.0f, 3.0f);

    const float thickness = calc_thickness(S, surf, ray_dir, t_far - tb);
    const V3 absorption = v3(expf(-0.45f * thickness * 8.0f), expf(-0.085f * thickness * 8.0f),
                             expf(-0.025f * thickness * 8.0f));
    // refract(rayDir, N, eta)
    const float eta = kIorAir / kIorWater;
    const float ni = dot3(N, ray_dir);
    const float k = 1.0f - eta * eta * (1.0f - ni * ni);
    V3 refr = k < 0.0f ? v3(0, 0, 0) : ray_dir * eta - N * (eta * ni + sqrtf(k));
    if (dot3(refr, refr) < 0.01f) refr = ray_dir;
    const V3 background = sample_sky(A.sky, A.sky_w, A.sky_h, normalize3(refr));

    const float sss_wrapped = fmaxf(0.0f, dot3(N, L) * 0.5f + 0.5f);
    const float sss_back = fmaxf(0.0f, dot3(-N, L));
    const float sss_factor = (sss_wrapped * 0.6f + sss_back * 0.4f) * (1.0f - expf(-thickness * 3.0f));
    const V3 scatter = v3(0.04f, 0.18f, 0.28f);
    const V3 sss = ((scatter * sun) * sss_factor) * 0.35f;

    float foam = smoothstepf(0.0f, 0.3f, thickness);
    foam *= smoothstepf(0.5f, 0.95f, N.y);
    const V3 refracted = background * absorption + sss;
    V3 water = mix3(refracted, reflection, F);
    const V3 foam_col = v3(0.92f, 0.96f, 1.0f) * (n_dot_l * 0.7f + 0.3f);
    water = mix3(water, foam_col, foam * 0.7f);
    water = water + scatter * 0.04f;
    water = v3(water.x / (water.x + 1.0f), water.y / (water.y + 1.0f), water.z / (water.z + 1.0f));
    *out = make_float4(water.x, water.y, water.z, 1.0f);
}

}  // namespace

cudaError_t raymarch(const RaymarchArgs& a, cudaStream_t stream) {
    dim3 grid((a.width + 15) / 16, (a.height + 7) / 8);
    k_raymarch<<<grid, 128, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace fe
