// fe_learned.cu — the learned warm start inside the step, and the capture of
// its training data from the plain solver.
//
// Before each of the two solves of a substep (after density_source, and after
// divergence_source):  features -> MLP (fe_mlp.cu) -> the solve's initial
// pressure (output 0 for the density solve, output 1 for the divergence
// solve).  After each solve the final pressure is recorded as the "last
// kappa" feature and, in capture mode, as the target of the captured
// particles (the other output's target is NaN: not trained).
//
// Normalisation.  With the Jacobi diagonal a_ii = -(dt / rho_i^2) alpha_i, one
// Jacobi step from zero gives p = -omega s_i rho_i^2 / (dt alpha_i), so
//   scale_i = rho_i^2 / (dt alpha_i) * (rho0 * 1e-3 / dt)
// maps a pressure to the units of sigma_i = s_i dt / (rho0 * 1e-3), the
// source term in 0.1 % density-error units.  Targets and the carried
// pressures are kappa / scale_i (0 where alpha_i, rho_i or dt <= 1e-6).
//
// Features (12, standardised with the model's statistics):
//   0 rho_i / rho0 - 1          1 alpha_i h^8 / m^2       2 sigma_i (this solve)
//   3 neighbour count / 32      4 last density kappa / scale_i
//   5 last divergence kappa / scale_i                    6 |v_i| dt / h
//   7..11 kernel-weighted neighbourhood moments of the source, orders 1..5:
//         sum_j W_ij t_j^k / sum_j W_ij with t_j = tanh(sigma_j / 4)
// ("last" = the most recent solve of that kind: at the divergence solve the
// density kappa is the one just computed in this substep).
#include <cuda_bf16.h>

#include "fe_common.cuh"
#include "fe_kernels.h"
#include "fe_neighbors.cuh"

namespace fe {

namespace {

__device__ __forceinline__ float kappa_scale(float rho, float alpha, float dt, float rho0) {
    if (!(alpha > kEpsR && rho > kEpsR && dt > kEpsR)) return 0.0f;
    return (rho * rho / (dt * alpha)) * (rho0 * 1e-3f / dt);
}

__device__ __forceinline__ float sigma_of(float s, float dt, float rho0) {
    return s * dt / (rho0 * 1e-3f);
}

__device__ __forceinline__ uint32_t sample_hash(uint32_t i, uint32_t seed) {
    uint32_t x = i * 2654435761u ^ (seed * 2246822519u + 0x9E3779B9u);
    x ^= x >> 15;
    x *= 2246822519u;
    x ^= x >> 13;
    return x;
}

}  // namespace

// Features of every particle before a solve (which = 0 density, 1
// divergence); network input rows in BF16; capture of a sample.
__global__ void __launch_bounds__(kBlock) k_features(Bufs B, LearnArgs L, int which) {
    uint32_t i, s, c;
    if (!chunk_of(B, i, s, c)) return;
    const DevParams& P = B.P[s];
    const float h = P.h, m = P.mass, dt = P.dt, rho0 = P.rho0;
    const f3 pi = xyz(__ldg(posb(B, i)));
    const float rho = B.rho[i], alpha = B.alpha[i];
    const float scale = kappa_scale(rho, alpha, dt, rho0);
    const float4 carry = L.carry[i];
    float f[12];
    f[0] = rho / rho0 - 1.0f;
    const float h2 = h * h, h4 = h2 * h2;
    f[1] = alpha * (h4 * h4) / (m * m);
    f[2] = sigma_of(B.src[i], dt, rho0);
    const uint32_t cnt = B.nbr_count[i];
    f[3] = (float)(cnt < 64u ? cnt : 64u) / 32.0f;
    f[4] = scale > 0.0f ? carry.x / scale : 0.0f;
    f[5] = scale > 0.0f ? carry.y / scale : 0.0f;
    // velocity the solve's source term used
    const float4* vel = (which == 0 || P.mode == 0u) ? B.vel_a : B.vel_b;
    const float4 v = vel[i];
    f[6] = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z) * dt / h;
    float wsum = 0.0f, mom[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    for_each_neighbor(
        B, P, i, pi, [&](uint32_t j) { return __ldg(B.src + j); },
        [&](uint32_t, f3 rv, float, float4, float sj) {
            float r = sqrtf(dot(rv, rv));
            float w = kernel_w(r, h);
            float t = tanhf(sigma_of(sj, dt, rho0) * 0.25f);
            float pw = t;
            wsum += w;
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                mom[k] += w * pw;
                pw *= t;
            }
        });
#pragma unroll
    for (int k = 0; k < 5; ++k) f[7 + k] = wsum > 0.0f ? mom[k] / wsum : 0.0f;

    if (L.learned) {
        uint32_t packed[8];
#pragma unroll
        for (int k = 0; k < 16; k += 2) {
            float a = k < 12 ? (f[k] - L.norm[k]) / L.norm[12 + k] : 0.0f;
            float b = k + 1 < 12 ? (f[k + 1] - L.norm[k + 1]) / L.norm[13 + k] : 0.0f;
            __nv_bfloat162 two = __floats2bfloat162_rn(a, b);
            packed[k / 2] = *reinterpret_cast<uint32_t*>(&two);
        }
        uint4* dst = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(L.xb) + (size_t)i * 16);
        dst[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
        dst[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
    }
    uint32_t slot = 0xFFFFFFFFu;
    if (L.capture && scale > 0.0f &&
        sample_hash(i, 2u * B.S[s].substeps + (uint32_t)which) % (L.cap_stride ? L.cap_stride : 1u) ==
            0u) {
        uint32_t k = atomicAdd(L.cap_count, 1u);
        if (k < L.cap_capacity) {
            slot = k;
#pragma unroll
            for (int q = 0; q < 12; ++q) L.cap_x[(size_t)k * 12 + q] = f[q];
            const float nan = __int_as_float(0x7fffffff);
            L.cap_y[2 * (size_t)k] = nan;      // the solve fills its own target;
            L.cap_y[2 * (size_t)k + 1] = nan;  // the other stays NaN (not trained)
        }
    }
    L.carry[i].w = __uint_as_float(slot);
}

// Applies the network's pressure to the solve about to start (output
// `which`, in normalised units, rescaled with the current state).
__global__ void __launch_bounds__(kBlock) k_warm_apply(Bufs B, LearnArgs L, int which) {
    uint32_t i, s, c;
    if (!chunk_of(B, i, s, c)) return;
    const DevParams& P = B.P[s];
    const float rho = B.rho[i];
    const float scale = kappa_scale(rho, B.alpha[i], P.dt, P.rho0);
    const float y = L.out[2 * (size_t)i + which] * L.norm[26 + which] + L.norm[24 + which];
    float p = y * scale;
    p = p > 0.0f ? p : 0.0f;  // pressures are clamped at 0 as in pressure_update
    B.prs[i] = p;
    posb(B, i)->w = pressure_over_rho2(p, rho);
}

// After a solve: the final pressure becomes the "last kappa" feature and, in
// capture mode, the training target of the particle's slot.
__global__ void __launch_bounds__(kBlock) k_after_solve(Bufs B, LearnArgs L, int which) {
    uint32_t i, s, c;
    if (!chunk_of(B, i, s, c)) return;
    const DevParams& P = B.P[s];
    const float p = B.prs[i];
    float4 cr = L.carry[i];
    if (which == 0)
        cr.x = p;
    else
        cr.y = p;
    const uint32_t slot = __float_as_uint(cr.w);
    if (L.capture && slot != 0xFFFFFFFFu && slot < L.cap_capacity) {
        const float scale = kappa_scale(B.rho[i], B.alpha[i], P.dt, P.rho0);
        L.cap_y[2 * (size_t)slot + which] = scale > 0.0f ? p / scale : 0.0f;
    }
    cr.w = __uint_as_float(0xFFFFFFFFu);
    L.carry[i] = cr;
}

// Carries the per-particle learned state through the re-sort: gather by the
// sorted index, then copy back.
__global__ void __launch_bounds__(kBlock) k_carry_gather(Bufs B, LearnArgs L) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B.n_total) return;
    uint32_t src = B.vals[i];
    if (src >= B.n_total) src = i;
    L.carry_tmp[i] = L.carry[src];
}

__global__ void __launch_bounds__(kBlock) k_carry_take(Bufs B, LearnArgs L) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B.n_total) return;
    L.carry[i] = L.carry_tmp[i];
}

}  // namespace fe
