// fe_features.cuh — the learned warm start's per-particle features, emitted
// by the two source-term passes (which already visit every neighbour).
//
// Normalisation.  With the Jacobi diagonal a_ii = -(dt / rho_i^2) alpha_i, one
// Jacobi step from zero gives p = -omega s_i rho_i^2 / (dt alpha_i), so
//   scale_i = rho_i^2 / (dt alpha_i) * (rho0 * 1e-3 / dt)
// maps a pressure to the units of sigma_i = s_i dt / (rho0 * 1e-3), the
// source term in 0.1 % density-error units.  The carried pressures enter as
// kappa / scale_i (0 where alpha_i, rho_i or dt <= 1e-6).  Targets: the
// density solve's final kappa / scale_i, and the divergence solve's final
// kappa minus the substep's density kappa (its start without the network),
// over scale_i.
//
// Features (12, standardised with the model's statistics before the network):
//   0  rho_i / rho0 - 1                    1  alpha_i h^8 / m^2
//   2  div_i dt / (rho0 1e-3)  (the velocity-divergence term of the source)
//   3  neighbour count / 32                4  last density kappa / scale_i
//   5  last divergence kappa / scale_i     6  |v_i| dt / h
//   7..11  the 5 lowest moments (orders 1..5) of the neighbours' density
//          residual, t_j = x / (1 + |x|) with x = 100 (rho_j / rho0 - 1),
//          weighted by -grad_factor / (h r) (the list's kernel-gradient
//          scale, >= 0): sum_j w_j t_j^k / sum_j w_j, as the density source
//          finds them at the start of the substep.  The divergence solve's
//          row carries the same five values through the mid-substep re-sort
//          (LearnArgs::mom, carry.z), so its features need no neighbour pass
//          of their own and are emitted by density_alpha.
// ("last" = the most recent solve of that kind: before the divergence solve
// the density kappa is the one just computed in this substep.)  The solve's
// own source term in the same units is a fixed linear combination of
// features 0 and 2 (-1000 f0 - f2 before the density solve, -f2 before the
// divergence solve), so it is not a feature of its own.
//
// Every operation is IEEE single precision in the order written (no fast
// division, no contraction), so the host oracle reproduces each feature and
// its BF16 row bit for bit.
#pragma once

#include <cuda_bf16.h>

#include "fe_common.cuh"

namespace fe {

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

constexpr int kMoments = 5;

// The density residual of one particle as the moments weigh it:
// t = x / (1 + |x|), x = 100 (rho / rho0 - 1).  It depends on the particle
// alone, so viscosity stores it once per particle (velocity_a's w) for the
// learned density source, which gathers it with the velocity.
__device__ __forceinline__ float density_residual_t(float rho, float rho0) {
    float x = 100.0f * (rho / rho0 - 1.0f);
    return x / (1.0f + fabsf(x));
}

// Running neighbourhood moments of the density residual (orders 1..5).
struct Moments {
    float w = 0.0f, m[kMoments] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    __device__ __forceinline__ void add(float g, float rho_j, float rho0) {
        add_t(g, density_residual_t(rho_j, rho0));
    }
    __device__ __forceinline__ void add_t(float g, float t) {
        float wj = -g;
        w += wj;
        float p = t;
#pragma unroll
        for (int k = 0; k < kMoments; ++k) {
            m[k] += wj * p;
            p *= t;
        }
    }
};

// The five moment features from the running sums.
__device__ __forceinline__ void moment_features(const Moments& mo, float fm[kMoments]) {
#pragma unroll
    for (int k = 0; k < kMoments; ++k) fm[k] = mo.w > 0.0f ? mo.m[k] / mo.w : 0.0f;
}

// Writes the network input row (learned mode) and captures a sample
// (capture mode) for particle i before solve `which` (0 density, 1
// divergence); fm = its five moment features.  Before the density solve the
// moments are also stored for the divergence solve (mom, carry.z).
__device__ __forceinline__ void emit_features(const Bufs& B, const LearnArgs& L,
                                              const DevParams& P, uint32_t i, uint32_t scene,
                                              int which, float div_i, f3 v,
                                              const float fm[kMoments]) {
    const float h = P.h, m = P.mass, dt = P.dt, rho0 = P.rho0;
    const float rho = B.rho[i], alpha = B.alpha[i];
    const float scale = kappa_scale(rho, alpha, dt, rho0);
    const float4 carry = L.carry[i];
    float f[12];
    f[0] = rho / rho0 - 1.0f;
    const float h2 = h * h, h4 = h2 * h2;
    f[1] = alpha * (h4 * h4) / (m * m);
    f[2] = sigma_of(div_i, dt, rho0);
    const uint32_t cnt = B.nbr_count[i];
    f[3] = (float)(cnt < 64u ? cnt : 64u) / 32.0f;
    f[4] = scale > 0.0f ? carry.x / scale : 0.0f;
    f[5] = scale > 0.0f ? carry.y / scale : 0.0f;
    f[6] = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z) * dt / h;
#pragma unroll
    for (int k = 0; k < kMoments; ++k) f[7 + k] = fm[k];
    if (which == 0) L.mom[i] = make_float4(fm[0], fm[1], fm[2], fm[3]);

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
        sample_hash(i, 2u * B.S[scene].substeps + (uint32_t)which) %
                (L.cap_stride ? L.cap_stride : 1u) == 0u) {
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
    // z: the fifth moment for the divergence solve (kept by that solve's
    // emission), w: the capture slot
    float2* zw = reinterpret_cast<float2*>(&L.carry[i]) + 1;
    *zw = make_float2(which == 0 ? fm[4] : carry.z, __uint_as_float(slot));
}

// Applies the network's pressure to the solve about to start (output
// `which`, in normalised units, rescaled with the current state).  Output 0
// is the density solve's kappa; output 1 is the divergence solve's kappa
// minus the density kappa of this substep (the start the divergence solve
// takes without the network, divergence_source_term.comp leaving p alone).
//
// The start is clamped from above.  With p1 = max(omega s_i / a_ii, 0) the
// first Jacobi iterate from zero, d_i = p1 / omega is the pressure that
// resolves particle i's source on its own (neighbours at zero pressure).  The
// density start is at most max(d_i, kappa_d,prev) (the particle's density
// kappa of the previous substep); the divergence start at most
// max(d_i, kappa_d) (this substep's density kappa, the start without the
// network).  scale_i grows as 1/alpha_i, so without a bound a small error of
// the network at a particle with few neighbours becomes a pressure far above
// anything the plain solver produces there, which the mean tolerance metric
// cannot see and which throws particles out at 10^4 m/s within a few hundred
// frames.  A bound that includes the previous divergence kappa, or a factor
// above 1, feeds such errors back from substep to substep and is not stable
// either.  Under the bound the start stays near or below the solution,
// where Jacobi approaches from the same side as the plain solver.
//
// Particles with fewer than kMinNeighbours neighbours (the free surface and
// splashes, where alpha is small, scale_i large and training samples few)
// keep the plain start.  Without this, a long adaptive-CFL run of the 262k
// dam break still threw single particles out at 10^2 - 10^3 m/s late in the
// run (a few over-pressured particles do not move the mean tolerance); with
// it the largest speed matches the plain solver's.
constexpr uint32_t kMinNeighbours = 16;
// y_std: the network's output `which` for particle i in standardised units.
__device__ __forceinline__ void warm_apply_particle(const Bufs& B, const LearnArgs& L,
                                                    const DevParams& P, uint32_t i, int which,
                                                    float y_std) {
    const float rho = B.rho[i], alpha = B.alpha[i];
    const float scale = kappa_scale(rho, alpha, P.dt, P.rho0);
    const float y = y_std * L.norm[26 + which] + L.norm[24 + which];
    const float4 carry = L.carry[i];
    const float base = which == 1 ? carry.x : 0.0f;
    // Comparisons rather than fminf/fmaxf, so that no signed zero depends on
    // how a maximum of -0 and +0 is taken: every value below is +0 or
    // positive, and NaN becomes 0.
    float p1 = 0.0f;
    if (alpha > kEpsR && rho > kEpsR) {
        const float a_ii = -(P.dt / (rho * rho)) * alpha;
        if (fabsf(a_ii) > 1e-20f) {
            const float q = (P.omega * B.src[i]) / a_ii;
            p1 = q > 0.0f ? q : 0.0f;
        }
    }
    const float d = p1 / P.omega;
    float p = B.nbr_count[i] < kMinNeighbours ? base : base + y * scale;
    p = p > 0.0f ? p : 0.0f;  // NaN -> 0; pressures are clamped at 0 as in pressure_update
    const float bound = d > carry.x ? d : carry.x;
    p = p < bound ? p : bound;
    B.prs[i] = p;
    posb(B, i)->w = pressure_over_rho2(p, rho);
}

// The scene of particle g (scenes are laid out back to back).
__device__ __forceinline__ uint32_t scene_of(const Bufs& B, uint32_t g) {
    uint32_t lo = 0, hi = B.n_scenes;   // first scene whose first particle is > g, minus one
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (B.P[mid].first <= g) lo = mid; else hi = mid;
    }
    return lo;
}

// After solve `which`: the final pressure becomes the particle's "last kappa"
// and, in capture mode, the training target of its sample slot (for the
// divergence solve relative to the substep's density kappa, as the warm start
// applies it).  Fused into the integration pass that follows each solve.
__device__ __forceinline__ void after_solve_particle(const Bufs& B, const LearnArgs& L,
                                                     const DevParams& P, uint32_t i, int which) {
    const float p = B.prs[i];
    float4 cr = L.carry[i];
    const float base = which == 1 ? cr.x : 0.0f;
    if (which == 0)
        cr.x = p;
    else
        cr.y = p;
    const uint32_t slot = __float_as_uint(cr.w);
    if (L.capture && slot != 0xFFFFFFFFu && slot < L.cap_capacity) {
        const float scale = kappa_scale(B.rho[i], B.alpha[i], P.dt, P.rho0);
        L.cap_y[2 * (size_t)slot + which] = scale > 0.0f ? (p - base) / scale : 0.0f;
    }
    cr.w = __uint_as_float(0xFFFFFFFFu);
    L.carry[i] = cr;
}

}  // namespace fe
