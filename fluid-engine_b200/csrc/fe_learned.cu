// fe_learned.cu — the learned warm start inside the step, and the capture of
// its training data from the plain solver.
//
// Before each of the two solves of a substep the source-term pass emits the
// features (fe_features.cuh), the network (fe_mlp.cu) maps them to the
// solve's initial pressure (output 0 for the density solve, output 1 for the
// divergence solve) and k_warm_apply installs it.  After each solve the
// integration pass records the final pressure as the "last kappa" feature
// and, in capture mode, as the target of the captured particles
// (after_solve_particle; the other output's target is NaN: not trained).
//
// Feature definitions and normalisation: fe_features.cuh.
#include <cuda_bf16.h>

#include "fe_common.cuh"
#include "fe_features.cuh"
#include "fe_kernels.h"
#include "fe_neighbors.cuh"

namespace fe {

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
__global__ void __launch_bounds__(kBlock) k_warm_apply(Bufs B, LearnArgs L, int which) {
    uint32_t i, s, c;
    if (!chunk_of(B, i, s, c)) return;
    const DevParams& P = B.P[s];
    const float rho = B.rho[i], alpha = B.alpha[i];
    const float scale = kappa_scale(rho, alpha, P.dt, P.rho0);
    const float y = L.out[2 * (size_t)i + which] * L.norm[26 + which] + L.norm[24 + which];
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

// Copies the re-sorted learned state back (k_reorder_carry gathered it into
// carry_tmp); FIXED mode does this inside k_take_pressure_carry.
__global__ void __launch_bounds__(kBlock) k_carry_take(Bufs B, LearnArgs L) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B.n_total) return;
    L.carry[i] = L.carry_tmp[i];
}

}  // namespace fe
