// fe_learned.cu — the learned warm start inside the step, and the capture of
// its training data from the plain solver.
//
// Before each of the two solves of a substep the source-term pass emits the
// features (fe_features.cuh), the network (fe_mlp.cu) maps them to the
// solve's initial pressure (output 0 for the density solve, output 1 for the
// divergence solve) and installs it in the same kernel (warm_apply_particle,
// fe_features.cuh, in the inference kernel's epilogue).  After each solve the
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

// Copies the re-sorted learned state back (k_reorder_carry gathered it into
// carry_tmp); FIXED mode does this inside k_take_pressure_carry, and after a
// substep's re-sort k_density_alpha_div_learn does it.
__global__ void __launch_bounds__(kBlock) k_carry_take(Bufs B, LearnArgs L) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B.n_total) return;
    L.carry[i] = L.carry_tmp[i];
}

}  // namespace fe
