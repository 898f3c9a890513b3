// fe_mlp.h — tensor-core MLP of the learned warm start (fe_mlp.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "fe_device.h"

namespace fe {
namespace mlp {

// Parameter layout (FP32 master and gradients, in this order):
//   w1 [64][16] (input columns 12..15 stay zero), w2 [64][64], w3 [2][64],
//   b1 [64], b2 [64], b3 [2].
// The BF16 weight copy holds w1, w2, w3 in the same order.
constexpr uint32_t kW1 = 64 * 16, kW2 = 64 * 64, kW3 = 2 * 64;
constexpr uint32_t kWeights = kW1 + kW2 + kW3;         // 5248
constexpr uint32_t kParams = kWeights + 64 + 64 + 2;   // 5378
constexpr uint32_t kFeatures = 12;

struct Params {
    const __nv_bfloat16 *w1, *w2, *w3;
    const float *b1, *b2, *b3;
};

struct Grads {
    float *w1, *w2, *w3, *b1, *b2, *b3;
    float* loss;
};

__host__ __device__ inline Params params_from(const __nv_bfloat16* wbf16, const float* master) {
    return Params{wbf16, wbf16 + kW1, wbf16 + kW1 + kW2, master + kWeights,
                  master + kWeights + 64, master + kWeights + 128};
}
__host__ __device__ inline Grads grads_from(float* g, float* loss) {
    return Grads{g, g + kW1, g + kW1 + kW2, g + kWeights, g + kWeights + 64, g + kWeights + 128,
                 loss};
}

size_t infer_smem_bytes();

// What the inference kernel needs to start a solve from its output in the
// same pass (the warm start of fe_features.cuh, warm_apply_particle):
// output `which` of particle g becomes its initial pressure.
struct ApplyArgs {
    Bufs B;
    LearnArgs L;
    int which;
};

// The inference kernel as a launch description (for CUDA-graph recording):
// arguments (Params, const __nv_bfloat16* X, float* out, uint32_t n,
// uint32_t* error_flags, ApplyArgs).  With `apply` the kernel also starts
// solve A.which from its output.  Sets the kernel's shared-memory attribute.
struct KernelLaunch {
    const void* func;
    dim3 grid, block;
    size_t smem;
};
// Inference grid: min(pairs of 128-row tiles, num_sms * ctas_per_sm) blocks
// of 256 threads looping over the pairs.  ctas_per_sm is accepted in
// 1..kInferMaxCtasPerSm; each block holds 128 TMEM columns, so at most 4
// run on an SM and larger values act as 4.
constexpr int kInferDefaultCtasPerSm = 4;
constexpr int kInferMaxCtasPerSm = 6;
cudaError_t infer_launch(uint32_t n, int num_sms, KernelLaunch* out,
                         int ctas_per_sm = kInferDefaultCtasPerSm, bool apply = false);
size_t train_smem_bytes();

// out[i][0..1] for the BF16 rows X[i][0..15], i < n.
cudaError_t infer(const Params& P, const __nv_bfloat16* X, float* out, uint32_t n,
                  uint32_t* error_flags, cudaStream_t stream, int num_sms,
                  int ctas_per_sm = kInferDefaultCtasPerSm);

// Writes d(loss)/d(params) of the mean squared error over the n samples to
// grad[kParams] and the summed squared error to grad[kParams].  Blocks sum
// their tiles into their own slice of part[min(tiles, num_sms)][kParams + 1],
// and the slices are added in block order: the same inputs give the same
// gradients bit for bit.
cudaError_t train_grads(const Params& P, const __nv_bfloat16* X, const float* Y, uint32_t n,
                        float* grad, float* part, uint32_t* error_flags, cudaStream_t stream,
                        int num_sms);

cudaError_t adam(float* master, float* grad, float* m, float* v, __nv_bfloat16* bf16_copy,
                 uint32_t count, uint32_t bf16_count, float lr, float beta1, float beta2, float eps,
                 uint32_t step, float weight_decay, cudaStream_t stream);

}  // namespace mlp
}  // namespace fe
