// fe_tune.h — the autotuner: measures the candidate shapes of the tunable
// kernels on the device and data they will run on, and picks the fastest.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "fe_mlp.h"
#include "fe_sort.h"

namespace fe {

constexpr int kMlpCtaCandidates = 4;
extern const int kMlpCtaChoices[kMlpCtaCandidates];

// Times radix_sort for every kRadixCandidates entry on a copy of
// (keys, vals) (n pairs, keys < 2^key_bits): one untimed run, then the
// median of `reps` CUDA-event timed runs, each on a fresh copy.  ms[k] gets
// candidate k's median; *best the fastest.  Allocates its working buffers
// and frees them before returning.
cudaError_t tune_radix(cudaStream_t stream, const uint32_t* keys, const uint32_t* vals,
                       uint32_t n, uint32_t key_bits, int reps, RadixConfig* best,
                       float ms[kRadixCandidateCount]);

// Times the MLP inference over n rows of X for each kMlpCtaChoices entry
// (blocks per SM of the persistent grid); out receives the network output.
cudaError_t tune_mlp(cudaStream_t stream, const mlp::Params& P, const __nv_bfloat16* X,
                     float* out, uint32_t n, uint32_t* error_flags, int num_sms, int reps,
                     int* best_ctas, float ms[kMlpCtaCandidates]);

// Process-wide choices for the standalone sort (fe_sort_pairs), per device
// and size class (ceil(log2 n), key_bits).  lookup returns false when the
// size class was never tuned.
bool sort_tuning_lookup(int device, uint32_t n, uint32_t key_bits, RadixConfig* out);
void sort_tuning_store(int device, uint32_t n, uint32_t key_bits, RadixConfig cfg);

}  // namespace fe
