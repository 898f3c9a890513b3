// fe_sort.h — radix and bitonic sorts of (key, value) pairs (fe_sort.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <initializer_list>

#include <cuda_runtime.h>

namespace fe {

// How the sorts enqueue work: eagerly on a stream, or as nodes of a CUDA
// graph being recorded (see Recorder in fe_api.cu).
struct SortLaunch {
    void* self;
    cudaError_t (*launch_fn)(void* self, const void* func, dim3 grid, dim3 block, size_t smem,
                             void** args);
    cudaError_t (*fill_fn)(void* self, uint32_t* p, uint32_t value, size_t count);

    cudaError_t launch(const void* func, dim3 grid, dim3 block, size_t smem,
                       std::initializer_list<const void*> args) const {
        void* a[16];
        size_t k = 0;
        for (const void* p : args) a[k++] = const_cast<void*>(p);
        return launch_fn(self, func, grid, block, smem, a);
    }
    cudaError_t fill(uint32_t* p, uint32_t value, size_t count) const {
        return fill_fn(self, p, value, count);
    }
};

// Shape of the onesweep passes: digit width in bits and keys per thread
// (a tile is 256 threads x items keys).  Every configuration produces the
// same stable sort; they differ in pass count, tiles in flight and shared
// memory per block.  The autotuner (fe_tune.cu) picks one per size.
struct RadixConfig {
    uint32_t digit_bits;  // 8 or 10
    uint32_t items;       // keys per thread
};
constexpr RadixConfig kRadixDefault{8, 16};
constexpr int kRadixCandidateCount = 5;
extern const RadixConfig kRadixCandidates[kRadixCandidateCount];
bool radix_config_valid(RadixConfig c);

// Number of passes for keys < 2^key_bits (key_bits 0 or > 32 = 32).
uint32_t radix_passes(uint32_t key_bits, uint32_t digit_bits = 8);

// 32-bit words of scratch radix_sort needs for n keys with configuration
// cfg, and the most any candidate configuration needs.
size_t radix_scratch_words(uint32_t n, uint32_t key_bits, RadixConfig cfg = kRadixDefault);
size_t radix_scratch_words_any(uint32_t n, uint32_t key_bits);

// Stable LSD radix sort of n pairs.  Ping-pongs between (keys, vals) and
// (tmp_keys, tmp_vals); *result_in_tmp tells where the sorted pairs are
// (true when the number of passes is odd).  error_flags gets bit 0x4 if a
// bounded look-back wait gave up.  cudaErrorInvalidValue for a
// configuration outside kRadixCandidates.
cudaError_t radix_sort(const SortLaunch& L, uint32_t* keys, uint32_t* vals, uint32_t* tmp_keys,
                       uint32_t* tmp_vals, uint32_t n, uint32_t key_bits, uint32_t* scratch,
                       uint32_t* error_flags, bool* result_in_tmp,
                       RadixConfig cfg = kRadixDefault);

// In-place bitonic network; n must be a power of two.
cudaError_t bitonic_sort(const SortLaunch& L, uint32_t* keys, uint32_t* vals, uint32_t n);

// Runs one look-back wait on a status word that is never published, with at
// most `limit` polls (clamped to the radix pass's own limit), on the current
// device; *flags_out receives the error flags it raised (0x4 = timed out).
cudaError_t lookback_wait_selftest(int limit, uint32_t* flags_out);

// The same wait, enqueued on `stream`, on a caller's status word (which must
// hold no published flag) with the timeout flag raised in *error_flags.
cudaError_t lookback_wait_on(uint32_t* status, uint32_t* error_flags, int limit,
                             cudaStream_t stream);

}  // namespace fe
