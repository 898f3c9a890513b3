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

// Number of 8-bit passes for keys < 2^key_bits (key_bits 0 or > 32 = 32).
uint32_t radix_passes(uint32_t key_bits);

// 32-bit words of scratch radix_sort needs for n keys.
size_t radix_scratch_words(uint32_t n, uint32_t key_bits);

// Stable LSD radix sort of n pairs.  Ping-pongs between (keys, vals) and
// (tmp_keys, tmp_vals); *result_in_tmp tells where the sorted pairs are
// (true when the number of passes is odd).  error_flags gets bit 0x4 if a
// bounded look-back wait gave up.
cudaError_t radix_sort(const SortLaunch& L, uint32_t* keys, uint32_t* vals, uint32_t* tmp_keys,
                       uint32_t* tmp_vals, uint32_t n, uint32_t key_bits, uint32_t* scratch,
                       uint32_t* error_flags, bool* result_in_tmp);

// In-place bitonic network; n must be a power of two.
cudaError_t bitonic_sort(const SortLaunch& L, uint32_t* keys, uint32_t* vals, uint32_t n);

}  // namespace fe
