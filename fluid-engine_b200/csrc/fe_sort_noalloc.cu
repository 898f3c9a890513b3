// fe_sort_noalloc.cu — the radix sort with its scratch in a static device
// array, for callers that cannot let the library allocate.
//
// fe_sort_pairs allocates scratch the first time it sees a size.  Some
// callers cannot accept that: a frame loop that must never stall (cudaMalloc
// and cudaFree synchronise the whole device), code recording work into a CUDA
// graph through stream capture in global mode (allocation calls are refused
// while such a capture is open), and host applications that budget every byte
// of device memory themselves and forbid libraries to allocate behind their
// back.  fe_sort_pairs_noalloc sorts with a scratch area that is a file-scope
// __device__ array: the CUDA runtime reserves it on each GPU when the library
// is loaded there, and it stays reserved until the process exits.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/fluid_step.h"
#include "fe_error.h"
#include "fe_kernels.h"
#include "fe_sort.h"

namespace {

constexpr uint32_t kMaxPairs = FE_SORT_NOALLOC_MAX_PAIRS;
constexpr uint32_t kMaxDevices = 64;

// Words of the radix scratch for the largest size (4 passes of 8 bits).
constexpr size_t kRadixWords =
    4u * 256u + 8u + 4u * ((kMaxPairs + 4095u) / 4096u) * 256u;
// Layout: ping-pong keys | ping-pong values | radix scratch | error flags.
constexpr size_t kWords = 2u * (size_t)kMaxPairs + kRadixWords + 8u;

// About 9 MiB per GPU.  Every call shares it; calls that overlap on the GPU
// race on it.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kWords];

std::mutex g_mutex;
uint32_t* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device.  In host code
// the symbol's name is only a host-side handle, never a device address, so
// the address is looked up once per device, with that device current.
cudaError_t scratch_for_current_device(uint32_t** out, int* device) {
    cudaError_t e = cudaGetDevice(device);
    if (e != cudaSuccess) return e;
    if (*device < 0 || (uint32_t)*device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[*device]) {
        uint32_t* p = nullptr;
        e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[*device] = p;
    }
    *out = g_scratch_ptr[*device];
    return cudaSuccess;
}

struct EagerLaunch {
    cudaStream_t stream;
};

cudaError_t launch_on_stream(void* self, const void* func, dim3 grid, dim3 block, size_t smem,
                             void** args) {
    return cudaLaunchKernel(func, grid, block, args, smem, static_cast<EagerLaunch*>(self)->stream);
}

cudaError_t fill_on_stream(void* self, uint32_t* p, uint32_t value, size_t count) {
    if (count == 0) return cudaSuccess;
    cudaStream_t s = static_cast<EagerLaunch*>(self)->stream;
    unsigned blocks = (unsigned)((count + 255) / 256 < 148 * 8 ? (count + 255) / 256 : 148 * 8);
    void* args[] = {&p, &value, &count};
    return cudaLaunchKernel((const void*)fe::k_fill_u32, dim3(blocks), dim3(256), args, 0, s);
}

}  // namespace

extern "C" FE_API fe_status fe_sort_pairs_noalloc(uint32_t* keys, uint32_t* values, uint32_t n,
                                                 uint32_t key_bits, void* stream_ptr) {
    if (n > kMaxPairs) {
        fe_set_error_message("fe_sort_pairs_noalloc: %u pairs exceed the static scratch "
                             "maximum of %u (FE_SORT_NOALLOC_MAX_PAIRS); use fe_sort_pairs",
                             n, kMaxPairs);
        return FE_ERR_CAPACITY;
    }
    if (key_bits > 32) {
        fe_set_error_message("fe_sort_pairs_noalloc: key_bits %u above 32", key_bits);
        return FE_ERR_INVALID_ARGUMENT;
    }
    if ((!keys || !values) && n > 0) {
        fe_set_error_message("fe_sort_pairs_noalloc: NULL keys or values");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (n < 2) return FE_OK;
    if (key_bits == 0) key_bits = 32;
    uint32_t* scratch = nullptr;
    int device = -1;
    cudaError_t e = scratch_for_current_device(&scratch, &device);
    if (e != cudaSuccess) {
        fe_set_error_message("fe_sort_pairs_noalloc: scratch set-up on device %d failed: %s",
                             device, cudaGetErrorString(e));
        return FE_ERR_CUDA;
    }
    uint32_t* tmp_keys = scratch;
    uint32_t* tmp_vals = scratch + kMaxPairs;
    uint32_t* radix_words = scratch + 2u * (size_t)kMaxPairs;
    uint32_t* flags = radix_words + kRadixWords;
    EagerLaunch ctx{(cudaStream_t)stream_ptr};
    fe::SortLaunch L{&ctx, launch_on_stream, fill_on_stream};
    e = L.fill(flags, 0u, 8);
    bool in_tmp = false;
    if (e == cudaSuccess)
        e = fe::radix_sort(L, keys, values, tmp_keys, tmp_vals, n, key_bits, radix_words, flags,
                           &in_tmp);
    if (e == cudaSuccess && in_tmp) {
        e = cudaMemcpyAsync(keys, tmp_keys, (size_t)n * 4, cudaMemcpyDeviceToDevice, ctx.stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(values, tmp_vals, (size_t)n * 4, cudaMemcpyDeviceToDevice,
                                ctx.stream);
    }
    if (e != cudaSuccess) {
        fe_set_error_message("fe_sort_pairs_noalloc: %s", cudaGetErrorString(e));
        return FE_ERR_CUDA;
    }
    return FE_OK;
}
