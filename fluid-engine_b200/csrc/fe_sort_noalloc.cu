// fe_sort_noalloc.cu — the radix sort with its scratch in a static device
// array, for callers that cannot let the library allocate.
//
// fe_sort_pairs allocates scratch the first time it sees a size.  Some
// callers cannot accept that: a frame loop that must never stall (cudaMalloc
// and cudaFree synchronise the whole device), and host applications that
// budget every byte of device memory themselves and forbid libraries to
// allocate behind their back.  fe_sort_pairs_noalloc sorts with a scratch area that is a file-scope
// __device__ array: the CUDA runtime reserves it on each GPU when the library
// is loaded there, and it stays reserved until the process exits.
#include <cuda.h>
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

// Per device: the CUDA context the address below was looked up in, and that
// address.  A device reset (cudaDeviceReset, or the primary context being
// destroyed and made again) loads the library's module anew, and the array
// may then live at another address; the context's unique ID tells a new
// context from the old one even if its handle value were reused.
struct ScratchAddress {
    unsigned long long ctx_id = 0;
    bool valid = false;
    uint32_t* ptr = nullptr;
};
ScratchAddress g_scratch[kMaxDevices];

// The driver's cuCtxGetCurrent and cuCtxGetId, fetched through the runtime
// (the library does not link the driver library directly).
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

cudaError_t current_context_id(unsigned long long* id) {
    if (!g_ctx_get_current || !g_ctx_get_id) {
        void* f1 = nullptr;
        void* f2 = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1);
        if (e != cudaSuccess) return e;
        e = cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2);
        if (e != cudaSuccess) return e;
        if (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2)
            return cudaErrorSymbolNotFound;
        g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
        g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f2);
    }
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return cudaErrorDeviceUninitialized;
    if (g_ctx_get_id(ctx, id) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
    return cudaSuccess;
}

// Device address of g_noalloc_scratch on the current device.  In host code
// the symbol's name is only a host-side handle, never a device address, so
// the address is looked up with the device current: on the first call in
// each CUDA context of a device (normally once per device per process).
cudaError_t scratch_for_current_device(uint32_t** out, int* device) {
    cudaError_t e = cudaGetDevice(device);
    if (e != cudaSuccess) return e;
    if (*device < 0 || (uint32_t)*device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mutex);
    ScratchAddress& a = g_scratch[*device];
    unsigned long long id = 0;
    if (a.valid && current_context_id(&id) == cudaSuccess && id == a.ctx_id) {
        *out = a.ptr;
        return cudaSuccess;
    }
    // First call in this context (the lookup also makes the device's primary
    // context current in a thread that has not used the runtime yet).
    uint32_t* p = nullptr;
    if ((e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch)) != cudaSuccess) return e;
    if ((e = current_context_id(&id)) != cudaSuccess) return e;
    a.ptr = p;
    a.ctx_id = id;
    a.valid = true;
    *out = p;
    return cudaSuccess;
}

// The error word of the last call inside the scratch (see the layout above).
uint32_t* flags_word(uint32_t* scratch) { return scratch + 2u * (size_t)kMaxPairs + kRadixWords; }

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
    uint32_t* flags = flags_word(scratch);
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

// The error word of the last fe_sort_pairs_noalloc call on the current
// device, copied in the order of `stream`.
extern "C" FE_API fe_status fe_sort_noalloc_flags(uint32_t* flags_out, void* stream_ptr) {
    if (!flags_out) {
        fe_set_error_message("fe_sort_noalloc_flags: NULL flags_out");
        return FE_ERR_INVALID_ARGUMENT;
    }
    uint32_t* scratch = nullptr;
    int device = -1;
    cudaError_t e = scratch_for_current_device(&scratch, &device);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(flags_out, flags_word(scratch), sizeof(uint32_t), cudaMemcpyDefault,
                            (cudaStream_t)stream_ptr);
    if (e != cudaSuccess) {
        fe_set_error_message("fe_sort_noalloc_flags on device %d: %s", device,
                             cudaGetErrorString(e));
        return FE_ERR_CUDA;
    }
    return FE_OK;
}

// Test hook: the radix pass's bounded look-back wait, run on a status word
// of the static scratch that nobody publishes, raising its timeout flag in
// the same error word a sort would.  No GPU fault is involved: the wait gives
// up after `limit` polls.
extern "C" FE_API fe_status fe_debug_noalloc_wait_timeout(uint32_t limit, void* stream_ptr) {
    if (limit == 0) {
        fe_set_error_message("fe_debug_noalloc_wait_timeout needs a non-zero limit");
        return FE_ERR_INVALID_ARGUMENT;
    }
    uint32_t* scratch = nullptr;
    int device = -1;
    cudaError_t e = scratch_for_current_device(&scratch, &device);
    cudaStream_t stream = (cudaStream_t)stream_ptr;
    uint32_t* flags = flags_word(scratch);
    if (e == cudaSuccess) e = cudaMemsetAsync(flags, 0, 8 * sizeof(uint32_t), stream);
    if (e == cudaSuccess)
        e = fe::lookback_wait_on(flags + 1, flags, (int)(limit < (1u << 30) ? limit : (1u << 30)),
                                 stream);
    if (e != cudaSuccess) {
        fe_set_error_message("fe_debug_noalloc_wait_timeout: %s", cudaGetErrorString(e));
        return FE_ERR_CUDA;
    }
    return FE_OK;
}
