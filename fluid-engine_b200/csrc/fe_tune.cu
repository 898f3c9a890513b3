// fe_tune.cu — the autotuner (no reference counterpart; the reference fixes
// its workgroup sizes and 8-bit digits in the shaders).
//
// Tunables, all with results independent of the choice:
//   * radix sort: digit width (8 or 10 bits) and keys per thread (4, 8, 16),
//     which set the number of passes, tiles in flight and shared memory per
//     block (fe_sort.cu);
//   * learned warm start: blocks per SM of the persistent inference grid.
// The neighbour-loop kernels are not tuned: their 256-particle chunks fix the
// order of the FP64 reductions that decide when the tolerance solver stops.
// Candidates are timed with CUDA events on the stream and data they will run
// on; the median of several runs decides.
#include "fe_tune.h"

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace fe {

const int kMlpCtaChoices[kMlpCtaCandidates] = {1, 2, 3, 4};

namespace {

struct StreamLaunch {
    cudaStream_t stream;
    static cudaError_t launch(void* self, const void* func, dim3 grid, dim3 block, size_t smem,
                              void** args) {
        return cudaLaunchKernel(func, grid, block, args, smem,
                                static_cast<StreamLaunch*>(self)->stream);
    }
    static cudaError_t fill(void* self, uint32_t* p, uint32_t value, size_t count) {
        // Only zero fills are requested by the sort.
        return cudaMemsetAsync(p, (int)(value & 0xFF), count * 4,
                               static_cast<StreamLaunch*>(self)->stream);
    }
};

float median(std::vector<float> v) {
    std::sort(v.begin(), v.end());
    return v[v.size() / 2];
}

struct Events {
    cudaEvent_t a = nullptr, b = nullptr;
    ~Events() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
    cudaError_t init() {
        cudaError_t e = cudaEventCreate(&a);
        return e != cudaSuccess ? e : cudaEventCreate(&b);
    }
};

}  // namespace

cudaError_t tune_radix(cudaStream_t stream, const uint32_t* keys, const uint32_t* vals,
                       uint32_t n, uint32_t key_bits, int reps, RadixConfig* best,
                       float ms[kRadixCandidateCount]) {
    *best = kRadixDefault;
    if (n < 2) return cudaSuccess;
    reps = std::max(reps, 1);
    uint32_t *wk = nullptr, *wv = nullptr, *tk = nullptr, *tv = nullptr, *scratch = nullptr;
    const size_t words = radix_scratch_words_any(n, key_bits) + 8;
    cudaError_t e = cudaSuccess;
    auto cleanup = [&]() {
        cudaFree(wk);
        cudaFree(wv);
        cudaFree(tk);
        cudaFree(tv);
        cudaFree(scratch);
    };
    if ((e = cudaMalloc(&wk, (size_t)n * 4)) != cudaSuccess ||
        (e = cudaMalloc(&wv, (size_t)n * 4)) != cudaSuccess ||
        (e = cudaMalloc(&tk, (size_t)n * 4)) != cudaSuccess ||
        (e = cudaMalloc(&tv, (size_t)n * 4)) != cudaSuccess ||
        (e = cudaMalloc(&scratch, words * 4)) != cudaSuccess) {
        cleanup();
        return e;
    }
    uint32_t* flags = scratch + (words - 8);
    Events ev;
    if ((e = ev.init()) != cudaSuccess) {
        cleanup();
        return e;
    }
    StreamLaunch sl{stream};
    SortLaunch L{&sl, &StreamLaunch::launch, &StreamLaunch::fill};
    float best_ms = 1e30f;
    for (int k = 0; k < kRadixCandidateCount && e == cudaSuccess; ++k) {
        const RadixConfig cfg = kRadixCandidates[k];
        std::vector<float> t;
        for (int r = 0; r <= reps && e == cudaSuccess; ++r) {
            if ((e = cudaMemcpyAsync(wk, keys, (size_t)n * 4, cudaMemcpyDeviceToDevice, stream)) ||
                (e = cudaMemcpyAsync(wv, vals, (size_t)n * 4, cudaMemcpyDeviceToDevice, stream)) ||
                (e = cudaMemsetAsync(flags, 0, 32, stream)))
                break;
            bool in_tmp = false;
            if ((e = cudaEventRecord(ev.a, stream)) ||
                (e = radix_sort(L, wk, wv, tk, tv, n, key_bits, scratch, flags, &in_tmp, cfg)) ||
                (e = cudaEventRecord(ev.b, stream)) || (e = cudaEventSynchronize(ev.b)))
                break;
            float x = 0.0f;
            if ((e = cudaEventElapsedTime(&x, ev.a, ev.b))) break;
            if (r > 0) t.push_back(x);  // run 0 warms caches and code
        }
        if (e != cudaSuccess) break;
        ms[k] = median(t);
        if (ms[k] < best_ms) {
            best_ms = ms[k];
            *best = cfg;
        }
    }
    cudaError_t s = cudaStreamSynchronize(stream);
    cleanup();
    return e != cudaSuccess ? e : s;
}

cudaError_t tune_mlp(cudaStream_t stream, const mlp::Params& P, const __nv_bfloat16* X,
                     float* out, uint32_t n, uint32_t* error_flags, int num_sms, int reps,
                     int* best_ctas, float ms[kMlpCtaCandidates]) {
    *best_ctas = mlp::kInferDefaultCtasPerSm;
    if (n == 0) return cudaSuccess;
    reps = std::max(reps, 1);
    Events ev;
    cudaError_t e = ev.init();
    if (e != cudaSuccess) return e;
    float best_ms = 1e30f;
    for (int k = 0; k < kMlpCtaCandidates; ++k) {
        std::vector<float> t;
        for (int r = 0; r <= reps; ++r) {
            if ((e = cudaEventRecord(ev.a, stream)) ||
                (e = mlp::infer(P, X, out, n, error_flags, stream, num_sms, kMlpCtaChoices[k])) ||
                (e = cudaEventRecord(ev.b, stream)) || (e = cudaEventSynchronize(ev.b)))
                return e;
            float x = 0.0f;
            if ((e = cudaEventElapsedTime(&x, ev.a, ev.b))) return e;
            if (r > 0) t.push_back(x);
        }
        ms[k] = median(t);
        if (ms[k] < best_ms) {
            best_ms = ms[k];
            *best_ctas = kMlpCtaChoices[k];
        }
    }
    return cudaSuccess;
}

namespace {

std::mutex g_tune_mutex;
std::map<std::tuple<int, uint32_t, uint32_t>, RadixConfig> g_sort_choice;

uint32_t size_class(uint32_t n) {
    uint32_t c = 0;
    while (c < 32 && (1u << c) < n) ++c;
    return c;
}

}  // namespace

bool sort_tuning_lookup(int device, uint32_t n, uint32_t key_bits, RadixConfig* out) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_sort_choice.find({device, size_class(n), key_bits});
    if (it == g_sort_choice.end()) return false;
    *out = it->second;
    return true;
}

void sort_tuning_store(int device, uint32_t n, uint32_t key_bits, RadixConfig cfg) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_sort_choice[{device, size_class(n), key_bits}] = cfg;
}

}  // namespace fe
