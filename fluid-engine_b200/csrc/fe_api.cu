// fe_api.cu — host driver and C ABI (include/fluid_step.h).
//
// A context is `GpuPhysicsData` + `ComputePipelines` (particle.rs:137-308,
// pipelines/mod.rs:78-124): it owns the device buffers, a CUDA stream and the
// recorded frame graphs.  Work is expressed once, through a Recorder that
// either launches on the stream (stage entry points, FE_STEP_NO_GRAPH) or
// appends kernel nodes to a CUDA graph — the counterpart of recording into
// the reference's AutoCommandBufferBuilder and submitting it.  Jacobi loops
// become conditional WHILE nodes whose condition the pressure-update kernel
// sets on the device, so a frame with a tolerance-driven solver runs without
// any host round trip.
#include <cuda_runtime.h>

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <tuple>
#include <utility>
#include <string>
#include <vector>

#include "../../include/fluid_step.h"
#include "fe_device.h"
#include "fe_error.h"
#include "fe_kernels.h"
#include "fe_mlp.h"
#include "fe_model.h"
#include "fe_sort.h"
#include "fe_raymarch.h"
#include "fe_splat.h"
#include "fe_tune.h"

using namespace fe;

// An NVTX range around each entry point that records or launches GPU work
// (the reference wraps each ComputeStep::execute in a Tracy span,
// renderer/mod.rs:279-340).  Like those spans, a range covers the host-side
// recording and launch; the device time is in the profiler's kernel rows.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

namespace {

thread_local std::string g_last_error;

void set_error_v(const char* fmt, va_list ap) {
    char buf[512];
    vsnprintf(buf, sizeof buf, fmt, ap);
    g_last_error = buf;
}

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    set_error_v(fmt, ap);
    va_end(ap);
}

#define FE_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                      __LINE__);                                                        \
            return e_ == cudaErrorMemoryAllocation ? FE_ERR_OUT_OF_MEMORY : FE_ERR_CUDA; \
        }                                                                               \
    } while (0)

uint32_t next_pow2(uint32_t n) {
    uint32_t t = 1;
    while (t < n) t <<= 1;
    return t;
}

uint32_t log2_ceil(uint64_t v) {
    uint32_t b = 0;
    while ((1ull << b) < v) ++b;
    return b;
}

bool finite3(const float* v) {
    return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]);
}

// ---------------------------------------------------------------------------
// Recorder: eager launches on a stream, or kernel nodes of a graph.
// ---------------------------------------------------------------------------
struct Recorder {
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;  // null: eager
    cudaGraph_t root = nullptr;   // graph owning conditional handles
    cudaGraphNode_t last = nullptr;

    cudaError_t launch(const void* func, dim3 grid, dim3 block, size_t smem, void** args) {
        if (!graph) return cudaLaunchKernel(func, grid, block, args, smem, stream);
        cudaKernelNodeParams p;
        std::memset(&p, 0, sizeof p);
        p.func = const_cast<void*>(func);
        p.gridDim = grid;
        p.blockDim = block;
        p.sharedMemBytes = (unsigned)smem;
        p.kernelParams = args;
        cudaGraphNode_t node;
        cudaError_t e = cudaGraphAddKernelNode(&node, graph, last ? &last : nullptr, last ? 1 : 0, &p);
        if (e == cudaSuccess) last = node;
        return e;
    }

    template <typename... KArgs, typename... Args>
    cudaError_t k(void (*func)(KArgs...), dim3 grid, dim3 block, Args... args) {
        std::tuple<KArgs...> values(static_cast<KArgs>(args)...);
        void* ptrs[sizeof...(KArgs) > 0 ? sizeof...(KArgs) : 1];
        fill_ptrs(values, ptrs, std::index_sequence_for<KArgs...>{});
        return launch((const void*)func, grid, block, 0, ptrs);
    }

    template <typename Tuple, size_t... I>
    static void fill_ptrs(Tuple& t, void** p, std::index_sequence<I...>) {
        ((p[I] = (void*)&std::get<I>(t)), ...);
    }

    // Device-to-device copy in recording order.
    cudaError_t copy(void* dst, const void* src, size_t bytes) {
        if (!graph) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream);
        cudaGraphNode_t node;
        cudaError_t e = cudaGraphAddMemcpyNode1D(&node, graph, last ? &last : nullptr,
                                                 last ? 1 : 0, dst, src, bytes,
                                                 cudaMemcpyDeviceToDevice);
        if (e == cudaSuccess) last = node;
        return e;
    }

    cudaError_t fill_u32(uint32_t* p, uint32_t v, size_t count) {
        if (count == 0) return cudaSuccess;
        size_t blocks = std::min<size_t>((count + 255) / 256, 148 * 8);
        return k(k_fill_u32, dim3((unsigned)blocks), dim3(256), p, v, count);
    }

    SortLaunch sort_launch() {
        SortLaunch L;
        L.self = this;
        L.launch_fn = [](void* self, const void* f, dim3 g, dim3 b, size_t smem, void** a) {
            return static_cast<Recorder*>(self)->launch(f, g, b, smem, a);
        };
        L.fill_fn = [](void* self, uint32_t* p, uint32_t v, size_t c) {
            return static_cast<Recorder*>(self)->fill_u32(p, v, c);
        };
        return L;
    }
};

// ---------------------------------------------------------------------------
// Parameters
// ---------------------------------------------------------------------------
fe_status validate(const fe_params* p) {
    if (!p) {
        set_error("params is NULL");
        return FE_ERR_INVALID_ARGUMENT;
    }
    const float scalars[] = {p->particle_radius, p->particle_mass, p->smoothing_radius,
                             p->target_density, p->viscosity, p->relax_factor, p->dt,
                             p->density_error_pct, p->divergence_error_pct, p->cfl_lambda,
                             p->cfl_min_dt, p->cfl_max_dt, p->cfl_growth,
                             p->density_tolerance, p->divergence_tolerance};
    for (float v : scalars)
        if (!std::isfinite(v)) {
            set_error("non-finite parameter");
            return FE_ERR_INVALID_ARGUMENT;
        }
    if (!finite3(p->gravity) || !finite3(p->box_min) || !finite3(p->box_max)) {
        set_error("non-finite gravity or box");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (!(p->smoothing_radius > 0.0f)) {
        set_error("smoothing_radius must be > 0");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (!(p->particle_mass > 0.0f) || !(p->target_density > 0.0f)) {
        set_error("particle_mass and target_density must be > 0");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (p->dt < 0.0f) {
        set_error("dt must be >= 0");
        return FE_ERR_INVALID_ARGUMENT;
    }
    for (int a = 0; a < 3; ++a)
        if (!(p->box_min[a] < p->box_max[a])) {
            set_error("box_min must be < box_max on every axis");
            return FE_ERR_INVALID_ARGUMENT;
        }
    if (p->sort_algorithm > FE_SORT_RADIX || p->mode > FE_MODE_FIXED ||
        p->solver > FE_SOLVER_TOLERANCE || p->warm_start > FE_WARM_LEARNED) {
        set_error("enum field out of range");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (p->solver == FE_SOLVER_TOLERANCE &&
        (p->max_iterations == 0 || p->min_iterations > p->max_iterations)) {
        set_error("tolerance solver needs 0 < max_iterations and min <= max");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (p->density_solver_iterations > 100000 || p->divergence_solver_iterations > 100000 ||
        p->max_iterations > 100000) {
        set_error("iteration counts above 100000");
        return FE_ERR_INVALID_ARGUMENT;
    }
    for (uint32_t r : p->reserved)
        if (r) {
            set_error("reserved fields must be zero");
            return FE_ERR_INVALID_ARGUMENT;
        }
    return FE_OK;
}

// Whether the reciprocal step of div_h (fe_common.cuh) returns the correctly
// rounded r / b for every significand m of r in [lo, hi) of [0, 2^23).
bool recip_division_exact_range(float b, uint32_t lo, uint32_t hi) {
    const float y = 1.0f / b;
    for (uint32_t m = lo; m < hi; ++m) {
        const uint32_t ab = 0x3f800000u | m;
        float a;
        std::memcpy(&a, &ab, 4);
        const float ref = a / b;
        const float q0 = a * y;
        const float q = std::fmaf(std::fmaf(-q0, b, a), y, q0);
        if (std::memcmp(&ref, &q, 4) != 0) return false;
    }
    return true;
}

// Whether, for the divisor b, that step is exact for every significand of r:
// checked over the 2^23 floats of [1, 2), since every step scales exactly
// with r's exponent.  About 50 ms of host time per new b, spread over up to
// 16 threads; the answer is kept per b.
bool recip_division_exact(float b) {
    if (!(b > 0.0f) || !std::isfinite(b) || !std::isnormal(b) || !std::isnormal(1.0f / b))
        return false;
    static std::mutex mu;
    static std::vector<std::pair<uint32_t, bool>> known;
    uint32_t key;
    std::memcpy(&key, &b, 4);
    std::lock_guard<std::mutex> lock(mu);
    for (const auto& kv : known)
        if (kv.first == key) return kv.second;
    const uint32_t total = 1u << 23;
    const uint32_t nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<char> ok(nt, 0);
    std::vector<std::thread> pool;
    for (uint32_t t = 0; t < nt; ++t)
        pool.emplace_back([&, t] {
            ok[t] = recip_division_exact_range(b, (uint32_t)((uint64_t)total * t / nt),
                                               (uint32_t)((uint64_t)total * (t + 1) / nt));
        });
    for (auto& th : pool) th.join();
    bool exact = true;
    for (char v : ok) exact = exact && v;
    known.emplace_back(key, exact);
    return exact;
}

DevParams to_device(const fe_params& p, uint32_t n, uint32_t T, uint32_t table_base,
                    uint32_t first) {
    DevParams d;
    std::memset(&d, 0, sizeof d);
    d.radius = p.particle_radius;
    d.mass = p.particle_mass;
    d.h = p.smoothing_radius;
    d.inv_h = 1.0f / p.smoothing_radius;
    d.h_recip_exact = recip_division_exact(p.smoothing_radius) ? 1u : 0u;
    d.rho0 = p.target_density;
    d.visc = p.viscosity;
    d.omega = p.relax_factor;
    d.dt = p.dt;
    d.gx = p.gravity[0];
    d.gy = p.gravity[1];
    d.gz = p.gravity[2];
    d.bminx = p.box_min[0];
    d.bminy = p.box_min[1];
    d.bminz = p.box_min[2];
    d.bmaxx = p.box_max[0];
    d.bmaxy = p.box_max[1];
    d.bmaxz = p.box_max[2];
    d.n = n;
    d.T = T;
    d.table_base = table_base;
    d.first = first;
    d.k_rho = p.density_solver_iterations;
    d.k_div = p.divergence_solver_iterations;
    d.use_cfl = p.use_cfl;
    d.use_thr = p.use_solver_error_threshold;
    d.eta_d_pct = p.density_error_pct;
    d.eta_v_pct = p.divergence_error_pct;
    d.cfl_lambda = p.cfl_lambda;
    d.cfl_min = p.cfl_min_dt;
    d.cfl_max = p.cfl_max_dt;
    d.cfl_growth = p.cfl_growth;
    d.mode = p.mode;
    d.solver = p.solver;
    d.tol_d = p.density_tolerance;
    d.tol_v = p.divergence_tolerance;
    d.min_it = p.min_iterations;
    d.max_it = p.max_iterations;
    d.warm = p.warm_start;
    return d;
}

}  // namespace

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
struct GraphEntry {
    uint64_t key;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
};

struct fe_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t n = 0, T = 0;  // particles, table slots (all scenes)
    std::vector<fe_params> params;  // host copy per scene
    std::vector<DevParams> dparams;
    Bufs B;
    uint32_t* tmp_keys = nullptr;
    uint32_t* tmp_vals = nullptr;
    uint32_t* sort_scratch = nullptr;
    uint4* upart = nullptr;
    uint32_t key_bits = 32;
    bool prepared = false;
    bool initialized = false;
    uint32_t last_substeps = 0;  // substeps of the last fe_step (fe_stats.substeps)
    std::vector<void*> allocations;
    std::vector<GraphEntry> graphs;
    SceneState* h_state = nullptr;   // pinned
    GlobalState* h_global = nullptr; // pinned
    // learned warm start / capture
    fe_model* model = nullptr;       // attached, not owned
    LearnArgs L{};
    bool capture = false;
    // test hook fe_debug_trace_learned: per solve slot, the network's input
    // rows (n x 32 B) and outputs (n x 8 B) as the warm start used them
    unsigned char* trace = nullptr;
    uint32_t trace_slots = 0, trace_cap = 0;

    // density splat: headless grid and the non-zero taps of the splat kernel
    uint32_t* splat_grid = nullptr;
    size_t splat_cap = 0;          // voxels allocated
    int splat_res[3] = {0, 0, 0};  // resolution of the last splat
    int4* splat_taps = nullptr;
    uint32_t splat_ntaps = 0;
    uint32_t* splat_hist = nullptr;    // particles per centre voxel
    size_t splat_hist_cap = 0;

    // raymarched image and its sky
    float4* sky = nullptr;
    size_t sky_cap = 0;
    int sky_w = 0, sky_h = 0;
    float4* image = nullptr;
    size_t image_cap = 0;
    int image_w = 0, image_h = 0;

    // fe_download_async: two device snapshots, the copy stream, and which
    // ticket each snapshot slot serves (0: none)
    cudaStream_t copy_stream = nullptr;
    void* snap[2] = {nullptr, nullptr};
    size_t snap_cap = 0;
    cudaEvent_t snap_ready[2] = {nullptr, nullptr};
    // fe_read_stats_async: two mapped host snapshots and their events
    StatsSnapshot* stats_host = nullptr;     // page-locked, mapped, 2 slots
    StatsSnapshot* stats_dev = nullptr;      // the same memory as the device sees it
    cudaEvent_t stats_done[2] = {nullptr, nullptr};
    uint64_t stats_tickets = 0;
    cudaEvent_t copy_done[2] = {nullptr, nullptr};
    uint64_t tickets = 0;
    uint64_t slot_ticket[2] = {0, 0};

    // tuned shapes (fe_autotune / fe_set_tuning)
    RadixConfig radix_cfg = kRadixDefault;
    int mlp_ctas = mlp::kInferDefaultCtasPerSm;
    // neighbour kernels, per FE_NBR_* group: threads per block, persistent
    uint32_t nbr_threads[FE_NBR_GROUPS] = {256, 256, 256, 256};
    uint32_t nbr_persistent[FE_NBR_GROUPS] = {0, 0, 0, 0};
    int num_sms = 148;

    bool learned() const { return params[0].warm_start == FE_WARM_LEARNED && model != nullptr; }
    bool carries() const { return L.carry != nullptr && (learned() || capture); }

    uint32_t sort_algorithm() const { return params[0].sort_algorithm; }
    bool fixed_mode() const { return params[0].mode == FE_MODE_FIXED; }
};

namespace {

// Test hooks (fe_debug_fail_allocation, fe_debug_poison_allocations).
std::atomic<uint32_t> g_fail_countdown{0};
std::atomic<int> g_poison{0};

template <class T>
fe_status dev_alloc(fe_ctx* c, T** out, size_t count) {
    void* p = nullptr;
    size_t bytes = std::max<size_t>(count * sizeof(T), 16);
    uint32_t k = g_fail_countdown.load();
    while (k != 0 && !g_fail_countdown.compare_exchange_weak(k, k - 1)) {
    }
    if (k == 1) {
        set_error("device allocation of %zu bytes failed (injected)", bytes);
        return FE_ERR_OUT_OF_MEMORY;
    }
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        set_error("cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
        return FE_ERR_OUT_OF_MEMORY;
    }
    if (g_poison.load() && cudaMemset(p, 0xFF, bytes) != cudaSuccess) {
        cudaFree(p);
        set_error("poisoning a new allocation failed");
        return FE_ERR_CUDA;
    }
    c->allocations.push_back(p);
    *out = static_cast<T*>(p);
    return FE_OK;
}

void release(fe_ctx* c) {
    if (!c) return;
    if (c->device >= 0) cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto& g : c->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
    }
    c->graphs.clear();
    for (void* p : c->allocations) cudaFree(p);
    c->allocations.clear();
    if (c->h_state) cudaFreeHost(c->h_state);
    if (c->h_global) cudaFreeHost(c->h_global);
    if (c->copy_stream) {
        cudaStreamSynchronize(c->copy_stream);
        cudaStreamDestroy(c->copy_stream);
    }
    for (int k = 0; k < 2; ++k) {
        if (c->snap_ready[k]) cudaEventDestroy(c->snap_ready[k]);
        if (c->copy_done[k]) cudaEventDestroy(c->copy_done[k]);
        if (c->stats_done[k]) cudaEventDestroy(c->stats_done[k]);
    }
    if (c->stats_host) cudaFreeHost(c->stats_host);
    if (c->stream) cudaStreamDestroy(c->stream);
}

dim3 chunk_grid(const fe_ctx* c) { return dim3(c->B.n_chunks); }

// The instantiation of a neighbour kernel for a block size (128, 256, 512)
// and persistence.
template <class... KArgs>
auto pick(void (*k128)(KArgs...), void (*k256)(KArgs...), void (*k512)(KArgs...), uint32_t t)
    -> void (*)(KArgs...) {
    return t == 128 ? k128 : t == 512 ? k512 : k256;
}
#define NBR_KERNEL_P(name, threads, persist)                                           \
    ((persist) ? pick(name<128, true>, name<256, true>, name<512, true>, (threads))   \
               : pick(name<128, false>, name<256, false>, name<512, false>, (threads)))
#define NBR_KERNEL(name, g) NBR_KERNEL_P(name, c->nbr_threads[g], c->nbr_persistent[g])

// Grid of a neighbour kernel of group g: one block per chunk step (a chunk,
// two chunks for 512 threads), or, persistent, as many blocks as fit on the
// GPU at once (each then strides over the chunk table).
struct NbrGrid {
    dim3 grid, block;
};
NbrGrid nbr_grid(const fe_ctx* c, int g, const void* func) {
    const uint32_t t = c->nbr_threads[g];
    const uint32_t per = t >= (uint32_t)kBlock ? t / kBlock : 1u;
    uint32_t blocks = (c->B.n_chunks + per - 1) / per;
    if (c->nbr_persistent[g]) {
        int resident = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, func, (int)t, 0) !=
                cudaSuccess ||
            resident < 1)
            resident = 1;
        blocks = std::min<uint32_t>(blocks, (uint32_t)resident * (uint32_t)c->num_sms);
    }
    return {dim3(blocks > 0 ? blocks : 1), dim3(t)};
}
dim3 flat_grid(uint32_t n) { return dim3((n + kBlock - 1) / kBlock); }

// ---------------------------------------------------------------------------
// Recording of the passes (shared by the stage calls and the frame graph).
// ---------------------------------------------------------------------------
fe_status rec_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return FE_OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? FE_ERR_OUT_OF_MEMORY : FE_ERR_CUDA;
}

#define REC(expr)                                              \
    do {                                                       \
        fe_status s_ = rec_check((expr), #expr);               \
        if (s_ != FE_OK) return s_;                            \
    } while (0)

// A neighbour kernel of group g with its tuned shape.
template <class... KArgs, class... Args>
fe_status rec_nbr(fe_ctx* c, Recorder& R, int g, void (*func)(KArgs...), Args... args) {
    const NbrGrid G = nbr_grid(c, g, (const void*)func);
    REC(R.k(func, G.grid, G.block, args...));
    return FE_OK;
}

// (128 or 256 threads: the shapes fe_set_tuning accepts for this group)
fe_status rec_density_alpha(fe_ctx* c, Recorder& R) {
    const int g = FE_NBR_DENSITY_ALPHA;
    const uint32_t t = c->nbr_threads[g];
    return rec_nbr(c, R, g,
                   c->nbr_persistent[g]
                       ? pick(k_density_alpha<128, true>, k_density_alpha<256, true>,
                              k_density_alpha<256, true>, t)
                       : pick(k_density_alpha<128, false>, k_density_alpha<256, false>,
                              k_density_alpha<256, false>, t),
                   c->B);
}

// density_alpha that also sums the divergence source (the mid-substep
// neighbour search's pass); with the learned state it also emits the
// divergence solve's features.
fe_status rec_density_alpha_div(fe_ctx* c, Recorder& R) {
    const int g = FE_NBR_DENSITY_ALPHA;
    const uint32_t t = c->nbr_threads[g];
    if (c->carries())
        return rec_nbr(c, R, g,
                       c->nbr_persistent[g]
                           ? pick(k_density_alpha_div_learn<128, true>,
                                  k_density_alpha_div_learn<256, true>,
                                  k_density_alpha_div_learn<256, true>, t)
                           : pick(k_density_alpha_div_learn<128, false>,
                                  k_density_alpha_div_learn<256, false>,
                                  k_density_alpha_div_learn<256, false>, t),
                       c->B, c->fixed_mode() ? 1 : 0, c->L);
    return rec_nbr(c, R, g,
                   c->nbr_persistent[g]
                       ? pick(k_density_alpha_div<128, true>, k_density_alpha_div<256, true>,
                              k_density_alpha_div<256, true>, t)
                       : pick(k_density_alpha_div<128, false>, k_density_alpha_div<256, false>,
                              k_density_alpha_div<256, false>, t),
                   c->B, c->fixed_mode() ? 1 : 0);
}

// Whether a shape may run group g.
bool nbr_shape_ok(int g, uint32_t threads, uint32_t persistent) {
    if (persistent > 1) return false;
    if (g == FE_NBR_PRESSURE_UPDATE) return threads == (uint32_t)kBlock;
    if (g == FE_NBR_DENSITY_ALPHA) return threads == 128 || threads == 256;
    return threads == 128 || threads == 256 || threads == 512;
}

fe_status rec_force(fe_ctx* c, Recorder& R, int which) {
    return rec_nbr(c, R, FE_NBR_PRESSURE_FORCE,
                   NBR_KERNEL(k_pressure_force, FE_NBR_PRESSURE_FORCE), c->B, which);
}

fe_status rec_update(fe_ctx* c, Recorder& R, int which, cudaGraphConditionalHandle h,
                     int use_handle) {
    return rec_nbr(c, R, FE_NBR_PRESSURE_UPDATE, k_pressure_update, c->B, which, h, use_handle);
}

// viscosity and the two source passes (plain or with the learned state)
fe_status rec_list_pass(fe_ctx* c, Recorder& R, int pass) {
    const int g = FE_NBR_LIST_PASSES;
    const int fixed = c->fixed_mode() ? 1 : 0;
    switch (pass) {
        case 0: return rec_nbr(c, R, g, NBR_KERNEL(k_viscosity, g), c->B);
        case 1:
            if (c->carries())
                return rec_nbr(c, R, g, NBR_KERNEL(k_density_source_learn, g), c->B, c->L);
            return rec_nbr(c, R, g, NBR_KERNEL(k_density_source, g), c->B);
        default:
            return rec_nbr(c, R, g, NBR_KERNEL(k_divergence_source, g), c->B, fixed);
    }
}

// NeighborSearch::execute (neighbor_search.rs:176-231).  take: end with the
// copy that makes the gathered pressures (FIXED mode) and learned carry
// current; the substep's search leaves it to density_alpha_div, which runs
// next and does it per particle.
fe_status rec_neighbor_search(fe_ctx* c, Recorder& R, bool take = true) {
    Bufs B = c->B;
    const bool radix = c->sort_algorithm() == FE_SORT_RADIX;
    uint32_t passes = radix_passes(c->key_bits, c->radix_cfg.digit_bits);
    // Radix ping-pongs through tmp; hashing into tmp when the pass count is
    // odd leaves the sorted entries in keys/vals.
    Bufs H = B;
    if (radix && (passes % 2 == 1)) {
        H.keys = c->tmp_keys;
        H.vals = c->tmp_vals;
    }
    REC(R.k(k_hash, chunk_grid(c), dim3(kBlock), H));
    SortLaunch L = R.sort_launch();
    if (radix) {
        bool in_tmp = false;
        REC(radix_sort(L, H.keys, H.vals, H.keys == B.keys ? c->tmp_keys : B.keys,
                       H.vals == B.vals ? c->tmp_vals : B.vals, c->n, c->key_bits,
                       c->sort_scratch, &B.G->flags, &in_tmp, c->radix_cfg));
    } else {
        REC(bitonic_sort(L, B.keys, B.vals, c->T));
    }
    REC(R.k(k_fill_cells, dim3(std::min<uint32_t>((c->T + 255) / 256, 148 * 8)), dim3(256),
            B.cells, (size_t)c->T));
    REC(R.k(k_offsets, flat_grid(c->n), dim3(kBlock), B));
    const int fixed = c->fixed_mode() ? 1 : 0;
    if (c->carries()) {
        // the learned state rides along with the gather and the copy-back
        REC(R.k(k_reorder_carry, flat_grid(c->n), dim3(kBlock), B, fixed, c->L));
        if (!take) return FE_OK;
        if (fixed)
            REC(R.k(k_take_pressure_carry, flat_grid(c->n), dim3(kBlock), B, c->L));
        else
            REC(R.k(k_carry_take, flat_grid(c->n), dim3(kBlock), B, c->L));
    } else {
        REC(R.k(k_reorder, flat_grid(c->n), dim3(kBlock), B, fixed));
        if (fixed && take) REC(R.k(k_take_pressure, flat_grid(c->n), dim3(kBlock), B));
    }
    return FE_OK;
}

fe_status rec_simple(fe_ctx* c, Recorder& R, void (*kern)(Bufs)) {
    REC(R.k(kern, chunk_grid(c), dim3(kBlock), c->B));
    return FE_OK;
}

fe_status rec_stats(fe_ctx* c, Recorder& R) {
    REC(R.k(k_stats, chunk_grid(c), dim3(kBlock), c->B, c->fixed_mode() ? 1 : 0, c->upart));
    if (c->B.n_scenes > 1)  // the per-scene finish, one block per scene
        REC(R.k(k_stats_finish, dim3(c->B.n_scenes), dim3(kBlock), c->B, c->upart));
    return FE_OK;
}

// One Jacobi solve.  Graph: begin kernel, WHILE node {force, update, the
// per-scene finish when the context holds several scenes, guard}, end
// kernel.  Eager: the same kernels with a host loop on the device flag.
fe_status rec_solve(fe_ctx* c, Recorder& R, int which) {
    Bufs B = c->B;
    if (!R.graph) {
        REC(R.k(k_solve_begin, dim3(1), dim3(32), B, which, (cudaGraphConditionalHandle)0, 0));
        for (uint32_t guard = 0; guard < 200001; ++guard) {
            uint32_t cond = 0;
            REC(cudaMemcpyAsync(&cond, &B.G->cond[which], sizeof cond, cudaMemcpyDeviceToHost,
                                R.stream));
            REC(cudaStreamSynchronize(R.stream));
            if (!cond) break;
            fe_status st;
            if ((st = rec_force(c, R, which))) return st;
            if ((st = rec_update(c, R, which, (cudaGraphConditionalHandle)0, 0))) return st;
            if (B.n_scenes > 1)
                REC(R.k(k_solve_finish, dim3(B.n_scenes), dim3(kBlock), B, which,
                        (cudaGraphConditionalHandle)0, 0));
        }
        REC(R.k(k_solve_end, dim3(1), dim3(32), B, which));
        return FE_OK;
    }
    cudaGraphConditionalHandle h;
    REC(cudaGraphConditionalHandleCreate(&h, R.root, 0, 0));
    REC(R.k(k_solve_begin, dim3(1), dim3(32), B, which, h, 1));
    // cudaGraphNodeParams has no default constructor (it holds a union);
    // zeroed storage gives the required all-zero reserved fields.
    alignas(cudaGraphNodeParams) unsigned char cp_storage[sizeof(cudaGraphNodeParams)] = {};
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cp_storage);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    REC(cudaGraphAddNode(&node, R.graph, R.last ? &R.last : nullptr, R.last ? 1 : 0, &cp));
    Recorder body;
    body.stream = R.stream;
    body.graph = cp.conditional.phGraph_out[0];
    body.root = R.root;
    fe_status st;
    if ((st = rec_force(c, body, which))) return st;
    if ((st = rec_update(c, body, which, h, 1))) return st;
    if (B.n_scenes > 1)  // the per-scene finish, one block per scene
        REC(body.k(k_solve_finish, dim3(B.n_scenes), dim3(kBlock), B, which, h, 1));
    REC(body.k(k_loop_guard, dim3(1), dim3(32), B, which, h));
    R.last = node;
    REC(R.k(k_solve_end, dim3(1), dim3(32), B, which));
    return FE_OK;
}

// Network inference on the feature rows (tensor-core kernel of fe_mlp.cu),
// which also starts solve `which` from its output (warm_apply_particle).
fe_status rec_mlp(fe_ctx* c, Recorder& R, int which) {
    mlp::KernelLaunch KL;
    REC(mlp::infer_launch(c->n, c->num_sms, &KL, c->mlp_ctas, true));
    mlp::Params P = c->model->params();
    const __nv_bfloat16* X = static_cast<const __nv_bfloat16*>(c->L.xb);
    float* out = c->L.out;
    uint32_t n = c->n;
    uint32_t* flags = &c->B.G->flags;
    mlp::ApplyArgs A{c->B, c->L, which};
    void* args[] = {&P, &X, &out, &n, &flags, &A};
    REC(R.launch(KL.func, KL.grid, KL.block, KL.smem, args));
    return FE_OK;
}

// Test hook: records the network's input rows and outputs of solve slot
// `slot` (2 x substep + which) into the trace buffer.
constexpr size_t kTraceBytesPerParticle = 16 * 2 + 2 * 4;
fe_status rec_trace(fe_ctx* c, Recorder& R, uint32_t slot) {
    if (slot >= c->trace_slots) return FE_OK;
    unsigned char* base = c->trace + (size_t)slot * c->n * kTraceBytesPerParticle;
    REC(R.copy(base, c->L.xb, (size_t)c->n * 32));
    REC(R.copy(base + (size_t)c->n * 32, c->L.out, (size_t)c->n * 8));
    return FE_OK;
}

// One substep of Renderer::step (renderer/mod.rs:289-337); k = its index in
// the frame.
fe_status rec_substep(fe_ctx* c, Recorder& R, uint32_t k, bool last) {
    Bufs B = c->B;
    const int fixed = c->fixed_mode() ? 1 : 0;
    fe_status s;
    if ((s = rec_list_pass(c, R, 0))) return s;
    if ((s = rec_list_pass(c, R, 1))) return s;
    if (c->learned()) {   // the network, which also starts the density solve
        if ((s = rec_mlp(c, R, 0))) return s;
        if ((s = rec_trace(c, R, 2 * k))) return s;
    }
    if ((s = rec_solve(c, R, 0))) return s;
    if (c->carries())
        REC(R.k(k_pressure_integration_learn, chunk_grid(c), dim3(kBlock), B, c->L));
    else if ((s = rec_simple(c, R, k_pressure_integration)))
        return s;
    if ((s = rec_neighbor_search(c, R, false))) return s;
    if ((s = rec_density_alpha_div(c, R))) return s;
    if (c->learned()) {   // ... and the divergence solve
        if ((s = rec_mlp(c, R, 1))) return s;
        if ((s = rec_trace(c, R, 2 * k + 1))) return s;
    }
    if ((s = rec_solve(c, R, 1))) return s;
    if (last) {   // the frame's stats ride in its last divergence integration
        if (c->carries())
            REC(R.k(k_divergence_integration_stats_learn, chunk_grid(c), dim3(kBlock), B, fixed,
                    c->L, c->upart));
        else
            REC(R.k(k_divergence_integration_stats, chunk_grid(c), dim3(kBlock), B, fixed,
                    c->upart));
        if (B.n_scenes > 1)  // the per-scene finish, one block per scene
            REC(R.k(k_stats_finish, dim3(B.n_scenes), dim3(kBlock), B, c->upart));
    } else if (c->carries()) {
        REC(R.k(k_divergence_integration_learn, chunk_grid(c), dim3(kBlock), B, fixed, c->L));
    } else {
        REC(R.k(k_divergence_integration, chunk_grid(c), dim3(kBlock), B, fixed));
    }
    REC(R.k(k_count_substep, dim3((B.n_scenes + 63) / 64), dim3(64), B));
    return FE_OK;
}

fe_status rec_frame(fe_ctx* c, Recorder& R, uint32_t n_substeps, bool init) {
    fe_status s;
    REC(R.k(k_frame_prologue, dim3((c->B.n_scenes + 63) / 64), dim3(64), c->B));
    if (init) {
        if ((s = rec_neighbor_search(c, R))) return s;
        if ((s = rec_density_alpha(c, R))) return s;
    }
    for (uint32_t k = 0; k < n_substeps; ++k)
        if ((s = rec_substep(c, R, k, k + 1 == n_substeps))) return s;
    return n_substeps ? FE_OK : rec_stats(c, R);
}

fe_status need_prepared(fe_ctx* c, const char* what) {
    if (!c) {
        set_error("%s: context is NULL", what);
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (!c->prepared) {
        set_error("%s: call prepare() before execute()", what);
        return FE_ERR_NOT_PREPARED;
    }
    if (cudaSetDevice(c->device) != cudaSuccess) {
        set_error("%s: cudaSetDevice failed", what);
        return FE_ERR_CUDA;
    }
    return FE_OK;
}

Recorder eager(fe_ctx* c) {
    Recorder R;
    R.stream = c->stream;
    return R;
}

fe_status upload_params(fe_ctx* c) {
    FE_CUDA(cudaMemcpyAsync(c->B.P, c->dparams.data(), sizeof(DevParams) * c->dparams.size(),
                            cudaMemcpyHostToDevice, c->stream));
    return FE_OK;
}

fe_status run_refresh_pr(fe_ctx* c) {
    Recorder R = eager(c);
    REC(R.k(k_refresh_pr, chunk_grid(c), dim3(kBlock), c->B));
    return FE_OK;
}

// Device location of a field: base pointer, element size and the distance
// between consecutive elements (position_b and the pressure acceleration are
// interleaved in 32-byte records).  Returns the host-side byte count.
size_t field_bytes(const fe_ctx* c, fe_field f, void** dptr, size_t* elem, size_t* pitch) {
    *pitch = 0;
    size_t n = c->n;
    switch (f) {
        case FE_FIELD_POSITION_A: *dptr = c->B.pos_a; *elem = 16; break;
        case FE_FIELD_POSITION_B: *dptr = c->B.pos_b; *elem = 16; break;
        case FE_FIELD_VELOCITY_A: *dptr = c->B.pa + 1; *elem = 16; *pitch = 32; break;
        case FE_FIELD_VELOCITY_B: *dptr = c->B.pv + 1; *elem = 16; *pitch = 32; break;
        case FE_FIELD_DENSITY: *dptr = c->B.rho; *elem = 4; break;
        case FE_FIELD_FACTOR: *dptr = c->B.alpha; *elem = 4; break;
        case FE_FIELD_SOURCE_TERM: *dptr = c->B.src; *elem = 4; break;
        case FE_FIELD_PRESSURE: *dptr = c->B.prs; *elem = 4; break;
        case FE_FIELD_PRESSURE_ACCEL: *dptr = c->B.rec + 1; *elem = 16; *pitch = 32; break;
        case FE_FIELD_ENTRY_HASH: *dptr = c->B.keys; *elem = 4; n = c->T; break;
        case FE_FIELD_ENTRY_INDEX: *dptr = c->B.vals; *elem = 4; n = c->T; break;
        case FE_FIELD_GRID_START: *dptr = c->B.cells; *elem = 4; *pitch = 8; n = c->T; break;
        case FE_FIELD_STATS: *dptr = c->B.S; *elem = 4; n = 3; break;
        case FE_FIELD_DENSITY_GRID:
            if (!c->splat_grid) {
                set_error("no density grid yet: call fe_density_splat first");
                return 0;
            }
            *dptr = c->splat_grid;
            *elem = 4;
            n = (size_t)c->splat_res[0] * c->splat_res[1] * c->splat_res[2];
            break;
        case FE_FIELD_IMAGE:
            if (!c->image) {
                set_error("no image yet: call fe_raymarch first");
                return 0;
            }
            *dptr = c->image;
            *elem = 16;
            n = (size_t)c->image_w * c->image_h;
            break;
        default: return 0;
    }
    if (*pitch == 0) *pitch = *elem;
    return n * *elem;
}

uint64_t graph_key(const fe_ctx* c, uint32_t n_substeps, bool init) {
    return (uint64_t)n_substeps | ((uint64_t)init << 32) | ((uint64_t)c->sort_algorithm() << 33) |
           ((uint64_t)c->fixed_mode() << 34) | ((uint64_t)c->learned() << 35) |
           ((uint64_t)c->capture << 36) | ((uint64_t)c->trace_slots << 40);
}

fe_status get_graph(fe_ctx* c, uint32_t n_substeps, bool init, cudaGraphExec_t* out) {
    uint64_t key = graph_key(c, n_substeps, init);
    for (auto& g : c->graphs)
        if (g.key == key) {
            *out = g.exec;
            return FE_OK;
        }
    GraphEntry g{key, nullptr, nullptr};
    FE_CUDA(cudaGraphCreate(&g.graph, 0));
    Recorder R;
    R.stream = c->stream;
    R.graph = g.graph;
    R.root = g.graph;
    fe_status s = rec_frame(c, R, n_substeps, init);
    if (s != FE_OK) {
        cudaGraphDestroy(g.graph);
        return s;
    }
    cudaError_t e = cudaGraphInstantiate(&g.exec, g.graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g.graph);
        set_error("cudaGraphInstantiate: %s", cudaGetErrorString(e));
        return FE_ERR_CUDA;
    }
    if (c->graphs.size() >= 8) {
        cudaStreamSynchronize(c->stream);
        cudaGraphExecDestroy(c->graphs.front().exec);
        cudaGraphDestroy(c->graphs.front().graph);
        c->graphs.erase(c->graphs.begin());
    }
    c->graphs.push_back(g);
    *out = g.exec;
    return FE_OK;
}

// fe_stats of one scene from its device state, the global flags and its dt.
void stats_from(const fe_ctx* c, const SceneState& S, const GlobalState& G, float dt, uint32_t n_p,
                fe_stats* out) {
    std::memset(out, 0, sizeof *out);
    out->max_speed_bits = S.stats[0];
    out->density_error_fp = S.stats[1];
    out->divergence_error_fp = S.stats[2];
    std::memcpy(&out->max_speed, &S.stats[0], 4);
    float n = (float)n_p;
    out->avg_density_error = (float)S.stats[1] / (1.0f * n);
    out->avg_divergence_error = (float)S.stats[2] / (10.0f * n);
    out->dt = dt;
    out->avg_density_error_f64 = S.stats_f64[0];
    out->avg_divergence_error_f64 = S.stats_f64[1];
    out->density_residual = S.last_metric[0];
    out->divergence_residual = S.last_metric[1];
    out->density_residual_max = S.last_metric_max[0];
    out->divergence_residual_max = S.last_metric_max[1];
    out->density_iterations = S.last_iters[0];
    out->divergence_iterations = S.last_iters[1];
    out->total_density_iterations = S.total_iters[0];
    out->total_divergence_iterations = S.total_iters[1];
    out->substeps = c->last_substeps;
    uint32_t flags = G.flags;  // cap hit and look-back timeout: any scene
    if (S.nonfinite) flags |= 0x8u;
    out->flags = flags;
}

fe_status collect_stats(fe_ctx* c, fe_stats* out, uint32_t scene = 0) {
    FE_CUDA(cudaMemcpyAsync(c->h_state + scene, c->B.S + scene, sizeof(SceneState),
                            cudaMemcpyDeviceToHost, c->stream));
    FE_CUDA(cudaMemcpyAsync(c->h_global, c->B.G, sizeof(GlobalState), cudaMemcpyDeviceToHost,
                            c->stream));
    DevParams dp;
    FE_CUDA(cudaMemcpyAsync(&dp, c->B.P + scene, sizeof dp, cudaMemcpyDeviceToHost, c->stream));
    FE_CUDA(cudaStreamSynchronize(c->stream));
    stats_from(c, c->h_state[scene], *c->h_global, dp.dt, dp.n, out);
    // host-side mirror of the device dt
    c->params[scene].dt = dp.dt;
    return FE_OK;
}


}  // namespace

void fe_set_error_message(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    set_error_v(fmt, ap);
    va_end(ap);
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

uint32_t fe_abi_version(void) { return FE_ABI_VERSION; }

const char* fe_status_string(fe_status s) {
    switch (s) {
        case FE_OK: return "FE_OK";
        case FE_ERR_INVALID_ARGUMENT: return "FE_ERR_INVALID_ARGUMENT";
        case FE_ERR_NOT_PREPARED: return "FE_ERR_NOT_PREPARED";
        case FE_ERR_CUDA: return "FE_ERR_CUDA";
        case FE_ERR_OUT_OF_MEMORY: return "FE_ERR_OUT_OF_MEMORY";
        case FE_ERR_NON_FINITE: return "FE_ERR_NON_FINITE";
        case FE_ERR_ITERATION_CAP: return "FE_ERR_ITERATION_CAP";
        case FE_ERR_TIMEOUT: return "FE_ERR_TIMEOUT";
        case FE_ERR_NO_DEVICE: return "FE_ERR_NO_DEVICE";
        case FE_ERR_CAPACITY: return "FE_ERR_CAPACITY";
        case FE_ERR_UNSUPPORTED: return "FE_ERR_UNSUPPORTED";
    }
    return "FE_ERR_UNKNOWN";
}

const char* fe_last_error(void) { return g_last_error.c_str(); }

void fe_default_params(fe_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof *p);
    const float radius = 0.020f;
    const float spacing = radius * 2.0f;
    p->particle_radius = radius;
    p->particle_mass = 1000.0f * (spacing * spacing * spacing);
    p->smoothing_radius = radius * 4.0f;
    p->target_density = 1000.0f;
    p->viscosity = 0.15f;
    p->relax_factor = 0.5f;
    p->dt = 0.005f;
    p->density_solver_iterations = 4;
    p->divergence_solver_iterations = 4;
    p->gravity[1] = -9.81f;
    p->box_min[0] = -1.5f;
    p->box_min[1] = 0.0f;
    p->box_min[2] = -1.0f;
    p->box_max[0] = 0.8f;
    p->box_max[1] = 4.0f;
    p->box_max[2] = 1.0f;
    p->grid_res[0] = p->grid_res[1] = p->grid_res[2] = 128;
    p->sort_algorithm = FE_SORT_RADIX;
    p->density_error_pct = 0.1f;
    p->divergence_error_pct = 0.5f;
    p->cfl_lambda = 0.4f;
    p->cfl_min_dt = 0.001f;
    p->cfl_max_dt = 0.05f;
    p->cfl_growth = 1.1f;
    p->mode = FE_MODE_REFERENCE;
    p->solver = FE_SOLVER_FIXED_ITERS;
    p->density_tolerance = 0.001f;
    p->divergence_tolerance = 0.001f;
    p->min_iterations = 2;
    p->max_iterations = 100;
    p->warm_start = FE_WARM_REFERENCE;
}

fe_status fe_validate_params(const fe_params* p) { return validate(p); }

namespace {

// The scenes of one context must share what is recorded once per frame for
// all of them: the sort (bitonic is single-scene), the buffer pairing mode
// and the warm start.  Everything else (physics, time step, solver and its
// tolerance) is per scene.
fe_status check_batch_uniform(const fe_params& a, const fe_params& b, uint32_t n_scenes) {
    if (n_scenes > 1 && (a.sort_algorithm != FE_SORT_RADIX || b.sort_algorithm != FE_SORT_RADIX)) {
        set_error("bitonic sort is single-scene only");
        return FE_ERR_UNSUPPORTED;
    }
    if (a.mode != b.mode || a.warm_start != b.warm_start || a.sort_algorithm != b.sort_algorithm) {
        set_error("scenes of one context must share mode, warm_start and sort_algorithm");
        return FE_ERR_INVALID_ARGUMENT;
    }
    return FE_OK;
}

// A context over n_scenes independent scenes laid out back to back: scene s
// owns particles [first_s, first_s + n_s), hash-table slots
// [base_s, base_s + T_s) with T_s = next_pow2(n_s), and ceil(n_s / 256)
// chunks of the chunk table.  Keys are base_s + hash_s, so one stable sort
// of all keys orders every scene by (hash, index) within its own range, and
// each scene's chunks, reductions and solver control are those it has alone.
fe_status create_ctx(const fe_params* params, const uint32_t* counts, uint32_t n_scenes,
                     const float* pos_xyz, const float* vel_xyz, int device, fe_ctx** out) {
    if (!out) {
        set_error("out is NULL");
        return FE_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    if (!params || !counts || n_scenes == 0) {
        set_error("params and counts must be given for at least one scene");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (n_scenes > FE_MAX_SCENES) {
        set_error("%u scenes above FE_MAX_SCENES (%u)", n_scenes, FE_MAX_SCENES);
        return FE_ERR_CAPACITY;
    }
    fe_status s;
    uint64_t n64 = 0, t64 = 0;
    for (uint32_t k = 0; k < n_scenes; ++k) {
        if ((s = validate(&params[k])) != FE_OK) return s;
        if ((s = check_batch_uniform(params[0], params[k], n_scenes)) != FE_OK) return s;
        if (counts[k] == 0 || counts[k] > FE_MAX_PARTICLES) {
            set_error("scene %u: particle count %u outside 1..%u", k, counts[k], FE_MAX_PARTICLES);
            return counts[k] == 0 ? FE_ERR_INVALID_ARGUMENT : FE_ERR_CAPACITY;
        }
        n64 += counts[k];
        t64 += next_pow2(counts[k]);
    }
    if (n64 > FE_MAX_PARTICLES || t64 > (1ull << 31)) {
        set_error("%llu particles (%llu table slots) above FE_MAX_PARTICLES",
                  (unsigned long long)n64, (unsigned long long)t64);
        return FE_ERR_CAPACITY;
    }
    const uint32_t n = (uint32_t)n64;
    if (!pos_xyz) {
        set_error("pos_xyz is NULL");
        return FE_ERR_INVALID_ARGUMENT;
    }
    for (size_t i = 0; i < (size_t)n * 3; ++i)
        if (!std::isfinite(pos_xyz[i]) || (vel_xyz && !std::isfinite(vel_xyz[i]))) {
            set_error("non-finite position or velocity at particle %zu", i / 3);
            return FE_ERR_NON_FINITE;
        }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        set_error("no CUDA device %d", device);
        return FE_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
        set_error("device %d is not sm_100 (Blackwell)", device);
        return FE_ERR_NO_DEVICE;
    }
    FE_CUDA(cudaSetDevice(device));
    fe_ctx* c = new fe_ctx();
    c->device = device;
    c->n = n;
    c->T = (uint32_t)t64;
    c->key_bits = log2_ceil(c->T);
    if (c->key_bits == 0) c->key_bits = 1;
    c->params.assign(params, params + n_scenes);
    std::vector<uint4> hc;
    {
        uint32_t first = 0, base = 0;
        for (uint32_t k = 0; k < n_scenes; ++k) {
            const uint32_t nk = counts[k], tk = next_pow2(nk);
            c->dparams.push_back(to_device(params[k], nk, tk, base, first));
            for (uint32_t q = 0; q * kBlock < nk; ++q)
                hc.push_back(make_uint4(first + q * kBlock, std::min<uint32_t>(kBlock, nk - q * kBlock),
                                        k, (uint32_t)hc.size()));
            first += nk;
            base += tk;
        }
    }
    auto fail = [&](fe_status st) {
        release(c);
        delete c;
        return st;
    };
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("cudaStreamCreate failed");
        return fail(FE_ERR_CUDA);
    }
    if (cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device) !=
            cudaSuccess ||
        c->num_sms < 1)
        c->num_sms = 1;
    Bufs& B = c->B;
    std::memset(&B, 0, sizeof B);
    const uint32_t nchunks = (uint32_t)hc.size();
    B.n_total = n;
    B.T_total = c->T;
    B.n_chunks = nchunks;
    B.n_scenes = n_scenes;
    uint4* chunks_d = nullptr;
    const size_t scratch_words = radix_scratch_words_any(n, c->key_bits);
    if ((s = dev_alloc(c, &B.pos_a, n)) || (s = dev_alloc(c, &B.pos_b, n)) ||
        (s = dev_alloc(c, &B.rec, 2 * (size_t)n)) ||
        (s = dev_alloc(c, &B.pa, 2 * (size_t)n)) || (s = dev_alloc(c, &B.pv, 2 * (size_t)n)) ||
        (s = dev_alloc(c, &B.rho, n)) ||
        (s = dev_alloc(c, &B.alpha, n)) || (s = dev_alloc(c, &B.src, n)) ||
        (s = dev_alloc(c, &B.prs, n)) || (s = dev_alloc(c, &B.prs_tmp, n)) ||
        (s = dev_alloc(c, &B.keys, c->T)) ||
        (s = dev_alloc(c, &B.vals, c->T)) || (s = dev_alloc(c, &B.cells, c->T)) ||
        (s = dev_alloc(c, &B.nbr_count, n)) || (s = dev_alloc(c, &B.nbr, (size_t)kNbrCap * n)) ||
        (s = dev_alloc(c, &chunks_d, nchunks)) || (s = dev_alloc(c, &B.P, n_scenes)) ||
        (s = dev_alloc(c, &B.S, n_scenes)) || (s = dev_alloc(c, &B.G, 1)) ||
        (s = dev_alloc(c, &B.partials, 2 * (size_t)nchunks)) ||
        (s = dev_alloc(c, &c->upart, nchunks)) || (s = dev_alloc(c, &c->tmp_keys, n)) ||
        (s = dev_alloc(c, &c->tmp_vals, n)) ||
        (s = dev_alloc(c, &c->sort_scratch, scratch_words)))
        return fail(s);
    B.chunks = chunks_d;
    if (cudaMallocHost(&c->h_state, sizeof(SceneState) * n_scenes) != cudaSuccess ||
        cudaMallocHost(&c->h_global, sizeof(GlobalState)) != cudaSuccess) {
        set_error("cudaMallocHost failed");
        return fail(FE_ERR_OUT_OF_MEMORY);
    }
    // Initial state (GpuPhysicsData::new): positions w = 1, velocities 0.
    std::vector<float4> h4(n);
    for (uint32_t i = 0; i < n; ++i)
        h4[i] = make_float4(pos_xyz[3 * i], pos_xyz[3 * i + 1], pos_xyz[3 * i + 2], 1.0f);
    auto setup = [&]() -> fe_status {
        FE_CUDA(cudaMemcpy(B.pos_a, h4.data(), (size_t)n * 16, cudaMemcpyHostToDevice));
        for (uint32_t i = 0; i < n; ++i)
            h4[i] = vel_xyz ? make_float4(vel_xyz[3 * i], vel_xyz[3 * i + 1], vel_xyz[3 * i + 2], 0.0f)
                            : make_float4(0, 0, 0, 0);
        FE_CUDA(cudaMemset(B.pa, 0, (size_t)n * 32));
        FE_CUDA(cudaMemcpy2D(B.pa + 1, 32, h4.data(), 16, 16, n, cudaMemcpyHostToDevice));
        FE_CUDA(cudaMemcpy(chunks_d, hc.data(), sizeof(uint4) * nchunks, cudaMemcpyHostToDevice));
        FE_CUDA(cudaMemset(B.rec, 0, (size_t)n * 32));
        FE_CUDA(cudaMemset(B.pos_b, 0, (size_t)n * 16));
        FE_CUDA(cudaMemset(B.pv, 0, (size_t)n * 32));
        for (void* p : {(void*)B.rho, (void*)B.alpha, (void*)B.src, (void*)B.prs,
                        (void*)B.prs_tmp, (void*)B.nbr_count})
            FE_CUDA(cudaMemset(p, 0, (size_t)n * 4));
        FE_CUDA(cudaMemset(B.keys, 0, (size_t)n * 4));
        FE_CUDA(cudaMemset(B.vals, 0, (size_t)n * 4));
        if (c->T > n) {  // sentinel tail of grid_entries (spatial_hash.comp:33-35)
            FE_CUDA(cudaMemset(B.keys + n, 0xFF, (size_t)(c->T - n) * 4));
            FE_CUDA(cudaMemset(B.vals + n, 0xFF, (size_t)(c->T - n) * 4));
        }
        FE_CUDA(cudaMemset(B.cells, 0xFF, (size_t)c->T * 8));
        FE_CUDA(cudaMemset(B.S, 0, sizeof(SceneState) * n_scenes));
        FE_CUDA(cudaMemset(B.G, 0, sizeof(GlobalState)));
        FE_CUDA(cudaMemcpy(B.P, c->dparams.data(), sizeof(DevParams) * n_scenes,
                           cudaMemcpyHostToDevice));
        fe_status st = run_refresh_pr(c);
        if (st != FE_OK) return st;
        FE_CUDA(cudaStreamSynchronize(c->stream));
        return FE_OK;
    };
    if ((s = setup()) != FE_OK) return fail(s);
    *out = c;
    return FE_OK;
}

}  // namespace

fe_status fe_create(const fe_params* params, uint32_t n, const float* pos_xyz,
                    const float* vel_xyz, int device, fe_ctx** out) {
    if (n == 0 || n > FE_MAX_PARTICLES) {
        if (out) *out = nullptr;
        set_error("particle count %u outside 1..%u", n, FE_MAX_PARTICLES);
        return n == 0 ? FE_ERR_INVALID_ARGUMENT : FE_ERR_CAPACITY;
    }
    return create_ctx(params, &n, 1, pos_xyz, vel_xyz, device, out);
}

fe_status fe_batch_create(const fe_params* params, const uint32_t* counts, uint32_t n_scenes,
                          const float* pos_xyz, const float* vel_xyz, int device, fe_ctx** out) {
    return create_ctx(params, counts, n_scenes, pos_xyz, vel_xyz, device, out);
}

fe_status fe_scene_count(const fe_ctx* c, uint32_t* out) {
    if (!c || !out) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    *out = c->B.n_scenes;
    return FE_OK;
}

fe_status fe_scene_table(const fe_ctx* c, uint32_t* first, uint32_t* count, uint32_t capacity) {
    if (!c || !first || !count) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (capacity < c->B.n_scenes) {
        set_error("capacity %u below the %u scenes", capacity, c->B.n_scenes);
        return FE_ERR_CAPACITY;
    }
    for (uint32_t k = 0; k < c->B.n_scenes; ++k) {
        first[k] = c->dparams[k].first;
        count[k] = c->dparams[k].n;
    }
    return FE_OK;
}

fe_status fe_destroy(fe_ctx* c) {
    if (!c) return FE_OK;
    release(c);
    delete c;
    return FE_OK;
}

namespace {

fe_status set_scene_params(fe_ctx* c, uint32_t first, uint32_t last, const fe_params* p) {
    fe_status s = validate(p);
    if (s != FE_OK) return s;
    const uint32_t ns = c->B.n_scenes;
    // Every scene must keep sharing what one frame records for all of them.
    for (uint32_t k = 0; k < ns; ++k) {
        if (k >= first && k < last) continue;
        if ((s = check_batch_uniform(c->params[k], *p, ns)) != FE_OK) return s;
    }
    if (ns > 1 && p->sort_algorithm != FE_SORT_RADIX) {
        set_error("bitonic sort is single-scene only");
        return FE_ERR_UNSUPPORTED;
    }
    FE_CUDA(cudaSetDevice(c->device));
    for (uint32_t k = first; k < last; ++k) {
        c->params[k] = *p;
        const DevParams& old = c->dparams[k];
        c->dparams[k] = to_device(*p, old.n, old.T, old.table_base, old.first);
    }
    return upload_params(c);
}

fe_status get_scene_params(const fe_ctx* c, uint32_t scene, fe_params* out) {
    fe_ctx* m = const_cast<fe_ctx*>(c);
    FE_CUDA(cudaSetDevice(c->device));
    DevParams dp;
    FE_CUDA(cudaMemcpyAsync(&dp, c->B.P + scene, sizeof dp, cudaMemcpyDeviceToHost, c->stream));
    FE_CUDA(cudaStreamSynchronize(c->stream));
    m->params[scene].dt = dp.dt;
    *out = c->params[scene];
    return FE_OK;
}

}  // namespace

fe_status fe_set_params(fe_ctx* c, const fe_params* p) {
    if (!c || !p) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    return set_scene_params(c, 0, c->B.n_scenes, p);
}

fe_status fe_set_scene_params(fe_ctx* c, uint32_t scene, const fe_params* p) {
    if (!c || !p) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (scene >= c->B.n_scenes) {
        set_error("scene %u of %u", scene, c->B.n_scenes);
        return FE_ERR_INVALID_ARGUMENT;
    }
    return set_scene_params(c, scene, scene + 1, p);
}

fe_status fe_get_params(const fe_ctx* c, fe_params* out) {
    if (!c || !out) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    return get_scene_params(c, 0, out);
}

fe_status fe_get_scene_params(const fe_ctx* c, uint32_t scene, fe_params* out) {
    if (!c || !out) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (scene >= c->B.n_scenes) {
        set_error("scene %u of %u", scene, c->B.n_scenes);
        return FE_ERR_INVALID_ARGUMENT;
    }
    return get_scene_params(c, scene, out);
}

fe_status fe_prepare(fe_ctx* c) {
    if (!c) {
        set_error("context is NULL");
        return FE_ERR_INVALID_ARGUMENT;
    }
    c->prepared = true;
    return FE_OK;
}

fe_status fe_get_size(const fe_ctx* c, uint32_t* n, uint32_t* t) {
    if (!c) {
        set_error("context is NULL");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (n) *n = c->n;
    if (t) *t = c->T;
    return FE_OK;
}

void* fe_get_stream(fe_ctx* c) { return c ? (void*)c->stream : nullptr; }

fe_status fe_synchronize(fe_ctx* c) {
    if (!c) {
        set_error("context is NULL");
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    FE_CUDA(cudaStreamSynchronize(c->stream));
    return FE_OK;
}

fe_status fe_upload(fe_ctx* c, fe_field f, const void* src, size_t bytes) {
    if (!c || !src) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    void* d;
    size_t elem, pitch;
    size_t need = field_bytes(c, f, &d, &elem, &pitch);
    if (need == 0 || bytes != need || f == FE_FIELD_STATS || f == FE_FIELD_GRID_START) {
        set_error("field %d: expected %zu bytes, got %zu (or read-only field)", (int)f, need, bytes);
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    FE_CUDA(cudaMemcpy2DAsync(d, pitch, src, elem, elem, need / elem, cudaMemcpyHostToDevice,
                              c->stream));
    if (f == FE_FIELD_POSITION_B) {  // keep the records' position copies
        FE_CUDA(cudaMemcpy2DAsync(c->B.rec, 32, src, 16, 16, c->n, cudaMemcpyHostToDevice,
                                  c->stream));
        FE_CUDA(cudaMemcpy2DAsync(c->B.pv, 32, src, 16, 16, c->n, cudaMemcpyHostToDevice,
                                  c->stream));
        FE_CUDA(cudaMemcpy2DAsync(c->B.pa, 32, src, 16, 16, c->n, cudaMemcpyHostToDevice,
                                  c->stream));
    }
    // pos_b.w caches p / rho^2 for pressure_force, the velocities' w rho.
    if (f == FE_FIELD_PRESSURE || f == FE_FIELD_DENSITY || f == FE_FIELD_POSITION_B ||
        f == FE_FIELD_VELOCITY_A || f == FE_FIELD_VELOCITY_B)
        return run_refresh_pr(c);
    return FE_OK;
}

fe_status fe_download(fe_ctx* c, fe_field f, void* dst, size_t bytes) {
    if (!c || !dst) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    void* d;
    size_t elem, pitch;
    size_t need = field_bytes(c, f, &d, &elem, &pitch);
    if (need == 0 && (f == FE_FIELD_DENSITY_GRID || f == FE_FIELD_IMAGE))
        return FE_ERR_INVALID_ARGUMENT;
    if (need == 0 || bytes != need) {
        set_error("field %d: expected %zu bytes, got %zu", (int)f, need, bytes);
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    FE_CUDA(cudaMemcpy2DAsync(dst, elem, d, pitch, elem, need / elem, cudaMemcpyDeviceToHost,
                              c->stream));
    FE_CUDA(cudaStreamSynchronize(c->stream));
    if (f == FE_FIELD_POSITION_B) {
        // The device keeps p / rho^2 in w; the reference's position_b.w is the
        // copied position_a.w, which is always 1 (particle.rs:171,
        // pressure_integration.comp:75).
        float* v = static_cast<float*>(dst);
        for (uint32_t i = 0; i < c->n; ++i) v[4 * i + 3] = 1.0f;
    }
    if (f == FE_FIELD_VELOCITY_A || f == FE_FIELD_VELOCITY_B) {
        // The device keeps the density in w; the reference's passes always
        // write the velocities' w as 0.
        float* v = static_cast<float*>(dst);
        for (uint32_t i = 0; i < c->n; ++i) v[4 * i + 3] = 0.0f;
    }
    return FE_OK;
}

// The reference's w of a float4 field whose device copy keeps other data
// in w: position_b.w = 1 (the copied position_a.w), the velocities' w = 0.
bool field_fixed_w(fe_field f, float* w) {
    if (f == FE_FIELD_POSITION_B) {
        *w = 1.0f;
        return true;
    }
    if (f == FE_FIELD_VELOCITY_A || f == FE_FIELD_VELOCITY_B) {
        *w = 0.0f;
        return true;
    }
    return false;
}

fe_status fe_download_async(fe_ctx* c, fe_field f, void* dst, size_t bytes, uint64_t* ticket) {
    if (!c || !dst || !ticket) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    void* d;
    size_t elem, pitch;
    size_t need = field_bytes(c, f, &d, &elem, &pitch);
    if (need == 0 || bytes != need) {
        set_error("field %d: expected %zu bytes, got %zu", (int)f, need, bytes);
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    if (!c->copy_stream) {
        FE_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        for (int k = 0; k < 2; ++k) {
            FE_CUDA(cudaEventCreateWithFlags(&c->snap_ready[k], cudaEventDisableTiming));
            FE_CUDA(cudaEventCreateWithFlags(&c->copy_done[k], cudaEventDisableTiming));
        }
    }
    if (need > c->snap_cap) {
        // earlier snapshots may still be copied out of the old buffers
        FE_CUDA(cudaStreamSynchronize(c->copy_stream));
        unsigned char *a = nullptr, *b = nullptr;
        fe_status st;
        if ((st = dev_alloc(c, &a, need)) != FE_OK || (st = dev_alloc(c, &b, need)) != FE_OK)
            return st;
        c->snap[0] = a;
        c->snap[1] = b;
        c->snap_cap = need;
        c->slot_ticket[0] = c->slot_ticket[1] = 0;
    }
    const uint64_t t = ++c->tickets;
    const int slot = (int)(t & 1u);
    // the slot's previous copy must have left the snapshot before it is
    // overwritten
    if (c->slot_ticket[slot]) FE_CUDA(cudaStreamWaitEvent(c->stream, c->copy_done[slot], 0));
    float w = 0.0f;
    const bool fix_w = field_fixed_w(f, &w);
    if (elem == 16) {
        Recorder R = eager(c);
        REC(R.k(k_snapshot4, flat_grid((uint32_t)(need / 16)), dim3(kBlock),
                static_cast<float4*>(c->snap[slot]), static_cast<const float4*>(d),
                (uint32_t)(pitch / 16), (uint32_t)(need / 16), fix_w ? 1 : 0, w));
    } else {
        FE_CUDA(cudaMemcpy2DAsync(c->snap[slot], elem, d, pitch, elem, need / elem,
                                  cudaMemcpyDeviceToDevice, c->stream));
    }
    FE_CUDA(cudaEventRecord(c->snap_ready[slot], c->stream));
    FE_CUDA(cudaStreamWaitEvent(c->copy_stream, c->snap_ready[slot], 0));
    FE_CUDA(cudaMemcpyAsync(dst, c->snap[slot], need, cudaMemcpyDeviceToHost, c->copy_stream));
    FE_CUDA(cudaEventRecord(c->copy_done[slot], c->copy_stream));
    c->slot_ticket[slot] = t;
    *ticket = t;
    return FE_OK;
}

fe_status fe_download_wait(fe_ctx* c, uint64_t ticket) {
    if (!c || ticket == 0 || ticket > c->tickets) {
        set_error("fe_download_wait: unknown ticket %llu", (unsigned long long)ticket);
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    // A slot serves tickets in increasing order, and each copy out of a slot
    // follows the one before it: waiting for the slot's latest copy covers
    // this ticket as well.
    FE_CUDA(cudaEventSynchronize(c->copy_done[ticket & 1u]));
    return FE_OK;
}

#define FE_STAGE(name, body)                                 \
    fe_status name(fe_ctx* c) {                              \
        NvtxRange range_(#name);                             \
        fe_status s_ = need_prepared(c, #name);              \
        if (s_ != FE_OK) return s_;                          \
        Recorder R = eager(c);                               \
        body;                                                \
    }

FE_STAGE(fe_neighbor_search, return rec_neighbor_search(c, R))
FE_STAGE(fe_density_alpha, return rec_density_alpha(c, R))
FE_STAGE(fe_viscosity,
         return rec_nbr(c, R, FE_NBR_LIST_PASSES,
                        NBR_KERNEL(k_viscosity, FE_NBR_LIST_PASSES), c->B))
FE_STAGE(fe_density_source,
         return rec_nbr(c, R, FE_NBR_LIST_PASSES,
                        NBR_KERNEL(k_density_source, FE_NBR_LIST_PASSES), c->B))
FE_STAGE(fe_pressure_force, return rec_force(c, R, -1))
FE_STAGE(fe_pressure_update, return rec_update(c, R, -1, (cudaGraphConditionalHandle)0, 0))
FE_STAGE(fe_pressure_integration, return rec_simple(c, R, k_pressure_integration))
FE_STAGE(fe_divergence_source,
         return rec_nbr(c, R, FE_NBR_LIST_PASSES,
                        NBR_KERNEL(k_divergence_source, FE_NBR_LIST_PASSES),
                        c->B, c->fixed_mode() ? 1 : 0))
FE_STAGE(fe_divergence_integration,
         REC(R.k(k_divergence_integration, chunk_grid(c), dim3(kBlock), c->B,
                 c->fixed_mode() ? 1 : 0));
         return FE_OK)
FE_STAGE(fe_stats_pass, return rec_stats(c, R))

// DensityTexturePipeline::execute after clear_color_image
// (renderer/mod.rs:385-390; density_texture.rs; splat_density.comp) into the
// context's headless grid.
fe_status fe_density_splat(fe_ctx* c) {
    NvtxRange range_("fe_density_splat");
    if (!c) {
        set_error("context is NULL");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (c->B.n_scenes != 1) {
        set_error("fe_density_splat: one grid per context; batches have one box per scene");
        return FE_ERR_UNSUPPORTED;
    }
    const fe_params& p = c->params[0];
    const int rx = p.grid_res[0], ry = p.grid_res[1], rz = p.grid_res[2];
    if (rx < 1 || ry < 1 || rz < 1 || rx > 1024 || ry > 1024 || rz > 1024) {
        set_error("grid_res %d x %d x %d outside 1..1024", rx, ry, rz);
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    const size_t voxels = (size_t)rx * ry * rz;
    if (voxels > c->splat_cap) {
        uint32_t* g = nullptr;
        fe_status s = dev_alloc(c, &g, voxels);
        if (s != FE_OK) return s;
        c->splat_grid = g;
        c->splat_cap = voxels;
    }
    if (!c->splat_taps) {
        // The splat's weights per voxel offset, evaluated once on the device;
        // the non-zero ones become the tap table (x fastest).
        constexpr int kAll = kSplatSide * kSplatSide * kSplatSide;
        uint32_t* w = nullptr;
        fe_status s = dev_alloc(c, &w, kAll);
        if (s != FE_OK) return s;
        FE_CUDA(splat_weights(w, c->stream));
        std::vector<uint32_t> hw(kAll);
        FE_CUDA(cudaMemcpyAsync(hw.data(), w, kAll * 4, cudaMemcpyDeviceToHost, c->stream));
        FE_CUDA(cudaStreamSynchronize(c->stream));
        std::vector<int4> taps;
        for (int t = 0; t < kAll; ++t)
            if (hw[t])
                taps.push_back(make_int4(t % kSplatSide - kSplatRadius,
                                         (t / kSplatSide) % kSplatSide - kSplatRadius,
                                         t / (kSplatSide * kSplatSide) - kSplatRadius, (int)hw[t]));
        int4* d = nullptr;
        if ((s = dev_alloc(c, &d, taps.size()))) return s;
        FE_CUDA(cudaMemcpy(d, taps.data(), taps.size() * sizeof(int4), cudaMemcpyHostToDevice));
        c->splat_taps = d;
        c->splat_ntaps = (uint32_t)taps.size();
    }
    c->splat_res[0] = rx;
    c->splat_res[1] = ry;
    c->splat_res[2] = rz;
    // Counts per centre voxel, then the convolution with the tap table
    // (fe_splat.cu).
    const int3 res = make_int3(rx, ry, rz);
    const size_t hist_n = (size_t)(rx + 1) * (ry + 1) * (rz + 1);
    if (hist_n > c->splat_hist_cap) {
        fe_status st0 = dev_alloc(c, &c->splat_hist, hist_n);
        if (st0 != FE_OK) return st0;
        c->splat_hist_cap = hist_n;
    }
    const float3 b0 = make_float3(p.box_min[0], p.box_min[1], p.box_min[2]);
    const float3 b1 = make_float3(p.box_max[0], p.box_max[1], p.box_max[2]);
    FE_CUDA(cudaMemsetAsync(c->splat_grid, 0, voxels * 4, c->stream));
    FE_CUDA(cudaMemsetAsync(c->splat_hist, 0, hist_n * 4, c->stream));
    FE_CUDA(splat_histogram(c->B.pos_a, c->n, b0, b1, res, c->splat_hist, c->stream));
    FE_CUDA(splat_convolve(c->splat_hist, res, c->splat_taps, c->splat_ntaps, c->splat_grid,
                           c->stream));
    return FE_OK;
}

fe_status fe_set_skybox(fe_ctx* c, const float* rgba, uint32_t width, uint32_t height) {
    if (!c || !rgba || width == 0 || height == 0) {
        set_error("skybox needs a context, pixels and a non-zero size");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (width > 16384 || height > 16384) {
        set_error("skybox %u x %u above 16384", width, height);
        return FE_ERR_CAPACITY;
    }
    FE_CUDA(cudaSetDevice(c->device));
    const size_t texels = (size_t)width * height;
    if (texels > c->sky_cap) {
        float4* p = nullptr;
        fe_status s = dev_alloc(c, &p, texels);
        if (s != FE_OK) return s;
        c->sky = p;
        c->sky_cap = texels;
    }
    FE_CUDA(cudaMemcpyAsync(c->sky, rgba, texels * 16, cudaMemcpyHostToDevice, c->stream));
    FE_CUDA(cudaStreamSynchronize(c->stream));
    c->sky_w = (int)width;
    c->sky_h = (int)height;
    return FE_OK;
}

// The water pass (water_pipeline.rs; raymarch.vert/.frag) of the last
// fe_density_splat grid into the context's RGBA32F image.
fe_status fe_raymarch(fe_ctx* c, const fe_camera* cam) {
    NvtxRange range_("fe_raymarch");
    if (!c || !cam) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (!c->splat_grid) {
        set_error("fe_raymarch: no density grid yet (fe_density_splat first)");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (!c->sky) {
        set_error("fe_raymarch: no skybox (fe_set_skybox first)");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (cam->width == 0 || cam->height == 0 || cam->width > 16384 || cam->height > 16384) {
        set_error("image %u x %u outside 1..16384", cam->width, cam->height);
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    const size_t pixels = (size_t)cam->width * cam->height;
    if (pixels > c->image_cap) {
        float4* p = nullptr;
        fe_status s = dev_alloc(c, &p, pixels);
        if (s != FE_OK) return s;
        c->image = p;
        c->image_cap = pixels;
    }
    c->image_w = (int)cam->width;
    c->image_h = (int)cam->height;
    const fe_params& p = c->params[0];
    RaymarchArgs a;
    a.grid = c->splat_grid;
    a.res = make_int3(c->splat_res[0], c->splat_res[1], c->splat_res[2]);
    a.sky = c->sky;
    a.sky_w = c->sky_w;
    a.sky_h = c->sky_h;
    std::memcpy(a.inv_view_proj, cam->inv_view_proj, sizeof a.inv_view_proj);
    a.cam = make_float3(cam->camera_pos[0], cam->camera_pos[1], cam->camera_pos[2]);
    a.box_min = make_float3(p.box_min[0], p.box_min[1], p.box_min[2]);
    a.box_max = make_float3(p.box_max[0], p.box_max[1], p.box_max[2]);
    a.width = (int)cam->width;
    a.height = (int)cam->height;
    a.out = c->image;
    FE_CUDA(raymarch(a, c->stream));
    return FE_OK;
}

fe_status fe_read_stats(fe_ctx* c, fe_stats* out) {
    if (!c || !out) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    return collect_stats(c, out);
}

fe_status fe_read_stats_async(fe_ctx* c, uint64_t* ticket) {
    if (!c || !ticket) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    if (!c->stats_host) {
        FE_CUDA(cudaHostAlloc(&c->stats_host, 2 * sizeof(StatsSnapshot), cudaHostAllocMapped));
        FE_CUDA(cudaHostGetDevicePointer((void**)&c->stats_dev, c->stats_host, 0));
        for (int k = 0; k < 2; ++k)
            FE_CUDA(cudaEventCreateWithFlags(&c->stats_done[k], cudaEventDisableTiming));
    }
    const uint64_t t = ++c->stats_tickets;
    const int slot = (int)(t & 1u);
    Recorder R = eager(c);
    REC(R.k(k_stats_snapshot, dim3(1), dim3(32), c->B, c->stats_dev + slot, 0u));
    FE_CUDA(cudaEventRecord(c->stats_done[slot], c->stream));
    *ticket = t;
    return FE_OK;
}

fe_status fe_stats_wait(fe_ctx* c, uint64_t ticket, fe_stats* out) {
    if (!c || !out || ticket == 0 || ticket > c->stats_tickets || ticket + 2 <= c->stats_tickets) {
        set_error("fe_stats_wait: unknown or overwritten ticket %llu",
                  (unsigned long long)ticket);
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    const int slot = (int)(ticket & 1u);
    FE_CUDA(cudaEventSynchronize(c->stats_done[slot]));
    const StatsSnapshot& snap = c->stats_host[slot];
    stats_from(c, snap.S, snap.G, snap.dt, snap.n, out);
    if (out->flags & 0x4u) {
        set_error("a bounded device wait timed out (look-back)");
        return FE_ERR_TIMEOUT;
    }
    if (out->flags & 0x8u) {
        set_error("non-finite velocity, density or source term in the stats pass");
        return FE_ERR_NON_FINITE;
    }
    return FE_OK;
}

fe_status fe_read_scene_stats(fe_ctx* c, uint32_t scene, fe_stats* out) {
    if (!c || !out) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (scene >= c->B.n_scenes) {
        set_error("scene %u of %u", scene, c->B.n_scenes);
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    return collect_stats(c, out, scene);
}

fe_status fe_step(fe_ctx* c, uint32_t n_substeps, uint32_t flags, fe_stats* out) {
    NvtxRange range_("fe_step");
    fe_status s = need_prepared(c, "fe_step");
    if (s != FE_OK) return s;
    if (n_substeps > 1024) {
        set_error("n_substeps %u above 1024", n_substeps);
        return FE_ERR_CAPACITY;
    }
    if (c->params[0].warm_start == FE_WARM_LEARNED && !c->model) {
        set_error("fe_step: warm_start = FE_WARM_LEARNED needs a model (fe_set_model)");
        return FE_ERR_UNSUPPORTED;
    }
    const bool init = (flags & FE_STEP_INIT_NS) || !c->initialized;
    c->last_substeps = n_substeps;
    if (flags & FE_STEP_NO_GRAPH) {
        Recorder R = eager(c);
        s = rec_frame(c, R, n_substeps, init);
        if (s != FE_OK) return s;
    } else {
        cudaGraphExec_t exec;
        s = get_graph(c, n_substeps, init, &exec);
        if (s != FE_OK) return s;
        FE_CUDA(cudaGraphLaunch(exec, c->stream));
    }
    c->initialized = true;
    if (!out) return FE_OK;
    s = collect_stats(c, out);
    if (s != FE_OK) return s;
    if (out->flags & 0x4u) {
        set_error("a bounded device wait timed out (look-back)");
        return FE_ERR_TIMEOUT;
    }
    if (out->flags & 0x8u) {
        set_error("non-finite velocity, density or source term in the stats pass");
        return FE_ERR_NON_FINITE;
    }
    return FE_OK;
}

// ---------------------------------------------------------------------------
// Learned warm start: model attachment and training-data capture.
// ---------------------------------------------------------------------------
static fe_status ensure_learn_buffers(fe_ctx* c) {
    if (c->L.carry) return FE_OK;
    fe_status s;
    __nv_bfloat16* xb = nullptr;
    if ((s = dev_alloc(c, &xb, (size_t)c->n * 16)) || (s = dev_alloc(c, &c->L.out, 2 * (size_t)c->n)) ||
        (s = dev_alloc(c, &c->L.carry_tmp, c->n)) || (s = dev_alloc(c, &c->L.mom, c->n)) ||
        (s = dev_alloc(c, &c->L.mom_tmp, c->n)))
        return s;
    float4* carry = nullptr;
    if ((s = dev_alloc(c, &carry, c->n))) return s;
    c->L.xb = xb;
    FE_CUDA(cudaMemsetAsync(c->L.mom, 0, (size_t)c->n * 16, c->stream));
    FE_CUDA(cudaMemsetAsync(c->L.mom_tmp, 0, (size_t)c->n * 16, c->stream));
    FE_CUDA(cudaMemsetAsync(carry, 0, (size_t)c->n * 16, c->stream));
    // no capture slot yet: w = all ones
    FE_CUDA(cudaMemset2DAsync(reinterpret_cast<char*>(carry) + 12, 16, 0xFF, 4, c->n, c->stream));
    FE_CUDA(cudaStreamSynchronize(c->stream));
    c->L.carry = carry;
    return FE_OK;
}

static void drop_graphs(fe_ctx* c) {
    cudaStreamSynchronize(c->stream);
    for (auto& g : c->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
    }
    c->graphs.clear();
}

extern "C" {

FE_API fe_status fe_set_model(fe_ctx* c, fe_model* model) {
    if (!c) {
        set_error("context is NULL");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (model && model->device != c->device) {
        set_error("model lives on device %d, context on %d", model->device, c->device);
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    fe_status s = ensure_learn_buffers(c);
    if (s != FE_OK) return s;
    drop_graphs(c);  // recorded graphs hold the previous model's pointers
    c->model = model;
    c->L.norm = model ? model->norm : nullptr;
    c->L.learned = model ? 1u : 0u;
    return FE_OK;
}

FE_API fe_status fe_capture_begin(fe_ctx* c, uint32_t capacity, uint32_t stride) {
    if (!c || capacity == 0 || stride == 0) {
        set_error("capacity and stride must be > 0");
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    fe_status s = ensure_learn_buffers(c);
    if (s != FE_OK) return s;
    if (c->L.cap_capacity < capacity) {
        if ((s = dev_alloc(c, &c->L.cap_x, (size_t)capacity * 12)) ||
            (s = dev_alloc(c, &c->L.cap_y, (size_t)capacity * 2)))
            return s;
        if (!c->L.cap_count && (s = dev_alloc(c, &c->L.cap_count, 4))) return s;
        c->L.cap_capacity = capacity;
    }
    FE_CUDA(cudaMemsetAsync(c->L.cap_count, 0, 4, c->stream));
    drop_graphs(c);
    c->L.cap_stride = stride;
    c->L.capture = 1;
    c->capture = true;
    return FE_OK;
}

FE_API fe_status fe_capture_read(fe_ctx* c, float* x, float* y, uint32_t rows, uint32_t* count) {
    if (!c || !count || (rows && (!x || !y))) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    uint32_t n = 0;
    if (c->L.cap_count) {
        FE_CUDA(cudaMemcpyAsync(&n, c->L.cap_count, 4, cudaMemcpyDeviceToHost, c->stream));
        FE_CUDA(cudaStreamSynchronize(c->stream));
    }
    if (n > c->L.cap_capacity) n = c->L.cap_capacity;
    *count = n;
    uint32_t k = n < rows ? n : rows;
    if (k) {
        FE_CUDA(cudaMemcpy(x, c->L.cap_x, (size_t)k * 12 * 4, cudaMemcpyDeviceToHost));
        FE_CUDA(cudaMemcpy(y, c->L.cap_y, (size_t)k * 2 * 4, cudaMemcpyDeviceToHost));
    }
    return FE_OK;
}

FE_API fe_status fe_capture_end(fe_ctx* c) {
    if (!c) {
        set_error("context is NULL");
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    drop_graphs(c);
    c->capture = false;
    c->L.capture = 0;
    return FE_OK;
}

FE_API fe_status fe_debug_trace_learned(fe_ctx* c, uint32_t slots) {
    if (!c) {
        set_error("fe_debug_trace_learned: context is NULL");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (slots > 64) {
        set_error("fe_debug_trace_learned: at most 64 solve slots");
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    if (slots > c->trace_cap) {
        unsigned char* p = nullptr;
        fe_status st = dev_alloc(c, &p, (size_t)slots * c->n * kTraceBytesPerParticle);
        if (st != FE_OK) return st;
        c->trace = p;
        c->trace_cap = slots;
    }
    c->trace_slots = slots;
    drop_graphs(c);
    return FE_OK;
}

FE_API fe_status fe_debug_read_trace(fe_ctx* c, uint32_t slot, uint16_t* rows, float* out) {
    if (!c || slot >= c->trace_slots) {
        set_error("fe_debug_read_trace: no such slot (trace %u slots)", c ? c->trace_slots : 0u);
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    const unsigned char* base = c->trace + (size_t)slot * c->n * kTraceBytesPerParticle;
    if (rows)
        FE_CUDA(cudaMemcpyAsync(rows, base, (size_t)c->n * 32, cudaMemcpyDeviceToHost,
                                c->stream));
    if (out)
        FE_CUDA(cudaMemcpyAsync(out, base + (size_t)c->n * 32, (size_t)c->n * 8,
                                cudaMemcpyDeviceToHost, c->stream));
    FE_CUDA(cudaStreamSynchronize(c->stream));
    return FE_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Standalone sort (device buffers).  Scratch per device, grown on demand;
// an event serialises users of the same scratch across streams.
// ---------------------------------------------------------------------------
namespace {
struct SortScratch {
    int device = -1;
    uint32_t cap = 0;
    uint32_t* tk = nullptr;
    uint32_t* tv = nullptr;
    uint32_t* words = nullptr;
    size_t nwords = 0;
    uint32_t* flags = nullptr;
    cudaEvent_t done = nullptr;
};
std::mutex g_sort_mutex;
SortScratch g_sort[16];
}  // namespace

namespace {

// The standalone sort; `forced` overrides the tuned (or default) radix shape.
fe_status sort_pairs_impl(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t key_bits,
                          int algorithm, void* stream_ptr, const RadixConfig* forced) {
    if ((!keys || !vals) && n > 0) {
        set_error("NULL keys or values");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (algorithm != FE_SORT_RADIX && algorithm != FE_SORT_BITONIC) {
        set_error("unknown sort algorithm %d", algorithm);
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (key_bits > 32) {
        set_error("key_bits %u above 32", key_bits);
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (n > FE_MAX_PARTICLES) {
        set_error("n %u above %u", n, FE_MAX_PARTICLES);
        return FE_ERR_CAPACITY;
    }
    if (n < 2) return FE_OK;
    if (algorithm == FE_SORT_BITONIC && (n & (n - 1))) {
        set_error("bitonic sort needs a power-of-two length (sorter.rs:57-60)");
        return FE_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t stream = (cudaStream_t)stream_ptr;
    Recorder R;
    R.stream = stream;
    SortLaunch L = R.sort_launch();
    if (algorithm == FE_SORT_BITONIC) {
        REC(bitonic_sort(L, keys, vals, n));
        return FE_OK;
    }
    int dev;
    FE_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 16) {
        set_error("device index %d unsupported", dev);
        return FE_ERR_NO_DEVICE;
    }
    std::lock_guard<std::mutex> lock(g_sort_mutex);
    SortScratch& S = g_sort[dev];
    const uint32_t kb = key_bits ? key_bits : 32;
    RadixConfig cfg = kRadixDefault;
    if (forced)
        cfg = *forced;
    else
        sort_tuning_lookup(dev, n, kb, &cfg);
    size_t words = radix_scratch_words(n, kb, cfg);
    if (S.cap < n || S.nwords < words) {
        if (S.done) FE_CUDA(cudaEventSynchronize(S.done));
        cudaFree(S.tk);
        cudaFree(S.tv);
        cudaFree(S.words);
        S.tk = S.tv = S.words = nullptr;
        uint32_t cap = std::max(n, S.cap);
        size_t nw = std::max(words, S.nwords);
        FE_CUDA(cudaMalloc(&S.tk, (size_t)cap * 4));
        FE_CUDA(cudaMalloc(&S.tv, (size_t)cap * 4));
        FE_CUDA(cudaMalloc(&S.words, (nw + 8) * 4));
        S.cap = cap;
        S.nwords = nw;
        S.flags = S.words + nw;
        FE_CUDA(cudaMemset(S.flags, 0, 32));
        if (!S.done) FE_CUDA(cudaEventCreateWithFlags(&S.done, cudaEventDisableTiming));
        S.device = dev;
    } else {
        FE_CUDA(cudaStreamWaitEvent(stream, S.done, 0));
    }
    // the error word reports this call only (fe_sort_flags reads it)
    REC(R.fill_u32(S.flags, 0u, 8));
    bool in_tmp = false;
    REC(radix_sort(L, keys, vals, S.tk, S.tv, n, kb, S.words, S.flags, &in_tmp, cfg));
    if (in_tmp) {
        FE_CUDA(cudaMemcpyAsync(keys, S.tk, (size_t)n * 4, cudaMemcpyDeviceToDevice, stream));
        FE_CUDA(cudaMemcpyAsync(vals, S.tv, (size_t)n * 4, cudaMemcpyDeviceToDevice, stream));
    }
    FE_CUDA(cudaEventRecord(S.done, stream));
    return FE_OK;
}

}  // namespace

fe_status fe_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t key_bits,
                        int algorithm, void* stream_ptr) {
    NvtxRange range_("fe_sort_pairs");
    return sort_pairs_impl(keys, vals, n, key_bits, algorithm, stream_ptr, nullptr);
}

// Error word of the last radix fe_sort_pairs on the current device, copied
// in the order of `stream` after that sort (0 before any radix sort).
fe_status fe_sort_flags(uint32_t* flags_out, void* stream_ptr) {
    if (!flags_out) {
        set_error("fe_sort_flags: NULL flags_out");
        return FE_ERR_INVALID_ARGUMENT;
    }
    int dev;
    FE_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 16) {
        set_error("device index %d unsupported", dev);
        return FE_ERR_NO_DEVICE;
    }
    cudaStream_t stream = (cudaStream_t)stream_ptr;
    std::lock_guard<std::mutex> lock(g_sort_mutex);
    SortScratch& S = g_sort[dev];
    if (!S.flags) {
        FE_CUDA(cudaMemsetAsync(flags_out, 0, sizeof(uint32_t), stream));
        return FE_OK;
    }
    FE_CUDA(cudaStreamWaitEvent(stream, S.done, 0));
    FE_CUDA(cudaMemcpyAsync(flags_out, S.flags, sizeof(uint32_t), cudaMemcpyDefault, stream));
    return FE_OK;
}

// ---------------------------------------------------------------------------
// Autotuning (fe_tune.cu).
// ---------------------------------------------------------------------------
namespace {

void fill_radix_report(fe_tune_report* r, const float* ms) {
    r->radix_candidates = kRadixCandidateCount;
    for (int k = 0; k < kRadixCandidateCount; ++k) {
        r->radix_digit_bits[k] = kRadixCandidates[k].digit_bits;
        r->radix_items[k] = kRadixCandidates[k].items;
        r->radix_ms[k] = ms[k];
    }
}

}  // namespace

// Neighbour-kernel shapes: every candidate of every group is timed on the
// context's current state (one untimed launch, then the median of 7 CUDA-
// event timed launches, eager, on the context stream).  Some of the timed
// passes write state (the sources reset the pressures, the update advances
// them), so the state is exported to host memory first and imported again
// at the end: the next frame starts from exactly the state it had.
constexpr uint32_t kNbrCandThreads[] = {128, 256, 512, 128, 256, 512};
constexpr uint32_t kNbrCandPersistent[] = {0, 0, 0, 1, 1, 1};
constexpr int kNbrCands = 6;

fe_status time_nbr_group(fe_ctx* c, int g, float* ms_out) {
    cudaEvent_t a = nullptr, b = nullptr;
    FE_CUDA(cudaEventCreate(&a));
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        set_error("cudaEventCreate failed");
        return FE_ERR_CUDA;
    }
    Recorder R = eager(c);
    auto launch = [&]() -> fe_status {
        switch (g) {
            case FE_NBR_DENSITY_ALPHA: return rec_density_alpha(c, R);
            case FE_NBR_LIST_PASSES: {
                fe_status st;
                for (int pass = 0; pass < 3; ++pass)
                    if ((st = rec_list_pass(c, R, pass)) != FE_OK) return st;
                return FE_OK;
            }
            case FE_NBR_PRESSURE_FORCE: return rec_force(c, R, -1);
            default: return rec_update(c, R, -1, (cudaGraphConditionalHandle)0, 0);
        }
    };
    std::vector<float> t;
    fe_status st = FE_OK;
    for (int rep = 0; rep < 8 && st == FE_OK; ++rep) {
        cudaEventRecord(a, c->stream);
        st = launch();
        cudaEventRecord(b, c->stream);
        if (st == FE_OK && cudaEventSynchronize(b) == cudaSuccess) {
            float v = 0.0f;
            cudaEventElapsedTime(&v, a, b);
            if (rep > 0) t.push_back(v);
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (st != FE_OK) return st;
    if (t.empty()) {
        set_error("neighbour tuning: timing failed");
        return FE_ERR_CUDA;
    }
    std::sort(t.begin(), t.end());
    *ms_out = t[t.size() / 2];
    return FE_OK;
}

fe_status tune_neighbour_kernels(fe_ctx* c, fe_tune_report* r) {
    size_t bytes = 0;
    fe_status st = fe_state_size(c, &bytes);
    if (st != FE_OK) return st;
    std::vector<unsigned char> snap(bytes);
    if ((st = fe_state_export(c, snap.data(), bytes)) != FE_OK) return st;
    r->nbr_candidates = kNbrCands;
    for (int k = 0; k < kNbrCands; ++k) {
        r->nbr_threads[k] = kNbrCandThreads[k];
        r->nbr_persistent[k] = kNbrCandPersistent[k];
    }
    uint32_t best_t[FE_NBR_GROUPS], best_p[FE_NBR_GROUPS];
    for (int g = 0; g < FE_NBR_GROUPS; ++g) {
        const uint32_t keep_t = c->nbr_threads[g], keep_p = c->nbr_persistent[g];
        float best = -1.0f;
        best_t[g] = keep_t;
        best_p[g] = keep_p;
        for (int k = 0; k < kNbrCands; ++k) {
            r->nbr_ms[g][k] = -1.0f;
            if (!nbr_shape_ok(g, kNbrCandThreads[k], kNbrCandPersistent[k])) continue;
            c->nbr_threads[g] = kNbrCandThreads[k];
            c->nbr_persistent[g] = kNbrCandPersistent[k];
            float ms = 0.0f;
            if ((st = time_nbr_group(c, g, &ms)) != FE_OK) break;
            r->nbr_ms[g][k] = ms;
            if (best < 0.0f || ms < best) {
                best = ms;
                best_t[g] = kNbrCandThreads[k];
                best_p[g] = kNbrCandPersistent[k];
            }
        }
        c->nbr_threads[g] = keep_t;
        c->nbr_persistent[g] = keep_p;
        if (st != FE_OK) break;
    }
    if (st == FE_OK)
        for (int g = 0; g < FE_NBR_GROUPS; ++g) {
            c->nbr_threads[g] = best_t[g];
            c->nbr_persistent[g] = best_p[g];
        }
    // the state as it was (the import rebuilds the neighbour list with the
    // chosen density_alpha shape: the same list)
    fe_status st2 = fe_state_import(c, snap.data(), bytes);
    drop_graphs(c);
    return st != FE_OK ? st : st2;
}

fe_status fe_autotune(fe_ctx* c, fe_tune_report* report) {
    if (!c) {
        set_error("context is NULL");
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    FE_CUDA(cudaStreamSynchronize(c->stream));
    fe_tune_report r;
    std::memset(&r, 0, sizeof r);
    // The sort is tuned on this context's own keys: the hashes of the
    // current positions (nearly sorted after the first frame), not random
    // keys, into temporary arrays.
    uint32_t *hk = nullptr, *hv = nullptr;
    if (cudaMalloc(&hk, (size_t)c->n * 4) != cudaSuccess ||
        cudaMalloc(&hv, (size_t)c->n * 4) != cudaSuccess) {
        cudaFree(hk);
        set_error("cudaMalloc of the tuning keys failed");
        return FE_ERR_OUT_OF_MEMORY;
    }
    Bufs H = c->B;
    H.keys = hk;
    H.vals = hv;
    k_hash<<<chunk_grid(c), kBlock, 0, c->stream>>>(H);
    cudaError_t e = cudaGetLastError();
    float ms[kRadixCandidateCount] = {};
    RadixConfig best = kRadixDefault;
    if (e == cudaSuccess) e = tune_radix(c->stream, hk, hv, c->n, c->key_bits, 7, &best, ms);
    cudaFree(hk);
    cudaFree(hv);
    if (e != cudaSuccess) {
        set_error("radix tuning: %s", cudaGetErrorString(e));
        return FE_ERR_CUDA;
    }
    fill_radix_report(&r, ms);
    int ctas = c->mlp_ctas;
    if (c->model && c->L.xb && c->L.out) {
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
        float mms[kMlpCtaCandidates] = {};
        e = tune_mlp(c->stream, c->model->params(), static_cast<const __nv_bfloat16*>(c->L.xb),
                     c->L.out, c->n, &c->B.G->flags, sms, 7, &ctas, mms);
        if (e != cudaSuccess) {
            set_error("network tuning: %s", cudaGetErrorString(e));
            return FE_ERR_CUDA;
        }
        r.mlp_candidates = kMlpCtaCandidates;
        for (int k = 0; k < kMlpCtaCandidates; ++k) {
            r.mlp_ctas_per_sm[k] = (uint32_t)kMlpCtaChoices[k];
            r.mlp_ms[k] = mms[k];
        }
    }
    drop_graphs(c);  // recorded frames hold the previous shapes
    c->radix_cfg = best;
    c->mlp_ctas = ctas;
    // (not while training data is captured: the learned source passes would
    // record extra samples while they are timed)
    if (c->initialized && !c->capture) {
        fe_status st = tune_neighbour_kernels(c, &r);
        if (st != FE_OK) return st;
    }
    r.chosen.radix_digit_bits = best.digit_bits;
    r.chosen.radix_items = best.items;
    r.chosen.mlp_ctas_per_sm = (uint32_t)ctas;
    for (int g = 0; g < FE_NBR_GROUPS; ++g) {
        r.chosen.nbr_threads[g] = c->nbr_threads[g];
        r.chosen.nbr_persistent[g] = c->nbr_persistent[g];
    }
    if (report) *report = r;
    return FE_OK;
}

fe_status fe_get_tuning(const fe_ctx* c, fe_tuning* out) {
    if (!c || !out) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    std::memset(out, 0, sizeof *out);
    out->radix_digit_bits = c->radix_cfg.digit_bits;
    out->radix_items = c->radix_cfg.items;
    out->mlp_ctas_per_sm = (uint32_t)c->mlp_ctas;
    for (int g = 0; g < FE_NBR_GROUPS; ++g) {
        out->nbr_threads[g] = c->nbr_threads[g];
        out->nbr_persistent[g] = c->nbr_persistent[g];
    }
    return FE_OK;
}

fe_status fe_set_tuning(fe_ctx* c, const fe_tuning* t) {
    if (!c || !t) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    RadixConfig cfg{t->radix_digit_bits, t->radix_items};
    if (!radix_config_valid(cfg)) {
        set_error("radix shape %u-bit digits x %u keys per thread is not a candidate",
                  t->radix_digit_bits, t->radix_items);
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (t->mlp_ctas_per_sm < 1 || t->mlp_ctas_per_sm > (uint32_t)mlp::kInferMaxCtasPerSm) {
        set_error("mlp_ctas_per_sm %u outside 1..%d", t->mlp_ctas_per_sm, mlp::kInferMaxCtasPerSm);
        return FE_ERR_INVALID_ARGUMENT;
    }
    uint32_t nt[FE_NBR_GROUPS];
    for (int g = 0; g < FE_NBR_GROUPS; ++g) {
        nt[g] = t->nbr_threads[g] ? t->nbr_threads[g] : (uint32_t)kBlock;
        if (!nbr_shape_ok(g, nt[g], t->nbr_persistent[g])) {
            set_error("neighbour group %d: %u threads per block, persistent %u is not a "
                      "candidate", g, t->nbr_threads[g], t->nbr_persistent[g]);
            return FE_ERR_INVALID_ARGUMENT;
        }
    }
    FE_CUDA(cudaSetDevice(c->device));
    drop_graphs(c);
    c->radix_cfg = cfg;
    c->mlp_ctas = (int)t->mlp_ctas_per_sm;
    for (int g = 0; g < FE_NBR_GROUPS; ++g) {
        c->nbr_threads[g] = nt[g];
        c->nbr_persistent[g] = t->nbr_persistent[g];
    }
    return FE_OK;
}

fe_status fe_autotune_sort(const uint32_t* keys, const uint32_t* vals, uint32_t n,
                           uint32_t key_bits, fe_tune_report* report) {
    if ((!keys || !vals) && n > 0) {
        set_error("NULL keys or values");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (key_bits > 32) {
        set_error("key_bits %u above 32", key_bits);
        return FE_ERR_INVALID_ARGUMENT;
    }
    const uint32_t kb = key_bits ? key_bits : 32;
    int dev = 0;
    FE_CUDA(cudaGetDevice(&dev));
    cudaStream_t st;
    FE_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    float ms[kRadixCandidateCount] = {};
    RadixConfig best = kRadixDefault;
    cudaError_t e = tune_radix(st, keys, vals, n, kb, 7, &best, ms);
    cudaStreamDestroy(st);
    if (e != cudaSuccess) {
        set_error("radix tuning: %s", cudaGetErrorString(e));
        return FE_ERR_CUDA;
    }
    sort_tuning_store(dev, n, kb, best);
    if (report) {
        std::memset(report, 0, sizeof *report);
        fill_radix_report(report, ms);
        report->chosen.radix_digit_bits = best.digit_bits;
        report->chosen.radix_items = best.items;
        report->chosen.mlp_ctas_per_sm = (uint32_t)mlp::kInferDefaultCtasPerSm;
    }
    return FE_OK;
}

fe_status fe_sort_pairs_config(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t key_bits,
                               uint32_t digit_bits, uint32_t items, void* stream) {
    RadixConfig cfg{digit_bits, items};
    if (!radix_config_valid(cfg)) {
        set_error("radix shape %u-bit digits x %u keys per thread is not a candidate",
                  digit_bits, items);
        return FE_ERR_INVALID_ARGUMENT;
    }
    return sort_pairs_impl(keys, vals, n, key_bits, FE_SORT_RADIX, stream, &cfg);
}

fe_status fe_sort_pairs_host(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t key_bits,
                             int algorithm) {
    if ((!keys || !vals) && n > 0) {
        set_error("NULL keys or values");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (n < 2) return FE_OK;
    uint32_t *dk = nullptr, *dv = nullptr;
    FE_CUDA(cudaMalloc(&dk, (size_t)n * 4));
    if (cudaMalloc(&dv, (size_t)n * 4) != cudaSuccess) {
        cudaFree(dk);
        set_error("cudaMalloc failed");
        return FE_ERR_OUT_OF_MEMORY;
    }
    fe_status s = FE_OK;
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMemcpyAsync(dk, keys, (size_t)n * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(dv, vals, (size_t)n * 4, cudaMemcpyHostToDevice, st) != cudaSuccess) {
        set_error("host-to-device copy failed");
        s = FE_ERR_CUDA;
    }
    if (s == FE_OK) s = fe_sort_pairs(dk, dv, n, key_bits, algorithm, st);
    uint32_t flags = 0;
    if (s == FE_OK && algorithm == FE_SORT_RADIX) s = fe_sort_flags(&flags, st);
    if (s == FE_OK &&
        (cudaMemcpyAsync(keys, dk, (size_t)n * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
         cudaMemcpyAsync(vals, dv, (size_t)n * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
         cudaStreamSynchronize(st) != cudaSuccess)) {
        set_error("device-to-host copy failed");
        s = FE_ERR_CUDA;
    }
    if (s == FE_OK && (flags & FE_STATS_LOOKBACK_TIMEOUT)) {
        set_error("fe_sort_pairs_host: a bounded look-back wait gave up; the output is not valid");
        s = FE_ERR_TIMEOUT;
    }
    if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    cudaFree(dk);
    cudaFree(dv);
    return s;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Checkpoint / resume (no reference counterpart: GpuPhysicsData,
// particle.rs:137-308, lives only as long as its Vulkan buffers).
// ---------------------------------------------------------------------------
namespace {

constexpr char kStateMagic[8] = {'F', 'E', 'S', 'T', 'A', 'T', 'E', '\0'};

struct StateHeader {
    char magic[8];
    uint32_t version, abi;
    uint32_t n, T, n_scenes, has_carry;
    uint32_t initialized, last_substeps;
    uint32_t size_params, size_devparams, size_scene, size_global;
    uint64_t bytes;  // the whole snapshot
};

struct Section {
    void* dev;
    size_t bytes;
};

// Device-resident state in snapshot order (after the header and the host
// parameter blocks).
std::vector<Section> state_sections(const fe_ctx* c, bool carry) {
    const size_t n = c->n, T = c->T, ns = c->B.n_scenes;
    const Bufs& B = c->B;
    std::vector<Section> v = {{B.P, sizeof(DevParams) * ns},
                              {B.S, sizeof(SceneState) * ns},
                              {B.G, sizeof(GlobalState)},
                              {B.pos_a, n * 16},
                              {B.pa, n * 32},
                              {B.pos_b, n * 16},
                              {B.pv, n * 32},
                              {B.rec, n * 32},
                              {B.rho, n * 4},
                              {B.alpha, n * 4},
                              {B.src, n * 4},
                              {B.prs, n * 4},
                              {B.keys, T * 4},
                              {B.vals, T * 4},
                              {B.cells, T * 8}};
    if (carry) v.push_back({c->L.carry, n * 16});
    return v;
}

size_t state_bytes(const fe_ctx* c, bool carry) {
    size_t b = sizeof(StateHeader) + sizeof(fe_params) * c->B.n_scenes;
    for (const Section& s : state_sections(c, carry)) b += s.bytes;
    return b;
}

// The learned warm start's carried state as a fresh context has it.
fe_status reset_carry(fe_ctx* c) {
    FE_CUDA(cudaMemsetAsync(c->L.carry, 0, (size_t)c->n * 16, c->stream));
    FE_CUDA(cudaMemset2DAsync(reinterpret_cast<char*>(c->L.carry) + 12, 16, 0xFF, 4, c->n,
                              c->stream));
    return FE_OK;
}

}  // namespace

extern "C" {

FE_API fe_status fe_state_size(const fe_ctx* c, size_t* bytes) {
    if (!c || !bytes) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    *bytes = state_bytes(c, c->L.carry != nullptr);
    return FE_OK;
}

FE_API fe_status fe_state_export(fe_ctx* c, void* dst, size_t bytes) {
    if (!c || !dst) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    const bool carry = c->L.carry != nullptr;
    const size_t need = state_bytes(c, carry);
    if (bytes < need) {
        set_error("snapshot needs %zu bytes, buffer has %zu", need, bytes);
        return FE_ERR_INVALID_ARGUMENT;
    }
    FE_CUDA(cudaSetDevice(c->device));
    const uint32_t ns = c->B.n_scenes;
    StateHeader hd;
    std::memset(&hd, 0, sizeof hd);
    std::memcpy(hd.magic, kStateMagic, sizeof hd.magic);
    hd.version = FE_STATE_VERSION;
    hd.abi = FE_ABI_VERSION;
    hd.n = c->n;
    hd.T = c->T;
    hd.n_scenes = ns;
    hd.has_carry = carry ? 1u : 0u;
    hd.initialized = c->initialized ? 1u : 0u;
    hd.last_substeps = c->last_substeps;
    hd.size_params = sizeof(fe_params);
    hd.size_devparams = sizeof(DevParams);
    hd.size_scene = sizeof(SceneState);
    hd.size_global = sizeof(GlobalState);
    hd.bytes = need;
    char* out = static_cast<char*>(dst);
    std::memcpy(out, &hd, sizeof hd);
    char* host_params = out + sizeof hd;
    char* p = host_params + sizeof(fe_params) * ns;
    char* dev_params = p;
    for (const Section& s : state_sections(c, carry)) {
        FE_CUDA(cudaMemcpyAsync(p, s.dev, s.bytes, cudaMemcpyDeviceToHost, c->stream));
        p += s.bytes;
    }
    FE_CUDA(cudaStreamSynchronize(c->stream));
    // the parameter blocks with dt as the device last set it (adaptive CFL)
    for (uint32_t k = 0; k < ns; ++k) {
        fe_params q = c->params[k];
        DevParams dp;
        std::memcpy(&dp, dev_params + sizeof(DevParams) * k, sizeof dp);
        q.dt = dp.dt;
        std::memcpy(host_params + sizeof(fe_params) * k, &q, sizeof q);
    }
    return FE_OK;
}

FE_API fe_status fe_state_import(fe_ctx* c, const void* src, size_t bytes) {
    if (!c || !src) {
        set_error("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    StateHeader hd;
    if (bytes < sizeof hd) {
        set_error("snapshot of %zu bytes is shorter than its header", bytes);
        return FE_ERR_INVALID_ARGUMENT;
    }
    std::memcpy(&hd, src, sizeof hd);
    const uint32_t ns = c->B.n_scenes;
    if (std::memcmp(hd.magic, kStateMagic, sizeof hd.magic) != 0 || hd.version != FE_STATE_VERSION ||
        hd.abi != FE_ABI_VERSION || hd.size_params != sizeof(fe_params) ||
        hd.size_devparams != sizeof(DevParams) || hd.size_scene != sizeof(SceneState) ||
        hd.size_global != sizeof(GlobalState) || hd.has_carry > 1u) {
        set_error("not a snapshot of this library version");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (hd.n != c->n || hd.T != c->T || hd.n_scenes != ns) {
        set_error("snapshot of %u particles / %u slots / %u scenes, context has %u / %u / %u",
                  hd.n, hd.T, hd.n_scenes, c->n, c->T, ns);
        return FE_ERR_INVALID_ARGUMENT;
    }
    const bool carry = hd.has_carry != 0;
    const size_t need = state_bytes(c, carry);
    if (hd.bytes != need || bytes < need) {
        set_error("snapshot should hold %zu bytes (header says %llu, buffer has %zu)", need,
                  (unsigned long long)hd.bytes, bytes);
        return FE_ERR_INVALID_ARGUMENT;
    }
    const char* in = static_cast<const char*>(src);
    const char* host_params = in + sizeof hd;
    const char* dev_params = host_params + sizeof(fe_params) * ns;
    std::vector<fe_params> params(ns);
    std::vector<DevParams> dparams(ns);
    for (uint32_t k = 0; k < ns; ++k) {
        std::memcpy(&params[k], host_params + sizeof(fe_params) * k, sizeof(fe_params));
        std::memcpy(&dparams[k], dev_params + sizeof(DevParams) * k, sizeof(DevParams));
        fe_status s = validate(&params[k]);
        if (s != FE_OK) return s;
        const DevParams& a = dparams[k];
        const DevParams& b = c->dparams[k];
        if (a.n != b.n || a.T != b.T || a.table_base != b.table_base || a.first != b.first) {
            set_error("scene %u: snapshot layout differs from the context's", k);
            return FE_ERR_INVALID_ARGUMENT;
        }
    }
    if (ns > 1 && params[0].sort_algorithm != FE_SORT_RADIX) {
        set_error("bitonic sort is single-scene only");
        return FE_ERR_UNSUPPORTED;
    }
    FE_CUDA(cudaSetDevice(c->device));
    fe_status s = FE_OK;
    const bool had_carry = c->L.carry != nullptr;
    if (carry && (s = ensure_learn_buffers(c)) != FE_OK) return s;
    // Recorded frame graphs stay valid: they reach the state through the
    // same device buffers, and their key covers everything the snapshot can
    // change in a frame's structure (first frame, mode, sort, warm start).
    // Only new learned-state buffers make them stale.
    if (!had_carry && c->L.carry) drop_graphs(c);
    FE_CUDA(cudaStreamSynchronize(c->stream));
    const char* p = dev_params;
    const char* global = nullptr;
    for (const Section& sec : state_sections(c, carry)) {
        if (sec.dev == c->B.G)
            global = p;
        else
            FE_CUDA(cudaMemcpyAsync(sec.dev, p, sec.bytes, cudaMemcpyHostToDevice, c->stream));
        p += sec.bytes;
    }
    if (!carry && c->L.carry && (s = reset_carry(c)) != FE_OK) return s;
    // The neighbour list is not part of a snapshot.  The last pass that
    // built it (density_alpha after the frame's last neighbour search) read
    // only the restored positions and cell table, so running it again
    // rebuilds the same list and rewrites the same densities, factors and
    // p / rho^2.  The global flags are restored after it.
    if (hd.initialized) {
        Recorder R = eager(c);
        if ((s = rec_density_alpha(c, R)) != FE_OK) return s;
    }
    FE_CUDA(cudaMemcpyAsync(c->B.G, global, sizeof(GlobalState), cudaMemcpyHostToDevice,
                            c->stream));
    FE_CUDA(cudaStreamSynchronize(c->stream));
    c->params = params;
    c->dparams = dparams;
    c->initialized = hd.initialized != 0;
    c->last_substeps = hd.last_substeps;
    c->prepared = true;
    return FE_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Test hooks.
// ---------------------------------------------------------------------------
extern "C" {

FE_API void fe_debug_fail_allocation(uint32_t k) { g_fail_countdown.store(k); }

FE_API void fe_debug_poison_allocations(int on) { g_poison.store(on ? 1 : 0); }

FE_API fe_status fe_debug_bounded_wait(int device, uint32_t limit, uint32_t* flags) {
    if (!flags || limit == 0) {
        set_error("fe_debug_bounded_wait needs flags and a non-zero limit");
        return FE_ERR_INVALID_ARGUMENT;
    }
    *flags = 0;
    FE_CUDA(cudaSetDevice(device));
    FE_CUDA(lookback_wait_selftest((int)std::min<uint32_t>(limit, 1u << 30), flags));
    if (*flags & 0x4u) {
        set_error("a bounded device wait timed out (look-back)");
        return FE_ERR_TIMEOUT;
    }
    return FE_OK;
}

}  // extern "C"
