// fe_sort.cu — key/value sorts for the neighbour search.
//
// Radix: stable LSD radix sort with 8-bit digits, ceil(key_bits / 8) passes.
// The reference runs count -> single-workgroup scan -> scatter per pass
// (radix_count.comp, radix_scan.comp, radix_reorder.comp; 12 dispatches for
// 4 passes).  Here one histogram kernel counts all passes' digits in a single
// read of the keys, and each pass is ONE kernel ("onesweep"): a block takes
// the next tile of 4096 keys from an atomic ticket, ranks them stably with
// warp match/ballot, publishes its per-digit counts and looks back over the
// preceding tiles' published counts (decoupled look-back) to find where each
// digit of the tile goes, then writes the tile out through shared memory.
// The permutation equals the reference's stable sort (cpu_radix_sort,
// sorter.rs:465-559).  Every wait on another block is bounded: after
// kMaxSpins polls the block records FE_STATS_LOOKBACK_TIMEOUT and moves on,
// so the kernel always terminates.
//
// Bitonic: the compare-exchange network of bitonic_sort.comp driven by the
// (h, step) loops of GpuSorter::execute (sorter.rs:73-115).  Stages whose
// pairs lie inside a 2048-entry tile run in shared memory, several per
// launch; the network and therefore the result are unchanged.
#include <cuda_runtime.h>

#include <cstdint>

#include "fe_sort.h"

namespace fe {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;  // 4096 keys per tile
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1;
constexpr int kMaxSpins = 1 << 22;

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.volatile.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Exclusive scan over 256 threads (one value each).  Returns the exclusive
// prefix; *total gets the sum.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* s_warp,
                                                         uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kWarps ? s_warp[lane] : 0;
        for (int o = 1; o < kWarps; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kWarps) s_warp[lane] = w;  // inclusive warp totals
    }
    __syncthreads();
    uint32_t warp_prefix = warp == 0 ? 0u : s_warp[warp - 1];
    *total = s_warp[kWarps - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

// One read of the keys: digit histograms of all passes.
__global__ void __launch_bounds__(kThreads) k_radix_hist(const uint32_t* __restrict__ keys,
                                                         uint32_t n, int passes,
                                                         uint32_t* __restrict__ hist) {
    __shared__ uint32_t s_hist[4][256];
    for (int t = threadIdx.x; t < 4 * 256; t += kThreads) (&s_hist[0][0])[t] = 0;
    __syncthreads();
    const uint32_t stride = gridDim.x * kThreads;
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
        uint32_t k = keys[i];
        for (int p = 0; p < passes; ++p) atomicAdd(&s_hist[p][(k >> (8 * p)) & 0xFF], 1u);
    }
    __syncthreads();
    for (int p = 0; p < passes; ++p) {
        uint32_t c = s_hist[p][threadIdx.x];
        if (c) atomicAdd(&hist[p * 256 + threadIdx.x], c);
    }
}

// One onesweep pass (see the file comment).
__global__ void __launch_bounds__(kThreads) k_radix_pass(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
    uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, uint32_t n, int shift,
    const uint32_t* __restrict__ hist, uint32_t* __restrict__ status,
    uint32_t* __restrict__ tile_counter, uint32_t* __restrict__ error_flags) {
    __shared__ uint32_t s_keys[kTile];
    __shared__ uint32_t s_vals[kTile];
    __shared__ uint32_t s_whist[kWarps][256];
    __shared__ uint32_t s_tile_start[256];
    __shared__ uint32_t s_dest_base[256];
    __shared__ uint32_t s_scan[kWarps];
    __shared__ uint32_t s_tile;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int d_self = threadIdx.x;  // digit owned by this thread in the digit phases
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    for (int t = threadIdx.x; t < kWarps * 256; t += kThreads) (&s_whist[0][0])[t] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t base = tile * kTile;

    // Load (warp-striped: item it of lane l at warp*32*kItems + it*32 + l).
    uint32_t key[kItems], val[kItems], rank[kItems];
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
        uint32_t pos = base + warp * 32 * kItems + it * 32 + lane;
        bool ok = pos < n;
        key[it] = ok ? keys_in[pos] : 0xFFFFFFFFu;
        val[it] = ok ? vals_in[pos] : 0u;
    }
    // Stable rank within the warp, items in position order.
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
        uint32_t d = (key[it] >> shift) & 0xFF;
        uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        int leader = __ffs(peers) - 1;
        uint32_t before = 0;
        if (lane == leader) {
            before = s_whist[warp][d];
            s_whist[warp][d] = before + __popc(peers);
        }
        before = __shfl_sync(0xFFFFFFFFu, before, leader);
        rank[it] = before + __popc(peers & lanemask_lt());
        __syncwarp();
    }
    __syncthreads();

    // Digit phase: warp offsets, tile digit counts and starts.
    uint32_t count = 0;
    for (int w = 0; w < kWarps; ++w) {
        uint32_t c = s_whist[w][d_self];
        s_whist[w][d_self] = count;
        count += c;
    }
    uint32_t total;
    uint32_t tile_start = block_exclusive_scan(count, s_scan, &total);
    s_tile_start[d_self] = tile_start;

    // Global digit base: exclusive scan of this pass's histogram.
    uint32_t gbase = block_exclusive_scan(hist[d_self], s_scan, &total);

    // Decoupled look-back for digit d_self.
    uint32_t* my = status + (size_t)tile * 256 + d_self;
    uint32_t excl = 0;
    if (tile == 0) {
        atomicExch(my, kFlagInc | count);
    } else {
        atomicExch(my, kFlagAgg | count);
        int pred = (int)tile - 1;
        int spins = 0;
        while (pred >= 0) {
            uint32_t v = ld_volatile(status + (size_t)pred * 256 + d_self);
            uint32_t flag = v & ~kValueMask;
            if (flag == 0) {
                if (++spins > kMaxSpins) {
                    atomicOr(error_flags, 0x4u);
                    break;
                }
                __nanosleep(32);
                continue;
            }
            excl += v & kValueMask;
            if (flag == kFlagInc) break;
            --pred;
        }
        atomicExch(my, kFlagInc | (excl + count));
    }
    s_dest_base[d_self] = gbase + excl - tile_start;
    __syncthreads();

    // Scatter into the tile-sorted order in shared memory.
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
        uint32_t d = (key[it] >> shift) & 0xFF;
        uint32_t q = s_tile_start[d] + s_whist[warp][d] + rank[it];
        s_keys[q] = key[it];
        s_vals[q] = val[it];
    }
    __syncthreads();

    // Write out in tile-sorted order (runs of equal digits are contiguous in
    // the output too).  Padding entries sort to the tail and are dropped.
    const uint32_t valid = n - base < (uint32_t)kTile ? n - base : (uint32_t)kTile;
    for (uint32_t q = threadIdx.x; q < valid; q += kThreads) {
        uint32_t k = s_keys[q];
        uint32_t dest = s_dest_base[(k >> shift) & 0xFF] + q;
        if (dest < n) {  // always true unless a look-back wait gave up
            keys_out[dest] = k;
            vals_out[dest] = s_vals[q];
        }
    }
}

// Bitonic compare-exchange of one (h, step) stage over global memory
// (bitonic_sort.comp:19-43).
__global__ void k_bitonic_global(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t h,
                                 uint32_t step) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n / 2) return;
    uint32_t left = (i / step) * step * 2 + (i % step);
    uint32_t right = left + step;
    uint32_t kl = keys[left], kr = keys[right];
    bool asc = (left & h) == 0u;
    if ((asc && kl > kr) || (!asc && kl < kr)) {
        keys[left] = kr;
        keys[right] = kl;
        uint32_t t = vals[left];
        vals[left] = vals[right];
        vals[right] = t;
    }
}

constexpr int kBitonicTile = 2048;  // entries per block in shared memory

// All stages (h, step) with h in [h_lo, h_hi] and step < kBitonicTile whose
// pairs lie in one 2048-entry tile: for h <= kBitonicTile every step, for a
// larger h only the steps below the tile size (h_lo == h_hi then).
__global__ void __launch_bounds__(1024) k_bitonic_local(uint32_t* keys, uint32_t* vals,
                                                        uint32_t n, uint32_t h_lo,
                                                        uint32_t h_hi) {
    __shared__ uint32_t sk[kBitonicTile];
    __shared__ uint32_t sv[kBitonicTile];
    const uint32_t base = blockIdx.x * kBitonicTile;
    for (int t = threadIdx.x; t < kBitonicTile; t += blockDim.x) {
        sk[t] = keys[base + t];
        sv[t] = vals[base + t];
    }
    __syncthreads();
    const uint32_t i = threadIdx.x;  // compare-exchange index within the tile
    for (uint32_t h = h_lo; h <= h_hi; h *= 2) {
        uint32_t first = h / 2 < (uint32_t)kBitonicTile / 2 ? h / 2 : (uint32_t)kBitonicTile / 2;
        for (uint32_t step = first; step > 0; step /= 2) {
            uint32_t l = (i / step) * step * 2 + (i % step);
            uint32_t r = l + step;
            uint32_t kl = sk[l], kr = sk[r];
            bool asc = ((base + l) & h) == 0u;
            if ((asc && kl > kr) || (!asc && kl < kr)) {
                sk[l] = kr;
                sk[r] = kl;
                uint32_t t = sv[l];
                sv[l] = sv[r];
                sv[r] = t;
            }
            __syncthreads();
        }
    }
    for (int t = threadIdx.x; t < kBitonicTile; t += blockDim.x) {
        keys[base + t] = sk[t];
        vals[base + t] = sv[t];
    }
}

}  // namespace

uint32_t radix_passes(uint32_t key_bits) {
    if (key_bits == 0 || key_bits > 32) key_bits = 32;
    return (key_bits + 7) / 8;
}

size_t radix_scratch_words(uint32_t n, uint32_t key_bits) {
    uint32_t passes = radix_passes(key_bits);
    size_t tiles = (n + kTile - 1) / kTile;
    // hist[passes*256] + counters[passes] (padded to 8) + status[passes*tiles*256]
    return (size_t)passes * 256 + 8 + (size_t)passes * tiles * 256;
}

cudaError_t radix_sort(const SortLaunch& L, uint32_t* keys, uint32_t* vals, uint32_t* tmp_keys,
                       uint32_t* tmp_vals, uint32_t n, uint32_t key_bits, uint32_t* scratch,
                       uint32_t* error_flags, bool* result_in_tmp) {
    *result_in_tmp = false;
    if (n <= 1) return cudaSuccess;
    const uint32_t passes = radix_passes(key_bits);
    const uint32_t tiles = (n + kTile - 1) / kTile;
    uint32_t* hist = scratch;
    uint32_t* counters = scratch + passes * 256;
    uint32_t* status = counters + 8;
    cudaError_t e = L.fill(scratch, 0u, radix_scratch_words(n, key_bits));
    if (e != cudaSuccess) return e;
    uint32_t hist_blocks = tiles < 4 * 148u ? tiles : 4 * 148u;
    int passes_i = (int)passes;
    e = L.launch((const void*)k_radix_hist, dim3(hist_blocks), dim3(kThreads), 0,
                 {(const void*)&keys, &n, &passes_i, &hist});
    if (e != cudaSuccess) return e;
    uint32_t* src_k = keys;
    uint32_t* src_v = vals;
    uint32_t* dst_k = tmp_keys;
    uint32_t* dst_v = tmp_vals;
    for (uint32_t p = 0; p < passes; ++p) {
        int shift = 8 * p;
        const uint32_t* hp = hist + p * 256;
        uint32_t* sp = status + (size_t)p * tiles * 256;
        uint32_t* cp = counters + p;
        e = L.launch((const void*)k_radix_pass, dim3(tiles), dim3(kThreads), 0,
                     {&src_k, &src_v, &dst_k, &dst_v, &n, &shift, &hp, &sp, &cp, &error_flags});
        if (e != cudaSuccess) return e;
        uint32_t* tk = src_k;
        uint32_t* tv = src_v;
        src_k = dst_k;
        src_v = dst_v;
        dst_k = tk;
        dst_v = tv;
    }
    *result_in_tmp = (passes % 2) == 1;
    return cudaSuccess;
}

cudaError_t bitonic_sort(const SortLaunch& L, uint32_t* keys, uint32_t* vals, uint32_t n) {
    if (n < 2) return cudaSuccess;
    if (n & (n - 1)) return cudaErrorInvalidValue;
    cudaError_t e;
    if (n <= (uint32_t)kBitonicTile) {
        // one block, all stages (tile = the whole array)
        uint32_t h_lo = 2, h_hi = n;
        // k_bitonic_local needs a full tile; run the global kernel instead
        for (uint32_t h = h_lo; h <= h_hi; h *= 2)
            for (uint32_t step = h / 2; step > 0; step /= 2) {
                uint32_t threads = n / 2;
                uint32_t blocks = (threads + 255) / 256;
                e = L.launch((const void*)k_bitonic_global, dim3(blocks), dim3(256), 0,
                             {&keys, &vals, &n, &h, &step});
                if (e != cudaSuccess) return e;
            }
        return cudaSuccess;
    }
    const uint32_t blocks_local = n / kBitonicTile;
    uint32_t h_lo = 2, h_hi = kBitonicTile;
    e = L.launch((const void*)k_bitonic_local, dim3(blocks_local), dim3(kBitonicTile / 2), 0,
                 {&keys, &vals, &n, &h_lo, &h_hi});
    if (e != cudaSuccess) return e;
    for (uint32_t h = 2 * kBitonicTile; h <= n; h *= 2) {
        for (uint32_t step = h / 2; step >= (uint32_t)kBitonicTile; step /= 2) {
            uint32_t blocks = (n / 2 + 255) / 256;
            e = L.launch((const void*)k_bitonic_global, dim3(blocks), dim3(256), 0,
                         {&keys, &vals, &n, &h, &step});
            if (e != cudaSuccess) return e;
        }
        e = L.launch((const void*)k_bitonic_local, dim3(blocks_local), dim3(kBitonicTile / 2), 0,
                     {&keys, &vals, &n, &h, &h});
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace fe
