// fe_sort.cu — key/value sorts for the neighbour search.
//
// Radix: stable LSD radix sort with b-bit digits (b = 8 or 10),
// ceil(key_bits / b) passes.  The reference runs count -> single-workgroup
// scan -> scatter per pass with 8-bit digits (radix_count.comp,
// radix_scan.comp, radix_reorder.comp; 12 dispatches for 4 passes).  Here one
// histogram kernel counts all passes' digits in a single read of the keys,
// and each pass is ONE kernel ("onesweep"): a block takes the next tile of
// 256 x items keys from an atomic ticket, ranks them stably with warp
// ballots, publishes its per-digit counts and looks back over the
// preceding tiles' published counts (decoupled look-back) to find where each
// digit of the tile goes, then writes the tile out through shared memory.
// Digit width and keys per thread are template parameters (RadixConfig); the
// result does not depend on them.
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

// One more poll of a look-back wait: false, with the look-back timeout flag
// raised, once `limit` polls are spent.
__device__ __forceinline__ bool lookback_backoff(int& spins, int limit, uint32_t* error_flags) {
    if (++spins > limit) {
        atomicOr(error_flags, 0x4u);
        return false;
    }
    __nanosleep(32);
    return true;
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
template <int kBits>
__global__ void __launch_bounds__(kThreads) k_radix_hist(const uint32_t* __restrict__ keys,
                                                         uint32_t n, int passes,
                                                         uint32_t* __restrict__ hist) {
    constexpr uint32_t kDig = 1u << kBits;
    __shared__ uint32_t s_hist[4][kDig];
    for (uint32_t t = threadIdx.x; t < 4 * kDig; t += kThreads) (&s_hist[0][0])[t] = 0;
    __syncthreads();
    const uint32_t stride = gridDim.x * kThreads;
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
        uint32_t k = keys[i];
        for (int p = 0; p < passes; ++p) atomicAdd(&s_hist[p][(k >> (kBits * p)) & (kDig - 1)], 1u);
    }
    __syncthreads();
    for (int p = 0; p < passes; ++p)
        for (uint32_t d = threadIdx.x; d < kDig; d += kThreads) {
            uint32_t c = s_hist[p][d];
            if (c) atomicAdd(&hist[p * kDig + d], c);
        }
}

// Shared-memory bytes of one pass block.
template <int kBits, int kItems>
constexpr size_t pass_smem_bytes() {
    return 4u * ((size_t)2 * kThreads * kItems + (size_t)kWarps * (1u << kBits) +
                 2u * (1u << kBits) + kWarps + 1);
}

// One onesweep pass (see the file comment) with kBits-bit digits and kItems
// keys per thread; thread t owns digits [t * kDpt, (t + 1) * kDpt) in the
// digit phases.
template <int kBits, int kItems>
constexpr int pass_min_blocks() {
    return (kBits > 8 && kItems > 8) ? 2 : 3;
}

template <int kBits, int kItems>
__global__ void __launch_bounds__(kThreads, pass_min_blocks<kBits, kItems>()) k_radix_pass(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
    uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, uint32_t n, int shift,
    const uint32_t* __restrict__ hist, uint32_t* __restrict__ status,
    uint32_t* __restrict__ tile_counter, uint32_t* __restrict__ error_flags) {
    constexpr uint32_t kDig = 1u << kBits;
    constexpr uint32_t kMask = kDig - 1;
    constexpr int kDpt = (int)(kDig / kThreads);
    constexpr int kTile = kThreads * kItems;
    extern __shared__ __align__(16) uint32_t smem[];
    uint32_t* s_keys = smem;
    uint32_t* s_vals = s_keys + kTile;
    uint32_t* s_whist = s_vals + kTile;            // [kWarps][kDig]
    uint32_t* s_tile_start = s_whist + kWarps * kDig;
    uint32_t* s_dest_base = s_tile_start + kDig;
    uint32_t* s_scan = s_dest_base + kDig;
    uint32_t* s_tile = s_scan + kWarps;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) *s_tile = atomicAdd(tile_counter, 1u);
    for (uint32_t t = threadIdx.x; t < kWarps * kDig; t += kThreads) s_whist[t] = 0;
    __syncthreads();
    const uint32_t tile = *s_tile;
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
    // Stable rank within the warp, items in position order.  The lanes with
    // the same digit are found with one ballot per digit bit (cheaper than a
    // match instruction on this part: the ranking chain dominates the pass).
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
        uint32_t d = (key[it] >> shift) & kMask;
        uint32_t peers = 0xFFFFFFFFu;
#pragma unroll
        for (int b = 0; b < kBits; ++b) {
            const uint32_t bal = __ballot_sync(0xFFFFFFFFu, (d >> b) & 1u);
            peers &= ((d >> b) & 1u) ? bal : ~bal;
        }
        int leader = __ffs(peers) - 1;
        uint32_t before = 0;
        if (lane == leader) {
            before = s_whist[warp * kDig + d];
            s_whist[warp * kDig + d] = before + __popc(peers);
        }
        before = __shfl_sync(0xFFFFFFFFu, before, leader);
        rank[it] = before + __popc(peers & lanemask_lt());
        __syncwarp();
    }
    __syncthreads();

    // Digit phase: warp offsets, tile digit counts and starts.
    const uint32_t d0 = threadIdx.x * kDpt;
    uint32_t count[kDpt];
    uint32_t tsum = 0, hsum = 0, hv[kDpt];
#pragma unroll
    for (int j = 0; j < kDpt; ++j) {
        uint32_t c = 0;
        for (int w = 0; w < kWarps; ++w) {
            uint32_t v = s_whist[w * kDig + d0 + j];
            s_whist[w * kDig + d0 + j] = c;
            c += v;
        }
        count[j] = c;
        tsum += c;
        hv[j] = hist[d0 + j];
        hsum += hv[j];
    }
    uint32_t total;
    uint32_t tile_prefix = block_exclusive_scan(tsum, s_scan, &total);
    uint32_t gprefix = block_exclusive_scan(hsum, s_scan, &total);

    // Publish this tile's per-digit counts before looking back, so that later
    // tiles can proceed.
#pragma unroll
    for (int j = 0; j < kDpt; ++j)
        atomicExch(status + (size_t)tile * kDig + d0 + j, (tile == 0 ? kFlagInc : kFlagAgg) | count[j]);
    uint32_t tstart = tile_prefix, gstart = gprefix;
#pragma unroll
    for (int j = 0; j < kDpt; ++j) {
        const uint32_t d = d0 + j;
        uint32_t excl = 0;
        if (tile > 0) {
            // Look back kLook predecessors per step: their status words are
            // loaded together, then consumed nearest first until an
            // inclusive prefix is found; an unpublished one (flag 0) is
            // re-polled from there.  Each step costs one memory latency
            // instead of kLook.
            constexpr int kLook = 8;
            int pred = (int)tile - 1;
            int spins = 0;
            bool done = false;
            while (!done && pred >= 0) {
                uint32_t v[kLook];
#pragma unroll
                for (int q = 0; q < kLook; ++q)
                    v[q] = pred - q >= 0 ? ld_volatile(status + (size_t)(pred - q) * kDig + d)
                                         : kFlagInc;  // below tile 0: nothing to add
                int used = 0;
                bool stalled = false;
#pragma unroll
                for (int q = 0; q < kLook; ++q) {
                    if (done || stalled) continue;
                    if (pred - q < 0) {
                        done = true;
                        continue;
                    }
                    const uint32_t flag = v[q] & ~kValueMask;
                    if (flag == 0) {
                        stalled = true;
                        continue;
                    }
                    excl += v[q] & kValueMask;
                    ++used;
                    if (flag == kFlagInc) done = true;
                }
                pred -= used;
                if (stalled && !done && !lookback_backoff(spins, kMaxSpins, error_flags)) break;
            }
            atomicExch(status + (size_t)tile * kDig + d, kFlagInc | (excl + count[j]));
        }
        s_tile_start[d] = tstart;
        s_dest_base[d] = gstart + excl - tstart;
        tstart += count[j];
        gstart += hv[j];
    }
    __syncthreads();

    // Scatter into the tile-sorted order in shared memory.
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
        uint32_t d = (key[it] >> shift) & kMask;
        uint32_t q = s_tile_start[d] + s_whist[warp * kDig + d] + rank[it];
        s_keys[q] = key[it];
        s_vals[q] = val[it];
    }
    __syncthreads();

    // Write out in tile-sorted order (runs of equal digits are contiguous in
    // the output too).  Padding entries sort to the tail and are dropped.
    const uint32_t valid = n - base < (uint32_t)kTile ? n - base : (uint32_t)kTile;
    for (uint32_t q = threadIdx.x; q < valid; q += kThreads) {
        uint32_t k = s_keys[q];
        uint32_t dest = s_dest_base[(k >> shift) & kMask] + q;
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

const RadixConfig kRadixCandidates[kRadixCandidateCount] = {
    {8, 4}, {8, 8}, {8, 16}, {10, 8}, {10, 16}};

bool radix_config_valid(RadixConfig c) {
    for (const RadixConfig& k : kRadixCandidates)
        if (k.digit_bits == c.digit_bits && k.items == c.items) return true;
    return false;
}

uint32_t radix_passes(uint32_t key_bits, uint32_t digit_bits) {
    if (key_bits == 0 || key_bits > 32) key_bits = 32;
    return (key_bits + digit_bits - 1) / digit_bits;
}

size_t radix_scratch_words(uint32_t n, uint32_t key_bits, RadixConfig cfg) {
    const uint32_t passes = radix_passes(key_bits, cfg.digit_bits);
    const size_t dig = (size_t)1 << cfg.digit_bits;
    const size_t tile = (size_t)kThreads * cfg.items;
    const size_t tiles = (n + tile - 1) / tile;
    // hist[passes*dig] + counters[passes] (padded to 8) + status[passes*tiles*dig]
    return (size_t)passes * dig + 8 + (size_t)passes * tiles * dig;
}

size_t radix_scratch_words_any(uint32_t n, uint32_t key_bits) {
    size_t w = 0;
    for (const RadixConfig& c : kRadixCandidates) {
        size_t x = radix_scratch_words(n, key_bits, c);
        w = x > w ? x : w;
    }
    return w;
}

namespace {

struct PassKernel {
    const void* pass;
    const void* hist;
    size_t smem;
};

template <int kBits, int kItems>
PassKernel pass_kernel() {
    return {(const void*)k_radix_pass<kBits, kItems>, (const void*)k_radix_hist<kBits>,
            pass_smem_bytes<kBits, kItems>()};
}

bool select_kernel(RadixConfig c, PassKernel* out) {
    if (c.digit_bits == 8 && c.items == 4) *out = pass_kernel<8, 4>();
    else if (c.digit_bits == 8 && c.items == 8) *out = pass_kernel<8, 8>();
    else if (c.digit_bits == 8 && c.items == 16) *out = pass_kernel<8, 16>();
    else if (c.digit_bits == 10 && c.items == 8) *out = pass_kernel<10, 8>();
    else if (c.digit_bits == 10 && c.items == 16) *out = pass_kernel<10, 16>();
    else return false;
    return true;
}

}  // namespace

cudaError_t radix_sort(const SortLaunch& L, uint32_t* keys, uint32_t* vals, uint32_t* tmp_keys,
                       uint32_t* tmp_vals, uint32_t n, uint32_t key_bits, uint32_t* scratch,
                       uint32_t* error_flags, bool* result_in_tmp, RadixConfig cfg) {
    *result_in_tmp = false;
    if (n <= 1) return cudaSuccess;
    PassKernel K;
    if (!select_kernel(cfg, &K)) return cudaErrorInvalidValue;
    if (K.smem > 48 * 1024) {
        // Opt-in above the default 48 KB; applies to the current device.
        cudaError_t a = cudaFuncSetAttribute(K.pass, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)K.smem);
        if (a != cudaSuccess) return a;
    }
    const uint32_t passes = radix_passes(key_bits, cfg.digit_bits);
    const uint32_t dig = 1u << cfg.digit_bits;
    const uint32_t tile = (uint32_t)kThreads * cfg.items;
    const uint32_t tiles = (n + tile - 1) / tile;
    uint32_t* hist = scratch;
    uint32_t* counters = scratch + passes * dig;
    uint32_t* status = counters + 8;
    cudaError_t e = L.fill(scratch, 0u, radix_scratch_words(n, key_bits, cfg));
    if (e != cudaSuccess) return e;
    uint32_t hist_tiles = (n + 4095) / 4096;
    uint32_t hist_blocks = hist_tiles < 4 * 148u ? hist_tiles : 4 * 148u;
    int passes_i = (int)passes;
    e = L.launch(K.hist, dim3(hist_blocks), dim3(kThreads), 0, {(const void*)&keys, &n, &passes_i, &hist});
    if (e != cudaSuccess) return e;
    uint32_t* src_k = keys;
    uint32_t* src_v = vals;
    uint32_t* dst_k = tmp_keys;
    uint32_t* dst_v = tmp_vals;
    for (uint32_t p = 0; p < passes; ++p) {
        int shift = (int)(cfg.digit_bits * p);
        const uint32_t* hp = hist + p * dig;
        uint32_t* sp = status + (size_t)p * tiles * dig;
        uint32_t* cp = counters + p;
        e = L.launch(K.pass, dim3(tiles), dim3(kThreads), K.smem,
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

namespace {
// A look-back wait on a status word that no block ever publishes: it gives
// up after `limit` polls through the same backoff as the radix pass.
__global__ void k_lookback_selftest(const uint32_t* status, uint32_t* error_flags, int limit) {
    int spins = 0;
    while ((ld_volatile(status) & ~kValueMask) == 0)
        if (!lookback_backoff(spins, limit, error_flags)) break;
}
}  // namespace

cudaError_t lookback_wait_selftest(int limit, uint32_t* flags_out) {
    uint32_t* d = nullptr;
    cudaError_t e = cudaMalloc(&d, 8);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemset(d, 0, 8)) == cudaSuccess) {
        k_lookback_selftest<<<1, 1>>>(d, d + 1, limit < kMaxSpins ? limit : kMaxSpins);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpy(flags_out, d + 1, 4, cudaMemcpyDeviceToHost);
    }
    cudaFree(d);
    return e;
}

cudaError_t lookback_wait_on(uint32_t* status, uint32_t* error_flags, int limit,
                             cudaStream_t stream) {
    k_lookback_selftest<<<1, 1, 0, stream>>>(status, error_flags,
                                             limit < kMaxSpins ? limit : kMaxSpins);
    return cudaGetLastError();
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
