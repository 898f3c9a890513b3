// fe_mlp.cu — the learned warm start: a 12 -> 64 -> 64 -> 2 MLP with SiLU,
// BF16 weights and activations, FP32 accumulation, on the 5th-generation
// tensor cores (tcgen05.mma, accumulators in tensor memory).
//
// One 128-thread block works on tiles of 128 samples.  Thread 0 issues the
// MMAs (cta_group::1, kind::f16, M = 128); operands live in shared memory in
// the canonical no-swizzle layouts; the accumulators sit in TMEM and every
// warp reads back its 32 rows with tcgen05.ld for the epilogue (bias, SiLU,
// BF16 rounding).  Training adds the backward pass on the same units:
// activation gradients as M = 128 products, weight gradients as products
// over the sample dimension with the feature dimension padded to M = 128,
// accumulated in TMEM across all tiles of the block; bias gradients and the
// loss are warp reductions.  Adam runs on the FP32 master weights.
//
// Every wait on an MMA completion is bounded: on time-out the block records
// FE_STATS_LOOKBACK_TIMEOUT in the error word, releases its TMEM and stops.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "fe_features.cuh"
#include "fe_mlp.h"

namespace fe {
namespace mlp {

namespace {

constexpr int kThreads = 128;
constexpr int kTile = 128;
constexpr uint32_t kMaxSpins = 1u << 24;

// ---------------------------------------------------------------------------
// Canonical K-major no-swizzle layout of a [rows x K] BF16 tile: 8 x 8
// element core matrices (8 rows of 16 bytes), K-groups 128 bytes apart
// (leading byte offset), 8-row groups K * 16 bytes apart (stride byte offset).
// Read as the transposed operand, the same bytes form the canonical
// MN-major layout with SBO = 128 and LBO = K * 16.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t off_k(uint32_t r, uint32_t k, uint32_t K) {
    return (r >> 3) * (K * 16u) + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}
// Transposed, feature-padded copy for the weight-gradient A operand:
// MN = feature (128 rows, zero beyond the real width), K = sample.
__device__ __forceinline__ uint32_t off_t(uint32_t s, uint32_t f) {
    return (s >> 3) * 2048u + (f >> 3) * 128u + (s & 7u) * 16u + (f & 7u) * 2u;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    return d;                // base offset 0, no swizzle
}

// Instruction descriptor of kind::f16: D F32, A and B BF16.
__host__ __device__ constexpr uint32_t idesc(uint32_t M, uint32_t N, uint32_t a_mn, uint32_t b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn << 15) | (b_mn << 16) | ((N >> 3) << 17) |
           ((M >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t id,
                                    uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(id), "r"(accumulate));
}

__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void bar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the given phase parity.  Returns false on time-out.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity) {
    uint32_t addr = smem_u32(bar);
    for (uint32_t spin = 0; spin < kMaxSpins; ++spin) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// The hardware tanh (PTX tanh.approx.f32: one special-function-unit op,
// about 2^-11 relative error, far below the network's BF16 rounding).
__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// SiLU z * sigmoid(z) with sigmoid(z) = (1 + tanh(z / 2)) / 2, i.e.
// s + s * tanh(s) for s = z / 2: one special-function op per activation
// instead of an exponential and a reciprocal, and one fused multiply-add.
__device__ __forceinline__ float silu_half(float s) { return __fmaf_rn(s, tanh_hw(s), s); }
__device__ __forceinline__ float silu(float z) { return silu_half(0.5f * z); }
__device__ __forceinline__ float silu_grad(float z) {
    const float sg = 0.5f + 0.5f * tanh_hw(0.5f * z);
    return sg * (1.0f + z * (1.0f - sg));
}

__device__ __forceinline__ void st_bf16(uint8_t* base, uint32_t off, float v) {
    *reinterpret_cast<__nv_bfloat16*>(base + off) = __float2bfloat16_rn(v);
}

// Shared-memory image of the weights (canonical K-major tiles).
struct SmemWeights {
    alignas(128) uint8_t w1[64 * 16 * 2];   // [64 out x 16 in]
    alignas(128) uint8_t w2[64 * 64 * 2];   // [64 out x 64 in]
    alignas(128) uint8_t w3[16 * 64 * 2];   // [16 out x 64 in], rows >= 2 zero
    float b1[64], b2[64], b3[16];
};

// Weights are stored row-major BF16 [out][in] (W3 with 2 real rows).
__device__ void load_weights(SmemWeights& W, const Params& P) {
    for (int t = threadIdx.x; t < 64 * 16; t += kThreads) {
        int o = t / 16, k = t % 16;
        *reinterpret_cast<__nv_bfloat16*>(W.w1 + off_k(o, k, 16)) = P.w1[t];
    }
    for (int t = threadIdx.x; t < 64 * 64; t += kThreads) {
        int o = t / 64, k = t % 64;
        *reinterpret_cast<__nv_bfloat16*>(W.w2 + off_k(o, k, 64)) = P.w2[t];
    }
    for (int t = threadIdx.x; t < 16 * 64; t += kThreads) {
        int o = t / 64, k = t % 64;
        __nv_bfloat16 v = o < 2 ? P.w3[o * 64 + k] : __float2bfloat16_rn(0.0f);
        *reinterpret_cast<__nv_bfloat16*>(W.w3 + off_k(o, k, 64)) = v;
    }
    for (int t = threadIdx.x; t < 64; t += kThreads) {
        W.b1[t] = P.b1[t];
        W.b2[t] = P.b2[t];
    }
    for (int t = threadIdx.x; t < 16; t += kThreads) W.b3[t] = t < 2 ? P.b3[t] : 0.0f;
}

struct TmemAlloc {
    uint32_t base;
};

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(slot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
}

__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols) {
    if (threadIdx.x < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols)
                     : "memory");
}

// TMEM address of (row block of this warp, column c).
__device__ __forceinline__ uint32_t lane_addr(uint32_t base, uint32_t col) {
    uint32_t warp = threadIdx.x >> 5;
    return base + ((warp * 32u) << 16) + col;
}

// Layer epilogue: 64 accumulator columns of this thread's row -> +bias ->
// SiLU -> BF16 into a K-major [128 x 64] tile; optionally keeps z.
__device__ __forceinline__ void epilogue_silu64(uint32_t taddr, const float* bias, uint8_t* out,
                                                uint32_t row) {
#pragma unroll
    for (int c0 = 0; c0 < 64; c0 += 16) {
        float v[16];
        tmem_ld16(taddr + c0, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) st_bf16(out, off_k(row, c0 + i, 64), silu(v[i] + bias[c0 + i]));
    }
}

constexpr int kInferThreads = 256;

__device__ __forceinline__ uint32_t lane_addr8(uint32_t base, uint32_t col) {
    uint32_t warp = threadIdx.x >> 5;
    return base + (((warp & 3u) * 32u) << 16) + col;
}

// 32 accumulator columns [c0, c0 + 32) of this warp's rows -> bias + SiLU ->
// BF16 into the K-major [128 x 64] tile.  Eight consecutive columns of a row
// are 16 contiguous bytes of the canonical layout: one 16-byte store each.
__device__ __forceinline__ void epilogue_half(uint32_t taddr, uint32_t c0, const float* bias,
                                              uint8_t* out, uint32_t row) {
#pragma unroll
    for (uint32_t cc = 0; cc < 32; cc += 16) {
        float v[16];
        tmem_ld16(taddr + c0 + cc, v);
#pragma unroll
        for (int g = 0; g < 16; g += 8) {
            uint32_t w[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t c = c0 + cc + g + 2 * j;
                // bias holds b / 2: fma(v, 1/2, b / 2) = (v + b) / 2 exactly as
                // the training kernel's 0.5f * (v + b) (halving is exact)
                __nv_bfloat162 two = __floats2bfloat162_rn(
                    silu_half(__fmaf_rn(v[g + 2 * j], 0.5f, bias[c])),
                    silu_half(__fmaf_rn(v[g + 2 * j + 1], 0.5f, bias[c + 1])));
                w[j] = *reinterpret_cast<uint32_t*>(&two);
            }
            *reinterpret_cast<uint4*>(out + off_k(row, c0 + cc + g, 64)) =
                make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

// ---------------------------------------------------------------------------
// Inference: out[i][0..1] = MLP(x_i) for n rows of X (BF16, 16 per row),
// on pairs of 128-row tiles: a block of 256 threads takes tiles 2p and
// 2p + 1 together (accumulators in TMEM columns [0, 64) and [64, 128));
// warps 0-3 serve the first tile's rows and warps 4-7 the second's, each
// warp all 64 columns of its 32 rows.  Each barrier and product round trip
// then serves 256 rows, and four blocks per SM keep eight tiles in flight.
// With kApply the epilogue also starts solve A.which from the output it has
// just written (warm_apply_particle).
// ---------------------------------------------------------------------------
struct InferPairSmem {
    SmemWeights W;
    alignas(128) uint8_t x[2][kTile * 16 * 2];
    alignas(128) uint8_t h[2][kTile * 64 * 2];
    alignas(8) uint64_t bar;
    uint32_t tmem_base;
};
constexpr int kInferPairMaxCtasPerSm = 4;   // 4 x 128 TMEM columns fill an SM

template <bool kApply>
__global__ void __launch_bounds__(kInferThreads) k_mlp_infer_pair(
    Params P, const __nv_bfloat16* __restrict__ X, float* __restrict__ out, uint32_t n,
    uint32_t* error_flags, ApplyArgs A) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    InferPairSmem& S = *reinterpret_cast<InferPairSmem*>(smem_raw);
    const uint32_t tid = threadIdx.x;
    const uint32_t warp = tid >> 5, lane = tid & 31u;
    const uint32_t sub = warp >> 2;                  // the tile of the pair this warp serves
    const uint32_t row = (warp & 3u) * 32u + lane;   // TMEM lane = sample row
    for (int t = tid; t < 64 * 16; t += kInferThreads)
        *reinterpret_cast<__nv_bfloat16*>(S.W.w1 + off_k(t / 16, t % 16, 16)) = P.w1[t];
    for (int t = tid; t < 64 * 64; t += kInferThreads)
        *reinterpret_cast<__nv_bfloat16*>(S.W.w2 + off_k(t / 64, t % 64, 64)) = P.w2[t];
    for (int t = tid; t < 16 * 64; t += kInferThreads) {
        int o = t / 64, k = t % 64;
        *reinterpret_cast<__nv_bfloat16*>(S.W.w3 + off_k(o, k, 64)) =
            o < 2 ? P.w3[o * 64 + k] : __float2bfloat16_rn(0.0f);
    }
    if (tid < 64) {  // hidden-layer biases halved for the epilogue's fused SiLU
        S.W.b1[tid] = 0.5f * P.b1[tid];
        S.W.b2[tid] = 0.5f * P.b2[tid];
    }
    if (tid < 16) S.W.b3[tid] = tid < 2 ? P.b3[tid] : 0.0f;
    if (tid == 0) bar_init(&S.bar);
    tmem_alloc(&S.tmem_base, 128);
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t d = S.tmem_base;
    const uint32_t ta = lane_addr8(d, 64u * sub);
    uint32_t phase = 0;
    bool ok = true;
    const uint32_t npairs = (n + 2 * kTile - 1) / (2 * kTile);
    const uint64_t dw1 = desc(smem_u32(S.W.w1), 128, 256);
    for (uint32_t pr = blockIdx.x; pr < npairs && ok; pr += gridDim.x) {
        // X rows of both tiles: 16 bytes per thread and step (row tid / 2,
        // half tid % 2), two steps
        for (uint32_t q = 0; q < 2; ++q) {
            const uint32_t r = tid >> 1, part = tid & 1u;
            const uint32_t g = (2 * pr + q) * kTile + r;
            uint4 a = make_uint4(0, 0, 0, 0);
            if (g < n) a = reinterpret_cast<const uint4*>(X + (size_t)g * 16)[part];
            *reinterpret_cast<uint4*>(S.x[q] + off_k(r, part * 8, 16)) = a;
        }
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc_after_sync();
            for (uint32_t q = 0; q < 2; ++q)
                mma(d + 64u * q, desc(smem_u32(S.x[q]), 128, 256), dw1, idesc(128, 64, 0, 0), 0);
            commit(&S.bar);
        }
        ok = __syncthreads_and(bar_wait(&S.bar, phase));
        phase ^= 1;
        tc_after_sync();
        if (ok) {
            epilogue_half(ta, 0, S.W.b1, S.h[sub], row);
            epilogue_half(ta, 32, S.W.b1, S.h[sub], row);
        }
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        if (tid == 0 && ok) {
            tc_after_sync();
            for (uint32_t q = 0; q < 2; ++q)
                for (uint32_t kk = 0; kk < 4; ++kk)
                    mma(d + 64u * q, desc(smem_u32(S.h[q]) + kk * 256, 128, 1024),
                        desc(smem_u32(S.W.w2) + kk * 256, 128, 1024), idesc(128, 64, 0, 0), kk > 0);
            commit(&S.bar);
        }
        ok = __syncthreads_and(ok && bar_wait(&S.bar, phase));
        phase ^= 1;
        tc_after_sync();
        if (ok) {
            epilogue_half(ta, 0, S.W.b2, S.h[sub], row);
            epilogue_half(ta, 32, S.W.b2, S.h[sub], row);
        }
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        if (tid == 0 && ok) {
            tc_after_sync();
            for (uint32_t q = 0; q < 2; ++q)
                for (uint32_t kk = 0; kk < 4; ++kk)
                    mma(d + 64u * q, desc(smem_u32(S.h[q]) + kk * 256, 128, 1024),
                        desc(smem_u32(S.W.w3) + kk * 256, 128, 1024), idesc(128, 16, 0, 0), kk > 0);
            commit(&S.bar);
        }
        ok = __syncthreads_and(ok && bar_wait(&S.bar, phase));
        phase ^= 1;
        tc_after_sync();
        if (ok) {
            float v[16];
            tmem_ld16(ta, v);
            const uint32_t g = (2 * pr + sub) * kTile + row;
            if (g < n) {
                const float o0 = v[0] + S.W.b3[0], o1 = v[1] + S.W.b3[1];
                reinterpret_cast<float2*>(out)[g] = make_float2(o0, o1);
                if (kApply)
                    warm_apply_particle(A.B, A.L, A.B.P[scene_of(A.B, g)], g, A.which,
                                        A.which == 0 ? o0 : o1);
            }
        }
        tc_before_sync();
        __syncthreads();
        tc_after_sync();
    }
    if (!ok && tid == 0) atomicOr(error_flags, 0x4u);
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    tmem_free(d, 128);
}

// ---------------------------------------------------------------------------
// Training step: gradients of the mean squared error over n samples
// (normalised targets; a NaN target masks that output of the sample),
// accumulated into grads (FP32, atomics, one add per parameter per block).  512 TMEM columns, one block per SM (the shared
// memory footprint keeps it so).
// ---------------------------------------------------------------------------
struct TrainSmem {
    SmemWeights W;
    alignas(128) uint8_t x[kTile * 16 * 2];
    alignas(128) uint8_t h1[kTile * 64 * 2];
    alignas(128) uint8_t h2[kTile * 64 * 2];
    alignas(128) uint8_t dout[kTile * 16 * 2];   // K-major [128 x 16]
    alignas(128) uint8_t dz[kTile * 64 * 2];     // K-major [128 x 64] (dZ2)
    alignas(128) uint8_t doutT[2048 * 16];       // transposed, padded to 128 features
    alignas(128) uint8_t dz2T[2048 * 16];
    alignas(128) uint8_t dz1T[2048 * 16];
    float db1[4][64], db2[4][64], db3[4][2];  // per warp: one writer each, summed in warp order
    float loss[4];
    alignas(8) uint64_t bar;
    uint32_t tmem_base;
};

__device__ __forceinline__ float warp_sum(float v) {
    for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, m);
    return v;
}

// Each block writes its gradient sums (kParams floats in the Grads layout,
// then the loss) to its own slice part[blockIdx.x][kParams + 1]; k_sum_parts
// adds the slices in block order, so the result does not depend on timing.
__global__ void __launch_bounds__(kThreads, 1) k_mlp_train(Params P, const __nv_bfloat16* __restrict__ X,
                                                          const float* __restrict__ Y, uint32_t n,
                                                          float inv_count, float* __restrict__ part,
                                                          uint32_t* error_flags) {
    Grads G = grads_from(part + (size_t)blockIdx.x * (kParams + 1),
                         part + (size_t)blockIdx.x * (kParams + 1) + kParams);
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
    const uint32_t tid = threadIdx.x;
    load_weights(S.W, P);
    // zero the padded transposes once: rows beyond the real width stay zero
    for (uint32_t t = tid; t < 2048 * 16 / 16; t += kThreads) {
        reinterpret_cast<uint4*>(S.doutT)[t] = make_uint4(0, 0, 0, 0);
        reinterpret_cast<uint4*>(S.dz2T)[t] = make_uint4(0, 0, 0, 0);
        reinterpret_cast<uint4*>(S.dz1T)[t] = make_uint4(0, 0, 0, 0);
    }
    for (uint32_t t = tid; t < 4 * 64; t += kThreads) (&S.db1[0][0])[t] = (&S.db2[0][0])[t] = 0.0f;
    if (tid < 8) (&S.db3[0][0])[tid] = 0.0f;
    if (tid < 4) S.loss[tid] = 0.0f;
    if (tid == 0) bar_init(&S.bar);
    tmem_alloc(&S.tmem_base, 512);
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tb = S.tmem_base;
    const uint32_t c_z1 = tb, c_z2 = tb + 64, c_o = tb + 128, c_dh = tb + 192;
    const uint32_t c_dw1 = tb + 256, c_dw2 = tb + 320, c_dw3 = tb + 384;
    uint32_t phase = 0;
    bool ok = true;
    uint32_t local_tiles = 0;
    const uint32_t ntiles = (n + kTile - 1) / kTile;
    const uint32_t row = tid;
    for (uint32_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++local_tiles) {
        const uint32_t g = tile * kTile + row;
        const bool valid = g < n;
        {
            uint4 a = make_uint4(0, 0, 0, 0), b = a;
            if (valid) {
                const uint4* src = reinterpret_cast<const uint4*>(X + (size_t)g * 16);
                a = src[0];
                b = src[1];
            }
            *reinterpret_cast<uint4*>(S.x + off_k(row, 0, 16)) = a;
            *reinterpret_cast<uint4*>(S.x + off_k(row, 8, 16)) = b;
        }
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        // ---- forward
        if (tid == 0) {
            tc_after_sync();
            mma(c_z1, desc(smem_u32(S.x), 128, 256), desc(smem_u32(S.W.w1), 128, 256),
                idesc(128, 64, 0, 0), 0);
            commit(&S.bar);
        }
        ok = __syncthreads_and(bar_wait(&S.bar, phase));
        phase ^= 1;
        tc_after_sync();
        if (ok) epilogue_silu64(lane_addr(c_z1, 0), S.W.b1, S.h1, row);
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        if (tid == 0 && ok) {
            tc_after_sync();
            for (uint32_t kk = 0; kk < 4; ++kk)
                mma(c_z2, desc(smem_u32(S.h1) + kk * 256, 128, 1024),
                    desc(smem_u32(S.W.w2) + kk * 256, 128, 1024), idesc(128, 64, 0, 0), kk > 0);
            commit(&S.bar);
        }
        ok = __syncthreads_and(ok && bar_wait(&S.bar, phase));
        phase ^= 1;
        tc_after_sync();
        if (ok) epilogue_silu64(lane_addr(c_z2, 0), S.W.b2, S.h2, row);
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        if (tid == 0 && ok) {
            tc_after_sync();
            for (uint32_t kk = 0; kk < 4; ++kk)
                mma(c_o, desc(smem_u32(S.h2) + kk * 256, 128, 1024),
                    desc(smem_u32(S.W.w3) + kk * 256, 128, 1024), idesc(128, 16, 0, 0), kk > 0);
            commit(&S.bar);
        }
        ok = __syncthreads_and(ok && bar_wait(&S.bar, phase));
        phase ^= 1;
        tc_after_sync();
        // ---- loss gradient dO = 2 (O - Y) / count (rows beyond n: 0)
        if (ok) {
            float v[16];
            tmem_ld16(lane_addr(c_o, 0), v);
            // A NaN target means "no target for this output" (masked).
            float e0 = 0.0f, e1 = 0.0f;
            if (valid) {
                const float y0 = Y[2 * (size_t)g], y1 = Y[2 * (size_t)g + 1];
                e0 = y0 == y0 ? v[0] + S.W.b3[0] - y0 : 0.0f;
                e1 = y1 == y1 ? v[1] + S.W.b3[1] - y1 : 0.0f;
            }
            float g0 = 2.0f * e0 * inv_count, g1 = 2.0f * e1 * inv_count;
            float l = warp_sum(e0 * e0 + e1 * e1);
            float s0 = warp_sum(g0), s1 = warp_sum(g1);
            if ((tid & 31) == 0) {
                S.loss[tid >> 5] += l;
                S.db3[tid >> 5][0] += s0;
                S.db3[tid >> 5][1] += s1;
            }
            for (int c = 0; c < 16; ++c) {
                float gv = c == 0 ? g0 : (c == 1 ? g1 : 0.0f);
                st_bf16(S.dout, off_k(row, c, 16), gv);
            }
            st_bf16(S.doutT, off_t(row, 0), g0);
            st_bf16(S.doutT, off_t(row, 1), g1);
        }
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        // ---- dH2 = dO . W3 ; dW3 += dO^T . H2
        if (tid == 0 && ok) {
            tc_after_sync();
            mma(c_dh, desc(smem_u32(S.dout), 128, 256), desc(smem_u32(S.W.w3), 1024, 128),
                idesc(128, 64, 0, 1), 0);
            for (uint32_t kk = 0; kk < 8; ++kk)
                mma(c_dw3, desc(smem_u32(S.doutT) + kk * 4096, 2048, 128),
                    desc(smem_u32(S.h2) + kk * 2048, 1024, 128), idesc(128, 64, 1, 1),
                    (local_tiles > 0 || kk > 0) ? 1u : 0u);
            commit(&S.bar);
        }
        ok = __syncthreads_and(ok && bar_wait(&S.bar, phase));
        phase ^= 1;
        tc_after_sync();
        // ---- dZ2 = dH2 * silu'(Z2)
        if (ok) {
#pragma unroll
            for (int c0 = 0; c0 < 64; c0 += 16) {
                float dh[16], z[16];
                tmem_ld16(lane_addr(c_dh, c0), dh);
                tmem_ld16(lane_addr(c_z2, c0), z);
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    float d = valid ? dh[i] * silu_grad(z[i] + S.W.b2[c0 + i]) : 0.0f;
                    st_bf16(S.dz, off_k(row, c0 + i, 64), d);
                    st_bf16(S.dz2T, off_t(row, c0 + i), d);
                    float s = warp_sum(d);
                    if ((tid & 31) == 0) S.db2[tid >> 5][c0 + i] += s;
                }
            }
        }
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        // ---- dH1 = dZ2 . W2 ; dW2 += dZ2^T . H1
        if (tid == 0 && ok) {
            tc_after_sync();
            for (uint32_t kk = 0; kk < 4; ++kk)
                mma(c_dh, desc(smem_u32(S.dz) + kk * 256, 128, 1024),
                    desc(smem_u32(S.W.w2) + kk * 2048, 1024, 128), idesc(128, 64, 0, 1), kk > 0);
            for (uint32_t kk = 0; kk < 8; ++kk)
                mma(c_dw2, desc(smem_u32(S.dz2T) + kk * 4096, 2048, 128),
                    desc(smem_u32(S.h1) + kk * 2048, 1024, 128), idesc(128, 64, 1, 1),
                    (local_tiles > 0 || kk > 0) ? 1u : 0u);
            commit(&S.bar);
        }
        ok = __syncthreads_and(ok && bar_wait(&S.bar, phase));
        phase ^= 1;
        tc_after_sync();
        // ---- dZ1 = dH1 * silu'(Z1)
        if (ok) {
#pragma unroll
            for (int c0 = 0; c0 < 64; c0 += 16) {
                float dh[16], z[16];
                tmem_ld16(lane_addr(c_dh, c0), dh);
                tmem_ld16(lane_addr(c_z1, c0), z);
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    float d = valid ? dh[i] * silu_grad(z[i] + S.W.b1[c0 + i]) : 0.0f;
                    st_bf16(S.dz1T, off_t(row, c0 + i), d);
                    float s = warp_sum(d);
                    if ((tid & 31) == 0) S.db1[tid >> 5][c0 + i] += s;
                }
            }
        }
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        // ---- dW1 += dZ1^T . X
        if (tid == 0 && ok) {
            tc_after_sync();
            for (uint32_t kk = 0; kk < 8; ++kk)
                mma(c_dw1, desc(smem_u32(S.dz1T) + kk * 4096, 2048, 128),
                    desc(smem_u32(S.x) + kk * 512, 256, 128), idesc(128, 16, 1, 1),
                    (local_tiles > 0 || kk > 0) ? 1u : 0u);
            commit(&S.bar);
        }
        ok = __syncthreads_and(ok && bar_wait(&S.bar, phase));
        phase ^= 1;
        tc_after_sync();
        tc_before_sync();
        __syncthreads();
    }
    // ---- write the block's gradient sums to its slice (rows 0..63 / 0..15
    // of TMEM for the weights; every element has one writer)
    if (ok && local_tiles > 0) {
        tc_after_sync();
        const uint32_t warp = tid >> 5;
        if (warp < 2) {
            float v[16];
            for (int c0 = 0; c0 < 64; c0 += 16) {
                tmem_ld16(lane_addr(c_dw2, c0), v);
                for (int i = 0; i < 16; ++i) G.w2[row * 64 + c0 + i] = v[i];
            }
            tmem_ld16(lane_addr(c_dw1, 0), v);
            for (int i = 0; i < 16; ++i) G.w1[row * 16 + i] = v[i];
        }
        if (warp == 0) {
            float v[16];
            for (int c0 = 0; c0 < 64; c0 += 16) {
                tmem_ld16(lane_addr(c_dw3, c0), v);
                if (row < 2)
                    for (int i = 0; i < 16; ++i) G.w3[row * 64 + c0 + i] = v[i];
            }
        }
        __syncthreads();
        for (uint32_t t = tid; t < 64; t += kThreads) {
            G.b1[t] = ((S.db1[0][t] + S.db1[1][t]) + S.db1[2][t]) + S.db1[3][t];
            G.b2[t] = ((S.db2[0][t] + S.db2[1][t]) + S.db2[2][t]) + S.db2[3][t];
        }
        if (tid < 2) G.b3[tid] = ((S.db3[0][tid] + S.db3[1][tid]) + S.db3[2][tid]) + S.db3[3][tid];
        if (tid == 0) *G.loss = ((S.loss[0] + S.loss[1]) + S.loss[2]) + S.loss[3];
    } else {
        // no tile (or a timed-out wait): an all-zero slice
        float* slice = part + (size_t)blockIdx.x * (kParams + 1);
        for (uint32_t t = tid; t < kParams + 1; t += kThreads) slice[t] = 0.0f;
    }
    if (!ok && tid == 0) atomicOr(error_flags, 0x4u);
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    tmem_free(tb, 512);
}

// Adam on the FP32 master weights; refreshes the BF16 copies.
__global__ void k_adam(float* __restrict__ master, float* __restrict__ grad, float* __restrict__ m,
                       float* __restrict__ v, __nv_bfloat16* __restrict__ bf16_copy,
                       uint32_t count, uint32_t bf16_count, float lr, float beta1, float beta2,
                       float eps, float bc1, float bc2, float weight_decay) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float g = grad[i] + weight_decay * master[i];
    float mi = beta1 * m[i] + (1.0f - beta1) * g;
    float vi = beta2 * v[i] + (1.0f - beta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    float w = master[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    master[i] = w;
    grad[i] = 0.0f;
    if (i < bf16_count) bf16_copy[i] = __float2bfloat16_rn(w);
}

}  // namespace

size_t infer_smem_bytes() { return sizeof(InferPairSmem) + 1024; }
size_t train_smem_bytes() { return sizeof(TrainSmem) + 1024; }

cudaError_t infer_launch(uint32_t n, int num_sms, KernelLaunch* out, int ctas_per_sm,
                         bool apply) {
    size_t smem = infer_smem_bytes();
    const void* func =
        apply ? (const void*)k_mlp_infer_pair<true> : (const void*)k_mlp_infer_pair<false>;
    cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    if (ctas_per_sm < 1 || ctas_per_sm > kInferMaxCtasPerSm) return cudaErrorInvalidValue;
    const int cps = ctas_per_sm < kInferPairMaxCtasPerSm ? ctas_per_sm : kInferPairMaxCtasPerSm;
    uint32_t tiles = (n + 2 * kTile - 1) / (2 * kTile);   // pairs of tiles
    const uint32_t cap = (uint32_t)(num_sms * cps);
    uint32_t grid = tiles < cap ? tiles : cap;
    out->func = func;
    out->grid = dim3(grid > 0 ? grid : 1);
    out->block = dim3(kInferThreads);
    out->smem = smem;
    return cudaSuccess;
}

cudaError_t infer(const Params& P, const __nv_bfloat16* X, float* out, uint32_t n,
                  uint32_t* error_flags, cudaStream_t stream, int num_sms, int ctas_per_sm) {
    if (n == 0) return cudaSuccess;
    KernelLaunch L;
    cudaError_t e = infer_launch(n, num_sms, &L, ctas_per_sm);
    if (e != cudaSuccess) return e;
    k_mlp_infer_pair<false><<<L.grid, L.block, L.smem, stream>>>(P, X, out, n, error_flags,
                                                                 ApplyArgs{});
    return cudaGetLastError();
}

namespace {
__global__ void k_sum_parts(const float* __restrict__ part, uint32_t blocks,
                            float* __restrict__ out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= kParams + 1) return;
    float s = 0.0f;
    for (uint32_t b = 0; b < blocks; ++b) s += part[(size_t)b * (kParams + 1) + t];
    out[t] = s;
}
}  // namespace

cudaError_t train_grads(const Params& P, const __nv_bfloat16* X, const float* Y, uint32_t n,
                        float* grad, float* part, uint32_t* error_flags, cudaStream_t stream,
                        int num_sms) {
    if (n == 0) return cudaSuccess;
    static bool configured = false;
    size_t smem = train_smem_bytes();
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    uint32_t tiles = (n + kTile - 1) / kTile;
    uint32_t grid = tiles < (uint32_t)num_sms ? tiles : (uint32_t)num_sms;
    k_mlp_train<<<grid, kThreads, smem, stream>>>(P, X, Y, n, 1.0f / (float)n, part, error_flags);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_sum_parts<<<(kParams + 1 + 255) / 256, 256, 0, stream>>>(part, grid, grad);
    return cudaGetLastError();
}

cudaError_t adam(float* master, float* grad, float* m, float* v, __nv_bfloat16* bf16_copy,
                 uint32_t count, uint32_t bf16_count, float lr, float beta1, float beta2, float eps,
                 uint32_t step, float weight_decay, cudaStream_t stream) {
    float bc1 = 1.0f - powf(beta1, (float)step);
    float bc2 = 1.0f - powf(beta2, (float)step);
    k_adam<<<(count + 255) / 256, 256, 0, stream>>>(master, grad, m, v, bf16_copy, count,
                                                    bf16_count, lr, beta1, beta2, eps, bc1, bc2,
                                                    weight_decay);
    return cudaGetLastError();
}

}  // namespace mlp
}  // namespace fe
