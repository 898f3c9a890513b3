// fe_common.cuh — device helpers shared by the DFSPH kernels.
//
// Numerics: this library is compiled with -fmad=false -prec-div=true
// -prec-sqrt=true -ftz=false, so every expression below rounds exactly as the
// host oracle does (IEEE single precision, one rounding per operation, in
// source order).  The shader formulas are restated from
// shaders/include/common.glsl.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "fe_device.h"

namespace fe {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr unsigned kFull = 0xFFFFFFFFu;
// GLSL `PI` of common.glsl:4 as a float literal.
constexpr float kPi = 3.1415926535897932384626433832795f;
constexpr float kEpsR = 1e-6f;

struct f3 {
    float x, y, z;
};
__device__ __forceinline__ f3 xyz(float4 v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ f3 sub(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 add(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 scale(float s, f3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ f3 scale_r(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
// dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z, as the oracle defines it.
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// get_cell_hash (common.glsl:30-35).
__device__ __forceinline__ uint32_t cell_hash(int cx, int cy, int cz, uint32_t table) {
    return (((uint32_t)cx * 73856093u) ^ ((uint32_t)cy * 19349663u) ^
            ((uint32_t)cz * 83492791u)) % table;
}

// get_cell_hash for a power-of-two table: x % T == x & (T - 1).
__device__ __forceinline__ uint32_t cell_hash_pow2(int cx, int cy, int cz, uint32_t mask) {
    return (((uint32_t)cx * 73856093u) ^ ((uint32_t)cy * 19349663u) ^
            ((uint32_t)cz * 83492791u)) & mask;
}

// ivec3(floor(p / h)): IEEE division, floor, saturating conversion (NaN -> 0).
__device__ __forceinline__ int cell_coord(float p, float h) {
    return __float2int_rz(floorf(p / h));
}

// 8 / (PI h^3), the normalisation of kernel_w and kernel_grad
// (common.glsl:40, 58).  Hoisting it out of a neighbour loop repeats the
// same two roundings, so the values are unchanged.
__device__ __forceinline__ float kernel_norm(float h) {
    float h3 = h * h * h;
    return 8.0f / (kPi * h3);
}

// kernel_w (common.glsl:38-54) for q = r / h and k = kernel_norm(h).  Both
// pieces of the spline are evaluated, each in the shader's operation order,
// and the result selected: the same value as the shader's branches (NaN
// included), without divergent branches in the neighbour loops.
__device__ __forceinline__ float kernel_w_q(float q, float k) {
    const float q2 = q * q;
    const float q3 = q2 * q;
    const float inner = k * (6.0f * q3 - 6.0f * q2 + 1.0f);
    const float omq = 1.0f - q;
    const float omq3 = omq * omq * omq;
    const float outer = k * 2.0f * omq3;
    const float w = q <= 0.5f ? inner : outer;
    return q >= 1.0f ? 0.0f : w;
}

// kernel_grad (common.glsl:56-73) as the scalar that multiplies r_vec, for
// q = r / h and k = kernel_norm(h); the pieces selected as in kernel_w_q.
// The division is skipped where the result is 0 (q >= 1 or r < 1e-6).
__device__ __forceinline__ float kernel_grad_scale_q(float q, float r, float h, float k) {
    if (q >= 1.0f || r < kEpsR) return 0.0f;
    const float inner = k * (18.0f * q * q - 12.0f * q);
    const float omq = 1.0f - q;
    const float outer = k * -6.0f * omq * omq;
    const float gf = q <= 0.5f ? inner : outer;
    return gf / (h * r);
}

// r / h, correctly rounded.  Where the host has checked, for this h, that
// the reciprocal step below returns the correctly rounded quotient for every
// significand of r (h_recip_exact), it is used: q0 = r (1/h) is within an
// ulp or two, e = r - q0 h is exact in one fused multiply-add, and
// q0 + e (1/h) rounds to r / h.  The steps scale exactly with r's exponent,
// so one binade of r covers every normal r (the neighbour loops see r = 0
// or r of at least about 1e-22, far from underflow).  Otherwise the IEEE
// division.  Both give the bits of the oracle's r / h.
__device__ __forceinline__ float div_h(float r, float h, float inv_h, uint32_t exact) {
    if (exact) {
        const float q0 = __fmul_rn(r, inv_h);
        return __fmaf_rn(__fmaf_rn(-q0, h, r), inv_h, q0);
    }
    return r / h;
}

// kernel_w (common.glsl:38-54).
__device__ __forceinline__ float kernel_w(float r, float h) {
    return kernel_w_q(r / h, kernel_norm(h));
}

// kernel_grad (common.glsl:56-73) as the scalar that multiplies r_vec.
__device__ __forceinline__ float kernel_grad_scale(float r, float h) {
    return kernel_grad_scale_q(r / h, r, h, kernel_norm(h));
}

// p / (rho * rho) for pressure_force, or NaN when rho <= 1e-6 (the shader
// skips such neighbours, pressure_force.comp:64).
__device__ __forceinline__ float pressure_over_rho2(float p, float rho) {
    return rho > kEpsR ? p / (rho * rho) : __int_as_float(0x7fffffff);
}

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// position_b and pressure acceleration of particle i (see Bufs).
__device__ __forceinline__ float4* posb(const Bufs& B, uint32_t i) { return B.pos_b + i; }
__device__ __forceinline__ float4* rec_pos(const Bufs& B, uint32_t i) {
    return B.rec + 2 * (size_t)i;
}
__device__ __forceinline__ float4* accp(const Bufs& B, uint32_t i) {
    return B.rec + 2 * (size_t)i + 1;
}
// velocity_a of particle i (second half of its position/velocity record).
__device__ __forceinline__ float4* vela(const Bufs& B, uint32_t i) {
    return B.pa + 2 * (size_t)i + 1;
}
// velocity_b of particle i (second half of its position/velocity record).
__device__ __forceinline__ float4* velb(const Bufs& B, uint32_t i) {
    return B.pv + 2 * (size_t)i + 1;
}

// Both halves of record i of a 32-byte record array in one 256-bit store.
__device__ __forceinline__ void st_pair(float4* base, uint32_t i, float4 a, float4 b) {
    float4* p = base + 2 * (size_t)i;
    asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "f"(a.x),
                 "f"(a.y), "f"(a.z), "f"(a.w), "f"(b.x), "f"(b.y), "f"(b.z), "f"(b.w)
                 : "memory");
}

// Both halves of record j of a 32-byte record array in one 256-bit
// read-only load.
__device__ __forceinline__ void ld_pair(const float4* base, uint32_t j, float4& a, float4& b) {
    const float4* p = base + 2 * (size_t)j;
    asm volatile("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z),
                   "=f"(b.w)
                 : "l"(p));
}

// Both halves of particle i's record in one 256-bit store: the 32-byte sector
// is written whole, so L2 never merges a half-written sector with DRAM.
__device__ __forceinline__ void st_record(const Bufs& B, uint32_t i, float4 pos, float4 acc) {
    float4* p = B.rec + 2 * (size_t)i;
    asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "f"(pos.x),
                 "f"(pos.y), "f"(pos.z), "f"(pos.w), "f"(acc.x), "f"(acc.y), "f"(acc.z), "f"(acc.w)
                 : "memory");
}

// Both halves of particle j's record in one 256-bit read-only load.
__device__ __forceinline__ void ld_record(const Bufs& B, uint32_t j, float4& pos, float4& acc) {
    const float4* p = B.rec + 2 * (size_t)j;
    asm volatile("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=f"(pos.x), "=f"(pos.y), "=f"(pos.z), "=f"(pos.w), "=f"(acc.x), "=f"(acc.y),
                   "=f"(acc.z), "=f"(acc.w)
                 : "l"(p));
}

// Fixed-order FP64 sum of one value per thread of a 256-thread block:
// warp halving tree (lane l + lane l^m, m = 16..1), then the 8 warp sums in a
// halving tree (m = 4, 2, 1).  Result valid in thread 0.  `smem` holds 8
// doubles.  The host oracle (fo_det_sum) reproduces this order.
__device__ __forceinline__ double block_tree256(double v, double* smem) {
    for (int m = 16; m >= 1; m >>= 1) v = v + __shfl_xor_sync(kFull, v, m);
    const int warp = threadIdx.x >> 5;
    if (lane_id() == 0) smem[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (warp == 0) {
        double w = lane_id() < 8 ? smem[lane_id()] : 0.0;
        for (int m = 4; m >= 1; m >>= 1) w = w + __shfl_xor_sync(kFull, w, m);
        r = w;
    }
    __syncthreads();
    return r;
}

// Maximum of one value per thread of a 256-thread block (order-free).
// Result valid in thread 0.
__device__ __forceinline__ double block_max256(double v, double* smem) {
    for (int m = 16; m >= 1; m >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, m));
    const int warp = threadIdx.x >> 5;
    if (lane_id() == 0) smem[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (warp == 0) {
        double w = lane_id() < 8 ? smem[lane_id()] : 0.0;
        for (int m = 4; m >= 1; m >>= 1) w = fmax(w, __shfl_xor_sync(kFull, w, m));
        r = w;
    }
    __syncthreads();
    return r;
}

// Final stage of the fixed-order sum over `chunks` partials: thread t adds
// partials t, t+256, ... in order, then block_tree256.  Valid in thread 0.
__device__ __forceinline__ double block_final_sum(const double* partials, uint32_t chunks,
                                                  double* smem) {
    double s = 0.0;
    for (uint32_t c = threadIdx.x; c < chunks; c += 256) s = s + __ldcg(partials + c);
    return block_tree256(s, smem);
}

// "Last block" ticket: returns true in every thread of the block that
// finished last.  Each block must have written its partials before calling.
__device__ __forceinline__ bool last_block_done(uint32_t* counter, uint32_t nblocks) {
    __shared__ bool s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = atomicAdd(counter, 1u);
        s_last = (t == nblocks - 1);
    }
    __syncthreads();
    if (s_last) __threadfence();
    return s_last;
}

}  // namespace fe
