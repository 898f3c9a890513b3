// fe_neighbors.cuh — particle/chunk mapping and the neighbour iteration
// shared by the DFSPH passes (fe_kernels.cu) and the learned warm start
// (fe_learned.cu).
#pragma once

#include "fe_common.cuh"

namespace fe {

__device__ __forceinline__ bool chunk_of(const Bufs& B, uint32_t& i, uint32_t& s,
                                         uint32_t& chunk) {
    chunk = blockIdx.x;
    uint4 c = B.chunks[chunk];
    s = c.z;
    i = c.x + threadIdx.x;
    return threadIdx.x < c.y;
}

// Block-size-agnostic particle loop of the neighbour kernels over the chunk
// table (the scene-offset table: every chunk is <= 256 consecutive particles
// of one scene).  A block of kThreads threads takes kThreads / 256 chunks at a
// time (512), or one chunk in 256 / kThreads passes (128); a grid smaller
// than the chunk count makes the kernel persistent: each block strides over
// the chunks until all are done.  Every warp covers 32 consecutive particles
// of one chunk, so warp-level cooperation and per-particle results are the
// same for every shape.  f(i, scene, live) is called by every thread of a
// warp together (live: i is a particle of the chunk).
template <int kThreads>
struct ParticleLoop {
    static_assert(kThreads == 128 || kThreads == 256 || kThreads == 512, "block size");
    static constexpr uint32_t kChunksPerStep = kThreads >= kBlock ? kThreads / kBlock : 1;
    static constexpr uint32_t kPasses = kThreads >= kBlock ? 1 : kBlock / kThreads;
};

// kPersist = false: the grid has one block per chunk step and the loop
// below runs once (compiled without the loop state).
template <int kThreads, bool kPersist, class F>
__device__ __forceinline__ void for_each_particle(const Bufs& B, F&& f) {
    using L = ParticleLoop<kThreads>;
    const uint32_t sub = kThreads >= kBlock ? threadIdx.x / kBlock : 0u;
    const uint32_t t = kThreads >= kBlock ? threadIdx.x % kBlock : threadIdx.x;
    auto step = [&](uint32_t c0) {
        const uint32_t c = c0 + sub;
        if (c >= B.n_chunks) return;   // whole warps: sub is uniform per 256 threads
        const uint4 cc = B.chunks[c];
#pragma unroll 1
        for (uint32_t k = 0; k < L::kPasses; ++k) {
            const uint32_t off = k * kThreads + t;
            f(cc.x + off, cc.z, off < cc.y);
        }
    };
    if constexpr (kPersist) {
        for (uint32_t c0 = blockIdx.x * L::kChunksPerStep; c0 < B.n_chunks;
             c0 += gridDim.x * L::kChunksPerStep)
            step(c0);
    } else {
        step(blockIdx.x * L::kChunksPerStep);
    }
}

// The bucket walk of the shaders (e.g. density_and_alpha.comp:31-63) over the
// {start, end} table.  f(j, r_vec, r2) is called for each candidate with
// r2 <= h*h, in walk order.
template <class F>
__device__ __forceinline__ void walk(const Bufs& B, const DevParams& P, f3 pi, F&& f) {
    const float h = P.h;
    const float h2 = h * h;
    const int cx = cell_coord(pi.x, h), cy = cell_coord(pi.y, h), cz = cell_coord(pi.z, h);
    for (int z = -1; z <= 1; ++z)
        for (int y = -1; y <= 1; ++y)
            for (int x = -1; x <= 1; ++x) {
                uint32_t k = P.table_base +
                             cell_hash_pow2((int)((uint32_t)cx + (uint32_t)x),
                                            (int)((uint32_t)cy + (uint32_t)y),
                                            (int)((uint32_t)cz + (uint32_t)z), P.T - 1u);
                uint2 cell = B.cells[k];
                if (cell.x == kEmpty) continue;
                for (uint32_t j = cell.x; j < cell.y; ++j) {
                    f3 rv = sub(pi, xyz(__ldg(posb(B, j))));
                    float r2 = dot(rv, rv);
                    if (r2 > h2) continue;
                    f(j, rv, r2);
                }
            }
}

// Streaming read of a neighbour-list entry: read once per pass, so it
// bypasses L1 and carries an evict-first L2 policy, leaving the caches to the
// gathered neighbour data.
__device__ __forceinline__ uint64_t evict_first_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ uint2 ld_list(const uint2* p, uint64_t pol) {
    uint2 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;"
                 : "=r"(v.x), "=r"(v.y)
                 : "l"(p), "l"(pol));
    return v;
}

// Neighbours with r > 1e-6 in walk order: f(j, r_vec, grad_scale, pos_j, d_j)
// where pos_j = pos_b[j] (w = p_j / rho_j^2) and d_j = gather(j).  List
// entries are consumed four at a time with all their loads issued before the
// arithmetic, which then runs strictly in list order.
template <class G, class F>
__device__ __forceinline__ void for_each_neighbor(const Bufs& B, const DevParams& P, uint32_t i,
                                                  f3 pi, G&& gather, F&& f) {
    const uint32_t cnt = B.nbr_count[i];
    if (cnt <= kNbrCap) {
        const uint2* e = B.nbr + i;
        const size_t stride = B.n_total;
        const uint64_t pol = evict_first_policy();
        uint32_t k = 0;
        for (; k + 4 <= cnt; k += 4) {
            uint2 v0 = ld_list(e + (k + 0) * stride, pol);
            uint2 v1 = ld_list(e + (k + 1) * stride, pol);
            uint2 v2 = ld_list(e + (k + 2) * stride, pol);
            uint2 v3 = ld_list(e + (k + 3) * stride, pol);
            float4 q0 = __ldg(posb(B, v0.x)), q1 = __ldg(posb(B, v1.x));
            float4 q2 = __ldg(posb(B, v2.x)), q3 = __ldg(posb(B, v3.x));
            auto d0 = gather(v0.x);
            auto d1 = gather(v1.x);
            auto d2 = gather(v2.x);
            auto d3 = gather(v3.x);
            f(v0.x, sub(pi, xyz(q0)), __uint_as_float(v0.y), q0, d0);
            f(v1.x, sub(pi, xyz(q1)), __uint_as_float(v1.y), q1, d1);
            f(v2.x, sub(pi, xyz(q2)), __uint_as_float(v2.y), q2, d2);
            f(v3.x, sub(pi, xyz(q3)), __uint_as_float(v3.y), q3, d3);
        }
        for (; k < cnt; ++k) {
            uint2 v = ld_list(e + k * stride, pol);
            float4 q = __ldg(posb(B, v.x));
            f(v.x, sub(pi, xyz(q)), __uint_as_float(v.y), q, gather(v.x));
        }
    } else {
        const float h = P.h;
        walk(B, P, pi, [&](uint32_t j, f3 rv, float r2) {
            float r = sqrtf(r2);
            if (r > kEpsR) f(j, rv, kernel_grad_scale(r, h), __ldg(posb(B, j)), gather(j));
        });
    }
}

struct NoData {};

// As for_each_neighbor, over a 32-byte record array whose first half of
// record j is a copy of position_b: f(r_vec, grad_scale, second_half_j), with
// both halves of j fetched by one 256-bit load.  B.rec (position,
// acceleration) for pressure_update, B.pv (position, velocity_b) for
// viscosity and the FIXED-mode divergence source.
template <class F>
__device__ __forceinline__ void for_each_neighbor_pair(const Bufs& B, const DevParams& P,
                                                       uint32_t i, f3 pi, const float4* recs,
                                                       F&& f) {
    const uint32_t cnt = B.nbr_count[i];
    if (cnt <= kNbrCap) {
        const uint2* e = B.nbr + i;
        const size_t stride = B.n_total;
        const uint64_t pol = evict_first_policy();
        uint32_t k = 0;
        for (; k + 4 <= cnt; k += 4) {
            uint2 v0 = ld_list(e + (k + 0) * stride, pol);
            uint2 v1 = ld_list(e + (k + 1) * stride, pol);
            uint2 v2 = ld_list(e + (k + 2) * stride, pol);
            uint2 v3 = ld_list(e + (k + 3) * stride, pol);
            float4 q0, a0, q1, a1, q2, a2, q3, a3;
            ld_pair(recs, v0.x, q0, a0);
            ld_pair(recs, v1.x, q1, a1);
            ld_pair(recs, v2.x, q2, a2);
            ld_pair(recs, v3.x, q3, a3);
            f(sub(pi, xyz(q0)), __uint_as_float(v0.y), a0);
            f(sub(pi, xyz(q1)), __uint_as_float(v1.y), a1);
            f(sub(pi, xyz(q2)), __uint_as_float(v2.y), a2);
            f(sub(pi, xyz(q3)), __uint_as_float(v3.y), a3);
        }
        for (; k < cnt; ++k) {
            uint2 v = ld_list(e + k * stride, pol);
            float4 q, a;
            ld_pair(recs, v.x, q, a);
            f(sub(pi, xyz(q)), __uint_as_float(v.y), a);
        }
    } else {
        const float h = P.h;
        walk(B, P, pi, [&](uint32_t j, f3 rv, float r2) {
            float r = sqrtf(r2);
            if (r > kEpsR) f(rv, kernel_grad_scale(r, h), __ldg(recs + 2 * (size_t)j + 1));
        });
    }
}

template <class F>
__device__ __forceinline__ void for_each_neighbor_record(const Bufs& B, const DevParams& P,
                                                         uint32_t i, f3 pi, F&& f) {
    for_each_neighbor_pair(B, P, i, pi, B.rec, f);
}

}  // namespace fe
