// fe_kernels.cu — the DFSPH passes as sm_100a kernels.
//
// One 256-thread block per chunk of <= 256 particles of one scene.  Each
// kernel restates one reference shader (cited per kernel); arithmetic is in
// the shader's order with no contraction (see fe_common.cuh), so results
// equal the host oracle bit for bit.
//
// Neighbour access.  density_alpha walks the 27 hash buckets exactly like the
// shaders (z, y, x offsets; bucket walk in sorted order; r^2 <= h^2) and, in
// the same pass, records for every particle the neighbours with r > 1e-6 in
// walk order together with the gradient scale grad_factor / (h r) of
// kernel_grad.  Positions do not move until the next neighbour search, so the
// ~18 later neighbour passes of the substep read this list (8 bytes per pair,
// coalesced: entry k of particle i at k * n_total + i) instead of re-walking
// ~216 candidates; they visit the same pairs in the same order and therefore
// produce identical sums.  A particle with more than kNbrCap neighbours keeps
// walking the buckets in every pass.
#include "fe_common.cuh"
#include "fe_features.cuh"
#include "fe_kernels.h"
#include "fe_neighbors.cuh"

namespace fe {

// ---------------------------------------------------------------------------
// Neighbour search: spatial_hash.comp, grid_offsets.comp, reorder.comp.
// ---------------------------------------------------------------------------
__global__ void k_fill_u32(uint32_t* p, uint32_t v, size_t count) {
    size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) p[i] = v;
}

__global__ void k_fill_cells(uint2* p, size_t count) {
    size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
        p[i] = make_uint2(kEmpty, kEmpty);
}

// spatial_hash.comp:23-36 (the sentinel tail is written once at creation and
// never changes).
__global__ void __launch_bounds__(kBlock) k_hash(Bufs B) {
    uint32_t i, s, c;
    if (!chunk_of(B, i, s, c)) return;
    const DevParams& P = B.P[s];
    float4 p = __ldg(B.pos_a + i);
    const float h = P.h;
    B.keys[i] = P.table_base + cell_hash_pow2(cell_coord(p.x, h), cell_coord(p.y, h),
                                              cell_coord(p.z, h), P.T - 1u);
    B.vals[i] = i;
}

// grid_offsets.comp:20-33, also recording where each bucket ends so that the
// walk needs no hash comparison.
__global__ void k_offsets(Bufs B) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B.n_total) return;
    uint32_t key = B.keys[i];
    if (key >= B.T_total) return;
    uint32_t prev = i == 0 ? kEmpty : B.keys[i - 1];
    uint32_t next = i + 1 == B.n_total ? kEmpty : B.keys[i + 1];
    if (key != prev) B.cells[key].x = i;
    if (key != next) B.cells[key].y = i + 1;
}

// reorder.comp:37-46.  FIXED mode also gathers the pressures into prs_tmp.
// The neighbour list of the old order is invalidated: until density_alpha
// rebuilds it, the neighbour passes walk the new buckets.
// kCarry: the learned warm start's per-particle state is gathered too.
// Every store is a whole aligned vector of a fully written array (no
// read-modify-write of pos_b, no half-written record): partial sectors
// made this pass about twice as slow.
template <bool kCarry>
__device__ __forceinline__ void reorder_body(const Bufs& B, int carry_pressure,
                                             const LearnArgs& L) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B.n_total) return;
    uint32_t src = B.vals[i];
    if (src >= B.n_total) src = i;  // unreachable for a valid permutation
    B.nbr_count[i] = kNbrCap + 1;
    // pos_b.w holds p / rho^2 of slot i (pressures and densities are not
    // permuted here): the value every pass that writes p or rho maintains,
    // recomputed from them.  The records' position half is written by
    // pressure_force, the only pass before pressure_update that needs it.
    float4 p = __ldg(B.pos_a + src);
    p.w = pressure_over_rho2(B.prs[i], B.rho[i]);
    *posb(B, i) = p;
    // position copy + velocity_b; then this slot's velocity_a record with the
    // new position copy (its velocity half is rewritten unchanged, so the
    // gathers of other threads read the same bytes either way)
    st_pair(B.pv, i, p, *vela(B, src));
    st_pair(B.pa, i, p, *vela(B, i));
    if (carry_pressure) B.prs_tmp[i] = B.prs[src];
    if (kCarry) {
        L.carry_tmp[i] = L.carry[src];
        L.mom_tmp[i] = L.mom[src];
    }
}

__global__ void __launch_bounds__(kBlock) k_reorder(Bufs B, int carry_pressure) {
    reorder_body<false>(B, carry_pressure, LearnArgs{});
}
__global__ void __launch_bounds__(kBlock) k_reorder_carry(Bufs B, int carry_pressure,
                                                          LearnArgs L) {
    reorder_body<true>(B, carry_pressure, L);
}

// FIXED mode: the gathered pressures become current; pr = p / rho^2 keeps
// matching the (not yet recomputed) densities.  kCarry: the gathered learned
// state too.
template <bool kCarry>
__device__ __forceinline__ void take_pressure_body(const Bufs& B, const LearnArgs& L) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B.n_total) return;
    float p = B.prs_tmp[i];
    B.prs[i] = p;
    posb(B, i)->w = pressure_over_rho2(p, B.rho[i]);
    if (kCarry) {
        L.carry[i] = L.carry_tmp[i];
    }
}

__global__ void __launch_bounds__(kBlock) k_take_pressure(Bufs B) {
    take_pressure_body<false>(B, LearnArgs{});
}
__global__ void __launch_bounds__(kBlock) k_take_pressure_carry(Bufs B, LearnArgs L) {
    take_pressure_body<true>(B, L);
}

// Snapshot of a float4 field for fe_download_async: element i of a field
// whose elements lie `stride` float4 apart, with w replaced by `w` when
// fix_w (the reference's w of that field; the device keeps other data there).
__global__ void __launch_bounds__(kBlock) k_snapshot4(float4* dst, const float4* src,
                                                      uint32_t stride, uint32_t n, int fix_w,
                                                      float w) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = src[(size_t)i * stride];
    if (fix_w) v.w = w;
    dst[i] = v;
}

// pr = p / rho^2, velocity_b's w = m / rho and velocity_a's w = the density
// residual t for all particles (after a host upload of p, rho, position_b or
// a velocity).  One block per chunk (t needs the scene's rho0).
__global__ void __launch_bounds__(kBlock) k_refresh_pr(Bufs B) {
    uint32_t i, s, c;
    if (!chunk_of(B, i, s, c)) return;
    posb(B, i)->w = pressure_over_rho2(B.prs[i], B.rho[i]);
    velb(B, i)->w = B.P[s].mass / B.rho[i];
    vela(B, i)->w = density_residual_t(B.rho[i], B.P[s].rho0);
}

// ---------------------------------------------------------------------------
// density_and_alpha.comp:14-72 + neighbour list.
//
// Two phases with the shader's summation order.  Phase 1 finds the in-range
// candidates (r^2 <= h^2, the shader's test) in walk order; phase 2 visits
// them in that order and does the expensive part (sqrt, kernel, gradient,
// list entry) with the lanes in lockstep.
//
// Phase 1 takes one of two forms, chosen per warp.  The lanes of a warp hold
// consecutive particles of the sorted order, and a run of lanes whose
// particles share a cell also shares that cell's 27 buckets.
//  * Few runs (bulk fluid, several particles per cell): cell-cooperative.
//    For each run the warp lays the 27 buckets end to end in walk order (z,
//    y, x offsets, each bucket's entries in sorted order) and visits the
//    candidates 32 at a time, one per lane: every lane tests its candidate
//    against each particle of the run, and the ballot of the lanes that pass
//    is that particle's in-range mask for the slab.  No lane idles on
//    another's longer bucket, and a candidate's position is loaded once per
//    run.  In phase 2 the set bits of a particle's masks, slab by slab and bit
//    by bit, are its candidates in walk order; the run's table of non-empty
//    buckets turns a bit back into a particle index.
//  * Many runs (spray, sparse cells): each lane walks its own 27 buckets and
//    records its in-range candidates.
// A particle with more than kStage in-range candidates, or a run with more
// than kMaxSlabs * 32 candidates, redoes everything in a single-phase walk.
// ---------------------------------------------------------------------------
constexpr int kStage = 44;
constexpr int kMaxSlabs = 16;
constexpr int kCoopRuns = 8;   // most runs per warp for the cooperative form

struct RunTable {
    uint32_t start[27];   // non-empty buckets in walk order: first entry
    uint16_t excl[28];    // place of the bucket's first entry in the run's row; [K] = row length
};

// Per-warp scratch: one form or the other.
union DensityScratch {
    struct {
        alignas(8) float rx[32];        // the run being tested: its particles' positions
        alignas(8) float ry[32];
        alignas(8) float rz[32];
        uint32_t mask[kMaxSlabs][32];
        RunTable table[kCoopRuns];
        uint32_t row[kMaxSlabs * 32];   // the run being tested: its candidates' indices
    } coop;
    uint32_t cand[kStage][32];
};

struct DensityAcc {
    float density = 0.0f, sum_grad_sq = 0.0f;
    f3 grad_sum = {0.0f, 0.0f, 0.0f};
    uint32_t cnt = 0;
    float div = 0.0f;   // kDiv: the divergence source's sum
    uint2* op = nullptr;   // the particle's next list slot
};

// kn = kernel_norm(h); q = r / h is shared by W and grad W.  The list entry
// goes to a.op, the particle's next slot (a.op advances by one row).  kDiv != 0 also
// sums divergence_source_term.comp's m (v_i - v_j) . grad W over the same
// pairs in the same order (vi, vj: the velocities that pass binds).
template <int kDiv>
__device__ __forceinline__ void density_term(DensityAcc& a, float m, const DevParams& P, float kn,
                                             uint32_t j, f3 rv, float r2, uint32_t stride,
                                             f3 vi, float4 vj) {
    const float h = P.h;
    float r = sqrtf(r2);
    float q = div_h(r, h, P.inv_h, P.h_recip_exact);
    float w = kernel_w_q(q, kn);
    a.density += m * w;
    if (r > kEpsR) {
        float g = 0.0f;   // kernel_grad_scale_q with r > 1e-6 known
        if (!(q >= 1.0f)) {
            const float inner = kn * (18.0f * q * q - 12.0f * q);
            const float omq = 1.0f - q;
            const float outer = kn * -6.0f * omq * omq;
            const float gf = q <= 0.5f ? inner : outer;
            g = gf / (h * r);
        }
        f3 grad = scale(g, rv);
        f3 mg = scale(m, grad);
        a.grad_sum = add(a.grad_sum, mg);
        a.sum_grad_sq += dot(mg, mg);
        if (kDiv) {
            f3 vd = sub(vi, xyz(vj));
            a.div += m * dot(vd, grad);
        }
        if (a.cnt < kNbrCap) {
            *a.op = make_uint2(j, __float_as_uint(g));
            a.op += stride;
        }
        ++a.cnt;
    }
}

// Neighbour j's position (and, kDiv, the velocity the fused divergence
// source binds: velocity_b's record in FIXED mode, velocity_a's in
// REFERENCE mode; both records start with a copy of position_b).
template <int kDiv>
__device__ __forceinline__ f3 neighbour_pos(const Bufs& B, uint32_t j, float4& vj) {
    if (kDiv == 0) return xyz(__ldg(posb(B, j)));
    float4 q;
    ld_pair(kDiv == 1 ? B.pv : B.pa, j, q, vj);
    return xyz(q);
}

// Cooperative phase 1 over the runs of one warp (see above).  Returns, for
// the calling lane, the table of its run (-1: single-phase walk) and its
// number of in-range candidates.
__device__ __forceinline__ void coop_candidates(const Bufs& B, const DevParams& P,
                                                DensityScratch& S, uint32_t heads, int n_live,
                                                int cx, int cy, int cz, float4 p4, int& my_table,
                                                uint32_t& n_in) {
    const int lane = lane_id();
    const float h = P.h;
    const float h2_wide = (h * h) * (1.0f + 0x1p-18f);
    const uint32_t lt_mask = (1u << lane) - 1u;
    int n_tables = 0;
    while (heads) {
        const int r0 = __ffs(heads) - 1;
        heads &= heads - 1;
        const int r1 = heads ? __ffs(heads) - 1 : n_live;
        const int rx = __shfl_sync(kFull, cx, r0), ry = __shfl_sync(kFull, cy, r0),
                  rz = __shfl_sync(kFull, cz, r0);
        // lane t < 27: bucket t of the walk
        uint32_t start = 0, len = 0;
        if (lane < 27) {
            const int x = lane % 3 - 1, y = (lane / 3) % 3 - 1, z = lane / 9 - 1;
            const uint32_t k = P.table_base +
                               cell_hash_pow2((int)((uint32_t)rx + (uint32_t)x),
                                              (int)((uint32_t)ry + (uint32_t)y),
                                              (int)((uint32_t)rz + (uint32_t)z), P.T - 1u);
            const uint2 cell = B.cells[k];
            if (cell.x != kEmpty) {
                start = cell.x;
                len = cell.y - cell.x;
            }
        }
        uint32_t incl = len;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t v = __shfl_up_sync(kFull, incl, d);
            if (lane >= d) incl += v;
        }
        const uint32_t excl = incl - len;
        const uint32_t total = __shfl_sync(kFull, incl, 31);
        const uint32_t nslab = (total + 31u) >> 5;
        const bool mine = lane >= r0 && lane < r1;
        if (nslab > (uint32_t)kMaxSlabs) continue;   // this run walks in phase 2
        if (mine) my_table = n_tables;
        RunTable& T = S.coop.table[n_tables++];
        const uint32_t nonempty = __ballot_sync(kFull, len != 0);
        if (len != 0) {
            const int slot = __popc(nonempty & lt_mask);
            T.start[slot] = start;
            T.excl[slot] = (uint16_t)excl;
        }
        if (lane == 0) T.excl[__popc(nonempty)] = (uint16_t)total;
        // the run's row: candidate c of the walk is particle row[c] (each
        // bucket's lane writes its entries)
        for (uint32_t u = 0; u < len; ++u) S.coop.row[excl + u] = start + u;
        if (mine) {
            S.coop.rx[lane - r0] = p4.x;
            S.coop.ry[lane - r0] = p4.y;
            S.coop.rz[lane - r0] = p4.z;
        }
        __syncwarp();
        for (uint32_t sl = 0; sl < nslab; ++sl) {
            const uint32_t cidx = (sl << 5) + (uint32_t)lane;
            const bool valid = cidx < total;
            const float4 q =
                valid ? __ldg(posb(B, S.coop.row[cidx])) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            // particle p's mask for this slab is the ballot; lane 0 stores it.
            // The test is a superset of the exact r^2 <= h^2 (contracted r^2
            // against h^2 (1 + 2^-18)); phase 2 applies the exact test.
            // two particles of the run per step in packed FP32 (the test
            // above; the contraction that packing allows is covered by the
            // widened bound), their coordinates read as pairs from the run's
            // position arrays
            uint64_t qx2, qy2, qz2;
            asm("mov.b64 %0, {%1, %1};" : "=l"(qx2) : "f"(q.x));
            asm("mov.b64 %0, {%1, %1};" : "=l"(qy2) : "f"(q.y));
            asm("mov.b64 %0, {%1, %1};" : "=l"(qz2) : "f"(q.z));
            const int cnt = r1 - r0;
            int p = 0;
#pragma unroll 1
            for (; p + 1 < cnt; p += 2) {
                const uint64_t ax = *reinterpret_cast<const uint64_t*>(&S.coop.rx[p]);
                const uint64_t ay = *reinterpret_cast<const uint64_t*>(&S.coop.ry[p]);
                const uint64_t az = *reinterpret_cast<const uint64_t*>(&S.coop.rz[p]);
                uint64_t dx, dy, dz, r2;
                asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(dx) : "l"(ax), "l"(qx2));
                asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(dy) : "l"(ay), "l"(qy2));
                asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(dz) : "l"(az), "l"(qz2));
                asm("mul.rn.f32x2 %0, %1, %1;" : "=l"(r2) : "l"(dz));
                asm("fma.rn.f32x2 %0, %1, %1, %2;" : "=l"(r2) : "l"(dy), "l"(r2));
                asm("fma.rn.f32x2 %0, %1, %1, %2;" : "=l"(r2) : "l"(dx), "l"(r2));
                float r2a, r2b;
                asm("mov.b64 {%0, %1}, %2;" : "=f"(r2a), "=f"(r2b) : "l"(r2));
                const uint32_t b0 = __ballot_sync(kFull, valid && !(r2a > h2_wide));
                const uint32_t b1 = __ballot_sync(kFull, valid && !(r2b > h2_wide));
                if (lane == 0) {
                    S.coop.mask[sl][r0 + p] = b0;
                    S.coop.mask[sl][r0 + p + 1] = b1;
                }
            }
            if (p < cnt) {
                const float dx = S.coop.rx[p] - q.x, dy = S.coop.ry[p] - q.y,
                            dz = S.coop.rz[p] - q.z;
                const float r2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
                const uint32_t bits = __ballot_sync(kFull, valid && !(r2 > h2_wide));
                if (lane == 0) S.coop.mask[sl][r0 + p] = bits;
            }
            __syncwarp();
            if (mine) n_in += __popc(S.coop.mask[sl][lane]);
        }
    }
}

// Blocks per SM the launch bounds ask for: 1024 resident threads per SM
// (at most 64 registers per thread), for every block size.
template <int kThreads>
constexpr int kMinBlocks = 1024 / kThreads;

// kDiv: 0 density and alpha only; 1 also the FIXED-mode divergence source
// (velocity_b), 2 also the REFERENCE-mode one (velocity_a) -- see
// density_term.
// kLearn (with kDiv): also the divergence solve's feature row, from this
// pass's density, factor, count and source and the moments carried from
// the substep's density source.
template <int kDiv, bool kLearn>
__device__ __forceinline__ void density_alpha_particle(const Bufs& B, DensityScratch& S,
                                                       uint32_t i, uint32_t s, bool live,
                                                       const LearnArgs& L) {
    const DevParams& P = B.P[s];
    const float m = P.mass, h = P.h;
    const float kn = kernel_norm(h);
    const int lane = lane_id();
    const float4 p4 = live ? __ldg(posb(B, i)) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const f3 pi = xyz(p4);
    const int cx = cell_coord(pi.x, h), cy = cell_coord(pi.y, h), cz = cell_coord(pi.z, h);

    // Runs: live lanes form a prefix; a run starts where the cell changes.
    const int px = __shfl_up_sync(kFull, cx, 1), py = __shfl_up_sync(kFull, cy, 1),
              pz = __shfl_up_sync(kFull, cz, 1);
    const bool head = live && (lane == 0 || cx != px || cy != py || cz != pz);
    const uint32_t heads = __ballot_sync(kFull, head);
    const int n_live = 32 - __clz(__ballot_sync(kFull, live));
    const bool coop = __popc(heads) <= kCoopRuns;
    int my_table = -1;
    uint32_t n1 = 0;
    if (coop) {
        coop_candidates(B, P, S, heads, n_live, cx, cy, cz, p4, my_table, n1);
    } else if (live) {
        walk(B, P, pi, [&](uint32_t j, f3, float) {
            if (n1 < (uint32_t)kStage) S.cand[n1][lane] = j;
            ++n1;
        });
    }
    __syncwarp();
    if (!live) return;

    uint2* out = B.nbr + i;
    const uint32_t stride = B.n_total;
    DensityAcc a;
    a.op = out;
    const f3 vi = kDiv ? xyz(__ldg(kDiv == 1 ? velb(B, i) : vela(B, i))) : f3{0.0f, 0.0f, 0.0f};
    float4 vj = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (coop && my_table >= 0) {
        const RunTable& T = S.coop.table[my_table];
        uint32_t sl = 0, bits = S.coop.mask[0][lane];
        uint32_t t = 0, cur_start = T.start[0], cur_excl = 0, next_excl = T.excl[1];
        for (uint32_t k = 0; k < n1; ++k) {
            while (bits == 0) bits = S.coop.mask[++sl][lane];
            const uint32_t cidx = (sl << 5) + (uint32_t)(__ffs(bits) - 1);
            bits &= bits - 1;
            while (cidx >= next_excl) {
                ++t;
                cur_start = T.start[t];
                cur_excl = next_excl;
                next_excl = T.excl[t + 1];
            }
            const uint32_t j = cur_start + (cidx - cur_excl);
            f3 rv = sub(pi, neighbour_pos<kDiv>(B, j, vj));
            const float r2 = dot(rv, rv);
            if (r2 > h * h) continue;   // the shader's test (phase 1 passed a superset)
            density_term<kDiv>(a, m, P, kn, j, rv, r2, stride, vi, vj);
        }
    } else if (!coop && n1 <= (uint32_t)kStage) {
        for (uint32_t k = 0; k < n1; ++k) {
            uint32_t j = S.cand[k][lane];
            f3 rv = sub(pi, neighbour_pos<kDiv>(B, j, vj));
            density_term<kDiv>(a, m, P, kn, j, rv, dot(rv, rv), stride, vi, vj);
        }
    } else {
        walk(B, P, pi, [&](uint32_t j, f3 rv, float r2) {
            if (kDiv) vj = __ldg(kDiv == 1 ? velb(B, j) : vela(B, j));
            density_term<kDiv>(a, m, P, kn, j, rv, r2, stride, vi, vj);
        });
    }
    if (kDiv) B.src[i] = -a.div;   // divergence_source_term.comp:58-60
    B.rho[i] = a.density;
    // velocity_b.w carries m / rho (the factor viscosity applies to each
    // neighbour's velocity, the same division done once per particle)
    velb(B, i)->w = m / a.density;
    float al = a.sum_grad_sq + dot(a.grad_sum, a.grad_sum);
    B.alpha[i] = al > kEpsR ? al : 0.0f;
    B.nbr_count[i] = a.cnt;
    // After the substep's re-sort this pass also makes the gathered state
    // current (what a separate copy pass did before): FIXED mode's pressure,
    // and the learned warm start's carry.
    float p_i;
    if (kDiv == 1) {
        p_i = B.prs_tmp[i];
        B.prs[i] = p_i;
    } else {
        p_i = B.prs[i];
    }
    posb(B, i)->w = pressure_over_rho2(p_i, a.density);
    if (a.cnt > kNbrCap) atomicOr(&B.G->flags, 0x2u);
    if (kLearn) {
        const float4 cr = L.carry_tmp[i];
        L.carry[i] = cr;
        // the substep's density-source moments, as the re-sort gathered them
        const float4 m4 = L.mom_tmp[i];
        const float fm[kMoments] = {m4.x, m4.y, m4.z, m4.w, cr.z};
        emit_features(B, L, P, i, s, 1, a.div, vi, fm);
    }
}

template <int kThreads, bool kPersist>
__global__ void __launch_bounds__(kThreads, kMinBlocks<kThreads>) k_density_alpha(Bufs B) {
    __shared__ DensityScratch scratch[kThreads / 32];
    DensityScratch& S = scratch[threadIdx.x >> 5];
    for_each_particle<kThreads, kPersist>(B, [&](uint32_t i, uint32_t s, bool live) {
        density_alpha_particle<0, false>(B, S, i, s, live, LearnArgs{});
    });
}

// density_alpha with the (plain) divergence source of the same substep
// summed in its pair loop: the divergence source needs exactly these pairs,
// gradients and order, and the neighbour's velocity shares a 32-byte record
// with the position copy the loop loads.  fixed: FIXED mode (velocity_b),
// else REFERENCE mode (velocity_a).  It runs right after the substep's
// re-sort and takes over that search's last copy: FIXED mode's gathered
// pressures (prs_tmp) become current here.
template <int kThreads, bool kPersist>
__global__ void __launch_bounds__(kThreads, kMinBlocks<kThreads>)
    k_density_alpha_div(Bufs B, int fixed) {
    __shared__ DensityScratch scratch[kThreads / 32];
    DensityScratch& S = scratch[threadIdx.x >> 5];
    if (fixed) {
        for_each_particle<kThreads, kPersist>(B, [&](uint32_t i, uint32_t s, bool live) {
            density_alpha_particle<1, false>(B, S, i, s, live, LearnArgs{});
        });
    } else {
        for_each_particle<kThreads, kPersist>(B, [&](uint32_t i, uint32_t s, bool live) {
            density_alpha_particle<2, false>(B, S, i, s, live, LearnArgs{});
        });
    }
}

// The same with the learned state: also the divergence solve's features,
// and the gathered carry (carry_tmp) becomes current here in both modes.
template <int kThreads, bool kPersist>
__global__ void __launch_bounds__(kThreads, kMinBlocks<kThreads>)
    k_density_alpha_div_learn(Bufs B, int fixed, LearnArgs L) {
    __shared__ DensityScratch scratch[kThreads / 32];
    DensityScratch& S = scratch[threadIdx.x >> 5];
    if (fixed) {
        for_each_particle<kThreads, kPersist>(B, [&](uint32_t i, uint32_t s, bool live) {
            density_alpha_particle<1, true>(B, S, i, s, live, L);
        });
    } else {
        for_each_particle<kThreads, kPersist>(B, [&](uint32_t i, uint32_t s, bool live) {
            density_alpha_particle<2, true>(B, S, i, s, live, L);
        });
    }
}

// ---------------------------------------------------------------------------
// viscosity.comp:17-66: velocity_b in, velocity_a out.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void viscosity_particle(const Bufs& B, uint32_t i, uint32_t s) {
    const DevParams& P = B.P[s];
    const float m = P.mass, h = P.h;
    const float kn = kernel_norm(h), inv_h = P.inv_h;
    const uint32_t exact = P.h_recip_exact;
    const f3 pi = xyz(__ldg(posb(B, i)));
    const f3 vi = xyz(__ldg(velb(B, i)));
    f3 sum = {0.0f, 0.0f, 0.0f};
    // velocity_b.w = m / rho_j (written by density_alpha): one 256-bit load of
    // the position/velocity record per neighbour
    for_each_neighbor_pair(
        B, P, i, pi, B.pv, [&](f3 rv, float, float4 vj) {
            float r2 = dot(rv, rv);
            float r = sqrtf(r2);
            float w = kernel_w_q(div_h(r, h, inv_h, exact), kn);
            f3 vd = sub(xyz(vj), vi);
            sum = add(sum, scale_r(scale(vj.w, vd), w));
        });
    f3 vv = add(vi, scale(P.visc, sum));
    f3 g = {P.gx, P.gy, P.gz};
    f3 vf = add(vv, scale_r(g, P.dt));
    // the whole position/velocity_a record; w = the slot's density residual
    // t (density_residual_t) for the learned density source
    st_pair(B.pa, i, make_float4(pi.x, pi.y, pi.z, 0.0f),
            make_float4(vf.x, vf.y, vf.z, density_residual_t(B.rho[i], P.rho0)));
}

template <int kThreads, bool kPersist>
__global__ void __launch_bounds__(kThreads, kMinBlocks<kThreads>) k_viscosity(Bufs B) {
    for_each_particle<kThreads, kPersist>(B, [&](uint32_t i, uint32_t s, bool live) {
        if (live) viscosity_particle(B, i, s);
    });
}

// ---------------------------------------------------------------------------
// density_source_term.comp:16-74 (velocities = velocity_a).  The kLearn
// variant also emits the warm-start features (same arithmetic for s and p).
// ---------------------------------------------------------------------------
struct VelRho {
    float4 v;
    float rho;
};

template <bool kLearn>
__device__ __forceinline__ void density_source_body(const Bufs& B, const LearnArgs& L,
                                                    uint32_t i, uint32_t s) {
    const DevParams& P = B.P[s];
    const float m = P.mass, dt = P.dt;
    const f3 pi = xyz(__ldg(posb(B, i)));
    const f3 vi = xyz(__ldg(vela(B, i)));
    float div = 0.0f;
    Moments mo;
    // velocity_a and (w) the density residual t of j from one load of its record
    for_each_neighbor_pair(B, P, i, pi, B.pa, [&](f3 rv, float g, float4 vj) {
        f3 grad = scale(g, rv);
        f3 vd = sub(vi, xyz(vj));
        div += m * dot(vd, grad);
        if (kLearn) mo.add_t(g, vj.w);   // velocity_a's w: the residual t of j
    });
    float rho_i = B.rho[i];
    float source = 0.0f;
    if (dt > kEpsR) source = ((P.rho0 - rho_i) / dt) - div;
    B.src[i] = source;
    B.prs[i] = 0.0f;
    posb(B, i)->w = pressure_over_rho2(0.0f, rho_i);
    if (kLearn) {
        float fm[kMoments];
        moment_features(mo, fm);
        emit_features(B, L, P, i, s, 0, div, vi, fm);
    }
}

template <int kThreads, bool kPersist>
__global__ void __launch_bounds__(kThreads, kMinBlocks<kThreads>) k_density_source(Bufs B) {
    for_each_particle<kThreads, kPersist>(B, [&](uint32_t i, uint32_t s, bool live) {
        if (live) density_source_body<false>(B, LearnArgs{}, i, s);
    });
}
template <int kThreads, bool kPersist>
__global__ void __launch_bounds__(kThreads, kMinBlocks<kThreads>)
    k_density_source_learn(Bufs B, LearnArgs L) {
    for_each_particle<kThreads, kPersist>(B, [&](uint32_t i, uint32_t s, bool live) {
        if (live) density_source_body<true>(B, L, i, s);
    });
}

// ---------------------------------------------------------------------------
// divergence_source_term.comp:14-61 (velocities = velocity_a in REFERENCE
// mode, velocity_b in FIXED mode).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void divergence_source_body(const Bufs& B, int fixed, uint32_t i,
                                                       uint32_t s) {
    const DevParams& P = B.P[s];
    const float m = P.mass;
    const f3 pi = xyz(__ldg(posb(B, i)));
    const f3 vi = xyz(__ldg(fixed ? velb(B, i) : vela(B, i)));
    float div = 0.0f;
    auto term = [&](f3 rv, float g, float4 vj) {
        f3 grad = scale(g, rv);
        f3 vd = sub(vi, xyz(vj));
        div += m * dot(vd, grad);
    };
    if (fixed) {
        // velocity_b from the position/velocity record
        for_each_neighbor_pair(B, P, i, pi, B.pv, [&](f3 rv, float g, float4 vj) { term(rv, g, vj); });
    } else {
        for_each_neighbor(
            B, P, i, pi, [&](uint32_t j) { return __ldg(vela(B, j)); },
            [&](uint32_t, f3 rv, float g, float4, float4 vj) { term(rv, g, vj); });
    }
    B.src[i] = -div;
}

// The stand-alone pass (the stage call; a frame sums it inside
// density_alpha, k_density_alpha_div).
template <int kThreads, bool kPersist>
__global__ void __launch_bounds__(kThreads, kMinBlocks<kThreads>) k_divergence_source(Bufs B,
                                                                                      int fixed) {
    for_each_particle<kThreads, kPersist>(B, [&](uint32_t i, uint32_t s, bool live) {
        if (live) divergence_source_body(B, fixed, i, s);
    });
}

// ---------------------------------------------------------------------------
// pressure_force.comp:15-78.  pr[j] = p_j / rho_j^2 (NaN when rho_j <= 1e-6)
// is maintained by every pass that writes p or rho.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pressure_force_particle(const Bufs& B, uint32_t i, uint32_t s) {
    const DevParams& P = B.P[s];
    const float m = P.mass;
    const float4 p4 = __ldg(posb(B, i));
    const f3 pi = xyz(p4);
    const float rho_i = B.rho[i], p_i = B.prs[i];
    float p_rho_i = 0.0f;
    if (rho_i > kEpsR) p_rho_i = p_i / (rho_i * rho_i);
    f3 acc = {0.0f, 0.0f, 0.0f};
    for_each_neighbor(
        B, P, i, pi, [&](uint32_t) { return NoData{}; },
        [&](uint32_t, f3 rv, float g, float4 qj, NoData) {
            float p_rho_j = qj.w;  // p_j / rho_j^2, NaN when rho_j <= 1e-6
            if (p_rho_j == p_rho_j) {
                f3 grad = scale(g, rv);
                float term = p_rho_i + p_rho_j;
                acc = add(acc, scale(m * term, grad));
            }
        });
    // the whole record: this particle's position for pressure_update's
    // gathers and its acceleration
    st_record(B, i, p4, make_float4(-acc.x, -acc.y, -acc.z, 0.0f));
}

template <int kThreads, bool kPersist>
__global__ void __launch_bounds__(kThreads, kMinBlocks<kThreads>) k_pressure_force(Bufs B,
                                                                                   int which) {
    for_each_particle<kThreads, kPersist>(B, [&](uint32_t i, uint32_t s, bool live) {
        if (live && !(which >= 0 && B.S[s].solve[which].done)) pressure_force_particle(B, i, s);
    });
}

// ---------------------------------------------------------------------------
// pressure_update.comp:18-84, plus the solver control of the tolerance loop.
// which = 0 (density solve), 1 (divergence solve), -1 (a bare stage call:
// no control).  The per-particle error of the pressure *before* this update
// is the projected-Jacobi step in residual units, with r_i = s_i - Ap_i:
// |r_i| where the update stays positive, p_i |a_ii| / omega where it clamps
// to 0 (0 for a particle at p = 0 that would go negative, i.e. complementary
// expansion), and 0 for rows the solver cannot act on (alpha or rho <= 1e-6).
// It vanishes only at the solution of the clamped system, so an over-
// estimated pressure counts as error as well as a missing one.  Times dt for
// the density solve, it is summed in the fixed FP64 order; the last block
// turns the per-scene sums into the metric, advances the iteration count and
// sets the loop condition.
// ---------------------------------------------------------------------------
// Index of scene sc's first chunk (chunks are laid out scene by scene): a
// block-wide sum of the chunk counts of the scenes before it.  `tmp` holds 8
// words.  Whole block.
__device__ __forceinline__ uint32_t scene_chunk_base(const Bufs& B, uint32_t sc, uint32_t* tmp) {
    uint32_t t = 0;
    for (uint32_t k = threadIdx.x; k < sc; k += kBlock) t += (B.P[k].n + kBlock - 1) / kBlock;
    for (int m = 16; m >= 1; m >>= 1) t += __shfl_xor_sync(kFull, t, m);
    if (lane_id() == 0) tmp[threadIdx.x >> 5] = t;
    __syncthreads();
    uint32_t r = 0;
    for (int w = 0; w < 8; ++w) r += tmp[w];
    __syncthreads();
    return r;
}

// Solver control of scene s after an iteration (whole block): the final
// fixed-order sum of its chunk partials, the metric, iteration count and
// done flag.  c0 = the scene's first chunk.
__device__ void solve_finish_scene(Bufs& B, int which, uint32_t s, uint32_t c0, double* smem) {
    const DevParams& P = B.P[s];
    SolveCtl& ctl = B.S[s].solve[which];
    uint32_t nchunks = (P.n + kBlock - 1) / kBlock;
    bool active = !ctl.done;
    double sum = 0.0, mx = 0.0;
    if (active && P.solver == 1u) {
        sum = block_final_sum(B.partials + c0, nchunks, smem);
        double m = 0.0;
        for (uint32_t k = threadIdx.x; k < nchunks; k += kBlock)
            m = fmax(m, __ldcg(B.partials + B.n_chunks + c0 + k));
        mx = block_max256(m, smem);
    }
    if (threadIdx.x == 0 && active) {
        ctl.iter += 1;
        if (P.solver == 1u) {
            double avg = sum / (double)P.n;
            if (which == 1) avg = avg * (double)P.dt;
            double metric = avg / (double)P.rho0;
            double metric_max = (which == 1 ? mx * (double)P.dt : mx) / (double)P.rho0;
            ctl.metric = metric;
            ctl.metric_max = metric_max;
            float tol = which == 0 ? P.tol_d : P.tol_v;
            if (ctl.iter >= P.min_it && metric <= (double)tol) {
                ctl.done = 1;
            } else if (ctl.iter >= P.max_it) {
                ctl.done = 1;
                ctl.cap_hit = 1;
            }
        } else {
            if (ctl.iter >= ctl.K) ctl.done = 1;
        }
    }
    __syncthreads();
}

// Sets the loop condition from every scene's done flag (thread 0).
__device__ __forceinline__ void solve_set_condition(Bufs& B, int which,
                                                    cudaGraphConditionalHandle handle,
                                                    int use_handle) {
    uint32_t any_open = 0;
    for (uint32_t s = 0; s < B.n_scenes; ++s)
        if (!__ldcg(&B.S[s].solve[which].done)) any_open = 1;
    B.G->cond[which] = any_open;
    if (use_handle) cudaGraphSetConditional(handle, any_open);
}

// Multi-scene contexts: the per-scene finish in parallel, one block per
// scene (the same per-scene code, so the same sums); the last block sets the
// loop condition.
__global__ void __launch_bounds__(kBlock) k_solve_finish(Bufs B, int which,
                                                         cudaGraphConditionalHandle handle,
                                                         int use_handle) {
    __shared__ double smem[8];
    __shared__ uint32_t tmp[8];
    const uint32_t s = blockIdx.x;
    const uint32_t c0 = scene_chunk_base(B, s, tmp);
    solve_finish_scene(B, which, s, c0, smem);
    if (last_block_done(&B.G->tickets[kTicketSolve], gridDim.x) && threadIdx.x == 0) {
        solve_set_condition(B, which, handle, use_handle);
        B.G->tickets[kTicketSolve] = 0;
    }
}

// One block per chunk, or a persistent grid whose blocks stride over the
// chunks (the per-chunk partials, and so the sums, are the same).
__global__ void __launch_bounds__(kBlock) k_pressure_update(Bufs B, int which,
                                                            cudaGraphConditionalHandle handle,
                                                            int use_handle) {
    __shared__ double smem[8];
    const bool control = which >= 0;
    for (uint32_t c = blockIdx.x; c < B.n_chunks; c += gridDim.x) {
        const uint4 cc = B.chunks[c];
        const uint32_t i = cc.x + threadIdx.x, s = cc.z;
        const bool valid = threadIdx.x < cc.y;
        const DevParams& P = B.P[s];
        const bool skip = control && B.S[s].solve[which].done;
        double e_sum_in = 0.0;
        if (valid && !skip) {
            const float m = P.mass, dt = P.dt, omega = P.omega;
            const f3 pi = xyz(__ldg(posb(B, i)));
            const f3 ai = xyz(*accp(B, i));
            float sum_ap = 0.0f;
            for_each_neighbor_record(B, P, i, pi, [&](f3 rv, float g, float4 aj) {
                f3 grad = scale(g, rv);
                f3 ad = sub(ai, xyz(aj));
                sum_ap += m * dot(ad, grad);
            });
            const float alpha_i = B.alpha[i], rho_i = B.rho[i], s_i = B.src[i], p_i = B.prs[i];
            float ap_i = dt * sum_ap;
            float error = s_i - ap_i;
            float p_new = p_i;
            float e = 0.0f;
            if (alpha_i > kEpsR && rho_i > kEpsR) {
                float a_ii = -(dt / (rho_i * rho_i)) * alpha_i;
                if (fabsf(a_ii) > 1e-20f) {
                    float corr = (omega * error) / a_ii;
                    float np = p_i + corr;
                    p_new = np > 0.0f ? np : 0.0f;
                    B.prs[i] = p_new;
                    e = np > 0.0f ? fabsf(error) : (p_i * fabsf(a_ii)) / omega;
                }
            }
            posb(B, i)->w = pressure_over_rho2(p_new, rho_i);
            if (control && P.solver == 1u) {
                if (which == 0) e = dt * e;
                e_sum_in = e > 0.0f ? (double)e : 0.0;  // NaN -> 0
            }
        }
        // Per-chunk partial of the fixed-order sum and the chunk's largest
        // error (uniform branch per block).
        if (control && !skip && P.solver == 1u) {
            double part = block_tree256(e_sum_in, smem);
            double mx = block_max256(e_sum_in, smem);
            if (threadIdx.x == 0) {
                B.partials[c] = part;
                B.partials[B.n_chunks + c] = mx;
            }
        }
    }
    if (!control) return;
    // One scene: its last block finishes the iteration.  Several scenes:
    // k_solve_finish does, one block per scene.
    if (B.n_scenes == 1 && last_block_done(&B.G->tickets[kTicketSolve], gridDim.x)) {
        solve_finish_scene(B, which, 0, 0, smem);
        if (threadIdx.x == 0) {
            solve_set_condition(B, which, handle, use_handle);
            B.G->tickets[kTicketSolve] = 0;
        }
    }
}

// Starts a solve: resets the per-scene control and sets the loop condition.
__global__ void k_solve_begin(Bufs B, int which, cudaGraphConditionalHandle handle,
                              int use_handle) {
    if (threadIdx.x != 0) return;
    uint32_t any_open = 0;
    uint32_t cap = 0;
    for (uint32_t s = 0; s < B.n_scenes; ++s) {
        const DevParams& P = B.P[s];
        SolveCtl& ctl = B.S[s].solve[which];
        uint32_t want = (P.solver == 1u) ? P.max_it
                                         : (which == 0 ? B.S[s].iters_rho : B.S[s].iters_div);
        cap = want > cap ? want : cap;
        ctl.iter = 0;
        ctl.cap_hit = 0;
        ctl.metric = 0.0;
        ctl.metric_max = 0.0;
        ctl.K = which == 0 ? B.S[s].iters_rho : B.S[s].iters_div;
        ctl.done = (P.solver == 1u) ? (P.max_it == 0u) : (ctl.K == 0u);
        if (!ctl.done) any_open = 1;
    }
    B.G->cond[which] = any_open;
    B.G->body_runs[which] = 0;
    B.G->body_cap[which] = cap + 2;
    if (use_handle) cudaGraphSetConditional(handle, any_open);
}

// Last node of a WHILE body: counts executions and ends the loop after a
// hard bound even if the solver control above misbehaved, so a frame graph
// always terminates.  Raises FE_STATS_LOOKBACK_TIMEOUT when it has to act.
__global__ void k_loop_guard(Bufs B, int which, cudaGraphConditionalHandle handle) {
    if (threadIdx.x != 0) return;
    uint32_t runs = ++B.G->body_runs[which];
    if (runs >= B.G->body_cap[which]) {
        cudaGraphSetConditional(handle, 0);
        B.G->cond[which] = 0;
        atomicOr(&B.G->flags, 0x4u);
    }
}

// Ends a solve: records iterations used, residual and cap hits.
__global__ void k_solve_end(Bufs B, int which) {
    if (threadIdx.x != 0) return;
    for (uint32_t s = 0; s < B.n_scenes; ++s) {
        SceneState& S = B.S[s];
        SolveCtl& ctl = S.solve[which];
        S.last_iters[which] = ctl.iter;
        S.last_metric[which] = ctl.metric;
        S.last_metric_max[which] = ctl.metric_max;
        S.total_iters[which] += ctl.iter;
        if (ctl.cap_hit) {
            S.cap_hits += 1;
            atomicOr(&B.G->flags, 0x1u);
        }
    }
}

// ---------------------------------------------------------------------------
// pressure_integration.comp:16-77: position_b in, position_a and velocity_a
// out.
// ---------------------------------------------------------------------------
template <bool kLearn>
__device__ __forceinline__ void pressure_integration_body(const Bufs& B, const LearnArgs& L) {
    uint32_t i, s, c;
    if (!chunk_of(B, i, s, c)) return;
    const DevParams& P = B.P[s];
    const float dt = P.dt, r = P.radius;
    const float rest = 0.5f, fric = 0.95f, eps = 0.001f;
    f3 pos = xyz(__ldg(posb(B, i)));
    const float4 v0 = *vela(B, i);
    f3 vel = xyz(v0);
    f3 ap = xyz(*accp(B, i));
    f3 nv = add(vel, scale_r(ap, dt));
    f3 np = add(pos, scale_r(nv, dt));
    if (np.y < P.bminy + r) {
        np.y = P.bminy + r + eps; nv.y *= -rest; nv.x *= fric; nv.z *= fric;
    } else if (np.y > P.bmaxy - r) {
        np.y = P.bmaxy - r - eps; nv.y *= -rest; nv.x *= fric; nv.z *= fric;
    }
    if (np.x < P.bminx + r) {
        np.x = P.bminx + r + eps; nv.x *= -rest; nv.y *= fric; nv.z *= fric;
    } else if (np.x > P.bmaxx - r) {
        np.x = P.bmaxx - r - eps; nv.x *= -rest; nv.y *= fric; nv.z *= fric;
    }
    if (np.z < P.bminz + r) {
        np.z = P.bminz + r + eps; nv.z *= -rest; nv.x *= fric; nv.y *= fric;
    } else if (np.z > P.bmaxz - r) {
        np.z = P.bmaxz - r - eps; nv.z *= -rest; nv.x *= fric; nv.y *= fric;
    }
    B.pos_a[i] = make_float4(np.x, np.y, np.z, 1.0f);
    *vela(B, i) = make_float4(nv.x, nv.y, nv.z, v0.w);
    if (kLearn) after_solve_particle(B, L, P, i, 0);
}

__global__ void __launch_bounds__(kBlock) k_pressure_integration(Bufs B) {
    pressure_integration_body<false>(B, LearnArgs{});
}
// + the density solve's after-solve bookkeeping of the learned warm start
__global__ void __launch_bounds__(kBlock) k_pressure_integration_learn(Bufs B, LearnArgs L) {
    pressure_integration_body<true>(B, L);
}

// divergence_integration.comp:14-43 (velocity; colour is render-only).
template <bool kLearn>
__device__ __forceinline__ void divergence_integration_body(const Bufs& B, int fixed,
                                                            const LearnArgs& L) {
    uint32_t i, s, c;
    if (!chunk_of(B, i, s, c)) return;
    const DevParams& P = B.P[s];
    float4* vel = fixed ? velb(B, i) : vela(B, i);
    const float4 v0 = *vel;
    f3 nv = add(xyz(v0), scale_r(xyz(*accp(B, i)), P.dt));
    *vel = make_float4(nv.x, nv.y, nv.z, v0.w);  // w (the density) is kept
    if (kLearn) after_solve_particle(B, L, P, i, 1);
}

__global__ void __launch_bounds__(kBlock) k_divergence_integration(Bufs B, int fixed) {
    divergence_integration_body<false>(B, fixed, LearnArgs{});
}
__global__ void __launch_bounds__(kBlock) k_divergence_integration_learn(Bufs B, int fixed,
                                                                          LearnArgs L) {
    divergence_integration_body<true>(B, fixed, L);
}

// ---------------------------------------------------------------------------
// stats.comp:18-30 + FP64 means.  Per-chunk partials, combined per scene by
// the last block (no fill pass needed, order fixed).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t fixed_point(float x, float scale) {
    float v = x * scale;
    if (!(v > 0.0f)) return 0u;
    if (v >= 10000.0f) return 10000u;
    return (uint32_t)v;
}

// The stats of scene sc from its chunk partials (whole block): two FP64
// sums in the fixed order, integer max and sums.  c0 = its first chunk.
__device__ void stats_finish_scene(Bufs& B, const uint4* upart, uint32_t sc, uint32_t c0,
                                   double* smem, uint32_t (*s_u)[8]) {
    const DevParams& Q = B.P[sc];
    uint32_t nch = (Q.n + kBlock - 1) / kBlock;
    // Two FP64 sums in the fixed order over this scene's chunks.
    double t1 = 0.0, t2 = 0.0;
    for (uint32_t k = threadIdx.x; k < nch; k += kBlock) {
        t1 = t1 + __ldcg(B.partials + 2 * (c0 + k));
        t2 = t2 + __ldcg(B.partials + 2 * (c0 + k) + 1);
    }
    double f1 = block_tree256(t1, smem);
    double f2 = block_tree256(t2, smem);
    // integer partials: max and wrapping sums, order-free
    uint32_t a = 0, b = 0, d = 0;
    for (uint32_t k = threadIdx.x; k < nch; k += kBlock) {
        uint4 u = __ldcg(upart + c0 + k);
        a = max(a, u.x);
        b += u.y;
        d += u.z;
    }
    for (int m = 16; m >= 1; m >>= 1) {
        a = max(a, __shfl_xor_sync(kFull, a, m));
        b += __shfl_xor_sync(kFull, b, m);
        d += __shfl_xor_sync(kFull, d, m);
    }
    if (lane_id() == 0) {
        s_u[0][threadIdx.x >> 5] = a;
        s_u[1][threadIdx.x >> 5] = b;
        s_u[2][threadIdx.x >> 5] = d;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        a = b = d = 0;
        for (int w = 0; w < 8; ++w) {
            a = max(a, s_u[0][w]);
            b += s_u[1][w];
            d += s_u[2][w];
        }
        SceneState& S = B.S[sc];
        S.stats[0] = a;
        S.stats[1] = b;
        S.stats[2] = d;
        S.stats_f64[0] = f1 / (double)Q.n;
        S.stats_f64[1] = f2 / (double)Q.n;
    }
    __syncthreads();
}

// The stats of one chunk (whole block): v = particle i's velocity (the one
// the pass binds), read by the caller.
__device__ __forceinline__ void stats_chunk(Bufs B, uint4* upart, bool valid, uint32_t i,
                                            uint32_t s, uint32_t c, float4 v) {
    __shared__ double smem[8];
    __shared__ uint32_t s_u[3][8];
    const DevParams& P = B.P[s];
    uint32_t mx = 0, s1 = 0, s2 = 0, bad = 0;
    double d1 = 0.0, d2 = 0.0;
    if (valid) {
        float speed = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
        mx = __float_as_uint(speed);
        float rho = B.rho[i], src = B.src[i];
        s1 = fixed_point(fabsf(rho - P.rho0), 1.0f);
        s2 = fixed_point(fabsf(src), 10.0f);
        d1 = fabs((double)rho - (double)P.rho0);
        d2 = fabs((double)src);
        bad = !(isfinite(speed) && isfinite(rho) && isfinite(src));
    }
    // integer parts: order-free
    for (int m = 16; m >= 1; m >>= 1) {
        mx = max(mx, __shfl_xor_sync(kFull, mx, m));
        s1 += __shfl_xor_sync(kFull, s1, m);
        s2 += __shfl_xor_sync(kFull, s2, m);
        bad |= __shfl_xor_sync(kFull, bad, m);
    }
    const int warp = threadIdx.x >> 5;
    if (lane_id() == 0) {
        s_u[0][warp] = mx;
        s_u[1][warp] = s1;
        s_u[2][warp] = s2;
    }
    if (bad) atomicOr(&B.S[s].nonfinite, 1u);
    double p1 = block_tree256(d1, smem);
    double p2 = block_tree256(d2, smem);
    if (threadIdx.x == 0) {
        uint32_t a = 0, b = 0, d = 0;
        for (int w = 0; w < 8; ++w) {
            a = max(a, s_u[0][w]);
            b += s_u[1][w];
            d += s_u[2][w];
        }
        upart[c] = make_uint4(a, b, d, 0);
        B.partials[2 * c] = p1;
        B.partials[2 * c + 1] = p2;
    }
    // One scene: its last block finishes.  Several scenes: k_stats_finish
    // does, one block per scene.
    if (B.n_scenes == 1 && last_block_done(&B.G->tickets[kTicketStats], gridDim.x)) {
        stats_finish_scene(B, upart, 0, 0, smem, s_u);
        if (threadIdx.x == 0) B.G->tickets[kTicketStats] = 0;
    }
}

__global__ void __launch_bounds__(kBlock) k_stats(Bufs B, int fixed, uint4* upart) {
    uint32_t i, s, c;
    const bool valid = chunk_of(B, i, s, c);
    const float4* vel = fixed ? velb(B, 0) : vela(B, 0);
    stats_chunk(B, upart, valid, i, s, c,
                valid ? vel[(size_t)i * 2u] : make_float4(0.0f, 0.0f, 0.0f, 0.0f));
}

// The substep's last divergence integration and the frame's stats in one
// pass: the stats read the velocity this pass has just written (the same
// value the stats pass would read back), and every other input of the stats
// is final by then.
template <bool kLearn>
__device__ __forceinline__ void divergence_integration_stats_body(const Bufs& B, int fixed,
                                                                  const LearnArgs& L,
                                                                  uint4* upart) {
    uint32_t i, s, c;
    const bool valid = chunk_of(B, i, s, c);
    float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (valid) {
        const DevParams& P = B.P[s];
        float4* vel = fixed ? velb(B, i) : vela(B, i);
        const float4 v0 = *vel;
        const f3 nv = add(xyz(v0), scale_r(xyz(*accp(B, i)), P.dt));
        v = make_float4(nv.x, nv.y, nv.z, v0.w);
        *vel = v;
        if (kLearn) after_solve_particle(B, L, P, i, 1);
    }
    stats_chunk(B, upart, valid, i, s, c, v);
}

__global__ void __launch_bounds__(kBlock) k_divergence_integration_stats(Bufs B, int fixed,
                                                                         uint4* upart) {
    divergence_integration_stats_body<false>(B, fixed, LearnArgs{}, upart);
}
__global__ void __launch_bounds__(kBlock) k_divergence_integration_stats_learn(Bufs B, int fixed,
                                                                               LearnArgs L,
                                                                               uint4* upart) {
    divergence_integration_stats_body<true>(B, fixed, L, upart);
}

__global__ void __launch_bounds__(kBlock) k_stats_finish(Bufs B, uint4* upart) {
    __shared__ double smem[8];
    __shared__ uint32_t s_u[3][8];
    const uint32_t sc = blockIdx.x;
    const uint32_t c0 = scene_chunk_base(B, sc, s_u[0]);
    stats_finish_scene(B, upart, sc, c0, smem, s_u);
}

// ---------------------------------------------------------------------------
// Frame prologue (renderer/mod.rs:231-267): adaptive CFL dt and early-exit
// iteration choice from the previous frame's stats.  One thread per scene.
// ---------------------------------------------------------------------------
__global__ void k_frame_prologue(Bufs B) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= B.n_scenes) return;
    DevParams& P = B.P[s];
    SceneState& S = B.S[s];
    float n = (float)P.n;
    float max_speed = __uint_as_float(S.stats[0]);
    float avg_de = (float)S.stats[1] / (1.0f * n);
    float avg_ve = (float)S.stats[2] / (10.0f * n);
    if (P.use_cfl && max_speed > 0.01f) {
        float cfl = (P.cfl_lambda * P.h) / max_speed;
        if (cfl < P.cfl_min) cfl = P.cfl_min;
        if (cfl > P.cfl_max) cfl = P.cfl_max;
        P.dt = fminf(cfl, P.dt * P.cfl_growth);
    }
    float rho0 = P.rho0;
    float thr_d = P.eta_d_pct / 100.0f * rho0;
    float thr_v = P.eta_v_pct / 100.0f * rho0;
    bool early = P.use_thr && P.solver == 0u;
    S.iters_rho = (early && avg_de < thr_d) ? 2u : P.k_rho;
    S.iters_div = (early && avg_ve < thr_v) ? 1u : P.k_div;
}

// fe_read_stats_async: scene `scene`'s stats, the global flags and its dt,
// in stream order, into mapped host memory (one thread; a few hundred
// bytes).
__global__ void k_stats_snapshot(Bufs B, StatsSnapshot* dst, uint32_t scene) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    dst->S = B.S[scene];
    dst->G = *B.G;
    dst->dt = B.P[scene].dt;
    dst->n = B.P[scene].n;
    __threadfence_system();
}

__global__ void k_count_substep(Bufs B) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < B.n_scenes) B.S[s].substeps += 1;
}

// The block sizes the autotuner chooses from.
// (density_alpha: 128 and 256 only; its per-warp scratch would exceed the
// 48 KB of static shared memory of a block at 512 threads)
#define FE_NBR_INSTANTIATE(T, P)                                                      \
    template __global__ void k_viscosity<T, P>(Bufs);                                 \
    template __global__ void k_density_source<T, P>(Bufs);                            \
    template __global__ void k_density_source_learn<T, P>(Bufs, LearnArgs);           \
    template __global__ void k_divergence_source<T, P>(Bufs, int);                    \
    template __global__ void k_pressure_force<T, P>(Bufs, int);
FE_NBR_INSTANTIATE(128, false)
FE_NBR_INSTANTIATE(256, false)
FE_NBR_INSTANTIATE(512, false)
FE_NBR_INSTANTIATE(128, true)
FE_NBR_INSTANTIATE(256, true)
FE_NBR_INSTANTIATE(512, true)
template __global__ void k_density_alpha<128, false>(Bufs);
template __global__ void k_density_alpha<256, false>(Bufs);
template __global__ void k_density_alpha<128, true>(Bufs);
template __global__ void k_density_alpha<256, true>(Bufs);
template __global__ void k_density_alpha_div<128, false>(Bufs, int);
template __global__ void k_density_alpha_div<256, false>(Bufs, int);
template __global__ void k_density_alpha_div<128, true>(Bufs, int);
template __global__ void k_density_alpha_div<256, true>(Bufs, int);
template __global__ void k_density_alpha_div_learn<128, false>(Bufs, int, LearnArgs);
template __global__ void k_density_alpha_div_learn<256, false>(Bufs, int, LearnArgs);
template __global__ void k_density_alpha_div_learn<128, true>(Bufs, int, LearnArgs);
template __global__ void k_density_alpha_div_learn<256, true>(Bufs, int, LearnArgs);

}  // namespace fe
