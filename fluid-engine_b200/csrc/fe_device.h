// fe_device.h — layout of the device-resident state of a context.
//
// A context holds one or more scenes (a batch).  Particles of all scenes are
// concatenated; scene s owns particles [first, first + n) before and after
// every sort, because its sort keys are table_base + cell hash with disjoint
// per-scene key ranges.  Every per-particle kernel runs one 256-thread block
// per *chunk*: at most 256 consecutive particles of a single scene
// (chunk table below), so scene parameters are uniform in a block and the
// fixed-order FP64 reductions see the same chunks as a standalone run of
// that scene.
#pragma once

#include <cstdint>

namespace fe {

constexpr int kBlock = 256;          // threads per block of particle kernels
constexpr uint32_t kNbrCap = 64;     // neighbour-list capacity per particle

// Parameters of one scene: `SimulationParams` (common.glsl:11-28) plus the
// frame-driver knobs.  Written by the host (fe_set_params) and, for dt, by
// the frame prologue kernel (adaptive CFL).
struct DevParams {
    float radius, mass, h, rho0;
    float visc, omega, dt;
    float inv_h;                        // 1 / h, correctly rounded (div_h)
    float gx, gy, gz, pad1;
    float bminx, bminy, bminz, pad2;
    float bmaxx, bmaxy, bmaxz, pad3;
    uint32_t n, T, table_base, first;   // scene layout in the batch
    uint32_t k_rho, k_div;              // configured Jacobi iterations
    uint32_t use_cfl, use_thr;
    float eta_d_pct, eta_v_pct;
    float cfl_lambda, cfl_min, cfl_max, cfl_growth;
    uint32_t mode, solver;
    float tol_d, tol_v;
    uint32_t min_it, max_it, warm;
    uint32_t h_recip_exact;             // div_h may divide by h through inv_h
};

// Jacobi solve control of one scene (index 0 = density, 1 = divergence).
struct SolveCtl {
    uint32_t iter;     // iterations done in the current solve
    uint32_t K;        // fixed-iteration target of this frame
    uint32_t done;     // scene finished this solve
    uint32_t cap_hit;  // tolerance solve stopped at max_it
    double metric;     // tolerance metric of the last iteration
    double metric_max; // largest per-particle error of the last iteration (same units)
};

struct SceneState {
    uint32_t stats[3];          // stats_buffer (stats.comp:8)
    uint32_t nonfinite;         // stats pass saw NaN/Inf
    double stats_f64[2];        // FP64 mean |rho-rho0|, mean |s|
    uint32_t iters_rho, iters_div;  // this frame's fixed-iteration choice
    SolveCtl solve[2];
    uint32_t last_iters[2];
    double last_metric[2];
    double last_metric_max[2];
    unsigned long long total_iters[2];
    uint32_t cap_hits;
    uint32_t substeps;
};

struct GlobalState {
    uint32_t flags;        // FE_STATS_* bits raised by device code
    uint32_t cond[2];      // last loop condition of each solve (eager mode)
    uint32_t pad;
    uint32_t tickets[8];   // last-block counters, reset by the last block
    uint32_t body_runs[2]; // loop-body executions of the current solve
    uint32_t body_cap[2];  // hard bound on body_runs (guard of the WHILE node)
};

enum Ticket : int { kTicketStats = 0, kTicketSolve = 1, kTicketHist = 2 };

// The stats of one scene as fe_read_stats_async captures them (written by
// k_stats_snapshot into page-locked, device-mapped host memory).
struct StatsSnapshot {
    SceneState S;
    GlobalState G;
    float dt;
    uint32_t n;
};

// Kernel-side view of every buffer of a context (passed by value).
struct Bufs {
    float4* pos_a;
    // 32-byte record per particle: pa[2i] = copy of position_b (xyz, written
    // with the whole record by reorder and viscosity), pa[2i+1] = velocity_a,
    // whose w carries the slot's density residual t = x / (1 + |x|),
    // x = 100 (rho / rho0 - 1), from viscosity on (read only by the learned
    // density source's moments).  The density source fetches a neighbour's
    // position, velocity and t with one 256-bit load.
    float4* pa;
    // 32-byte record per particle: pv[2i] = copy of position_b (xyz, written
    // by reorder), pv[2i+1] = velocity_b with the slot's m / rho in w
    // (written by density_alpha, kept by the FIXED-mode divergence
    // integration).  Viscosity and the FIXED-mode divergence source fetch a
    // neighbour's position, velocity and density with one 256-bit load.
    float4* pv;
    // position_b; w holds p / rho^2 (NaN when rho <= 1e-6) for pressure_force.
    float4* pos_b;
    // 32-byte record per particle: rec[2i] = copy of position_b (xyz),
    // rec[2i+1] = pressure acceleration, both written by pressure_force with
    // one 256-bit store.  pressure_update fetches both halves of a neighbour
    // with one 256-bit load.
    float4* rec;
    float *rho, *alpha, *src, *prs, *prs_tmp;
    uint32_t *keys, *vals;      // grid_entries (hash, index), T_total
    uint2* cells;               // {start, end} per table slot, T_total
    uint32_t* nbr_count;        // per particle; > kNbrCap = walk instead
    uint2* nbr;                 // nbr[k * n_total + i] = {j, grad scale bits}
    const uint4* chunks;        // {first, count, scene, chunk-in-scene}
    DevParams* P;
    SceneState* S;
    GlobalState* G;
    double* partials;           // per-chunk FP64 partial sums (2 per chunk)
    uint32_t n_total, T_total, n_chunks, n_scenes;
};

// Learned warm start and training-data capture (fe_learned.cu).
// carry[i] travels with particle i through every re-sort:
//   x = final pressure of the last density solve, y = of the last
//   divergence solve, z = the fifth neighbourhood moment of the substep
//   (feature 11), w = capture slot of the solve in progress (bits; ~0 none).
// mom[i] = features 7..10 (the first four moments), with z above the
// moments the density source computed at the substep's start; the
// divergence solve's features reuse them after the mid-substep re-sort,
// reading the re-sorted copy mom_tmp (nothing reads mom again before the
// next density source rewrites it, so it is not copied back).
struct LearnArgs {
    const float* norm;          // model standardisation: x mean[12], std[12], y mean[2], std[2]
    void* xb;                   // BF16 feature rows [n][16] (network input)
    float* out;                 // network output [n][2] (standardised)
    float4* carry;
    float4* carry_tmp;
    float4* mom;
    float4* mom_tmp;
    float* cap_x;               // captured raw features [capacity][12]
    float* cap_y;               // captured normalised targets [capacity][2]
    uint32_t* cap_count;
    uint32_t cap_capacity;
    uint32_t cap_stride;        // sample one particle in cap_stride (hashed)
    uint32_t capture;           // 1: record samples this frame
    uint32_t learned;           // 1: apply the network's pressures
};

}  // namespace fe
