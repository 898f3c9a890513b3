// fe_oracle.cpp — CPU oracle of the DFSPH step.
//
// TEST INFRASTRUCTURE ONLY: the checker for libfluidstep.so, never shipped
// with it.  Every pass cites the shader it restates (paths are relative to
// the reference project).  Compile with -ffp-contract=off so that
// `a * b + c` stays two roundings, as written in the shaders.
//
// Semantics decided here (the GLSL leaves them to the driver):
//   - dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z, left to right;
//   - length(v) = sqrt(dot(v, v));
//   - float -> int conversion saturates and maps NaN to 0 (CUDA cvt.rzi);
//   - GLSL literals without suffix are float (PI = 3.14159274f).

#include "fe_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <new>
#include <type_traits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;

// ---------------------------------------------------------------------------
// Small vector type with the shaders' component-wise semantics.
// ---------------------------------------------------------------------------
template <class R>
struct V3 {
    R x, y, z;
};
template <class R>
struct V4 {
    R x, y, z, w;
};
template <class R>
inline V3<R> sub(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R>
inline V3<R> add(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R>
inline V3<R> scale(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R>
inline V3<R> scale_r(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R>
inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R>
inline V3<R> xyz(const V4<R>& v) { return {v.x, v.y, v.z}; }

template <class R>
inline int32_t to_int_sat(R v) {
    if (!(v == v)) return 0;
    if (v >= R(2147483647.0)) return 2147483647;
    if (v <= R(-2147483648.0)) return (int32_t)0x80000000u;
    return (int32_t)v;
}

// Constants of the shaders as their own type.
template <class R>
struct K;
template <>
struct K<float> {
    static float pi() { return 3.1415926535897932384626433832795f; }
    static float eps_r() { return 1e-6f; }
};
template <>
struct K<double> {
    static double pi() { return 3.1415926535897932384626433832795; }
    static double eps_r() { return 1e-6; }
};

// get_cell_hash (shaders/include/common.glsl:30-35).
inline uint32_t cell_hash(int32_t cx, int32_t cy, int32_t cz, uint32_t table) {
    const uint32_t p1 = 73856093u, p2 = 19349663u, p3 = 83492791u;
    return (((uint32_t)cx * p1) ^ ((uint32_t)cy * p2) ^ ((uint32_t)cz * p3)) % table;
}

// kernel_w (common.glsl:38-54).
template <class R>
inline R kernel_w(R r, R h) {
    R q = r / h;
    if (q >= R(1)) return R(0);
    R h3 = h * h * h;
    R k = R(8) / (K<R>::pi() * h3);
    if (q <= R(0.5)) {
        R q2 = q * q;
        R q3 = q2 * q;
        return k * (R(6) * q3 - R(6) * q2 + R(1));
    } else {
        R omq = R(1) - q;
        R omq3 = omq * omq * omq;
        return k * R(2) * omq3;
    }
}

// kernel_grad (common.glsl:56-73), split into the scalar factor
// grad_factor / (h * r) that multiplies r_vec.
template <class R>
inline R kernel_grad_scale(R r, R h) {
    R q = r / h;
    if (q >= R(1) || r < K<R>::eps_r()) return R(0);
    R h3 = h * h * h;
    R k = R(8) / (K<R>::pi() * h3);
    R gf;
    if (q <= R(0.5)) {
        gf = k * (R(18) * q * q - R(12) * q);
    } else {
        R omq = R(1) - q;
        gf = k * R(-6) * omq * omq;
    }
    return gf / (h * r);
}

int g_threads = 0;  // 0 = OpenMP default

inline int nthreads() {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

// ---------------------------------------------------------------------------
// Fixed-order FP64 sum.  The GPU reduces per-particle doubles in this exact
// order: chunks of 256 particles (one 256-thread block), inside a chunk a
// halving tree over each warp of 32 (lane l adds lane l+m, m = 16..1), then a
// halving tree over the 8 warp sums (m = 4, 2, 1); the chunk sums are added by
// a single 256-thread block, thread t summing chunks t, t+256, ... in order,
// followed by the same 256-wide tree.
// ---------------------------------------------------------------------------
double tree256(double* a) {  // a[256], destroyed
    double w[8];
    for (int wi = 0; wi < 8; ++wi) {
        double* v = a + 32 * wi;
        for (int m = 16; m >= 1; m >>= 1)
            for (int l = 0; l < m; ++l) v[l] = v[l] + v[l + m];
        w[wi] = v[0];
    }
    for (int m = 4; m >= 1; m >>= 1)
        for (int l = 0; l < m; ++l) w[l] = w[l] + w[l + m];
    return w[0];
}

double det_sum(const double* vals, size_t n) {
    size_t chunks = (n + 255) / 256;
    std::vector<double> part(chunks);
#pragma omp parallel for schedule(static) num_threads(nthreads())
    for (long long c = 0; c < (long long)chunks; ++c) {
        double a[256];
        for (int t = 0; t < 256; ++t) {
            size_t i = (size_t)c * 256 + t;
            a[t] = i < n ? vals[i] : 0.0;
        }
        part[c] = tree256(a);
    }
    double a[256];
    for (int t = 0; t < 256; ++t) {
        double s = 0.0;
        for (size_t c = t; c < chunks; c += 256) s = s + part[c];
        a[t] = s;
    }
    return tree256(a);
}

// ---------------------------------------------------------------------------
// Sorting.
// ---------------------------------------------------------------------------
// cpu_radix_sort (src/renderer/pipelines/sorter.rs:465-559).
void radix_mirror(uint32_t* keys, uint32_t* vals, uint32_t n) {
    const size_t WG = 256, EPI = 8;
    size_t num_wg = (n + WG * EPI - 1) / (WG * EPI);
    std::vector<uint32_t> ak(keys, keys + n), av(vals, vals + n), bk(n), bv(n);
    for (uint32_t pass = 0; pass < 4; ++pass) {
        uint32_t shift = pass * 8;
        bool even = pass % 2 == 0;
        std::vector<uint32_t>& sk = even ? ak : bk;
        std::vector<uint32_t>& sv = even ? av : bv;
        std::vector<uint32_t>& dk = even ? bk : ak;
        std::vector<uint32_t>& dv = even ? bv : av;
        std::vector<uint32_t> counts(256 * num_wg, 0);
        for (size_t wg = 0; wg < num_wg; ++wg) {
            uint32_t local[256] = {0};
            for (size_t lid = 0; lid < WG; ++lid) {
                size_t base = wg * WG * EPI + lid * EPI;
                for (size_t i = 0; i < EPI; ++i) {
                    size_t idx = base + i;
                    if (idx >= n) break;
                    local[(sk[idx] >> shift) & 0xFF]++;
                }
            }
            for (int d = 0; d < 256; ++d) counts[d * num_wg + wg] = local[d];
        }
        uint32_t sums[256];
        for (size_t lid = 0; lid < 256; ++lid) {
            uint32_t running = 0;
            for (size_t i = lid * num_wg; i < lid * num_wg + num_wg; ++i) {
                uint32_t v = counts[i];
                counts[i] = running;
                running += v;
            }
            sums[lid] = running;
        }
        for (size_t stride = 1; stride < 256; stride *= 2) {
            uint32_t prev[256];
            std::memcpy(prev, sums, sizeof(prev));
            for (size_t lid = stride; lid < 256; ++lid) sums[lid] += prev[lid - stride];
        }
        for (size_t lid = 0; lid < 256; ++lid) {
            uint32_t off = lid == 0 ? 0 : sums[lid - 1];
            for (size_t i = lid * num_wg; i < lid * num_wg + num_wg; ++i) counts[i] += off;
        }
        for (size_t wg = 0; wg < num_wg; ++wg)
            for (size_t lid = 0; lid < WG; ++lid) {
                size_t base = wg * WG * EPI + lid * EPI;
                for (size_t i = 0; i < EPI; ++i) {
                    size_t idx = base + i;
                    if (idx >= n) break;
                    uint32_t d = (sk[idx] >> shift) & 0xFF;
                    uint32_t dest = counts[d * num_wg + wg]++;
                    dk[dest] = sk[idx];
                    dv[dest] = sv[idx];
                }
            }
    }
    std::memcpy(keys, ak.data(), sizeof(uint32_t) * n);
    std::memcpy(vals, av.data(), sizeof(uint32_t) * n);
}

// Parallel stable LSD radix sort (the CPU baseline): per-thread block
// histograms, a digit-major scan, then a stable scatter per block.
void radix_parallel(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t key_bits) {
    if (n < 2) return;
    if (key_bits == 0 || key_bits > 32) key_bits = 32;
    uint32_t passes = (key_bits + 7) / 8;
    int T = nthreads();
    std::vector<uint32_t> tk(n), tv(n);
    uint32_t* sk = keys;
    uint32_t* sv = vals;
    uint32_t* dk = tk.data();
    uint32_t* dv = tv.data();
    std::vector<uint32_t> hist((size_t)T * 256);
    for (uint32_t pass = 0; pass < passes; ++pass) {
        uint32_t shift = pass * 8;
        std::fill(hist.begin(), hist.end(), 0u);
#pragma omp parallel num_threads(T)
        {
#ifdef _OPENMP
            int t = omp_get_thread_num();
#else
            int t = 0;
#endif
            size_t lo = (size_t)n * t / T, hi = (size_t)n * (t + 1) / T;
            uint32_t* h = hist.data() + (size_t)t * 256;
            for (size_t i = lo; i < hi; ++i) h[(sk[i] >> shift) & 0xFF]++;
#pragma omp barrier
#pragma omp single
            {
                uint32_t run = 0;
                for (int d = 0; d < 256; ++d)
                    for (int tt = 0; tt < T; ++tt) {
                        uint32_t c = hist[(size_t)tt * 256 + d];
                        hist[(size_t)tt * 256 + d] = run;
                        run += c;
                    }
            }
            for (size_t i = lo; i < hi; ++i) {
                uint32_t d = (sk[i] >> shift) & 0xFF;
                uint32_t dest = h[d]++;
                dk[dest] = sk[i];
                dv[dest] = sv[i];
            }
        }
        std::swap(sk, dk);
        std::swap(sv, dv);
    }
    if (sk != keys) {
        std::memcpy(keys, sk, sizeof(uint32_t) * n);
        std::memcpy(vals, sv, sizeof(uint32_t) * n);
    }
}

// bitonic_sort.comp:19-43 driven by GpuSorter::execute (sorter.rs:73-115).
void bitonic(uint32_t* keys, uint32_t* vals, uint32_t n) {
    for (uint32_t h = 2; h <= n; h *= 2) {
        for (uint32_t step = h / 2; step > 0; step /= 2) {
#pragma omp parallel for schedule(static) num_threads(nthreads()) if (n >= (1u << 16))
            for (long long ii = 0; ii < (long long)(n / 2); ++ii) {
                uint32_t i = (uint32_t)ii;
                uint32_t left = (i / step) * step * 2 + (i % step);
                uint32_t right = left + step;
                uint32_t kl = keys[left], kr = keys[right];
                bool asc = (left & h) == 0u;
                if ((asc && kl > kr) || (!asc && kl < kr)) {
                    std::swap(keys[left], keys[right]);
                    std::swap(vals[left], vals[right]);
                }
            }
        }
    }
}

uint32_t next_pow2(uint32_t n) {
    uint32_t t = 1;
    while (t < n) t <<= 1;
    return t;
}

inline uint32_t fixed_point(float x, float scale) {
    // min(uint(x * scale), 10000u) of stats.comp:26,29 with a defined result
    // for NaN (0) and for values beyond the uint range (10000).
    float v = x * scale;
    if (!(v > 0.0f)) return 0u;
    if (v >= 10000.0f) return 10000u;
    return (uint32_t)v;
}

// ---------------------------------------------------------------------------
// The state: GpuPhysicsData (particle.rs:137-161) on the host.
// ---------------------------------------------------------------------------
struct Base {
    virtual ~Base() {}
    fe_params p{};
    uint32_t n = 0, T = 0;
    std::vector<uint32_t> ekey, eidx, grid_start;
    uint32_t stats[3] = {0, 0, 0};
    double stats_f64[2] = {0, 0};
    fe_stats last{};
    bool initialized = false;
    // frame-driver state (renderer/mod.rs:231-267)
    uint32_t iters_rho = 0, iters_div = 0;
    virtual int neighbor_search() = 0;
    virtual void density_alpha() = 0;
    virtual void viscosity() = 0;
    virtual void density_source() = 0;
    virtual void pressure_force() = 0;
    double last_max = 0.0;  // largest per-particle error of the last residual pass
    virtual double pressure_update(bool want_residual, bool divergence) = 0;
    virtual void pressure_integration() = 0;
    virtual void divergence_source() = 0;
    virtual void divergence_integration() = 0;
    virtual void stats_pass() = 0;
    virtual int download(int field, void* dst, size_t bytes) const = 0;
    virtual int download_f64(int field, double* dst, size_t count) const = 0;
    virtual int upload(int field, const void* src, size_t bytes) = 0;

    // Learned warm start (no reference counterpart; restates
    // fe_features.cuh, fe_learned.cu and the carry through reorder of the
    // CUDA library).  The network itself is not restated: its per-particle
    // outputs for each solve of the next frame are given (net_out), the
    // features it was fed are kept (rows) for comparison.
    bool learned = false;
    float norm[28] = {};
    uint32_t net_slots = 0;        // solves with outputs given for the next frame
    std::vector<float> net_out;    // [slot][n][2], standardised outputs
    std::vector<uint16_t> rows;    // [slot][n][16], BF16 network inputs of the last frame
    uint32_t cur_substep = 0;      // substep of the frame being computed
    bool net_missing = false;      // a solve had no given outputs
    virtual void warm_apply(int which) = 0;
    virtual void after_solve(int which) = 0;
};

// __float2bfloat16_rn: round to nearest even; NaN -> the canonical 0x7FFF.
inline uint16_t bf16_rn(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7FFFFFFFu) > 0x7F800000u) return 0x7FFFu;
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

template <class R>
struct State : Base {
    std::vector<V4<R>> pos_a, pos_b, vel_a, vel_b, acc;
    std::vector<R> rho, alpha, src, prs, prs_tmp;
    // learned warm start: carry[i] = {last density kappa, last divergence
    // kappa, -, -} travelling with particle i; neighbours with r > 1e-6 per
    // particle from the last density_alpha (duplicates of a doubly visited
    // bucket counted twice, like the walk)
    std::vector<V4<R>> carry, carry_tmp;
    // the five moment features of the substep's density source, carried
    // through the mid-substep re-sort for the divergence solve's row
    std::vector<std::array<R, 5>> mom, mom_tmp;
    std::vector<uint32_t> nbr_count;

    R h() const { return (R)p.smoothing_radius; }
    R mass() const { return (R)p.particle_mass; }
    R dt() const { return (R)p.dt; }

    // Velocity array bound to the divergence passes and stats.
    std::vector<V4<R>>& vel_div() { return p.mode == FE_MODE_FIXED ? vel_b : vel_a; }

    inline void cell_of(const V4<R>& q, int32_t c[3]) const {
        R hh = h();
        c[0] = to_int_sat(std::floor(q.x / hh));
        c[1] = to_int_sat(std::floor(q.y / hh));
        c[2] = to_int_sat(std::floor(q.z / hh));
    }

    // The neighbour walk shared by all particle passes (e.g.
    // density_and_alpha.comp:31-63): z, y, x offsets; bucket start from
    // grid_start; walk while the sorted hash matches; skip r2 > h*h.
    template <class F>
    inline void for_neighbors(uint32_t i, F&& f) const {
        const V4<R>& pi = pos_b[i];
        int32_t c[3];
        cell_of(pi, c);
        R hh = h();
        R h2 = hh * hh;
        for (int z = -1; z <= 1; ++z)
            for (int y = -1; y <= 1; ++y)
                for (int x = -1; x <= 1; ++x) {
                    uint32_t k = cell_hash((int32_t)((uint32_t)c[0] + (uint32_t)x),
                                           (int32_t)((uint32_t)c[1] + (uint32_t)y),
                                           (int32_t)((uint32_t)c[2] + (uint32_t)z), T);
                    uint32_t s = grid_start[k];
                    if (s == kEmpty) continue;
                    for (uint32_t j = s; j < n; ++j) {
                        if (ekey[j] != k) break;
                        V3<R> rv = sub(xyz(pi), xyz(pos_b[j]));
                        R r2 = dot(rv, rv);
                        if (r2 > h2) continue;
                        f(j, rv, r2);
                    }
                }
    }

    // NeighborSearch::execute (neighbor_search.rs:176-231).
    int neighbor_search() override {
        // spatial_hash.comp:23-36 over T threads.
#pragma omp parallel for schedule(static) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)T; ++ii) {
            uint32_t i = (uint32_t)ii;
            if (i < n) {
                int32_t c[3];
                cell_of(pos_a[i], c);
                ekey[i] = cell_hash(c[0], c[1], c[2], T);
                eidx[i] = i;
            } else {
                ekey[i] = kEmpty;
                eidx[i] = kEmpty;
            }
        }
        if (p.sort_algorithm == FE_SORT_RADIX)
            radix_parallel(ekey.data(), eidx.data(), T, 32);
        else
            bitonic(ekey.data(), eidx.data(), T);
        // fill_buffer(grid_start, 0xFFFFFFFF) + grid_offsets.comp:20-33.
        std::fill(grid_start.begin(), grid_start.end(), kEmpty);
#pragma omp parallel for schedule(static) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)T; ++ii) {
            uint32_t i = (uint32_t)ii;
            uint32_t key = ekey[i];
            if (key == kEmpty) continue;
            uint32_t prev = i == 0 ? kEmpty : ekey[i - 1];
            if (key != prev) grid_start[key] = i;
        }
        // reorder.comp:37-46 (FIXED mode also carries the pressures).
        bool fixed = p.mode == FE_MODE_FIXED;
#pragma omp parallel for schedule(static) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            uint32_t s = eidx[i];
            pos_b[i] = pos_a[s];
            vel_b[i] = vel_a[s];
            if (fixed) prs_tmp[i] = prs[s];
            if (learned) {
                carry_tmp[i] = carry[s];
                mom_tmp[i] = mom[s];
            }
        }
        if (fixed) std::swap(prs, prs_tmp);
        if (learned) {
            std::swap(carry, carry_tmp);
            std::swap(mom, mom_tmp);
        }
        return 0;
    }

    // density_and_alpha.comp:14-72.
    void density_alpha() override {
        R m = mass(), hh = h();
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            R density = 0, sum_grad_sq = 0;
            V3<R> grad_sum{0, 0, 0};
            uint32_t cnt = 0;
            for_neighbors(i, [&](uint32_t, V3<R> rv, R r2) {
                R r = std::sqrt(r2);
                R w = kernel_w(r, hh);
                density += m * w;
                if (r > K<R>::eps_r()) {
                    V3<R> grad = scale(kernel_grad_scale(r, hh), rv);
                    V3<R> mg = scale(m, grad);
                    grad_sum = add(grad_sum, mg);
                    sum_grad_sq += dot(mg, mg);
                    ++cnt;
                }
            });
            nbr_count[i] = cnt;
            rho[i] = density;
            R a = sum_grad_sq + dot(grad_sum, grad_sum);
            alpha[i] = a > K<R>::eps_r() ? a : R(0);
        }
    }

    // viscosity.comp:17-66: reads velocity_b, writes velocity_a
    // (viscosity.rs:49-52).
    void viscosity() override {
        R m = mass(), hh = h(), nu = (R)p.viscosity, d = dt();
        V3<R> g{(R)p.gravity[0], (R)p.gravity[1], (R)p.gravity[2]};
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            V3<R> sum{0, 0, 0};
            V3<R> vi = xyz(vel_b[i]);
            for_neighbors(i, [&](uint32_t j, V3<R>, R r2) {
                R r = std::sqrt(r2);
                R w = kernel_w(r, hh);
                if (r > K<R>::eps_r()) {
                    V3<R> vd = sub(xyz(vel_b[j]), vi);
                    sum = add(sum, scale_r(scale(m / rho[j], vd), w));
                }
            });
            V3<R> vv = add(vi, scale(nu, sum));
            V3<R> vf = add(vv, scale_r(g, d));
            vel_a[i] = {vf.x, vf.y, vf.z, R(0)};
        }
    }

    // density_source_term.comp:16-74 (velocities = velocity_a,
    // density_source_term.rs:48).
    void density_source() override {
        R m = mass(), hh = h(), d = dt(), rho0 = (R)p.target_density;
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            V3<R> vi = xyz(vel_a[i]);
            R div = 0;
            Moments mo;
            for_neighbors(i, [&](uint32_t j, V3<R> rv, R r2) {
                R r = std::sqrt(r2);
                if (r > K<R>::eps_r()) {
                    R g = kernel_grad_scale(r, hh);
                    V3<R> grad = scale(g, rv);
                    V3<R> vd = sub(vi, xyz(vel_a[j]));
                    div += m * dot(vd, grad);
                    if (learned) mo.add(g, rho[j], rho0);
                }
            });
            R source = 0;
            if (d > K<R>::eps_r()) source = ((rho0 - rho[i]) / d) - div;
            src[i] = source;
            prs[i] = 0;
            if (learned) {
                for (int k = 0; k < 5; ++k) mom[i][k] = mo.w > R(0) ? mo.m[k] / mo.w : R(0);
                emit_row(i, 0, div, vi, mom[i].data());
            }
        }
    }

    // ---- learned warm start ------------------------------------------------
    // Moments of order 1..5 of the neighbours' density residual
    // (fe_features.cuh, Moments::add): t = x / (1 + |x|), x = 100 (rho_j /
    // rho0 - 1), weighted by -grad_factor / (h r).
    struct Moments {
        R w = 0, m[5] = {0, 0, 0, 0, 0};
        void add(R g, R rho_j, R rho0) {
            R x = R(100) * (rho_j / rho0 - R(1));
            R t = x / (R(1) + std::fabs(x));
            R wj = -g;
            w += wj;
            R pw = t;
            for (int k = 0; k < 5; ++k) {
                m[k] += wj * pw;
                pw *= t;
            }
        }
    };

    // kappa_scale (fe_features.cuh): rho^2 / (dt alpha) * (rho0 1e-3 / dt).
    R kappa_scale(R rho_i, R al, R d, R rho0) const {
        R eps = K<R>::eps_r();
        if (!(al > eps && rho_i > eps && d > eps)) return R(0);
        return (rho_i * rho_i / (d * al)) * (rho0 * R(1e-3f) / d);
    }

    // emit_features (fe_features.cuh): the 12 features of particle i before
    // solve `which`, standardised with the model's statistics, as the BF16
    // row the network reads; fm = its five moment features (the density
    // source's, carried for the divergence solve).
    void emit_row(uint32_t i, int which, R div, V3<R> v, const R* fm) {
        uint32_t slot = 2u * cur_substep + (uint32_t)which;
        if (slot >= net_slots) return;
        R hh = h(), m = mass(), d = dt(), rho0 = (R)p.target_density;
        R rho_i = rho[i], al = alpha[i];
        R sc = kappa_scale(rho_i, al, d, rho0);
        R f[12];
        f[0] = rho_i / rho0 - R(1);
        R h2 = hh * hh, h4 = h2 * h2;
        f[1] = al * (h4 * h4) / (m * m);
        f[2] = div * d / (rho0 * R(1e-3f));
        uint32_t cnt = nbr_count[i];
        f[3] = (R)(cnt < 64u ? cnt : 64u) / R(32);
        f[4] = sc > R(0) ? carry[i].x / sc : R(0);
        f[5] = sc > R(0) ? carry[i].y / sc : R(0);
        f[6] = std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z) * d / hh;
        for (int k = 0; k < 5; ++k) f[7 + k] = fm[k];
        uint16_t* row = rows.data() + ((size_t)slot * n + i) * 16;
        for (int k = 0; k < 16; ++k) {
            R a = k < 12 ? (f[k] - (R)norm[k]) / (R)norm[12 + k] : R(0);
            row[k] = bf16_rn((float)a);
        }
    }

    // warm_apply_particle (fe_features.cuh, run in the network's epilogue):
    // the solve's start from the network's output, clamped to
    // [0, max(d_i, carried density kappa)]; particles with fewer than 16
    // neighbours keep the plain start.
    void warm_apply(int which) override {
        uint32_t slot = 2u * cur_substep + (uint32_t)which;
        if (slot >= net_slots) {
            net_missing = true;
            return;
        }
        const float* out = net_out.data() + (size_t)slot * n * 2;
        R d = dt(), omega = (R)p.relax_factor, rho0 = (R)p.target_density;
        R eps = K<R>::eps_r();
#pragma omp parallel for schedule(static) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            R rho_i = rho[i], al = alpha[i];
            R sc = kappa_scale(rho_i, al, d, rho0);
            R y = (R)out[2 * (size_t)i + which] * (R)norm[26 + which] + (R)norm[24 + which];
            R base = which == 1 ? carry[i].x : R(0);
            R p1 = 0;
            if (al > eps && rho_i > eps) {
                R a_ii = -(d / (rho_i * rho_i)) * al;
                if (std::fabs(a_ii) > R(1e-20)) {
                    R q = (omega * src[i]) / a_ii;
                    p1 = q > R(0) ? q : R(0);
                }
            }
            R dd = p1 / omega;
            R pr = nbr_count[i] < 16u ? base : base + y * sc;
            pr = pr > R(0) ? pr : R(0);
            R bound = dd > carry[i].x ? dd : carry[i].x;
            prs[i] = pr < bound ? pr : bound;
        }
    }

    // after_solve_particle (fe_features.cuh): the solve's final pressure
    // becomes the particle's last kappa of that kind.
    void after_solve(int which) override {
#pragma omp parallel for schedule(static) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)n; ++ii) {
            if (which == 0)
                carry[ii].x = prs[ii];
            else
                carry[ii].y = prs[ii];
        }
    }

    // divergence_source_term.comp:14-61 (velocities = velocity_a in
    // REFERENCE mode, divergence_source_term.rs:47).
    void divergence_source() override {
        R m = mass(), hh = h();
        const std::vector<V4<R>>& vel = vel_div();
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            V3<R> vi = xyz(vel[i]);
            R div = 0;
            for_neighbors(i, [&](uint32_t j, V3<R> rv, R r2) {
                R r = std::sqrt(r2);
                if (r > K<R>::eps_r()) {
                    V3<R> grad = scale(kernel_grad_scale(r, hh), rv);
                    V3<R> vd = sub(vi, xyz(vel[j]));
                    div += m * dot(vd, grad);
                }
            });
            src[i] = -div;
            if (learned) emit_row(i, 1, div, vi, mom[i].data());
        }
    }

    // pressure_force.comp:15-78.
    void pressure_force() override {
        R m = mass(), hh = h(), eps = K<R>::eps_r();
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            R rho_i = rho[i], p_i = prs[i];
            R p_rho_i = 0;
            if (rho_i > eps) p_rho_i = p_i / (rho_i * rho_i);
            V3<R> acc_sum{0, 0, 0};
            for_neighbors(i, [&](uint32_t j, V3<R> rv, R r2) {
                R r = std::sqrt(r2);
                if (r > eps) {
                    R rho_j = rho[j], p_j = prs[j];
                    if (rho_j > eps) {
                        V3<R> grad = scale(kernel_grad_scale(r, hh), rv);
                        R p_rho_j = p_j / (rho_j * rho_j);
                        R term = p_rho_i + p_rho_j;
                        acc_sum = add(acc_sum, scale(m * term, grad));
                    }
                }
            });
            acc[i] = {-acc_sum.x, -acc_sum.y, -acc_sum.z, R(0)};
        }
    }

    // pressure_update.comp:18-84.  With want_residual, also returns the
    // fixed-order FP64 sum of the per-particle error of the pressure *before*
    // this update (tolerance solver, no reference counterpart): the
    // projected-Jacobi step in residual units, r_i = s_i - Ap_i, is |r_i|
    // where the update stays positive, p_i |a_ii| / omega where it clamps to
    // 0, and 0 for rows the update skips; times dt for the density solve.
    std::vector<double> resid;
    double pressure_update(bool want_residual, bool divergence) override {
        R m = mass(), hh = h(), d = dt(), omega = (R)p.relax_factor, eps = K<R>::eps_r();
        if (want_residual) resid.assign(n, 0.0);
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            V3<R> ai = xyz(acc[i]);
            R alpha_i = alpha[i], rho_i = rho[i], s_i = src[i], p_i = prs[i];
            R sum_ap = 0;
            for_neighbors(i, [&](uint32_t j, V3<R> rv, R r2) {
                R r = std::sqrt(r2);
                if (r > eps) {
                    V3<R> grad = scale(kernel_grad_scale(r, hh), rv);
                    V3<R> ad = sub(ai, xyz(acc[j]));
                    sum_ap += m * dot(ad, grad);
                }
            });
            R ap_i = d * sum_ap;
            R error = s_i - ap_i;
            R e = 0;
            if (alpha_i > eps && rho_i > eps) {
                R a_ii = -(d / (rho_i * rho_i)) * alpha_i;
                if (std::fabs(a_ii) > R(1e-20)) {
                    R corr = (omega * error) / a_ii;
                    R np = p_i + corr;
                    prs[i] = np > R(0) ? np : R(0);  // max(x, 0.0), NaN -> 0
                    e = np > R(0) ? std::fabs(error) : (p_i * std::fabs(a_ii)) / omega;
                }
            }
            if (want_residual) {
                if (!divergence) e = d * e;
                resid[i] = e > R(0) ? (double)e : 0.0;
            }
        }
        if (want_residual) {
            double mx = 0.0;
            for (double v : resid) mx = std::max(mx, v);  // order-free
            last_max = mx;
        }
        return want_residual ? det_sum(resid.data(), n) : 0.0;
    }

    // pressure_integration.comp:16-77: reads position_b, writes position_a
    // and velocity_a in place (pressure_integration_pipeline.rs:49-53).
    void pressure_integration() override {
        R d = dt(), r = (R)p.particle_radius;
        V3<R> mn{(R)p.box_min[0], (R)p.box_min[1], (R)p.box_min[2]};
        V3<R> mx{(R)p.box_max[0], (R)p.box_max[1], (R)p.box_max[2]};
        const R rest = R(0.5), fric = R(0.95), e = R(0.001);
#pragma omp parallel for schedule(static) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            V3<R> pos = xyz(pos_b[i]);
            V3<R> vel = xyz(vel_a[i]);
            V3<R> ap = xyz(acc[i]);
            V3<R> nv = add(vel, scale_r(ap, d));
            V3<R> np = add(pos, scale_r(nv, d));
            if (np.y < mn.y + r) {
                np.y = mn.y + r + e; nv.y *= -rest; nv.x *= fric; nv.z *= fric;
            } else if (np.y > mx.y - r) {
                np.y = mx.y - r - e; nv.y *= -rest; nv.x *= fric; nv.z *= fric;
            }
            if (np.x < mn.x + r) {
                np.x = mn.x + r + e; nv.x *= -rest; nv.y *= fric; nv.z *= fric;
            } else if (np.x > mx.x - r) {
                np.x = mx.x - r - e; nv.x *= -rest; nv.y *= fric; nv.z *= fric;
            }
            if (np.z < mn.z + r) {
                np.z = mn.z + r + e; nv.z *= -rest; nv.x *= fric; nv.y *= fric;
            } else if (np.z > mx.z - r) {
                np.z = mx.z - r - e; nv.z *= -rest; nv.x *= fric; nv.y *= fric;
            }
            pos_a[i] = {np.x, np.y, np.z, R(1)};
            vel_a[i] = {nv.x, nv.y, nv.z, R(0)};
        }
    }

    // divergence_integration.comp:14-43 (velocity part; the colour output is
    // render-only).
    void divergence_integration() override {
        R d = dt();
        std::vector<V4<R>>& vel = vel_div();
#pragma omp parallel for schedule(static) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            V3<R> nv = add(xyz(vel[i]), scale_r(xyz(acc[i]), d));
            vel[i] = {nv.x, nv.y, nv.z, R(0)};
        }
    }

    // StatsPipeline::execute (stats_pipeline.rs:54-66): fill(0) +
    // stats.comp:18-30, plus FP64 means of |ρ-ρ0| and |s|.
    void stats_pass() override {
        const std::vector<V4<R>>& vel = vel_div();
        uint32_t mx = 0;
        uint64_t s1 = 0, s2 = 0;
        std::vector<double> d1(n), d2(n);
        float rho0f = p.target_density;
#pragma omp parallel for schedule(static) num_threads(nthreads()) reduction(max : mx) reduction(+ : s1, s2)
        for (long long ii = 0; ii < (long long)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            float vx = (float)vel[i].x, vy = (float)vel[i].y, vz = (float)vel[i].z;
            float speed = std::sqrt(vx * vx + vy * vy + vz * vz);
            uint32_t bits;
            std::memcpy(&bits, &speed, 4);
            mx = std::max(mx, bits);
            float de = std::fabs((float)rho[i] - rho0f);
            s1 += fixed_point(de, 1.0f);
            float ve = std::fabs((float)src[i]);
            s2 += fixed_point(ve, 10.0f);
            d1[i] = std::fabs((double)rho[i] - (double)p.target_density);
            d2[i] = std::fabs((double)src[i]);
        }
        stats[0] = mx;
        stats[1] = (uint32_t)s1;  // the reference's u32 atomics wrap alike
        stats[2] = (uint32_t)s2;
        stats_f64[0] = det_sum(d1.data(), n) / (double)n;
        stats_f64[1] = det_sum(d2.data(), n) / (double)n;
    }

    // ---- field transfer --------------------------------------------------
    const void* field_ptr(int f, size_t& count, int& kind) const {
        // kind: 0 = R scalar, 1 = V4<R>, 2 = uint32
        switch (f) {
            case FE_FIELD_POSITION_A: kind = 1; count = n; return pos_a.data();
            case FE_FIELD_POSITION_B: kind = 1; count = n; return pos_b.data();
            case FE_FIELD_VELOCITY_A: kind = 1; count = n; return vel_a.data();
            case FE_FIELD_VELOCITY_B: kind = 1; count = n; return vel_b.data();
            case FE_FIELD_DENSITY: kind = 0; count = n; return rho.data();
            case FE_FIELD_FACTOR: kind = 0; count = n; return alpha.data();
            case FE_FIELD_SOURCE_TERM: kind = 0; count = n; return src.data();
            case FE_FIELD_PRESSURE: kind = 0; count = n; return prs.data();
            case FE_FIELD_PRESSURE_ACCEL: kind = 1; count = n; return acc.data();
            case FE_FIELD_ENTRY_HASH: kind = 2; count = T; return ekey.data();
            case FE_FIELD_ENTRY_INDEX: kind = 2; count = T; return eidx.data();
            case FE_FIELD_GRID_START: kind = 2; count = T; return grid_start.data();
            case FE_FIELD_STATS: kind = 2; count = 3; return stats;
        }
        return nullptr;
    }
    int download(int f, void* dst, size_t bytes) const override {
        size_t count;
        int kind;
        const void* src_ptr = field_ptr(f, count, kind);
        if (!src_ptr || !dst) return FE_ERR_INVALID_ARGUMENT;
        size_t elems = kind == 1 ? count * 4 : count;
        if (bytes != elems * 4) return FE_ERR_INVALID_ARGUMENT;
        if (kind == 2) {
            std::memcpy(dst, src_ptr, bytes);
        } else {
            const R* s = (const R*)src_ptr;
            float* d = (float*)dst;
            for (size_t i = 0; i < elems; ++i) d[i] = (float)s[i];
        }
        return 0;
    }
    int download_f64(int f, double* dst, size_t count_req) const override {
        size_t count;
        int kind;
        const void* src_ptr = field_ptr(f, count, kind);
        if (!src_ptr || !dst || kind == 2) return FE_ERR_INVALID_ARGUMENT;
        size_t elems = kind == 1 ? count * 4 : count;
        if (count_req != elems) return FE_ERR_INVALID_ARGUMENT;
        const R* s = (const R*)src_ptr;
        for (size_t i = 0; i < elems; ++i) dst[i] = (double)s[i];
        return 0;
    }
    int upload(int f, const void* src_in, size_t bytes) override {
        size_t count;
        int kind;
        void* dst = const_cast<void*>(field_ptr(f, count, kind));
        if (!dst || !src_in) return FE_ERR_INVALID_ARGUMENT;
        size_t elems = kind == 1 ? count * 4 : count;
        if (bytes != elems * 4) return FE_ERR_INVALID_ARGUMENT;
        if (kind == 2) {
            std::memcpy(dst, src_in, bytes);
        } else {
            const float* s = (const float*)src_in;
            R* d = (R*)dst;
            for (size_t i = 0; i < elems; ++i) d[i] = (R)s[i];
        }
        return 0;
    }
};

template <class R>
Base* make_state(const fe_params* params, uint32_t n, const float* pos, const float* vel) {
    State<R>* s = new (std::nothrow) State<R>();
    if (!s) return nullptr;
    s->p = *params;
    s->n = n;
    s->T = next_pow2(n);
    s->pos_a.resize(n);
    s->pos_b.resize(n);
    s->vel_a.resize(n);
    s->vel_b.resize(n);
    s->acc.assign(n, {0, 0, 0, 0});
    s->rho.assign(n, 0);
    s->alpha.assign(n, 0);
    s->src.assign(n, 0);
    s->prs.assign(n, 0);
    s->prs_tmp.assign(n, 0);
    s->carry.assign(n, {0, 0, 0, 0});
    s->mom.assign(n, {0, 0, 0, 0, 0});
    s->mom_tmp.assign(n, {0, 0, 0, 0, 0});
    s->carry_tmp.assign(n, {0, 0, 0, 0});
    s->nbr_count.assign(n, 0);
    s->ekey.assign(s->T, 0);
    s->eidx.assign(s->T, 0);
    s->grid_start.assign(s->T, 0);
    for (uint32_t i = 0; i < n; ++i) {
        s->pos_a[i] = {(R)pos[3 * i], (R)pos[3 * i + 1], (R)pos[3 * i + 2], R(1)};
        s->pos_b[i] = {0, 0, 0, 0};
        if (vel)
            s->vel_a[i] = {(R)vel[3 * i], (R)vel[3 * i + 1], (R)vel[3 * i + 2], R(0)};
        else
            s->vel_a[i] = {0, 0, 0, 0};
        s->vel_b[i] = {0, 0, 0, 0};
    }
    return s;
}

// ---------------------------------------------------------------------------
// Frame driver.
// ---------------------------------------------------------------------------
// Prologue of Renderer::step (renderer/mod.rs:231-267): adaptive CFL dt and
// the early-exit iteration choice, both from the previous frame's stats.
void frame_prologue(Base* s) {
    fe_params& p = s->p;
    float n = (float)s->n;
    float max_speed;
    std::memcpy(&max_speed, &s->stats[0], 4);
    float avg_de = (float)s->stats[1] / (1.0f * n);
    float avg_ve = (float)s->stats[2] / (10.0f * n);
    if (p.use_cfl && max_speed > 0.01f) {
        float h = p.smoothing_radius;
        float cfl = (p.cfl_lambda * h) / max_speed;
        // f32::clamp(min, max)
        if (cfl < p.cfl_min_dt) cfl = p.cfl_min_dt;
        if (cfl > p.cfl_max_dt) cfl = p.cfl_max_dt;
        p.dt = std::fmin(cfl, p.dt * p.cfl_growth);
    }
    float rho0 = p.target_density;
    float thr_d = p.density_error_pct / 100.0f * rho0;
    float thr_v = p.divergence_error_pct / 100.0f * rho0;
    bool early = p.use_solver_error_threshold && p.solver == FE_SOLVER_FIXED_ITERS;
    s->iters_rho = (early && avg_de < thr_d) ? 2u : p.density_solver_iterations;
    s->iters_div = (early && avg_ve < thr_v) ? 1u : p.divergence_solver_iterations;
}

// The tolerance metric from the residual sum: mean density error over ρ0
// (density solve) and mean dρ/dt · dt over ρ0 (divergence solve).  The device computes the same expression in double.
double solver_metric(Base* s, double sum, bool divergence) {
    double avg = sum / (double)s->n;
    if (divergence) avg = avg * (double)s->p.dt;
    return avg / (double)s->p.target_density;
}

// One Jacobi solve: fixed count, or the tolerance loop.
uint32_t solve(Base* s, bool divergence, double* residual_out, bool* cap_hit,
               double* residual_max_out) {
    const fe_params& p = s->p;
    if (p.solver == FE_SOLVER_FIXED_ITERS) {
        uint32_t k = divergence ? s->iters_div : s->iters_rho;
        for (uint32_t it = 0; it < k; ++it) {
            s->pressure_force();
            s->pressure_update(false, divergence);
        }
        *residual_out = 0.0;
        *residual_max_out = 0.0;
        return k;
    }
    double tol = divergence ? (double)p.divergence_tolerance : (double)p.density_tolerance;
    uint32_t it = 0;
    double metric = 0.0;
    for (;;) {
        s->pressure_force();
        double sum = s->pressure_update(true, divergence);
        ++it;
        metric = solver_metric(s, sum, divergence);
        if (it >= p.min_iterations && metric <= tol) break;
        if (it >= p.max_iterations) {
            *cap_hit = true;
            break;
        }
    }
    *residual_out = metric;
    double mx = s->last_max;
    if (divergence) mx = mx * (double)p.dt;
    *residual_max_out = mx / (double)p.target_density;
    return it;
}

void substep(Base* s, fe_stats* acc_stats, bool* cap_hit) {
    double r;
    s->viscosity();
    s->density_source();
    if (s->learned) s->warm_apply(0);
    double rm = 0.0;
    uint32_t kr = solve(s, false, &r, cap_hit, &rm);
    acc_stats->density_residual_max = rm;
    acc_stats->density_iterations = kr;
    acc_stats->total_density_iterations += kr;
    acc_stats->density_residual = r;
    s->pressure_integration();
    if (s->learned) s->after_solve(0);
    s->neighbor_search();
    s->density_alpha();
    s->divergence_source();
    if (s->learned) s->warm_apply(1);
    uint32_t kd = solve(s, true, &r, cap_hit, &rm);
    acc_stats->divergence_residual_max = rm;
    acc_stats->divergence_iterations = kd;
    acc_stats->total_divergence_iterations += kd;
    acc_stats->divergence_residual = r;
    s->divergence_integration();
    if (s->learned) s->after_solve(1);
}

void fill_stats(Base* s, fe_stats* out) {
    out->max_speed_bits = s->stats[0];
    out->density_error_fp = s->stats[1];
    out->divergence_error_fp = s->stats[2];
    std::memcpy(&out->max_speed, &s->stats[0], 4);
    float n = (float)s->n;
    out->avg_density_error = (float)s->stats[1] / (1.0f * n);
    out->avg_divergence_error = (float)s->stats[2] / (10.0f * n);
    out->avg_density_error_f64 = s->stats_f64[0];
    out->avg_divergence_error_f64 = s->stats_f64[1];
    out->dt = s->p.dt;
}

}  // namespace

struct fo_ctx {
    Base* s;
};

extern "C" {

fo_ctx* fo_create(const fe_params* params, uint32_t n, const float* pos_xyz,
                  const float* vel_xyz, int fp64) {
    if (!params || !pos_xyz || n == 0 || n > FE_MAX_PARTICLES) return nullptr;
    fo_ctx* c = new (std::nothrow) fo_ctx;
    if (!c) return nullptr;
    c->s = fp64 ? make_state<double>(params, n, pos_xyz, vel_xyz)
                : make_state<float>(params, n, pos_xyz, vel_xyz);
    if (!c->s) {
        delete c;
        return nullptr;
    }
    return c;
}

void fo_destroy(fo_ctx* c) {
    if (!c) return;
    delete c->s;
    delete c;
}

int fo_set_params(fo_ctx* c, const fe_params* p) {
    if (!c || !p) return FE_ERR_INVALID_ARGUMENT;
    c->s->p = *p;
    return 0;
}
int fo_get_params(const fo_ctx* c, fe_params* out) {
    if (!c || !out) return FE_ERR_INVALID_ARGUMENT;
    *out = c->s->p;
    return 0;
}
uint32_t fo_table_size(const fo_ctx* c) { return c ? c->s->T : 0; }

int fo_neighbor_search(fo_ctx* c) { return c->s->neighbor_search(); }
int fo_density_alpha(fo_ctx* c) { c->s->density_alpha(); return 0; }
int fo_viscosity(fo_ctx* c) { c->s->viscosity(); return 0; }
int fo_density_source(fo_ctx* c) { c->s->density_source(); return 0; }
int fo_pressure_force(fo_ctx* c) { c->s->pressure_force(); return 0; }
int fo_pressure_update(fo_ctx* c) { c->s->pressure_update(false, false); return 0; }
int fo_pressure_integration(fo_ctx* c) { c->s->pressure_integration(); return 0; }
int fo_divergence_source(fo_ctx* c) { c->s->divergence_source(); return 0; }
int fo_divergence_integration(fo_ctx* c) { c->s->divergence_integration(); return 0; }
int fo_stats_pass(fo_ctx* c) {
    c->s->stats_pass();
    fill_stats(c->s, &c->s->last);
    return 0;
}
int fo_read_stats(const fo_ctx* c, fe_stats* out) {
    if (!c || !out) return FE_ERR_INVALID_ARGUMENT;
    *out = c->s->last;
    return 0;
}

int fo_step(fo_ctx* c, uint32_t n_substeps, uint32_t flags, fe_stats* out) {
    if (!c) return FE_ERR_INVALID_ARGUMENT;
    Base* s = c->s;
    frame_prologue(s);
    if ((flags & FE_STEP_INIT_NS) || !s->initialized) {
        s->neighbor_search();
        s->density_alpha();
        s->initialized = true;
    }
    fe_stats st = s->last;
    st.density_iterations = st.divergence_iterations = 0;
    bool cap_hit = false;
    if (s->learned) s->rows.assign((size_t)s->net_slots * s->n * 16, 0);
    for (uint32_t k = 0; k < n_substeps; ++k) {
        s->cur_substep = k;
        substep(s, &st, &cap_hit);
    }
    s->cur_substep = 0;
    if (s->learned) s->net_slots = 0;  // outputs are given per frame
    s->stats_pass();
    fill_stats(s, &st);
    st.substeps = n_substeps;
    st.flags = cap_hit ? FE_STATS_ITERATION_CAP_HIT : 0u;
    s->last = st;
    if (out) *out = st;
    return 0;
}

int fo_set_learned(fo_ctx* c, const float* norm28) {
    if (!c) return FE_ERR_INVALID_ARGUMENT;
    Base* s = c->s;
    s->learned = norm28 != nullptr;
    if (norm28) std::memcpy(s->norm, norm28, sizeof s->norm);
    s->net_slots = 0;
    return 0;
}

int fo_set_network_outputs(fo_ctx* c, uint32_t slots, const float* out) {
    if (!c || !c->s->learned || (slots && !out)) return FE_ERR_INVALID_ARGUMENT;
    Base* s = c->s;
    s->net_out.assign(out, out + (size_t)slots * s->n * 2);
    s->net_slots = slots;
    s->net_missing = false;
    return 0;
}

int fo_get_feature_rows(const fo_ctx* c, uint32_t slot, uint16_t* rows) {
    if (!c || !rows) return FE_ERR_INVALID_ARGUMENT;
    const Base* s = c->s;
    size_t per = (size_t)s->n * 16;
    if ((size_t)(slot + 1) * per > s->rows.size()) return FE_ERR_INVALID_ARGUMENT;
    std::memcpy(rows, s->rows.data() + slot * per, per * sizeof(uint16_t));
    return 0;
}

int fo_learned_missing_outputs(const fo_ctx* c) { return c && c->s->net_missing ? 1 : 0; }

int fo_download(const fo_ctx* c, int field, void* dst, size_t bytes) {
    if (!c) return FE_ERR_INVALID_ARGUMENT;
    return c->s->download(field, dst, bytes);
}
int fo_download_f64(const fo_ctx* c, int field, double* dst, size_t count) {
    if (!c) return FE_ERR_INVALID_ARGUMENT;
    return c->s->download_f64(field, dst, count);
}
int fo_upload(fo_ctx* c, int field, const void* src, size_t bytes) {
    if (!c) return FE_ERR_INVALID_ARGUMENT;
    return c->s->upload(field, src, bytes);
}

void fo_sort_radix_mirror(uint32_t* keys, uint32_t* values, uint32_t n) {
    radix_mirror(keys, values, n);
}
void fo_sort_radix_parallel(uint32_t* keys, uint32_t* values, uint32_t n, uint32_t key_bits) {
    radix_parallel(keys, values, n, key_bits);
}
int fo_sort_bitonic(uint32_t* keys, uint32_t* values, uint32_t n) {
    if (n == 0 || (n & (n - 1))) return FE_ERR_INVALID_ARGUMENT;
    bitonic(keys, values, n);
    return 0;
}
double fo_det_sum(const double* values, size_t n) { return det_sum(values, n); }

// splat_density.comp:11-51, loop by loop: every particle whose normalised
// position uvw lies in [0, 1]^3 adds uint(200 (1 - (d/8)^2)^3) to each grid
// voxel at offset (x, y, z), d = length(vec3(x, y, z)) < 8, from its centre
// ivec3(uvw * grid_res).  out[res_z][res_y][res_x] is cleared first (the
// clear_color_image of renderer/mod.rs:387-389).
void fo_splat_density(const float* pos4, uint32_t n, const fe_params* p, uint32_t* out) {
    const int rx = p->grid_res[0], ry = p->grid_res[1], rz = p->grid_res[2];
    std::fill(out, out + (size_t)rx * ry * rz, 0u);
    const int radius = 8;
    const float r = (float)radius;
    const float sx = p->box_max[0] - p->box_min[0], sy = p->box_max[1] - p->box_min[1],
                sz = p->box_max[2] - p->box_min[2];
    for (uint32_t i = 0; i < n; ++i) {
        const float u = (pos4[4 * i] - p->box_min[0]) / sx;
        const float v = (pos4[4 * i + 1] - p->box_min[1]) / sy;
        const float w = (pos4[4 * i + 2] - p->box_min[2]) / sz;
        if (u < 0.0f || v < 0.0f || w < 0.0f || u > 1.0f || v > 1.0f || w > 1.0f) continue;
        const int cx = to_int_sat<float>(u * (float)rx), cy = to_int_sat<float>(v * (float)ry),
                  cz = to_int_sat<float>(w * (float)rz);
        for (int z = -radius; z <= radius; ++z)
            for (int y = -radius; y <= radius; ++y)
                for (int x = -radius; x <= radius; ++x) {
                    const int X = cx + x, Y = cy + y, Z = cz + z;
                    if (X < 0 || Y < 0 || Z < 0 || X >= rx || Y >= ry || Z >= rz) continue;
                    const float fx = (float)x, fy = (float)y, fz = (float)z;
                    const float dist = std::sqrt((fx * fx + fy * fy) + fz * fz);
                    if (dist < r) {
                        const float x_norm = dist / r;
                        float weight = 1.0f - x_norm * x_norm;
                        weight = (weight * weight) * weight;
                        out[((size_t)Z * ry + Y) * rx + X] += (uint32_t)(weight * 200.0f);
                    }
                }
    }
}

// raymarch.frag:1-215, restated for one ray per pixel (see fo_raymarch in
// fe_oracle.h for the conventions).  Transcendentals are the host's libm.
namespace rm {
struct V {
    float x, y, z;
};
inline V v(float x, float y, float z) { return {x, y, z}; }
inline V add(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V sub(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V mul(V a, V b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V muls(V a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V divv(V a, V b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline float dot(V a, V b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline V normalize(V a) {
    float l = std::sqrt(dot(a, a));
    return {a.x / l, a.y / l, a.z / l};
}
inline float mix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline V mixv(V a, V b, float t) { return {mix(a.x, b.x, t), mix(a.y, b.y, t), mix(a.z, b.z, t)}; }
inline float clampf(float x, float lo, float hi) { return std::fmin(std::fmax(x, lo), hi); }
inline float smoothstep(float e0, float e1, float x) {
    float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
struct Grid {
    const uint32_t* g;
    int rx, ry, rz;
    V bmin, bmax;
    float fetch(int x, int y, int z) const {
        x = std::min(std::max(x, 0), rx - 1);
        y = std::min(std::max(y, 0), ry - 1);
        z = std::min(std::max(z, 0), rz - 1);
        return (float)g[((size_t)z * ry + y) * rx + x];
    }
    float density(V p) const {  // getDensity
        V uvw = divv(sub(p, bmin), sub(bmax, bmin));
        if (uvw.x < 0.0f || uvw.y < 0.0f || uvw.z < 0.0f || uvw.x > 1.0f || uvw.y > 1.0f ||
            uvw.z > 1.0f)
            return 0.0f;
        float gx = uvw.x * (float)rx - 0.5f, gy = uvw.y * (float)ry - 0.5f,
              gz = uvw.z * (float)rz - 0.5f;
        float fx = std::floor(gx), fy = std::floor(gy), fz = std::floor(gz);
        int ix = to_int_sat<float>(fx), iy = to_int_sat<float>(fy), iz = to_int_sat<float>(fz);
        float tx = gx - fx, ty = gy - fy, tz = gz - fz;
        float v0 = mix(mix(fetch(ix, iy, iz), fetch(ix + 1, iy, iz), tx),
                       mix(fetch(ix, iy + 1, iz), fetch(ix + 1, iy + 1, iz), tx), ty);
        float v1 = mix(mix(fetch(ix, iy, iz + 1), fetch(ix + 1, iy, iz + 1), tx),
                       mix(fetch(ix, iy + 1, iz + 1), fetch(ix + 1, iy + 1, iz + 1), tx), ty);
        return std::fmax(0.0f, (mix(v0, v1, tz) - 300.0f) * 1.0f);
    }
};
inline V sky(const float* s, int w, int h, V dir) {  // sampleSkybox, bilinear clamp-to-edge
    dir = normalize(dir);
    float u = std::atan2(dir.z, dir.x) * 0.15915f + 0.5f;
    float vv = std::asin(clampf(dir.y, -1.0f, 1.0f)) * 0.31831f + 0.5f;
    float x = u * (float)w - 0.5f, y = vv * (float)h - 0.5f;
    float x0f = std::floor(x), y0f = std::floor(y);
    float ax = x - x0f, ay = y - y0f;
    int x0 = to_int_sat<float>(x0f), y0 = to_int_sat<float>(y0f);
    auto at = [&](int xi, int yi) {
        xi = std::min(std::max(xi, 0), w - 1);
        yi = std::min(std::max(yi, 0), h - 1);
        const float* c = s + 4 * ((size_t)yi * w + xi);
        return v(c[0], c[1], c[2]);
    };
    V c0 = mixv(at(x0, y0), at(x0 + 1, y0), ax), c1 = mixv(at(x0, y0 + 1), at(x0 + 1, y0 + 1), ax);
    return mixv(c0, c1, ay);
}
}  // namespace rm

void fo_raymarch(const uint32_t* grid, int rx, int ry, int rz, const float* sky4, int sky_w,
                 int sky_h, const float* inv_view_proj, const float* cam_pos,
                 const float* box_min, const float* box_max, int width, int height, float* out) {
    using namespace rm;
    const float* M = inv_view_proj;
    V size = v(box_max[0] - box_min[0], box_max[1] - box_min[1], box_max[2] - box_min[2]);
    V center = v(box_min[0] + size.x * 0.5f, box_min[1] + size.y * 0.5f, box_min[2] + size.z * 0.5f);
    V scale = v(std::sqrt(size.x * size.x), std::sqrt(size.y * size.y), std::sqrt(size.z * size.z));
    Grid G{grid, rx, ry, rz, sub(center, muls(scale, 0.5f)), add(center, muls(scale, 0.5f))};
    const V cam = v(cam_pos[0], cam_pos[1], cam_pos[2]);
    const V L = normalize(v(0.4f, 1.0f, 0.3f));
    const V sun = v(1.0f, 0.95f, 0.85f), scatter = v(0.04f, 0.18f, 0.28f);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads())
    for (int py = 0; py < height; ++py)
        for (int px = 0; px < width; ++px) {
            float* o = out + 4 * ((size_t)py * width + px);
            float nx = ((float)px + 0.5f) / (float)width * 2.0f - 1.0f;
            float ny = ((float)py + 0.5f) / (float)height * 2.0f - 1.0f;
            float w4[4];
            for (int r = 0; r < 4; ++r) w4[r] = ((M[r] * nx + M[4 + r] * ny) + M[8 + r] * 1.0f) + M[12 + r] * 1.0f;
            V rd = normalize(sub(v(w4[0] / w4[3], w4[1] / w4[3], w4[2] / w4[3]), cam));
            V t1 = divv(sub(G.bmin, cam), rd), t2 = divv(sub(G.bmax, cam), rd);
            float tn = std::fmax(std::fmax(std::fmin(t1.x, t2.x), std::fmin(t1.y, t2.y)), std::fmin(t1.z, t2.z));
            float tf = std::fmin(std::fmin(std::fmax(t1.x, t2.x), std::fmax(t1.y, t2.y)), std::fmax(t1.z, t2.z));
            o[0] = o[1] = o[2] = o[3] = 0.0f;
            if (tn > tf || tf < 0.0f) continue;
            float step = 0.007f * std::fmax(std::fmax(scale.x, scale.y), scale.z);
            float tc = std::fmax(tn, 0.0f);
            bool hit = false;
            for (int i = 0; i < 96; i++) {
                if (tc > tf) break;
                if (G.density(add(cam, muls(rd, tc))) > 0.01f) {
                    hit = true;
                    break;
                }
                tc += step;
            }
            if (!hit) continue;
            float ta = tc - step, tb = tc;
            for (int i = 0; i < 8; i++) {
                float m = (ta + tb) * 0.5f;
                if (G.density(add(cam, muls(rd, m))) > 0.01f) tb = m;
                else ta = m;
            }
            V sp = add(cam, muls(rd, tb));
            const float e = 0.018f;
            V n = normalize(v(G.density(add(sp, v(e, 0, 0))) - G.density(sub(sp, v(e, 0, 0))),
                              G.density(add(sp, v(0, e, 0))) - G.density(sub(sp, v(0, e, 0))),
                              G.density(add(sp, v(0, 0, e))) - G.density(sub(sp, v(0, 0, e)))));
            V N = normalize(v(-n.x, -n.y, -n.z));
            if (dot(N, N) < 0.5f) N = v(0.0f, 1.0f, 0.0f);
            V Vw = v(-rd.x, -rd.y, -rd.z);
            V H = normalize(add(L, Vw));
            float ndv = std::fmax(dot(N, Vw), 0.0f), ndl = std::fmax(dot(N, L), 0.0f),
                  ndh = std::fmax(dot(N, H), 0.0f);
            float f0 = std::pow((1.0f - 1.333f) / (1.0f + 1.333f), 2.0f);
            float F = clampf(f0 + (1.0f - f0) * std::pow(clampf(1.0f - ndv, 0.0f, 1.0f), 5.0f), 0.0f, 1.0f);
            V refl = sub(rd, muls(N, 2.0f * dot(N, rd)));
            V reflection = sky(sky4, sky_w, sky_h, refl);
            float a = 0.04f * 0.04f, a2 = a * a, dd = ndh * ndh * (a2 - 1.0f) + 1.0f;
            float spec = a2 / (3.14159f * dd * dd) * ndl;
            reflection = add(reflection, muls(sun, clampf(spec * 0.15f, 0.0f, 3.0f)));
            float thickness = 0.0f, t = 0.0f, tmax = tf - tb;
            for (int i = 0; i < 64 && t < tmax; i++, t += 0.015f)
                if (G.density(add(sp, muls(rd, t))) > 0.01f) thickness += 0.015f;
            V absorption = v(std::exp(-0.45f * thickness * 8.0f), std::exp(-0.085f * thickness * 8.0f),
                             std::exp(-0.025f * thickness * 8.0f));
            float eta = 1.0f / 1.333f, ni = dot(N, rd), k = 1.0f - eta * eta * (1.0f - ni * ni);
            V refr = k < 0.0f ? v(0, 0, 0) : sub(muls(rd, eta), muls(N, eta * ni + std::sqrt(k)));
            if (dot(refr, refr) < 0.01f) refr = rd;
            V background = sky(sky4, sky_w, sky_h, normalize(refr));
            float sw = std::fmax(0.0f, dot(N, L) * 0.5f + 0.5f);
            float sb = std::fmax(0.0f, dot(v(-N.x, -N.y, -N.z), L));
            float sf = (sw * 0.6f + sb * 0.4f) * (1.0f - std::exp(-thickness * 3.0f));
            V sss = muls(muls(mul(scatter, sun), sf), 0.35f);
            float foam = smoothstep(0.0f, 0.3f, thickness) * smoothstep(0.5f, 0.95f, N.y);
            V refracted = add(mul(background, absorption), sss);
            V water = mixv(refracted, reflection, F);
            water = mixv(water, muls(v(0.92f, 0.96f, 1.0f), ndl * 0.7f + 0.3f), foam * 0.7f);
            water = add(water, muls(scatter, 0.04f));
            o[0] = water.x / (water.x + 1.0f);
            o[1] = water.y / (water.y + 1.0f);
            o[2] = water.z / (water.z + 1.0f);
            o[3] = 1.0f;
        }
}

int fo_set_threads(int t) {
    g_threads = t;
    return nthreads();
}
int fo_get_threads(void) { return nthreads(); }

}  // extern "C"
