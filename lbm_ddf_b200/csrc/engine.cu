// engine.cu — single-case engine behind the C ABI of include/lbm_ddf.h.
//
// Device state of one case (all in HBM, allocated once at lbm_create):
//   f, g  : 27 populations each, structure of arrays, population k at
//           base + k*ps, node idx = (iz*LY + iy)*LX + ix (reference order),
//           ps = nodes rounded up to 128 elements so that every population
//           row starts 256-byte aligned;
//   phip  : previous-step temperature per node (FP64 for F64 storage, else FP32);
//   scratch: per-block partial sums of the observables reduction and the
//           reduced result.
// The layout flag `swapped` records which AA layout the populations are in.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "internal.h"
#include "rowstep.cuh"
#include "step.cuh"

using namespace lbm;

namespace {
thread_local std::string g_last_error;
}  // namespace

namespace lbm_internal {

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

size_t store_bytes(int storage) {
    switch (storage) {
    case LBM_STORE_F64: return 8;
    case LBM_STORE_F32: return 4;
    case LBM_STORE_F16S:
    case LBM_STORE_BF16S: return 2;
    default: return 0;
    }
}

}  // namespace lbm_internal

using namespace lbm_internal;

namespace {
constexpr int kObs = lbm::kObsTerms;   // partial sums per block (step.cuh add_obs_terms)
constexpr int kObsThreads = 256;
constexpr int kStepThreads = 128;
}  // namespace

// ---------------------------------------------------------------------------
// device kernels besides the step
// ---------------------------------------------------------------------------
namespace lbm {

// Per-block partial sums, in FP64, of
//   0 uy*phi  1 |u|^2  2 ux  3 uy  4 uz  5 phi
//   6..8  phi on the planes iy = 0, 1, 2
//   9..11 phi on the planes iy = LY-1, LY-2, LY-3
//   12 number of nodes with a non-finite moment
//
// split: the moments as the 16-bit BGK step kernel forms them (split_moments),
// so these observables match those it reduces when it steps; else as the
// node update forms them.
template <class S, bool SWAPPED, bool PERIODIC>
__global__ void __launch_bounds__(kObsThreads) obs_kernel(const StepArgs<S> a, double *__restrict__ partial,
                                                          int split) {
    using R = typename Codec<S>::R;
    double acc[kObs];
#pragma unroll
    for (int k = 0; k < kObs; k++) acc[k] = 0.0;
    for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < a.nodes; n += gridDim.x * blockDim.x) {
        const Node g = make_node<PERIODIC>(a, n);
        if constexpr (elem_stride<S>() == 2) {
            if (split) {
                add_obs_terms(acc, split_moments<S, SWAPPED, PERIODIC>(a, g), g.iy, a.ly);
                continue;
            }
        }
        R fr[Q], gr[Q];
        // rows away from the plates (and a closed box's z walls): no y or z
        // boundary tests (uniform over a warp whenever LX is a multiple of
        // 32); FP64 keeps one path (two do not fit its registers)
        if (sizeof(S) < 8 && SWAPPED && yz_interior<PERIODIC>(g))
            gather<S, SWAPPED, kRowInside>(a, g, fr, gr);
        else
            gather<S, SWAPPED, kNoneInside>(a, g, fr, gr);
        const Moments<R> m = node_moments<S>(a, fr, gr, n);
        add_obs_terms(acc, m, g.iy, a.ly);
    }
    __shared__ double red[kObs][kObsThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kObs; k++) {
        double v = warp_sum(acc[k]);
        if (lane == 0) red[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < kObs) {
        double s = 0.0;
        for (int w = 0; w < kObsThreads / 32; w++) s += red[threadIdx.x][w];
        partial[(size_t)blockIdx.x * kObs + threadIdx.x] = s;
    }
}

struct ObsConsts {
    double nodes, plane, ly, diff, dT, visc;
    int64_t step;
};

// Sums the block partials in a fixed order (deterministic: warp w sums
// quantity w, lane l the blocks l, l + 32, ..., then a butterfly over the
// lanes) and forms the observables: Nu_bulk of src/output.cu:228-233;
// Nu_top/bottom of :236-256 written with plane sums,
// <(3T0 - 4T1 + T2)/2> = (3<T0> - 4<T1> + <T2>)/2.  Launch: kObs warps.
// The body of obs_finalize, for a block of kObs warps; `partial` is read
// through L2 (it may have been written by other blocks of the same launch).
__device__ __forceinline__ void finalize_observables(const double *__restrict__ partial, int nblocks,
                                                     const ObsConsts &c, lbm_observables *__restrict__ out) {
    __shared__ double tot[kObs];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32) s += __ldcg(partial + (size_t)b * kObs + w);
    s = warp_sum(s);
    if (lane == 0) tot[w] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        const double uyT = tot[0] / c.nodes;
        out->step = c.step;
        out->nu_bulk = 1.0 + uyT * c.ly / (c.diff * c.dT);
        const double b0 = tot[6] / c.plane, b1 = tot[7] / c.plane, b2 = tot[8] / c.plane;
        const double t0 = tot[9] / c.plane, t1 = tot[10] / c.plane, t2 = tot[11] / c.plane;
        const double dTdy_bot = (-3.0 * b0 + 4.0 * b1 - b2) / 2.0;
        const double dTdy_top = (3.0 * t0 - 4.0 * t1 + t2) / 2.0;
        out->nu_top = -dTdy_top * c.ly / c.dT;
        out->nu_bottom = -dTdy_bot * c.ly / c.dT;
        const double usq = tot[1] / c.nodes;
        out->ke = 0.5 * usq;
        out->re = sqrt(usq) * c.ly / c.visc;
        out->ux_mean = tot[2] / c.nodes;
        out->uy_mean = tot[3] / c.nodes;
        out->uz_mean = tot[4] / c.nodes;
        out->phi_mean = tot[5] / c.nodes;
        out->diverged = tot[12] > 0.0 ? 1 : 0;
        out->reserved = 0;
    }
}

__global__ void __launch_bounds__(32 * kObs) obs_finalize(const double *__restrict__ partial, int nblocks,
                                                          ObsConsts c, lbm_observables *__restrict__ out) {
    finalize_observables(partial, nblocks, c, out);
}

// The per-warp rows a fused step kernel wrote, summed in blocks of
// kRowChunk rows into one partial row each, then (by the block that finishes
// last) the partial rows into the observables, as obs_finalize forms them.
// Thread t of a block reads the chunk's words t, t + 32 kObs, ...: coalesced,
// and all of term t % kObs, rows t / kObs + 32 i; the 32 threads of a term
// are then added by a butterfly in row order.  A fixed order, so the result
// is deterministic.  `done` counts the blocks that have written their
// partial row; the last one resets it to 0 for the next launch.  Launch: kObs
// warps per block.
constexpr int kRowChunk = 1024;
__global__ void __launch_bounds__(32 * kObs) obs_rows_reduce(const double *__restrict__ rows, int nrows,
                                                             double *__restrict__ partial,
                                                             unsigned *__restrict__ done, ObsConsts c,
                                                             lbm_observables *__restrict__ out) {
    __shared__ double red[32 * kObs];
    __shared__ bool last;
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int r0 = blockIdx.x * kRowChunk;
    const int words = (min(nrows, r0 + kRowChunk) - r0) * kObs;
    const double *chunk = rows + (size_t)r0 * kObs;
    double s = 0.0;
    for (int e = t; e < words; e += 32 * kObs) s += chunk[e];
    red[t] = s;
    __syncthreads();
    const double v = warp_sum(red[lane * kObs + w]);   // term w, rows lane + 32 i
    if (lane == 0) partial[(size_t)blockIdx.x * kObs + w] = v;
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    finalize_observables(partial, gridDim.x, c, out);
    if (t == 0) *done = 0u;
}

// Vertical profile, src/output.cu:336-368: one block per xz plane iy.
template <class S, bool SWAPPED, bool PERIODIC>
__global__ void __launch_bounds__(kObsThreads) profile_kernel(const StepArgs<S> a, double *__restrict__ out) {
    using R = typename Codec<S>::R;
    const int iy = blockIdx.x;
    double acc[5] = {0, 0, 0, 0, 0};
    const uint32_t cnt = (uint32_t)a.lx * (uint32_t)a.lz;
    for (uint32_t t = threadIdx.x; t < cnt; t += blockDim.x) {
        const uint32_t iz = t / (uint32_t)a.lx, ix = t - iz * (uint32_t)a.lx;
        const uint32_t n = (iz * (uint32_t)a.ly + (uint32_t)iy) * (uint32_t)a.lx + ix;
        const Node g = make_node<PERIODIC>(a, n);
        R fr[Q], gr[Q];
        gather<S, SWAPPED>(a, g, fr, gr);
        const Moments<R> m = node_moments<S>(a, fr, gr, n);
        acc[0] += (double)m.ux;
        acc[1] += (double)m.uy;
        acc[2] += (double)m.uz;
        acc[3] += (double)m.phi;
        acc[4] += (double)m.phi * (double)m.phi;
    }
    __shared__ double red[5][kObsThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 5; k++) {
        double v = warp_sum(acc[k]);
        if (lane == 0) red[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s[5];
        for (int k = 0; k < 5; k++) {
            s[k] = 0.0;
            for (int w = 0; w < (int)(blockDim.x / 32); w++) s[k] += red[k][w];
        }
        const double c = (double)cnt;
        const double ap = s[3] / c;
        out[5 * iy + 0] = s[0] / c;
        out[5 * iy + 1] = s[1] / c;
        out[5 * iy + 2] = s[2] / c;
        out[5 * iy + 3] = ap;
        out[5 * iy + 4] = sqrt(s[4] / c - ap * ap);
    }
}

// One population (which 0 = f, 1 = g; index k), decoded, natural order.
template <class S, bool SWAPPED, bool PERIODIC>
__global__ void export_pop_kernel(const StepArgs<S> a, int which, int k, double *__restrict__ out) {
    using C = Codec<S>;
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.nodes) return;
    const Node g = make_node<PERIODIC>(a, n);
    double v = 0.0;
    Unroll<0, Q>::run([&](auto kk) {
        constexpr int K = decltype(kk)::value;
        if (K == k) {
            // 16-bit storage: g/w is stored relative to the conduction
            // profile at the location read (step.cuh shift0)
            float sh = 0.f;
            if constexpr (elem_stride<S>() == 2) sh = shift0(a, g) + read_shift_delta<SWAPPED, K, kNoneInside>(a, g);
            if (which)
                v = (double)C::template g_in<K>(load_pop<S, SWAPPED, K, false, 1>(a, g),
                                                elem_stride<S>() == 2 ? (typename C::R)sh : a.t0);
            else
                v = (double)C::template f_in<K>(load_pop<S, SWAPPED, K, false, 0>(a, g), a.t0);
        }
    });
    out[n] = v;
}

// rho, ux, uy, uz, phi as the reference's macrovar leaves them (src/macrovar.cu:3-34).
template <class S, bool SWAPPED, bool PERIODIC>
__global__ void export_macro_kernel(const StepArgs<S> a, double *__restrict__ out /* 5 x nodes */) {
    using R = typename Codec<S>::R;
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.nodes) return;
    const Node g = make_node<PERIODIC>(a, n);
    R fr[Q], gr[Q];
    gather<S, SWAPPED>(a, g, fr, gr);
    const Moments<R> m = node_moments<S>(a, fr, gr, n);
    const size_t N = a.nodes;
    out[n] = (double)m.rho;
    out[N + n] = (double)m.ux;
    out[2 * N + n] = (double)m.uy;
    out[3 * N + n] = (double)m.uz;
    out[4 * N + n] = (double)m.phi;
}

// Writes one population in the natural layout from FP64 values.
template <class S>
__global__ void import_pop_kernel(const StepArgs<S> a, int which, int k, const double *__restrict__ in) {
    using C = Codec<S>;
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.nodes) return;
    const double v = in[n];
    // 16-bit storage: shifted by the conduction profile at this node (natural layout)
    const uint32_t q = a.div_lx.div(n);
    const int iy = (int)(q - a.div_ly.div(q) * (uint32_t)a.ly);
    const float sh = fmaf(-(float)iy, (float)a.t_dy, (float)a.t_top);
    Unroll<0, Q>::run([&](auto kk) {
        constexpr int K = decltype(kk)::value;
        if (K == k) {
            using R = typename C::R;
            if (which)
                a.st(1, K, n) = C::template g_out<K>((R)v, elem_stride<S>() == 2 ? (R)sh : a.t0);
            else
                a.st(0, K, n) = C::template f_out<K>((R)v, a.t0);
        }
    });
}

template <class S>
__global__ void import_phip_kernel(const StepArgs<S> a, const double *__restrict__ in) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.nodes) return;
    a.phip[n] = (typename Codec<S>::P)in[n];
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// Conduction (mode 1), rest (mode 0, src/initial.cu:208-241) or given
// temperature (mode 2: T = a.phip[n], copied there by the caller) state.
// Temperatures are formed in FP64 with explicit round-to-nearest operations,
// in the order T = T_hot - ((T_hot - T_cold) * iy) / (LY - 1.0), then
// T + amplitude*(2u - 1), so every build gives the same bits.
template <class S>
__global__ void init_kernel(const StepArgs<S> a, int mode, uint64_t seed_key, double amplitude, double t_hot,
                            double t_cold, const typename Codec<S>::P *temperature) {
    using C = Codec<S>;
    using R = typename C::R;
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.nodes) return;
    double t = 0.5;
    const uint32_t q = a.div_lx.div(n);
    const uint32_t z = a.div_ly.div(q);
    const int iy = (int)(q - z * (uint32_t)a.ly);
    // 16-bit storage: g/w stored relative to the conduction profile here (step.cuh shift0)
    const float sh = fmaf(-(float)iy, (float)a.t_dy, (float)a.t_top);
    if (mode == 1) {
        const uint64_t r = splitmix64(seed_key + (uint64_t)n);
        const double u = (double)(r >> 11) * (1.0 / 9007199254740992.0);
        t = __dsub_rn(t_hot, __ddiv_rn(__dmul_rn(__dsub_rn(t_hot, t_cold), (double)iy), __dsub_rn((double)a.ly, 1.0)));
        t = __dadd_rn(t, __dmul_rn(amplitude, __dsub_rn(__dmul_rn(2.0, u), 1.0)));
    } else if (mode == 2) {
        t = (double)temperature[n];
    }
    Unroll<0, Q>::run([&](auto kk) {
        constexpr int K = decltype(kk)::value;
        const double gk = __dmul_rn(wd(K), t);
        a.st(0, K, n) = C::template f_out<K>((R)0, a.t0);
        a.st(1, K, n) = C::template g_out<K>((R)gk, elem_stride<S>() == 2 ? (R)sh : a.t0);
    });
    a.phip[n] = (typename C::P)t;
}

// Counts dividends a for which div_by(a, b, RN(1/b)) differs from the
// hardware's correctly rounded a / b: random signs, 52-bit mantissas and
// exponents in [-60, 10].
__global__ void division_check_kernel(double b, double y, uint64_t n, uint64_t key, unsigned long long *bad) {
    unsigned long long cnt = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = splitmix64(key + i);
        const double m = 1.0 + (double)(r >> 12) * (1.0 / 4503599627370496.0);
        const int e = (int)((r & 0x7f) % 71) - 60;
        double a = scalbn(m, e);
        if ((r >> 7) & 1) a = -a;
        if (div_by(a, b, y) != __ddiv_rn(a, b)) cnt++;
    }
    if (cnt) atomicAdd(bad, cnt);
}

}  // namespace lbm

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------


namespace lbm_internal {

int check_params(const lbm_params *p) {
    if (!p) return fail(LBM_ERR_ARG, "params is NULL");
    if (p->lx < 2 || p->ly < 3 || p->lz < 2)
        return fail(LBM_ERR_ARG, "grid must be at least 2 x 3 x 2 (LY >= 3 for the plate gradients)");
    const double nodes = (double)p->lx * (double)p->ly * (double)p->lz;
    if (nodes > 2147483647.0) return fail(LBM_ERR_ARG, "more than 2^31-1 nodes in one case");
    if (p->sides != LBM_SIDES_WALL && p->sides != LBM_SIDES_PERIODIC) return fail(LBM_ERR_ARG, "bad sides");
    if (store_bytes(p->storage) == 0) return fail(LBM_ERR_ARG, "bad storage");
    // 16-bit pair rows are addressed with 32-bit indices below 9 padded rows
    if (store_bytes(p->storage) == 2 && 9.0 * (double)round_up((int64_t)nodes, 128) >= 4294967296.0)
        return fail(LBM_ERR_ARG, "16-bit storage holds at most 477,218,560 nodes per case (FP32 beyond)");
    if (!(p->rayleigh > 0) || !(p->prandtl > 0)) return fail(LBM_ERR_ARG, "Ra and Pr must be positive");
    if (!(p->t_hot > p->t_cold)) return fail(LBM_ERR_ARG, "T_hot must exceed T_cold");
    if (!(p->gravity * p->beta > 0)) return fail(LBM_ERR_ARG, "gravity*beta must be positive");
    return LBM_OK;
}

void derive(const lbm_params *p, lbm_derived *d) {
    const double ly = (double)p->ly;
    d->visc = ly * std::sqrt(p->gravity * p->beta * (p->t_hot - p->t_cold) * ly * p->prandtl / p->rayleigh);
    d->tau = 3.0 * d->visc + 0.5;
    d->u0 = std::sqrt(p->gravity * p->beta * (p->t_hot - p->t_cold) * ly);
    d->diff = d->visc / p->prandtl;
    d->tauc = 3.0 * d->diff + 0.5;
    d->t0 = 0.5 * (p->t_cold + p->t_hot);
}

}  // namespace lbm_internal

namespace {

// Most blocks of the observables reduction: 8 per SM of a 148-SM B200.  The
// fixed array of lbm_observables_noalloc has this many rows, so it covers
// every grid on every device.
constexpr int kObsMaxBlocks = 148 * 8;

// SM count of `device` (148 if it cannot be read, e.g. without a GPU)
int sm_count_of(int device) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0) {
        cudaGetLastError();
        return 148;
    }
    return sms;
}

// Reduction blocks for a grid: one per 256 nodes, at most 8 per SM of the
// device and never more than kObsMaxBlocks.
int obs_blocks_for(int64_t nodes, int sms) {
    const int64_t b = (nodes + kObsThreads - 1) / kObsThreads;
    const int64_t cap = std::min<int64_t>((int64_t)sms * 8, kObsMaxBlocks);
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, cap));
}

template <class S> StepArgs<S> make_args(const lbm_case *c) {
    using R = typename Codec<S>::R;
    StepArgs<S> a;
    for (int k = 0; k < Q; k++) {
        a.fl[k] = a.fs[k] = (S *)c->f + (size_t)k * (size_t)c->ps * elem_stride<S>();
        a.gl[k] = a.gs[k] = (S *)c->g + (size_t)k * (size_t)c->ps * elem_stride<S>();
    }
    for (int b = 0; b < 3; b++)
        a.pairs[b] = a.pairs_st[b] = (S *)c->f + (size_t)(9 * b) * (size_t)c->ps * elem_stride<S>();
    a.pair_row = (uint32_t)c->ps;
    a.obs_rows = nullptr;
    a.phip = (typename Codec<S>::P *)c->phip;
    a.lx = c->p.lx;
    a.ly = c->p.ly;
    a.lz = c->p.lz;
    a.nodes = (uint32_t)c->nodes;
    a.div_lx = FastDiv((uint32_t)c->p.lx);
    a.div_ly = FastDiv((uint32_t)c->p.ly);
    a.tau = (R)c->d.tau;
    a.tauc = (R)c->d.tauc;
    a.rcp_tau = (R)(1.0 / c->d.tau);
    a.rcp_tauc = (R)(1.0 / c->d.tauc);
    a.rcp_rt = (R)(1.0 / (1.0 / 3.0));
    a.omega_f = (R)(1.0 / c->d.tau);
    a.omega_g = (R)(1.0 / c->d.tauc);
    a.force_fac = (R)(1.0 - 0.5 / c->d.tau);
    a.gb = (R)(c->p.gravity * c->p.beta);
    a.t0 = (R)c->d.t0;
    a.t_top = (R)(c->p.t_hot - (c->p.t_hot - c->p.t_cold) * 0.5 / c->p.ly);
    a.t_dy = (R)((c->p.t_hot - c->p.t_cold) / c->p.ly);
    a.t_hot = (R)c->p.t_hot;
    a.t_cold = (R)c->p.t_cold;
    a.use_phi_fix = c->rest_phi ? 1 : 0;
    a.phi_fix = (R)0.5;
    return a;
}

inline unsigned grid_for(int64_t nodes, int threads) { return (unsigned)((nodes + threads - 1) / threads); }

// Calls fn(tag<S>) for the case's storage type.
template <class Fn> int with_storage(const lbm_case *c, Fn &&fn) {
    switch (c->p.storage) {
    case LBM_STORE_F64: return fn((double *)nullptr);
    case LBM_STORE_F32: return fn((float *)nullptr);
    case LBM_STORE_F16S: return fn((__half *)nullptr);
    case LBM_STORE_BF16S: return fn((__nv_bfloat16 *)nullptr);
    }
    return fail(LBM_ERR_ARG, "bad storage");
}

// Whether the case steps on step16_split_kernel (16-bit storage, BGK): 64
// nodes per block there, 128 in step_kernel.
bool split_step(const lbm_case *c) { return interleaved(c) && c->collision == LBM_COLLISION_BGK; }
int step_blocks(const lbm_case *c) {
    if (split_step(c)) return (int)grid_for(c->nodes, 64);
    return (int)grid_for(c->nodes, c->p.storage == LBM_STORE_F32 ? node_threads<float>() : kStepThreads);
}
// rows of observables sums an observed step writes: one per warp of the node
// kernel, one per warp pair of the 16-bit split kernel
int obs_rows_of(const lbm_case *c) {
    if (split_step(c)) return step_blocks(c) * 2;
    return step_blocks(c) * ((c->p.storage == LBM_STORE_F32 ? node_threads<float>() : kStepThreads) / 32);
}

template <class S, bool SW, bool PER, bool OBS = false>
void launch_step_t(const lbm_case *c, const StepArgs<S> &a, cudaStream_t st) {
    // 16-bit storage, BGK: one node's update split over two warps
    if constexpr (sizeof(S) == 2) {
        if (c->collision == LBM_COLLISION_BGK) {
            step16_split_kernel<S, SW, PER, OBS><<<grid_for(c->nodes, 64), 128, 0, st>>>(a);
            return;
        }
    }
    constexpr int threads = node_threads<S>();
    const unsigned grid = grid_for(c->nodes, threads);
    if (c->collision == LBM_COLLISION_REGULARIZED)
        step_kernel<S, SW, PER, LBM_COLLISION_REGULARIZED, OBS><<<grid, threads, 0, st>>>(a);
    else
        step_kernel<S, SW, PER, LBM_COLLISION_BGK, OBS><<<grid, threads, 0, st>>>(a);
}

// One node-kernel step that also writes the observables of the state it
// reads as per-warp rows into a.obs_rows.
template <class S> void launch_step_observed(const lbm_case *c, const StepArgs<S> &a, cudaStream_t st) {
    const bool per = c->p.sides == LBM_SIDES_PERIODIC;
    if (c->swapped) {
        if (per) launch_step_t<S, true, true, true>(c, a, st);
        else launch_step_t<S, true, false, true>(c, a, st);
    } else {
        if (per) launch_step_t<S, false, true, true>(c, a, st);
        else launch_step_t<S, false, false, true>(c, a, st);
    }
}

// Whether the row-staged kernel (rowstep.cuh) can run this case: periodic
// sides, rows of 32-256 nodes whose bytes are a multiple of 16, FP32 or FP64
// storage (16-bit storage interleaves f and g, which the row staging does
// not handle; its node kernel already moves both in one 32-bit access).
bool row_eligible(const lbm_case *c) {
    const size_t sb = store_bytes(c->p.storage);
    return !interleaved(c) && c->p.sides == LBM_SIDES_PERIODIC && c->p.lx >= 32 && c->p.lx <= 256 &&
           ((size_t)c->p.lx * sb) % 16 == 0;
}

// LBM_KERNEL_AUTO runs the node kernel: on B200 it measured faster than the
// row-staged kernel, whose bulk copies do not raise the bandwidth the node
// kernel already reaches.
bool use_row_kernel(const lbm_case *c) { return c->kernel == LBM_KERNEL_ROW; }

template <class S, bool SW, int PITCH>
cudaError_t launch_row_p(const lbm_case *c, const StepArgs<S> &a, cudaStream_t st) {
    // The shared-memory attribute belongs to the function in one device's
    // context: one bit per device (per instantiation), set once it is applied.
    static std::atomic<uint64_t> configured{0};
    const size_t smem = row_smem_bytes<S>(PITCH);
    const uint64_t bit = c->p.device < 64 ? uint64_t(1) << c->p.device : 0;
    if (!(configured.load(std::memory_order_acquire) & bit)) {
        cudaError_t e = cudaFuncSetAttribute(row_step_kernel<S, SW, PITCH>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured.fetch_or(bit, std::memory_order_release);
    }
    row_step_kernel<S, SW, PITCH><<<(unsigned)(c->p.ly * c->p.lz), (unsigned)c->p.lx, smem, st>>>(a, c->d_err,
                                                                                             c->debug_extra_tx);
    return cudaPeekAtLastError();
}

template <class S, bool SW> cudaError_t launch_row_t(const lbm_case *c, const StepArgs<S> &a, cudaStream_t st) {
    if (c->p.lx <= 64) return launch_row_p<S, SW, 64>(c, a, st);
    if (c->p.lx <= 128) return launch_row_p<S, SW, 128>(c, a, st);
    return launch_row_p<S, SW, 256>(c, a, st);
}

// One step of the case's kernel; returns the launch's error, if any.
template <class S> cudaError_t launch_step(const lbm_case *c, const StepArgs<S> &a, cudaStream_t st) {
    if constexpr (elem_stride<S>() == 1) {
        if (use_row_kernel(c)) return c->swapped ? launch_row_t<S, true>(c, a, st) : launch_row_t<S, false>(c, a, st);
    }
    const bool per = c->p.sides == LBM_SIDES_PERIODIC;
    if (c->swapped) {
        if (per) launch_step_t<S, true, true>(c, a, st);
        else launch_step_t<S, true, false>(c, a, st);
    } else {
        if (per) launch_step_t<S, false, true>(c, a, st);
        else launch_step_t<S, false, false>(c, a, st);
    }
    return cudaPeekAtLastError();
}

// Dispatch a (SWAPPED, PERIODIC)-templated launch for the case's current layout.
#define LBM_DISPATCH_LAYOUT(c, KERNEL, GRID, BLOCK, STREAM, ...)                         \
    do {                                                                                  \
        const bool per_ = (c)->p.sides == LBM_SIDES_PERIODIC;                             \
        if ((c)->swapped) {                                                               \
            if (per_) KERNEL<S, true, true><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__);      \
            else KERNEL<S, true, false><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__);          \
        } else {                                                                          \
            if (per_) KERNEL<S, false, true><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__);     \
            else KERNEL<S, false, false><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__);         \
        }                                                                                 \
    } while (0)

// Launches obs_kernel over case c's state (layout and sides as c says) into
// `partial` and returns the blocks it ran: at most `cap` (the partial rows
// there are) and at most the blocks `sms` SMs hold at once, so that the
// grid-stride loop runs in one wave (8 blocks per SM asked of a kernel that
// fits 5 would run a second, partly idle wave).
template <class S, bool SW, bool PER> int obs_resident() {
    static const int resident = [] {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, obs_kernel<S, SW, PER>, kObsThreads, 0) !=
                cudaSuccess ||
            n <= 0) {
            cudaGetLastError();
            n = 1;
        }
        return n;
    }();
    return resident;
}
template <class S>
int launch_obs(const lbm_case *c, const StepArgs<S> &a, double *partial, int cap, int sms, int split,
               cudaStream_t st) {
    const bool per = c->p.sides == LBM_SIDES_PERIODIC;
    const int resident = c->swapped ? (per ? obs_resident<S, true, true>() : obs_resident<S, true, false>())
                                    : (per ? obs_resident<S, false, true>() : obs_resident<S, false, false>());
    const int blocks = std::max(1, std::min(cap, sms * resident));
    LBM_DISPATCH_LAYOUT(c, obs_kernel, blocks, kObsThreads, st, a, partial, split);
    return blocks;
}

int check_case(const lbm_case *c, bool need_state) {
    if (!c) return fail(LBM_ERR_ARG, "case is NULL");
    if (need_state && !c->initialised) return fail(LBM_ERR_STATE, "case has no state yet (init or load first)");
    return LBM_OK;
}

// Calls that change a case's state or layout: not while it is a batch
// member (the batch's descriptors and captured graphs describe its layout).
int check_mutable(const lbm_case *c, bool need_state) {
    const int rc = check_case(c, need_state);
    if (rc) return rc;
    if (c->batch) return fail(LBM_ERR_STATE, "case is a batch member: remove it from the batch first");
    return LBM_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char *lbm_last_error(void) { return g_last_error.c_str(); }
int lbm_abi_version(void) { return LBM_DDF_ABI_VERSION; }

int lbm_derive(const lbm_params *p, lbm_derived *out) {
    int rc = check_params(p);
    if (rc) return rc;
    if (!out) return fail(LBM_ERR_ARG, "out is NULL");
    derive(p, out);
    return LBM_OK;
}

int lbm_case_bytes(const lbm_params *p, uint64_t *bytes) {
    int rc = check_params(p);
    if (rc) return rc;
    if (!bytes) return fail(LBM_ERR_ARG, "bytes is NULL");
    const int64_t nodes = (int64_t)p->lx * p->ly * p->lz;
    const int64_t ps = round_up(nodes, 128);
    const uint64_t pop = 2ull * Q * (uint64_t)ps * store_bytes(p->storage);
    const uint64_t carry = (uint64_t)round_up(nodes, 128) * (p->storage == LBM_STORE_F64 ? 8 : 4);
    // the reduction rows at their most (the device's SM count is not needed)
    const uint64_t scratch = (uint64_t)obs_blocks_for(nodes, 1 << 20) * kObs * 8 + 256;
    *bytes = pop + carry + scratch;
    return LBM_OK;
}

int lbm_create(const lbm_params *p, lbm_case **out) {
    int rc = check_params(p);
    if (rc) return rc;
    if (!out) return fail(LBM_ERR_ARG, "out is NULL");
    *out = nullptr;
    lbm_case *c = new (std::nothrow) lbm_case();
    if (!c) return fail(LBM_ERR_NOMEM, "host allocation failed");
    c->p = *p;
    derive(p, &c->d);
    c->nodes = (int64_t)p->lx * p->ly * p->lz;
    c->ps = round_up(c->nodes, 128);
    DeviceGuard dg(p->device);
    c->sms = sm_count_of(p->device);
    c->obs_blocks = obs_blocks_for(c->nodes, c->sms);
    const size_t sb = store_bytes(p->storage);
    const size_t pop_bytes = (size_t)Q * (size_t)c->ps * sb;
    const size_t carry_bytes = (size_t)c->ps * (p->storage == LBM_STORE_F64 ? 8 : 4);
    cudaError_t e;
    if (interleaved(c)) {   // one array of (f, g) pairs; g starts one element in
        e = cudaMalloc(&c->f, 2 * pop_bytes);
        if (e == cudaSuccess) c->g = (char *)c->f + sb;
    } else {
        e = cudaMalloc(&c->f, pop_bytes);
        if (e == cudaSuccess) e = cudaMalloc(&c->g, pop_bytes);
    }
    if (e == cudaSuccess) e = cudaMalloc(&c->phip, carry_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&c->partial, (size_t)c->obs_blocks * kObs * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&c->d_obs, sizeof(lbm_observables));
    if (e == cudaSuccess) e = cudaMalloc(&c->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, sizeof(int));
    if (e != cudaSuccess) {
        cudaGetLastError();
        lbm_destroy(c);
        return fail(e == cudaErrorMemoryAllocation ? LBM_ERR_NOMEM : LBM_ERR_CUDA,
                    std::string("device allocation failed: ") + cudaGetErrorString(e));
    }
    *out = c;
    return LBM_OK;
}

int lbm_destroy(lbm_case *c) {
    if (!c) return LBM_OK;
    if (c->batch) batch_forget(c->batch, c);
    DeviceGuard dg(c->p.device);
    cudaFree(c->f);
    if (!interleaved(c)) cudaFree(c->g);
    cudaFree(c->phip);
    cudaFree(c->partial);
    cudaFree(c->d_obs);
    cudaFree(c->d_err);
    cudaFree(c->obs_rows);
    cudaFree(c->obs_series);
    delete c;
    return LBM_OK;
}

// mode 0: rest state; 1: seeded conduction state; 2: from `temperature`
// (one carried-temperature value per node, readable by the device).
static int init_common(lbm_case *c, int mode, uint64_t seed, double amplitude, void *stream,
                       const void *temperature = nullptr) {
    int rc = check_mutable(c, false);
    if (rc) return rc;
    DeviceGuard dg(c->p.device);
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t key = [&] {
        uint64_t x = seed + 0x9E3779B97F4A7C15ull;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        return x ^ (x >> 31);
    }();
    rc = with_storage(c, [&](auto tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        const StepArgs<S> a = make_args<S>(c);
        init_kernel<S><<<grid_for(c->nodes, 256), 256, 0, st>>>(
            a, mode, key, amplitude, c->p.t_hot, c->p.t_cold, (const typename Codec<S>::P *)temperature);
        return LBM_OK;
    });
    if (rc) return rc;
    CUDA_TRY(cudaGetLastError());
    // returns with the state written, so later work on any stream sees it
    CUDA_TRY(cudaStreamSynchronize(st));
    c->swapped = false;
    c->step = 0;
    c->initialised = true;
    c->rest_phi = mode == 0;
    return LBM_OK;
}

int lbm_init_rest(lbm_case *c, void *stream) { return init_common(c, 0, 0, 0.0, stream); }

int lbm_init_conduction(lbm_case *c, uint64_t seed, double amplitude, void *stream) {
    return init_common(c, 1, seed, amplitude, stream);
}

int lbm_init_temperature(lbm_case *c, const void *temperature, void *stream) {
    int rc = check_mutable(c, false);
    if (rc) return rc;
    if (!temperature) return fail(LBM_ERR_ARG, "temperature is NULL");
    DeviceGuard dg(c->p.device);
    // Memory this device can read (its own, or page-locked host memory
    // mapped into its address space, as cudaHostAlloc gives under unified
    // addressing): the init kernel reads the field itself, host memory over
    // PCIe while it writes the populations to HBM, so the transfer and the
    // initialisation overlap.  Anything else (pageable memory, another
    // device's): copied into the carried-temperature array first.
    const void *direct = nullptr;
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, temperature) == cudaSuccess) {
        if ((at.type == cudaMemoryTypeDevice && at.device == c->p.device) || at.type == cudaMemoryTypeHost ||
            at.type == cudaMemoryTypeManaged)
            direct = at.devicePointer;
    } else {
        cudaGetLastError();   // an unknown pointer is not an error here: it is copied
    }
    if (direct) return init_common(c, 2, 0, 0.0, stream, direct);
    const size_t bytes = (size_t)c->nodes * (c->p.storage == LBM_STORE_F64 ? sizeof(double) : sizeof(float));
    CUDA_TRY(cudaMemcpyAsync(c->phip, temperature, bytes, cudaMemcpyDefault, (cudaStream_t)stream));
    return init_common(c, 2, 0, 0.0, stream, c->phip);
}

int lbm_load_ref_state(lbm_case *c, const double *rho, const double *ux, const double *uy, const double *uz,
                       const double *phi, const double *f, const double *g) {
    (void)rho; (void)ux; (void)uz; (void)phi;
    int rc = check_mutable(c, false);
    if (rc) return rc;
    if (!uy || !f || !g) return fail(LBM_ERR_ARG, "uy, f and g are required");
    DeviceGuard dg(c->p.device);
    const int64_t N = c->nodes;
    // Previous-step temperature from uy = sum(c_y f) + g*beta*(phi_prev - t0)/2.
    // For FP64 storage the estimate is nudged, one ulp at a time, until the
    // device's own formula, jy + 0.5*(gb*(phi_prev - t0)), gives back the
    // file's uy bit for bit, so the first step uses the velocity the
    // reference would use.
    std::vector<double> pp((size_t)N);
    const double gb = c->p.gravity * c->p.beta;
    const double t0 = c->d.t0;
    const bool exact = c->p.storage == LBM_STORE_F64;
    for (int64_t i = 0; i < N; i++) {
        double jy = 0.0;
        for (int k = 0; k < Q; k++) {
            if (cy(k) > 0) jy += f[(size_t)k * N + i];
            if (cy(k) < 0) jy -= f[(size_t)k * N + i];
        }
        double p = t0 + 2.0 * (uy[i] - jy) / gb;
        if (exact && std::isfinite(p)) {
            for (int it = 0; it < 64; it++) {
                const volatile double h = gb * (p - t0);
                const volatile double u = jy + 0.5 * h;
                if (u == uy[i]) break;
                p = std::nextafter(p, u < uy[i] ? INFINITY : -INFINITY);
            }
        }
        pp[(size_t)i] = p;
    }
    double *stage = nullptr;
    CUDA_TRY(cudaMalloc(&stage, (size_t)N * sizeof(double)));
    rc = with_storage(c, [&](auto tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        const StepArgs<S> a = make_args<S>(c);
        for (int which = 0; which < 2; which++)
            for (int k = 0; k < Q; k++) {
                const double *src = (which ? g : f) + (size_t)k * N;
                cudaError_t e = cudaMemcpy(stage, src, (size_t)N * sizeof(double), cudaMemcpyHostToDevice);
                if (e != cudaSuccess) return fail(LBM_ERR_CUDA, cudaGetErrorString(e));
                import_pop_kernel<S><<<grid_for(N, 256), 256>>>(a, which, k, stage);
            }
        cudaError_t e = cudaMemcpy(stage, pp.data(), (size_t)N * sizeof(double), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return fail(LBM_ERR_CUDA, cudaGetErrorString(e));
        import_phip_kernel<S><<<grid_for(N, 256), 256>>>(a, stage);
        return LBM_OK;
    });
    cudaError_t e = cudaDeviceSynchronize();
    cudaFree(stage);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(LBM_ERR_CUDA, cudaGetErrorString(e));
    c->swapped = false;
    c->step = 0;
    c->initialised = true;
    c->rest_phi = false;
    return LBM_OK;
}

int lbm_store_ref_state(lbm_case *c, double *rho, double *ux, double *uy, double *uz, double *phi, double *f,
                        double *g) {
    int rc = check_case(c, true);
    if (rc) return rc;
    DeviceGuard dg(c->p.device);
    const int64_t N = c->nodes;
    CUDA_TRY(cudaDeviceSynchronize());
    double *stage = nullptr;
    CUDA_TRY(cudaMalloc(&stage, (size_t)N * 5 * sizeof(double)));
    rc = with_storage(c, [&](auto tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        const StepArgs<S> a = make_args<S>(c);
        if (rho || ux || uy || uz || phi) {
            LBM_DISPATCH_LAYOUT(c, export_macro_kernel, grid_for(N, 256), 256, (cudaStream_t)0, a, stage);
            double *dst[5] = {rho, ux, uy, uz, phi};
            for (int k = 0; k < 5; k++)
                if (dst[k]) {
                    cudaError_t e = cudaMemcpy(dst[k], stage + (size_t)k * N, (size_t)N * sizeof(double),
                                               cudaMemcpyDeviceToHost);
                    if (e != cudaSuccess) return fail(LBM_ERR_CUDA, cudaGetErrorString(e));
                }
        }
        for (int which = 0; which < 2; which++) {
            double *dst = which ? g : f;
            if (!dst) continue;
            for (int k = 0; k < Q; k++) {
                LBM_DISPATCH_LAYOUT(c, export_pop_kernel, grid_for(N, 256), 256, (cudaStream_t)0, a, which, k,
                                    stage);
                cudaError_t e = cudaMemcpy(dst + (size_t)k * N, stage, (size_t)N * sizeof(double),
                                           cudaMemcpyDeviceToHost);
                if (e != cudaSuccess) return fail(LBM_ERR_CUDA, cudaGetErrorString(e));
            }
        }
        return LBM_OK;
    });
    cudaError_t e = cudaGetLastError();
    cudaFree(stage);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(LBM_ERR_CUDA, cudaGetErrorString(e));
    return LBM_OK;
}

int lbm_step(lbm_case *c, int32_t nsteps, void *stream) {
    int rc = check_mutable(c, true);
    if (rc) return rc;
    if (nsteps < 0) return fail(LBM_ERR_ARG, "nsteps < 0");
    DeviceGuard dg(c->p.device);
    cudaStream_t st = (cudaStream_t)stream;
    rc = with_storage(c, [&](auto tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        StepArgs<S> a = make_args<S>(c);
        for (int s = 0; s < nsteps; s++) {
            const cudaError_t e = launch_step<S>(c, a, st);
            if (e != cudaSuccess) {
                c->step += s;   // the steps launched before the failure
                cudaGetLastError();
                return fail(LBM_ERR_CUDA, cudaGetErrorString(e));
            }
            c->swapped = !c->swapped;
            c->rest_phi = false;
            a.use_phi_fix = 0;
        }
        c->step += nsteps;
        return LBM_OK;
    });
    if (rc) return rc;
    CUDA_TRY(cudaGetLastError());
    return LBM_OK;
}

}  // extern "C"

// Enqueues on `st` the observables reduction of case c's current state into
// dst (device memory): two kernels, no synchronisation.
int lbm_internal::enqueue_observables(const lbm_case *c, lbm_observables *dst, cudaStream_t st) {
    return with_storage(c, [&](auto tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        const StepArgs<S> a = make_args<S>(c);
        const int blocks = launch_obs<S>(c, a, c->partial, c->obs_blocks, c->sms, split_step(c) ? 1 : 0, st);
        ObsConsts k;
        k.nodes = (double)c->nodes;
        k.plane = (double)c->p.lx * (double)c->p.lz;
        k.ly = (double)c->p.ly;
        k.diff = c->d.diff;
        k.dT = c->p.t_hot - c->p.t_cold;
        k.visc = c->d.visc;
        k.step = c->step;
        obs_finalize<<<1, 32 * kObs, 0, st>>>(c->partial, blocks, k, dst);
        return LBM_OK;
    });
}

// Enqueues on `st` one node-kernel step of case c from layout `swapped`
// (whatever c->swapped says: a batch enqueues several steps of a member
// before its host-side layout flag moves); changes nothing on the host.
int lbm_internal::enqueue_case_step(const lbm_case *c, bool swapped, cudaStream_t st) {
    return with_storage(c, [&](auto tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        StepArgs<S> a = make_args<S>(c);
        a.use_phi_fix = 0;   // batch members have taken their first step
        const bool per = c->p.sides == LBM_SIDES_PERIODIC;
        if (swapped) {
            if (per) launch_step_t<S, true, true>(c, a, st);
            else launch_step_t<S, true, false>(c, a, st);
        } else {
            if (per) launch_step_t<S, false, true>(c, a, st);
            else launch_step_t<S, false, false>(c, a, st);
        }
        const cudaError_t e = cudaPeekAtLastError();
        return e == cudaSuccess ? LBM_OK : fail(LBM_ERR_CUDA, cudaGetErrorString(e));
    });
}

extern "C" {

int lbm_get_observables(lbm_case *c, lbm_observables *out, void *stream) {
    int rc = check_case(c, true);
    if (rc) return rc;
    if (!out) return fail(LBM_ERR_ARG, "out is NULL");
    DeviceGuard dg(c->p.device);
    cudaStream_t st = (cudaStream_t)stream;
    rc = enqueue_observables(c, c->d_obs, st);
    if (rc) return rc;
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(out, c->d_obs, sizeof(lbm_observables), cudaMemcpyDeviceToHost, st));
    int err = 0;
    CUDA_TRY(cudaMemcpyAsync(&err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (err) return fail(LBM_ERR_CUDA, "a step kernel gave up waiting for its shared-memory copies");
    if (out->diverged) return fail(LBM_ERR_DIVERGED, "NaN/Inf in the macroscopic fields");
    return LBM_OK;
}

// lbm_step_observed (wait = true) and lbm_step_observed_async (false).
static int step_observed(lbm_case *c, int32_t nsteps, lbm_observables *out, void *stream, bool wait) {
    int rc = check_mutable(c, true);
    if (rc) return rc;
    if (nsteps < 0) return fail(LBM_ERR_ARG, "nsteps < 0");
    if (nsteps > 0 && !out) return fail(LBM_ERR_ARG, "out is NULL");
    if (use_row_kernel(c))
        return fail(LBM_ERR_ARG, "steps with observables run on the node kernel; the case's step kernel is set to ROW");
    if (nsteps == 0) return LBM_OK;
    DeviceGuard dg(c->p.device);
    cudaStream_t st = (cudaStream_t)stream;
    // one row per warp of the node kernel (per warp pair of the 16-bit BGK
    // kernel): room for the most rows, whichever kernel the case uses now
    const int rows = obs_rows_of(c);
    const int parts = (rows + kRowChunk - 1) / kRowChunk;
    const int max_rows = (int)grid_for(c->nodes, kStepThreads) * (kStepThreads / 32);
    const int max_parts = (max_rows + kRowChunk - 1) / kRowChunk;
    if (!c->obs_rows) {   // per-warp rows, the chunk partials, the count of chunks done
        const size_t bytes = (size_t)(max_rows + max_parts) * kObs * sizeof(double);
        CUDA_TRY(cudaMalloc(&c->obs_rows, bytes + sizeof(double)));
        CUDA_TRY(cudaMemsetAsync((char *)c->obs_rows + bytes, 0, sizeof(double), st));
    }
    if (nsteps > c->obs_series_cap) {
        if (c->obs_series) {
            CUDA_TRY(cudaStreamSynchronize(st));
            cudaFree(c->obs_series);
            c->obs_series = nullptr;
            c->obs_series_cap = 0;
        }
        CUDA_TRY(cudaMalloc(&c->obs_series, (size_t)nsteps * sizeof(lbm_observables)));
        c->obs_series_cap = nsteps;
    }
    double *partial = c->obs_rows + (size_t)max_rows * kObs;
    unsigned *done = (unsigned *)(partial + (size_t)max_parts * kObs);
    rc = with_storage(c, [&](auto tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        StepArgs<S> a = make_args<S>(c);
        a.obs_rows = c->obs_rows;
        ObsConsts k;
        k.nodes = (double)c->nodes;
        k.plane = (double)c->p.lx * (double)c->p.lz;
        k.ly = (double)c->p.ly;
        k.diff = c->d.diff;
        k.dT = c->p.t_hot - c->p.t_cold;
        k.visc = c->d.visc;
        for (int s = 0; s < nsteps; s++) {
            k.step = c->step + s;   // the state this step starts from
            launch_step_observed<S>(c, a, st);
            obs_rows_reduce<<<parts, 32 * kObs, 0, st>>>(c->obs_rows, rows, partial, done, k, c->obs_series + s);
            c->swapped = !c->swapped;
            c->rest_phi = false;
            a.use_phi_fix = 0;
        }
        return LBM_OK;
    });
    if (rc) return rc;
    c->step += nsteps;
    CUDA_TRY(cudaGetLastError());
    // in stream order before the next call's kernels rewrite obs_series
    CUDA_TRY(cudaMemcpyAsync(out, c->obs_series, (size_t)nsteps * sizeof(lbm_observables), cudaMemcpyDefault, st));
    if (!wait) return LBM_OK;
    CUDA_TRY(cudaStreamSynchronize(st));
    for (int s = 0; s < nsteps; s++)
        if (out[s].diverged) return fail(LBM_ERR_DIVERGED, "NaN/Inf in the macroscopic fields");
    return LBM_OK;
}

int lbm_step_observed(lbm_case *c, int32_t nsteps, lbm_observables *out, void *stream) {
    return step_observed(c, nsteps, out, stream, true);
}

int lbm_step_observed_async(lbm_case *c, int32_t nsteps, lbm_observables *out, void *stream) {
    return step_observed(c, nsteps, out, stream, false);
}

int lbm_get_profile(lbm_case *c, double *out, void *stream) {
    int rc = check_case(c, true);
    if (rc) return rc;
    if (!out) return fail(LBM_ERR_ARG, "out is NULL");
    DeviceGuard dg(c->p.device);
    cudaStream_t st = (cudaStream_t)stream;
    double *dprof = nullptr;
    CUDA_TRY(cudaMalloc(&dprof, (size_t)5 * c->p.ly * sizeof(double)));
    rc = with_storage(c, [&](auto tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        const StepArgs<S> a = make_args<S>(c);
        LBM_DISPATCH_LAYOUT(c, profile_kernel, c->p.ly, kObsThreads, st, a, dprof);
        return LBM_OK;
    });
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, dprof, (size_t)5 * c->p.ly * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(dprof);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(LBM_ERR_CUDA, cudaGetErrorString(e));
    return LBM_OK;
}

// Checkpoint image: header, f, g, phip (each region 256-byte aligned).
struct CheckpointHeader {
    char magic[8];          // "LBMDDF3\0" (16-bit states: interleaved (f, g) pairs, g shifted by the conduction profile)
    lbm_params p;
    int64_t step;
    int32_t swapped;
    int32_t flags;          // bit 0: next step uses the rest state's phi = 0.5
    int64_t ps;
};

static uint64_t ckpt_layout(const lbm_case *c, uint64_t *off_f, uint64_t *off_g, uint64_t *off_p,
                            uint64_t *pop_bytes, uint64_t *carry_bytes) {
    const uint64_t hb = (uint64_t)round_up(sizeof(CheckpointHeader), 256);
    *pop_bytes = (uint64_t)Q * (uint64_t)c->ps * store_bytes(c->p.storage);
    *carry_bytes = (uint64_t)c->ps * (c->p.storage == LBM_STORE_F64 ? 8 : 4);
    *off_f = hb;
    *off_g = hb + *pop_bytes;
    *off_p = hb + 2 * *pop_bytes;
    return *off_p + *carry_bytes;
}

int lbm_checkpoint_bytes(const lbm_case *c, uint64_t *bytes) {
    if (!c || !bytes) return fail(LBM_ERR_ARG, "NULL argument");
    uint64_t a, b, d, e, f;
    *bytes = ckpt_layout(c, &a, &b, &d, &e, &f);
    return LBM_OK;
}

int lbm_save_state(lbm_case *c, void *host, uint64_t bytes, void *stream) {
    int rc = check_case(c, true);
    if (rc) return rc;
    uint64_t of, og, op, pb, cb;
    const uint64_t need = ckpt_layout(c, &of, &og, &op, &pb, &cb);
    if (!host || bytes < need) return fail(LBM_ERR_ARG, "checkpoint buffer missing or too small");
    DeviceGuard dg(c->p.device);
    CheckpointHeader h;
    std::memset(&h, 0, sizeof h);
    std::memcpy(h.magic, "LBMDDF3", 8);
    h.p = c->p;
    h.step = c->step;
    h.swapped = c->swapped ? 1 : 0;
    h.flags = c->rest_phi ? 1 : 0;
    h.ps = c->ps;
    std::memcpy(host, &h, sizeof h);
    cudaStream_t st = (cudaStream_t)stream;
    char *b = (char *)host;
    if (interleaved(c)) {   // the f and g regions are one array of pairs
        CUDA_TRY(cudaMemcpyAsync(b + of, c->f, 2 * pb, cudaMemcpyDeviceToHost, st));
    } else {
        CUDA_TRY(cudaMemcpyAsync(b + of, c->f, pb, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaMemcpyAsync(b + og, c->g, pb, cudaMemcpyDeviceToHost, st));
    }
    CUDA_TRY(cudaMemcpyAsync(b + op, c->phip, cb, cudaMemcpyDeviceToHost, st));
    return LBM_OK;
}

int lbm_restore_state(lbm_case *c, const void *host, uint64_t bytes, void *stream) {
    int rc = check_mutable(c, false);
    if (rc) return rc;
    uint64_t of, og, op, pb, cb;
    const uint64_t need = ckpt_layout(c, &of, &og, &op, &pb, &cb);
    if (!host || bytes < need) return fail(LBM_ERR_ARG, "checkpoint buffer missing or too small");
    CheckpointHeader h;
    std::memcpy(&h, host, sizeof h);
    if (std::memcmp(h.magic, "LBMDDF3", 8) != 0) return fail(LBM_ERR_ARG, "not an engine checkpoint");
    if (h.p.lx != c->p.lx || h.p.ly != c->p.ly || h.p.lz != c->p.lz || h.p.storage != c->p.storage ||
        h.p.sides != c->p.sides || h.ps != c->ps || h.p.rayleigh != c->p.rayleigh || h.p.prandtl != c->p.prandtl ||
        h.p.beta != c->p.beta || h.p.gravity != c->p.gravity || h.p.t_hot != c->p.t_hot || h.p.t_cold != c->p.t_cold)
        return fail(LBM_ERR_ARG, "checkpoint was taken from a case with other parameters");
    DeviceGuard dg(c->p.device);
    cudaStream_t st = (cudaStream_t)stream;
    const char *b = (const char *)host;
    if (interleaved(c)) {
        CUDA_TRY(cudaMemcpyAsync(c->f, b + of, 2 * pb, cudaMemcpyHostToDevice, st));
    } else {
        CUDA_TRY(cudaMemcpyAsync(c->f, b + of, pb, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(c->g, b + og, pb, cudaMemcpyHostToDevice, st));
    }
    CUDA_TRY(cudaMemcpyAsync(c->phip, b + op, cb, cudaMemcpyHostToDevice, st));
    c->step = h.step;
    c->swapped = h.swapped != 0;
    c->rest_phi = (h.flags & 1) != 0;
    c->initialised = true;
    return LBM_OK;
}

// ---------------------------------------------------------------------------
// Observables without allocating.
//
// For callers that hold their populations in memory they manage themselves
// and may not allocate device memory from this library: code that runs while
// a CUDA stream is being captured into a graph, a serving loop whose whole
// HBM budget is accounted for up front, or a host thread that must not block
// (cudaMalloc and cudaFree synchronise the device).  The reduction's block
// partial sums live in this fixed device array instead of an allocation; the
// array is part of the library image, so every GPU that loads the library
// holds it (kNoAllocRows x 13 doubles = 123 KB) until the process exits.
// ---------------------------------------------------------------------------
constexpr int kNoAllocRows = kObsMaxBlocks;   // most reduction blocks one call runs
static_assert(kNoAllocRows >= kObsMaxBlocks, "the fixed array must hold every reduction row");
static __device__ __align__(256) double g_noalloc_partials[kNoAllocRows * kObs];

namespace {
std::mutex g_noalloc_mu;
void *g_noalloc_ptr[256];               // device address of the array, per device ordinal
int g_noalloc_sms[256];                 // SM count, per device ordinal

// Looks up the array's device address (and the SM count) once per device,
// with that device current; host code cannot use the symbol itself as a
// device address.
int noalloc_scratch(int device, double **out, int *sms) {
    if (device < 0 || device >= 256) return fail(LBM_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_partials);
        if (e != cudaSuccess || !ptr)
            return fail(LBM_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_partials): ") +
                                          cudaGetErrorString(e));
        g_noalloc_sms[device] = sm_count_of(device);
        g_noalloc_ptr[device] = ptr;
    }
    *out = (double *)g_noalloc_ptr[device];
    *sms = g_noalloc_sms[device];
    return LBM_OK;
}
}  // namespace

int lbm_observables_noalloc(const lbm_params *p, const void *f, const void *g, const void *phi_prev,
                            uint64_t pop_stride, int32_t swapped, int64_t step, lbm_observables *out_dev,
                            void *stream) {
    int rc = check_params(p);
    if (rc) return rc;
    if (!f || !g || !phi_prev || !out_dev) return fail(LBM_ERR_ARG, "f, g, phi_prev and out_dev are required");
    const int64_t nodes = (int64_t)p->lx * p->ly * p->lz;
    if ((int64_t)pop_stride < nodes) return fail(LBM_ERR_ARG, "pop_stride is smaller than the node count");
    if (p->storage == LBM_STORE_F16S || p->storage == LBM_STORE_BF16S) {
        // one array of (f, g) pairs: g is f's partner element, and the pair
        // rows are addressed with 32-bit indices below 9 * pop_stride
        if ((const char *)g != (const char *)f + store_bytes(p->storage))
            return fail(LBM_ERR_ARG, "16-bit storage interleaves f and g: pass g = f + 1 element");
        if (9ull * pop_stride >= (1ull << 32))
            return fail(LBM_ERR_ARG, "16-bit storage: pop_stride must be below 477,218,589 pairs");
    } else if (pop_stride > (1ull << 40)) {
        return fail(LBM_ERR_ARG, "pop_stride too large");
    }
    DeviceGuard dg(p->device);
    double *scratch = nullptr;
    int sms = 0;
    rc = noalloc_scratch(p->device, &scratch, &sms);
    if (rc) return rc;
    const int cap = obs_blocks_for(nodes, sms);   // <= kObsMaxBlocks = the array's rows
    lbm_case view;               // a stack view of the caller's buffers; owns nothing
    view.p = *p;
    derive(p, &view.d);
    view.nodes = nodes;
    view.ps = (int64_t)pop_stride;
    view.step = step;
    view.swapped = swapped != 0;
    view.initialised = true;
    view.f = const_cast<void *>(f);
    view.g = const_cast<void *>(g);
    view.phip = const_cast<void *>(phi_prev);
    cudaStream_t st = (cudaStream_t)stream;
    rc = with_storage(&view, [&](auto tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        const StepArgs<S> a = make_args<S>(&view);
        const lbm_case *c = &view;
        // 16-bit storage: the moments as the BGK step kernel forms them
        const int blocks = launch_obs<S>(c, a, scratch, cap, sms, interleaved(c) ? 1 : 0, st);
        ObsConsts k;
        k.nodes = (double)nodes;
        k.plane = (double)p->lx * (double)p->lz;
        k.ly = (double)p->ly;
        k.diff = view.d.diff;
        k.dT = p->t_hot - p->t_cold;
        k.visc = view.d.visc;
        k.step = step;
        obs_finalize<<<1, 32 * kObs, 0, st>>>(scratch, blocks, k, out_dev);
        return LBM_OK;
    });
    view.f = view.g = view.phip = nullptr;
    if (rc) return rc;
    CUDA_TRY(cudaGetLastError());
    return LBM_OK;
}

int lbm_selfcheck_division(int device, double divisor, uint64_t n, uint64_t seed, uint64_t *mismatches) {
    if (!mismatches || !(divisor > 0) || !std::isfinite(divisor)) return fail(LBM_ERR_ARG, "bad arguments");
    DeviceGuard dg(device);
    unsigned long long *d = nullptr;
    CUDA_TRY(cudaMalloc(&d, sizeof(unsigned long long)));
    cudaError_t e = cudaMemset(d, 0, sizeof(unsigned long long));
    if (e == cudaSuccess) {
        division_check_kernel<<<148 * 8, 256>>>(divisor, 1.0 / divisor, n, seed, d);
        e = cudaGetLastError();
    }
    unsigned long long h = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof h, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(LBM_ERR_CUDA, cudaGetErrorString(e));
    *mismatches = h;
    return LBM_OK;
}

int lbm_set_step_kernel(lbm_case *c, int32_t kind) {
    if (!c) return fail(LBM_ERR_ARG, "case is NULL");
    if (kind != LBM_KERNEL_AUTO && kind != LBM_KERNEL_NODE && kind != LBM_KERNEL_ROW)
        return fail(LBM_ERR_ARG, "unknown step kernel");
    if (kind == LBM_KERNEL_ROW && !row_eligible(c))
        return fail(LBM_ERR_ARG, "the row-staged kernel needs FP32 or FP64 storage, periodic sides, "
                                 "32 <= LX <= 256 and LX*element size a multiple of 16 bytes");
    if (kind == LBM_KERNEL_ROW && c->collision != LBM_COLLISION_BGK)
        return fail(LBM_ERR_ARG, "the row-staged kernel collides with BGK only");
    c->kernel = kind;
    return LBM_OK;
}

int lbm_debug_row_wait_extra_bytes(lbm_case *c, uint32_t bytes) {
    if (!c) return fail(LBM_ERR_ARG, "case is NULL");
    if (bytes % 16 != 0 || bytes > 4096) return fail(LBM_ERR_ARG, "bytes must be a multiple of 16, at most 4096");
    c->debug_extra_tx = bytes;
    return LBM_OK;
}

int lbm_set_collision(lbm_case *c, int32_t model) {
    if (!c) return fail(LBM_ERR_ARG, "case is NULL");
    if (model != LBM_COLLISION_BGK && model != LBM_COLLISION_REGULARIZED)
        return fail(LBM_ERR_ARG, "unknown collision model");
    if (c->batch) return fail(LBM_ERR_STATE, "case is a batch member: remove it from the batch first");
    if (model != LBM_COLLISION_BGK && use_row_kernel(c))
        return fail(LBM_ERR_ARG, "the regularised collision runs on the node kernel; the case's step kernel is "
                                 "set to ROW");
    c->collision = model;
    return LBM_OK;
}

int lbm_get_collision(const lbm_case *c, int32_t *model) {
    if (!c || !model) return fail(LBM_ERR_ARG, "NULL argument");
    *model = c->collision;
    return LBM_OK;
}

int lbm_get_step_kernel(const lbm_case *c, int32_t *kind) {
    if (!c || !kind) return fail(LBM_ERR_ARG, "NULL argument");
    *kind = use_row_kernel(c) ? LBM_KERNEL_ROW : LBM_KERNEL_NODE;
    return LBM_OK;
}

int lbm_get_params(const lbm_case *c, lbm_params *p, lbm_derived *d, int64_t *step) {
    if (!c) return fail(LBM_ERR_ARG, "case is NULL");
    if (p) *p = c->p;
    if (d) *d = c->d;
    if (step) *step = c->step;
    return LBM_OK;
}

}  // extern "C"
