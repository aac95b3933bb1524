// pair16.cuh — the fused step for 16-bit storage with two nodes per thread.
//
// Same update and AA layouts as step_kernel (step.cuh), for FP16S / BF16S
// populations and periodic sides.  A thread owns the node pair (x, x+1), x
// even, so every population row is accessed as 32-bit words holding both
// nodes' values: 128 bytes per warp request instead of 64, half as many load
// and store instructions, and two conversions per instruction.  The two
// nodes are collided one after the other in FP32; the inputs of the second
// stay packed in the same registers that receive the first one's outputs.
//
// Swapped layout.  Population k of the pair comes from nodes x - c_kx and
// x + 1 - c_kx.  For c_kx = 0 that is one aligned word; for c_kx = +1 it is
// the high half of word (x-2, x-1) and the low half of word (x, x+1), for
// c_kx = -1 the high half of (x, x+1) and the low half of (x+2, x+3) (x
// periodic).  Outputs with c_Ix != 0 land on (x + c_Ix, x + 1 + c_Ix): the
// aligned word they fall into is completed with the neighbouring pair's
// value, taken from the adjacent lane with one shuffle when that lane holds
// the neighbouring pair of the same row, and written as a 16-bit half by
// each side otherwise (at warp and row ends).
//
// Eligibility (host): 16-bit storage, periodic sides, LX even.
#pragma once

#include "step.cuh"

namespace lbm {

template <class S> struct Pair;

template <> struct Pair<__half> {
    using S2 = __half2;
    __device__ __forceinline__ static float lo(S2 v) { return __low2float(v); }
    __device__ __forceinline__ static float hi(S2 v) { return __high2float(v); }
    __device__ __forceinline__ static S2 pack(float a, float b) { return __floats2half2_rn(a, b); }
    __device__ __forceinline__ static __half rn(float a) { return __float2half_rn(a); }
    __device__ __forceinline__ static S2 make(__half a, __half b) { return __halves2half2(a, b); }
    __device__ __forceinline__ static __half low(S2 v) { return __low2half(v); }
    __device__ __forceinline__ static __half high(S2 v) { return __high2half(v); }
};

template <> struct Pair<__nv_bfloat16> {
    using S2 = __nv_bfloat162;
    __device__ __forceinline__ static float lo(S2 v) { return __low2float(v); }
    __device__ __forceinline__ static float hi(S2 v) { return __high2float(v); }
    __device__ __forceinline__ static S2 pack(float a, float b) { return __floats2bfloat162_rn(a, b); }
    __device__ __forceinline__ static __nv_bfloat16 rn(float a) { return __float2bfloat16_rn(a); }
    __device__ __forceinline__ static S2 make(__nv_bfloat16 a, __nv_bfloat16 b) { return __halves2bfloat162(a, b); }
    __device__ __forceinline__ static __nv_bfloat16 low(S2 v) { return __low2bfloat16(v); }
    __device__ __forceinline__ static __nv_bfloat16 high(S2 v) { return __high2bfloat16(v); }
};

// Stored value <-> FP32 population (the F16S / BF16S shift of lattice.cuh).
template <int K, bool G> __device__ __forceinline__ float dec16(float h, float t0) {
    return G ? (float)wd(K) * (h + t0) : (float)wd(K) * h;
}
template <int I, bool G> __device__ __forceinline__ float enc16(float v, float t0) {
    return G ? fmaf(v, (float)winv(I), -t0) : v * (float)winv(I);
}

// The update of node pair `pr` (nodes 2pr, 2pr+1).  All 32 lanes of the warp
// must call it together (pairs past the end of the grid are inactive lanes);
// `a` is StepArgs or any accessor with the same members (BatchCase).
template <class S, bool SWAPPED, class A>
__device__ __forceinline__ void update_pair(const A &a, uint32_t pr) {
    using P = Pair<S>;
    using S2 = typename P::S2;
    const uint32_t n0 = 2u * pr;                                  // the pair's even node
    const bool active = n0 < a.nodes;
    const int lane = threadIdx.x & 31;
    // geometry of the pair (inactive lanes take node 0 and touch no memory)
    const Node g = make_node<true>(a, active ? n0 : 0u);
    const int32_t x0 = g.ix;
    const int32_t dxm2 = x0 == 0 ? a.lx - 2 : -2;                 // word (x-2, x-1), periodic
    const int32_t dxp2 = x0 + 2 == a.lx ? 2 - a.lx : 2;           // word (x+2, x+3)
    const bool y_lo = g.vym, y_hi = g.vyp;

    S2 fq[Q], gq[Q];
    if (active) {
        Unroll<0, Q>::run([&](auto kk) {
            constexpr int K = decltype(kk)::value;
            constexpr int DY = -cy(K), DZ = -cz(K);
            const bool in = DY < 0 ? y_lo : DY > 0 ? y_hi : true;
            if (!SWAPPED || !in) {
                const uint32_t w = n0 >> 1;
                fq[K] = reinterpret_cast<const S2 *>(a.ld_row(0, K))[w];
                gq[K] = reinterpret_cast<const S2 *>(a.ld_row(1, K))[w];
            } else {
                const int32_t base = (int32_t)n0 + disp<0, DY, DZ>(g);   // node (x, y - c_y, z - c_z)
                const S2 *fr = reinterpret_cast<const S2 *>(a.ld_row(0, opp(K)));
                const S2 *gr = reinterpret_cast<const S2 *>(a.ld_row(1, opp(K)));
                if (cx(K) == 0) {
                    fq[K] = fr[base >> 1];
                    gq[K] = gr[base >> 1];
                } else if (cx(K) > 0) {   // (x-1, x): high of (x-2, x-1), low of (x, x+1)
                    const S2 fm = fr[(base + dxm2) >> 1], f0 = fr[base >> 1];
                    const S2 gm = gr[(base + dxm2) >> 1], g0 = gr[base >> 1];
                    fq[K] = P::make(P::high(fm), P::low(f0));
                    gq[K] = P::make(P::high(gm), P::low(g0));
                } else {                  // (x+1, x+2): high of (x, x+1), low of (x+2, x+3)
                    const S2 f0 = fr[base >> 1], fp = fr[(base + dxp2) >> 1];
                    const S2 g0 = gr[base >> 1], gp = gr[(base + dxp2) >> 1];
                    fq[K] = P::make(P::high(f0), P::low(fp));
                    gq[K] = P::make(P::high(g0), P::low(gp));
                }
            }
        });
    } else {
        Unroll<0, Q>::run([&](auto kk) {
            constexpr int K = decltype(kk)::value;
            fq[K] = P::pack(0.f, 0.f);
            gq[K] = P::pack(0.f, 0.f);
        });
    }

    // collide node x (HALF = 0, low halves), then node x+1 (HALF = 1); each
    // output goes into the half just read: for the natural layout into word
    // opp(I) (its slot), for the swapped layout into word I (its direction)
    Unroll<0, 2>::run([&](auto hh) {
        constexpr int HALF = decltype(hh)::value;
        float fr[Q], gr[Q];
        Unroll<0, Q>::run([&](auto kk) {
            constexpr int K = decltype(kk)::value;
            fr[K] = dec16<K, false>(HALF ? P::hi(fq[K]) : P::lo(fq[K]), a.t0);
            gr[K] = dec16<K, true>(HALF ? P::hi(gq[K]) : P::lo(gq[K]), a.t0);
        });
        const uint32_t n = n0 + HALF;
        Moments<float> m = moments(fr, gr, (float)a.phip[active ? n : 0], a.gb, a.t0);
        if (a.use_phi_fix) m.phi = a.phi_fix;
        collide_fast(fr, gr, m, a.omega_f, a.omega_g, a.force_fac, a.gb, a.t0);
        if (active) a.phip[n] = m.phi;
        Unroll<0, Q>::run([&](auto ii) {
            constexpr int I = decltype(ii)::value;
            constexpr int DY = cy(I);
            const bool out_y = DY < 0 ? !y_lo : DY > 0 ? !y_hi : false;
            float gv = gr[I];
            if (DY != 0 && out_y) gv = abb<I>(gv, DY < 0 ? a.t_hot : a.t_cold, m.rho);
            constexpr int W = SWAPPED ? I : opp(I);
            const auto fh = P::rn(enc16<I, false>(fr[I], a.t0));
            const auto gh = P::rn(enc16<I, true>(gv, a.t0));
            if (HALF == 0) {
                fq[W] = P::make(fh, P::high(fq[W]));
                gq[W] = P::make(gh, P::high(gq[W]));
            } else {
                fq[W] = P::make(P::low(fq[W]), fh);
                gq[W] = P::make(P::low(gq[W]), gh);
            }
        });
    });

    // stores
    const bool left_ok = lane > 0 && x0 > 0;              // lane - 1 holds pair (x-2, x-1) of this row
    const bool right_ok = lane < 31 && x0 + 2 < a.lx;     // lane + 1 holds pair (x+2, x+3) of this row
    Unroll<0, Q>::run([&](auto ii) {
        constexpr int I = decltype(ii)::value;
        constexpr int DX = cx(I), DY = cy(I), DZ = cz(I);
        const bool out_y = DY < 0 ? !y_lo : DY > 0 ? !y_hi : false;
        const S2 fv = fq[I], gv = gq[I];
        if (!SWAPPED) {
            if (active) {
                reinterpret_cast<S2 *>(a.st_row(0, I))[n0 >> 1] = fv;
                reinterpret_cast<S2 *>(a.st_row(1, I))[n0 >> 1] = gv;
            }
            return;
        }
        if (DX == 0) {
            // aligned: the pair itself (bounce-back to slot opp(I)) or the same
            // x in the destination row (slot I)
            if (active) {
                if (out_y) {
                    reinterpret_cast<S2 *>(a.st_row(0, opp(I)))[n0 >> 1] = fv;
                    reinterpret_cast<S2 *>(a.st_row(1, opp(I)))[n0 >> 1] = gv;
                } else {
                    const int32_t dst = (int32_t)n0 + disp<0, DY, DZ>(g);
                    reinterpret_cast<S2 *>(a.st_row(0, I))[dst >> 1] = fv;
                    reinterpret_cast<S2 *>(a.st_row(1, I))[dst >> 1] = gv;
                }
            }
            return;
        }
        // x-shifted directions: every lane takes part in the shuffle, before
        // any branch that depends on the lane (warps may straddle two rows)
        const S2 fn = DX > 0 ? __shfl_up_sync(0xffffffffu, fv, 1) : __shfl_down_sync(0xffffffffu, fv, 1);
        const S2 gn = DX > 0 ? __shfl_up_sync(0xffffffffu, gv, 1) : __shfl_down_sync(0xffffffffu, gv, 1);
        if (!active) return;
        if (out_y) {   // bounce-back: the pair itself, slot opp(I)
            reinterpret_cast<S2 *>(a.st_row(0, opp(I)))[n0 >> 1] = fv;
            reinterpret_cast<S2 *>(a.st_row(1, opp(I)))[n0 >> 1] = gv;
            return;
        }
        // destinations x + DX and x + 1 + DX in row (y + DY, z + DZ)
        const int32_t row = (int32_t)n0 - x0 + disp<0, DY, DZ>(g);   // node (0, y + DY, z + DZ)
        S *fd = a.st_row(0, I) + row;
        S *gd = a.st_row(1, I) + row;
        if (DX > 0) {
            // word (x, x+1) gets (B of the left pair, A of this pair);
            // this pair's B goes to the low half of word (x+2, x+3)
            if (left_ok) {
                reinterpret_cast<S2 *>(fd)[x0 >> 1] = P::make(P::high(fn), P::low(fv));
                reinterpret_cast<S2 *>(gd)[x0 >> 1] = P::make(P::high(gn), P::low(gv));
            } else {
                fd[x0 + 1] = P::low(fv);
                gd[x0 + 1] = P::low(gv);
            }
            if (!right_ok) {
                const int32_t xr = x0 + 2 == a.lx ? 0 : x0 + 2;
                fd[xr] = P::high(fv);
                gd[xr] = P::high(gv);
            }
        } else {
            // word (x, x+1) gets (B of this pair, A of the right pair);
            // this pair's A goes to the high half of word (x-2, x-1)
            if (right_ok) {
                reinterpret_cast<S2 *>(fd)[x0 >> 1] = P::make(P::high(fv), P::low(fn));
                reinterpret_cast<S2 *>(gd)[x0 >> 1] = P::make(P::high(gv), P::low(gn));
            } else {
                fd[x0] = P::high(fv);
                gd[x0] = P::high(gv);
            }
            if (!left_ok) {
                const int32_t xl = x0 == 0 ? a.lx - 1 : x0 - 1;
                fd[xl] = P::low(fv);
                gd[xl] = P::low(gv);
            }
        }
    });
}

template <class S, bool SWAPPED>
__global__ void __launch_bounds__(128, 3) pair16_kernel(const StepArgs<S> a) {
    update_pair<S, SWAPPED>(a, blockIdx.x * blockDim.x + threadIdx.x);
}

}  // namespace lbm
