// step.cuh — the fused LBM-DDF time step: moments, BGK collision of f with the
// Boussinesq force, BGK collision of g, and streaming with halfway bounce-back
// and anti-bounce-back plates, for one node per thread, in place (AA pattern).
//
// What one step computes is the reference's six-launch step
// (Summer536/LBM_DDF src/main.cu:27-46):
//   forcing     F_y = g*beta*(phi^{n-1} - t0)                    src/macrovar.cu:36-47
//   collide f   BGK to feq(rho, u) + (1 - 1/(2 tau)) F_y 3(c_y - u_y) feq(1, u)
//                                                               src/collision.cu:3-33
//   collide g   BGK to geq = w phi (1 + 3c.u + 4.5(c.u)^2 - 1.5u^2)  src/collision.cu:52-64
//   stream f/g  with the wall rules of src/streaming.cu:59-124, 183-250
//   macrovar    rho = sum f, u = sum c f + F/2, phi = sum g      src/macrovar.cu:3-34
// fused into a single pass.  The moments of step n are recomputed from the
// populations at the start of step n+1; the only extra per-node state is the
// previous-step temperature phi^{n-1} ("phip"), because the stored velocity of
// the reference carries the force of the previous step (u^n = sum c f^n +
// g*beta*(phi^{n-1} - t0)/2) and the anti-bounce-back uses rho^{n-1}.
//
// AA pattern (Bailey et al., ICPP 2009).  One array per distribution holds
// the populations in one of two layouts:
//   natural : slot k of node x holds f_k(x) after streaming;
//   swapped : slot k of node x holds the post-collision f*_{opp k}(x), not
//             yet streamed.
// From natural, a step reads slot k of x and writes f*_i to slot opp(i) of x
// (all accesses local).  From swapped, a step reads population k of x from
// slot opp(k) of x - c_k, and writes f*_i to slot i of x + c_i (the set of
// locations a node reads is the set it writes, so no two threads touch the
// same word).  Walls: a population that would leave the box through a wall
// is kept at the node, in the slot its reflection is read from next step,
// with the anti-bounce-back transform applied when it is written; the
// rho^{n-1} this needs is the pre-collision density of the same node.
//
// Wall precedence (reference "last write wins", src/streaming.cu:59-124,
// 183-250, faces applied x-, x+, y-, y+, z-, z+): for g a population that
// crosses a z face is bounced back plainly even if it also crosses a y face;
// otherwise crossing a y face gives anti-bounce-back.  For f every rule is the
// same plain bounce-back.
#pragma once

#include "../../include/lbm_ddf.h"
#include "lattice.cuh"

namespace lbm {

template <class S> struct StepArgs {
    using R = typename Codec<S>::R;
    using P = typename Codec<S>::P;
    // Base address of each population row (row k of f at fl[k]; for 16-bit
    // storage the rows hold (f, g) pairs and gl[k] = fl[k] + 1 element, see
    // elem_stride).  Kernel parameters live in the constant bank, so an
    // access costs one multiply-add of a 32-bit node index onto a constant,
    // whatever the case's size.
    S *fl[Q];
    S *gl[Q];
    // The same addresses again, used only for the stores.  In the
    // natural-layout step every store address equals a load address; forming
    // it from separate bases keeps the compiler from holding all 54 load
    // addresses live across the collision (which costs ~110 registers).
    S *fs[Q];
    S *gs[Q];
    P *phip;           // previous-step temperature, one per node
    int32_t lx, ly, lz;
    uint32_t nodes;
    FastDiv div_lx, div_ly;
    R tau, tauc;       // relaxation times (the FP64 path divides by them)
    R rcp_tau, rcp_tauc, rcp_rt;   // their correctly rounded reciprocals, and that of 1/3
    R omega_f;         // 1/tau
    R omega_g;         // 1/tauc
    R force_fac;       // 1 - 1/(2 tau)
    R gb;              // gravity*beta
    R t0, t_hot, t_cold;
    // 16-bit storage shifts g/w by the conduction profile at the node a value
    // is stored at, T_c(iy) = t_top - iy * t_dy (see stored_shift)
    R t_top, t_dy;
    // The reference's rest state (src/initial.cu:218-240) stores phi = 0.5
    // while its populations w_i * 0.5 sum to 0.5 - 2^-54; its first step
    // collides with the stored 0.5.  When set, the moments use phi_fix
    // instead of sum(g) (one step after lbm_init_rest).
    int32_t use_phi_fix;
    R phi_fix;

    // population rows: loads (f, g) and stores (f, g)
    __device__ __forceinline__ S *ld_row(int which, int k) const { return which ? gl[k] : fl[k]; }
    __device__ __forceinline__ S *st_row(int which, int k) const { return which ? gs[k] : fs[k]; }
    // population k of node j (the accessor interface update_node uses); the
    // index keeps its type (unsigned node, signed displaced node), which
    // the register allocation of the update is sensitive to
    template <class I> __device__ __forceinline__ const S *ldp(int which, int k, I j) const {
        if constexpr (elem_stride<S>() == 1) return ld_row(which, k) + j;
        else return ld_row(which, k) + 2u * (uint32_t)j;
    }
    template <class I> __device__ __forceinline__ S ld(int which, int k, I j) const { return *ldp(which, k, j); }
    template <class I> __device__ __forceinline__ S &st(int which, int k, I j) const {
        if constexpr (elem_stride<S>() == 1) return st_row(which, k)[j];
        else return st_row(which, k)[2u * (uint32_t)j];
    }
    // 16-bit storage: the (f_k, g_k) pair of node j as one 32-bit word.
    // The pair array is addressed in three blocks of nine rows, pair
    // (k mod 9) * pair_row + j of block k / 9, with a 32-bit index (one
    // multiply-add and one wide add per access; on B200 this ran 18% faster
    // than the per-row bases above, which FP32 and FP64 keep: for them the
    // same indexing measured within 1%).  The index stays below
    // 9 pair_row < 2^32 for every case the C ABI accepts in 16-bit storage.
    template <class I, class SS = S> __device__ __forceinline__ typename Pack16<SS>::T ld2(int k, I j) const {
        return reinterpret_cast<const typename Pack16<SS>::T *>(pairs[k / 9])[(uint32_t)(k % 9) * pair_row +
                                                                              (uint32_t)j];
    }
    template <class I, class SS = S> __device__ __forceinline__ typename Pack16<SS>::T &st2(int k, I j) const {
        return reinterpret_cast<typename Pack16<SS>::T *>(pairs_st[k / 9])[(uint32_t)(k % 9) * pair_row +
                                                                           (uint32_t)j];
    }
    double *obs_rows;  // fused observables: one row of kObsTerms sums per warp (else unused)
    S *pairs[3];       // 16-bit storage: rows 0, 9 and 18 of the (f, g) pair array
    S *pairs_st[3];    // the same, for the stores (see fs)
    uint32_t pair_row; // pairs per row (the padded node count)
};

// Geometry of one node: coordinates, and node-index displacements to the
// neighbours along each axis (periodic wrap folded in), with validity flags.
struct Node {
    uint32_t n;
    int32_t ix, iy, iz;
    int32_t dxm, dxp, dym, dyp, dzm, dzp;
    bool vxm, vxp, vym, vyp, vzm, vzp;
};

template <bool PERIODIC, class A>
__device__ __forceinline__ Node make_node(const A &a, uint32_t n) {
    Node g;
    g.n = n;
    uint32_t q = a.div_lx.div(n);
    g.ix = (int32_t)(n - q * (uint32_t)a.lx);
    uint32_t z = a.div_ly.div(q);
    g.iy = (int32_t)(q - z * (uint32_t)a.ly);
    g.iz = (int32_t)z;
    const int32_t plane = a.lx * a.ly;
    g.dym = -a.lx;
    g.dyp = a.lx;
    g.vym = g.iy > 0;
    g.vyp = g.iy < a.ly - 1;
    if (PERIODIC) {
        g.dxm = g.ix > 0 ? -1 : a.lx - 1;
        g.dxp = g.ix < a.lx - 1 ? 1 : 1 - a.lx;
        g.dzm = g.iz > 0 ? -plane : (a.lz - 1) * plane;
        g.dzp = g.iz < a.lz - 1 ? plane : (1 - a.lz) * plane;
        g.vxm = g.vxp = g.vzm = g.vzp = true;
    } else {
        g.dxm = -1;
        g.dxp = 1;
        g.dzm = -plane;
        g.dzp = plane;
        g.vxm = g.ix > 0;
        g.vxp = g.ix < a.lx - 1;
        g.vzm = g.iz > 0;
        g.vzp = g.iz < a.lz - 1;
    }
    return g;
}

// displacement (in nodes) and validity of the neighbour x + (DX, DY, DZ)
template <int DX, int DY, int DZ>
__device__ __forceinline__ int32_t disp(const Node &g) {
    return (DX < 0 ? g.dxm : DX > 0 ? g.dxp : 0) + (DY < 0 ? g.dym : DY > 0 ? g.dyp : 0) +
           (DZ < 0 ? g.dzm : DZ > 0 ? g.dzp : 0);
}
template <int DX, int DY, int DZ>
__device__ __forceinline__ bool inside(const Node &g) {
    return (DX < 0 ? g.vxm : DX > 0 ? g.vxp : true) && (DY < 0 ? g.vym : DY > 0 ? g.vyp : true) &&
           (DZ < 0 ? g.vzm : DZ > 0 ? g.vzp : true);
}
// Which neighbours a node update may take as inside the box without a test
// (the INTERIOR template argument of the gathers and scatters):
//   kNoneInside: none, every neighbour is tested;
//   kRowInside:  those along y and z (0 < iy < LY-1, and periodic sides or
//                0 < iz < LZ-1): only the x neighbour is tested, which is a
//                compile-time true with periodic sides and a per-lane select
//                at the x walls of a closed box;
//   kAllInside:  all of them (a closed box's rows whose warp holds no x-wall
//                node: with LX a multiple of 32, all but the first and last
//                warp of a row);
//   kRowLoWall, kRowHiWall: as kRowInside, in a closed box's warp whose
//                x-wall nodes, if any, all lie at x = 0 (Lo) or all at
//                x = LX-1 (Hi): only the x neighbour on that side is tested
//                (the first and last warp of a row, with LX a multiple of 32
//                and at least 64).
constexpr int kNoneInside = 0, kRowInside = 1, kAllInside = 2, kRowLoWall = 3, kRowHiWall = 4;
template <int INTERIOR, int DX, int DY, int DZ>
__device__ __forceinline__ bool inside_t(const Node &g) {
    if constexpr (INTERIOR == kAllInside) return true;
    else if constexpr (INTERIOR == kRowInside) return DX < 0 ? g.vxm : DX > 0 ? g.vxp : true;
    else if constexpr (INTERIOR == kRowLoWall) return DX < 0 ? g.vxm : true;
    else if constexpr (INTERIOR == kRowHiWall) return DX > 0 ? g.vxp : true;
    else return inside<DX, DY, DZ>(g);
}
// whether every neighbour of a node taking this path is inside (so the
// swapped layout reads every population from, and writes it to, the
// neighbouring planes: the 16-bit update's plane-shift fold applies)
template <int INTERIOR, bool PERIODIC> constexpr bool all_inside() {
    return INTERIOR == kAllInside || (INTERIOR == kRowInside && PERIODIC);
}

// Whether node g's neighbours along y and z are all inside the box (the
// INTERIOR case of inside_t); uniform over a warp whenever LX is a multiple
// of 32.
template <bool PERIODIC> __device__ __forceinline__ bool yz_interior(const Node &g) {
    return g.vym && g.vyp && (PERIODIC || (g.vzm && g.vzp));
}

// The path of node g's update (the INTERIOR argument, see inside_t):
// kRowInside for rows whose y and z neighbours are inside, kAllInside for
// those of a closed box when no active lane of the warp lies at an x wall
// (decided over the warp, so a warp takes one path), else kNoneInside.
// In the natural layout every access is at the node itself, so kAllInside
// would compile to kRowInside's code again: with SWAPPED false it is not
// returned, which keeps a third copy of the update out of the kernel (in the
// issue-bound 16-bit split kernel a larger body measured slower).
template <bool PERIODIC, bool SWAPPED = true> __device__ __forceinline__ int node_path(const Node &g) {
    if (!yz_interior<PERIODIC>(g)) return kNoneInside;
    if constexpr (!PERIODIC && SWAPPED) {
        if (__all_sync(__activemask(), g.vxm && g.vxp)) return kAllInside;
    }
    return kRowInside;
}
// node_path, with a closed box's warps at one x wall told apart (kRowLoWall,
// kRowHiWall), for updates that take those paths (the node kernel's swapped
// layout; in the 16-bit split kernel the two extra paths measured 12% slower
// on the swapped closed-box step).
template <bool PERIODIC> __device__ __forceinline__ int node_path_x(const Node &g) {
    if (!yz_interior<PERIODIC>(g)) return kNoneInside;
    if constexpr (!PERIODIC) {
        const unsigned active = __activemask();
        const bool lo_in = __all_sync(active, g.vxm), hi_in = __all_sync(active, g.vxp);
        if (lo_in && hi_in) return kAllInside;
        if (hi_in) return kRowLoWall;
        if (lo_in) return kRowHiWall;
        return kNoneInside;   // a warp at both x walls (rows shorter than 64 or not whole warps)
    }
    return kRowInside;
}

// Population k (of f when WHICH = 0, of g when 1) of node g at the current
// time, from either layout.  `a` supplies the addresses: a.ldp(which, k,
// node).  In the swapped layout the value sits at the neighbour x - c_K
// (population opp(K)) when that is inside the box, else at the node itself
// (population K, bounce-back); the address is chosen by a select, so a warp
// whose lanes differ (one holding an x-wall node) still issues one load
// rather than two half-masked ones.
template <class S, bool SWAPPED, int K, int INTERIOR = kNoneInside, int WHICH = 0, class A>
__device__ __forceinline__ S load_pop(const A &a, const Node &g) {
    if (!SWAPPED) return a.ld(WHICH, K, g.n);
    constexpr int DX = -cx(K), DY = -cy(K), DZ = -cz(K);
    const bool in = inside_t<INTERIOR, DX, DY, DZ>(g);
    return *(in ? a.ldp(WHICH, opp(K), (int32_t)g.n + disp<DX, DY, DZ>(g)) : a.ldp(WHICH, K, g.n));
}

// The (f_k, g_k) pair that node g collides in this step, as load_pop finds
// each value, with one 32-bit load.  (Here a branch: the address select of
// load_pop measured 3% slower in the 16-bit closed-box swapped step.)
template <class S, bool SWAPPED, int K, int INTERIOR, class A>
__device__ __forceinline__ typename Pack16<S>::T load_pair(const A &a, const Node &g) {
    if (!SWAPPED) return a.ld2(K, g.n);
    constexpr int DX = -cx(K), DY = -cy(K), DZ = -cz(K);
    if (inside_t<INTERIOR, DX, DY, DZ>(g)) return a.ld2(opp(K), (int32_t)g.n + disp<DX, DY, DZ>(g));
    return a.ld2(K, g.n);
}

// 16-bit storage keeps g_i / w_i - T_c at every location, T_c(iy) =
// T_hot - (T_hot - T_cold) (iy + 1/2) / LY the conduction profile at the
// plane of the node the value is stored at (halfway walls: the plates sit
// half a node outside the first and last planes).  Near the plates, where Nu
// is measured, g/w is then close to the stored shift and 16-bit rounding
// small against the plane-to-plane temperature step; with one constant
// shift it was up to 2^-11 (FP16) and 2^-8 (BF16) there.  Inside a node
// update the g values are kept relative to the node's own T_c (shift0); a
// value read from or written to a neighbour's plane differs from that by
// a multiple of t_dy:
//   read (swapped layout, population K from x - c_K): + c_Ky t_dy
//   write (swapped layout, population I to x + c_I):   + c_Iy t_dy
// and by nothing at the node itself (natural layout, bounce-back).
template <class A> __device__ __forceinline__ float shift0(const A &a, const Node &g) {
    return fmaf(-(float)g.iy, (float)a.t_dy, (float)a.t_top);
}
template <bool SWAPPED, int K, int INTERIOR, class A>
__device__ __forceinline__ float read_shift_delta(const A &a, const Node &g) {
    constexpr int DX = -cx(K), DY = -cy(K), DZ = -cz(K);
    if constexpr (!SWAPPED || DY == 0) return 0.f;
    else return inside_t<INTERIOR, DX, DY, DZ>(g) ? (float)cy(K) * (float)a.t_dy : 0.f;
}
template <bool SWAPPED, int I, int INTERIOR, class A>
__device__ __forceinline__ float write_shift_delta(const A &a, const Node &g) {
    constexpr int DX = cx(I), DY = cy(I), DZ = cz(I);
    if constexpr (!SWAPPED || DY == 0) return 0.f;
    else return inside_t<INTERIOR, DX, DY, DZ>(g) ? (float)cy(I) * (float)a.t_dy : 0.f;
}

template <class S, bool SWAPPED, int INTERIOR = kNoneInside, class A>
__device__ __forceinline__ void gather(const A &a, const Node &g, typename Codec<S>::R (&fr)[Q],
                                       typename Codec<S>::R (&gr)[Q]) {
    using C = Codec<S>;
    float s0 = 0.f;
    if constexpr (elem_stride<S>() == 2) s0 = shift0(a, g);
    Unroll<0, Q>::run([&](auto kk) {
        constexpr int K = decltype(kk)::value;
        if constexpr (elem_stride<S>() == 2) {   // (f, g) pairs: f_i = w_i fh, g_i = w_i (gh + T_c at the location)
            // explicit rounding: the compiler cannot fuse these products into
            // the moment sums in one kernel and not in another, so every
            // kernel that gathers (the step, the observables) forms the same
            // FP32 moments
            const float2 v = Pack16<S>::unpack(load_pair<S, SWAPPED, K, INTERIOR>(a, g));
            fr[K] = __fmul_rn((float)wd(K), v.x);
            gr[K] = __fmul_rn((float)wd(K), __fadd_rn(v.y, __fadd_rn(s0, read_shift_delta<SWAPPED, K, INTERIOR>(a, g))));
        } else {
            fr[K] = C::template f_in<K>(load_pop<S, SWAPPED, K, INTERIOR, 0>(a, g), a.t0);
            gr[K] = C::template g_in<K>(load_pop<S, SWAPPED, K, INTERIOR, 1>(a, g), a.t0);
        }
    });
}

// Moments of the populations at one node.  u carries the previous step's
// half force, as the reference's stored velocity does (src/macrovar.cu:28-30).
template <class R> struct Moments {
    R rho, ux, uy, uz, phi;
};

template <class R>
__device__ __forceinline__ Moments<R> moments(const R (&fr)[Q], const R (&gr)[Q], R phip, R gb, R t0) {
    Moments<R> m;
    R rho = 0, jx = 0, jy = 0, jz = 0, phi = 0;
    Unroll<0, Q>::run([&](auto kk) {
        constexpr int K = decltype(kk)::value;
        rho += fr[K];
        if (cx(K) > 0) jx += fr[K];
        if (cx(K) < 0) jx -= fr[K];
        if (cy(K) > 0) jy += fr[K];
        if (cy(K) < 0) jy -= fr[K];
        if (cz(K) > 0) jz += fr[K];
        if (cz(K) < 0) jz -= fr[K];
        phi += gr[K];
    });
    m.rho = rho;
    m.ux = jx;
    if constexpr (std::is_same<R, float>::value)   // explicit rounding: the same in every kernel
        m.uy = __fadd_rn(jy, __fmul_rn(0.5f, __fmul_rn(gb, __fsub_rn(phip, t0))));
    else   // FP64: as written, the rounding the reference build has (bitwise parity)
        m.uy = jy + R(0.5) * (gb * (phip - t0));
    m.uz = jz;
    m.phi = phi;
    return m;
}

template <class S, class A>
__device__ __forceinline__ Moments<typename Codec<S>::R> node_moments(const A &a,
                                                                     const typename Codec<S>::R (&fr)[Q],
                                                                     const typename Codec<S>::R (&gr)[Q],
                                                                     uint32_t n) {
    using R = typename Codec<S>::R;
    Moments<R> m = moments(fr, gr, (R)a.phip[n], a.gb, a.t0);
    if (a.use_phi_fix) m.phi = a.phi_fix;
    return m;
}

// BGK collision of f (with the buoyancy force) and g, in place on fr/gr,
// in FP32: the same equilibria with the divisions by 1/3 and tau folded into
// multiplications and every multiply-add left to the compiler.
template <class R>
__device__ __forceinline__ void collide_fast(R (&fr)[Q], R (&gr)[Q], const Moments<R> &m, R omega_f, R omega_g,
                                             R force_fac, R gb, R t0) {
    const R uv = R(3) * (m.ux * m.ux + m.uy * m.uy + m.uz * m.uz);
    const R fy = gb * (m.phi - t0);           // force of this step, from phi^{n-1}
    const R kf = R(3) * force_fac * fy;
    Unroll<0, Q>::run([&](auto kk) {
        constexpr int K = decltype(kk)::value;
        constexpr R w = R(wd(K));
        R cu = R(0);
        if (cx(K) > 0) cu += m.ux;
        if (cx(K) < 0) cu -= m.ux;
        if (cy(K) > 0) cu += m.uy;
        if (cy(K) < 0) cu -= m.uy;
        if (cz(K) > 0) cu += m.uz;
        if (cz(K) < 0) cu -= m.uz;
        const R eu = R(3) * cu;
        const R p = eu + R(0.5) * (eu * eu - uv);   // velocity part of the equilibria
        const R feq = w * (m.rho + p);
        const R feq0 = w * (R(1) + p);
        const R fo = fr[K];
        fr[K] = fo - omega_f * (fo - feq) + kf * (R(cy(K)) - m.uy) * feq0;
        const R go = gr[K];
        gr[K] = go - omega_g * (go - m.phi * feq0);
    });
}

// Round-to-nearest operations the compiler never fuses or reorders: code
// written with them rounds identically in every kernel that inlines it.
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

// Paired FP32 operations (two lanes in one instruction on sm_100): each lane
// rounds exactly as the scalar operation, so code written with them gives
// the scalar code's bits.
__device__ __forceinline__ float2 splat(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// Regularised BGK (Latt and Chopard, Math. Comput. Simul. 72 (2006)
// 165-168), an option beside the reference's BGK for relaxation times near
// 1/2.  Same equilibria and force term as collide_fast; the non-equilibrium
// part that relaxes is replaced by its projection on the second-order
// Hermite polynomial for f and the first-order one for g:
//   f_i* = feq_i + (1 - 1/tau) 4.5 w_i (c_i c_i : Pi - tr(Pi)/3) + force_i,
//          Pi = sum_i c_i c_i f_i - (rho/3 I + u u)
//   g_i* = geq_i + (1 - 1/tau_c) 3 w_i c_i . j,   j = sum_i c_i g_i - phi u
// (rho/3 I + u u and phi u are the equilibria's own second and first
// moments on D3Q27).  rho, u and phi are unchanged, as in BGK; at tau = 1 the
// two models coincide.  Every operation is an explicit round-to-nearest one,
// so a case gives bitwise the same result in the single-case and the batch
// kernels, in FP64 and FP32.
template <class R>
__device__ __forceinline__ void collide_reg(R (&fr)[Q], R (&gr)[Q], const Moments<R> &m, R omega_f, R omega_g,
                                            R force_fac, R gb, R t0) {
    R sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0, jx = 0, jy = 0, jz = 0;
    Unroll<0, Q>::run([&](auto kk) {
        constexpr int K = decltype(kk)::value;
        constexpr int X = cx(K), Y = cy(K), Z = cz(K);
        const R f = fr[K], g = gr[K];
        if (X != 0) sxx = add_rn(sxx, f);
        if (Y != 0) syy = add_rn(syy, f);
        if (Z != 0) szz = add_rn(szz, f);
        if (X * Y > 0) sxy = add_rn(sxy, f);
        if (X * Y < 0) sxy = sub_rn(sxy, f);
        if (X * Z > 0) sxz = add_rn(sxz, f);
        if (X * Z < 0) sxz = sub_rn(sxz, f);
        if (Y * Z > 0) syz = add_rn(syz, f);
        if (Y * Z < 0) syz = sub_rn(syz, f);
        if (X > 0) jx = add_rn(jx, g);
        if (X < 0) jx = sub_rn(jx, g);
        if (Y > 0) jy = add_rn(jy, g);
        if (Y < 0) jy = sub_rn(jy, g);
        if (Z > 0) jz = add_rn(jz, g);
        if (Z < 0) jz = sub_rn(jz, g);
    });
    const R third = R(1) / R(3);
    const R rho3 = mul_rn(m.rho, third);
    const R pxx = fma_rn(-m.ux, m.ux, sub_rn(sxx, rho3));
    const R pyy = fma_rn(-m.uy, m.uy, sub_rn(syy, rho3));
    const R pzz = fma_rn(-m.uz, m.uz, sub_rn(szz, rho3));
    const R pxy2 = mul_rn(R(2), fma_rn(-m.ux, m.uy, sxy));
    const R pxz2 = mul_rn(R(2), fma_rn(-m.ux, m.uz, sxz));
    const R pyz2 = mul_rn(R(2), fma_rn(-m.uy, m.uz, syz));
    const R tr3 = mul_rn(add_rn(add_rn(pxx, pyy), pzz), third);
    jx = fma_rn(-m.phi, m.ux, jx);
    jy = fma_rn(-m.phi, m.uy, jy);
    jz = fma_rn(-m.phi, m.uz, jz);
    const R keep_f = mul_rn(R(4.5), sub_rn(R(1), omega_f)), keep_g = mul_rn(R(3), sub_rn(R(1), omega_g));
    const R uv = mul_rn(R(3), fma_rn(m.uz, m.uz, fma_rn(m.uy, m.uy, mul_rn(m.ux, m.ux))));
    const R kf = mul_rn(mul_rn(R(3), force_fac), mul_rn(gb, sub_rn(m.phi, t0)));
    Unroll<0, Q>::run([&](auto kk) {
        constexpr int K = decltype(kk)::value;
        constexpr int X = cx(K), Y = cy(K), Z = cz(K);
        constexpr R w = R(wd(K));
        R cu = R(0), cj = R(0), qpi = -tr3;
        if (X > 0) { cu = add_rn(cu, m.ux); cj = add_rn(cj, jx); qpi = add_rn(qpi, pxx); }
        if (X < 0) { cu = sub_rn(cu, m.ux); cj = sub_rn(cj, jx); qpi = add_rn(qpi, pxx); }
        if (Y > 0) { cu = add_rn(cu, m.uy); cj = add_rn(cj, jy); qpi = add_rn(qpi, pyy); }
        if (Y < 0) { cu = sub_rn(cu, m.uy); cj = sub_rn(cj, jy); qpi = add_rn(qpi, pyy); }
        if (Z > 0) { cu = add_rn(cu, m.uz); cj = add_rn(cj, jz); qpi = add_rn(qpi, pzz); }
        if (Z < 0) { cu = sub_rn(cu, m.uz); cj = sub_rn(cj, jz); qpi = add_rn(qpi, pzz); }
        if (X * Y > 0) qpi = add_rn(qpi, pxy2);
        if (X * Y < 0) qpi = sub_rn(qpi, pxy2);
        if (X * Z > 0) qpi = add_rn(qpi, pxz2);
        if (X * Z < 0) qpi = sub_rn(qpi, pxz2);
        if (Y * Z > 0) qpi = add_rn(qpi, pyz2);
        if (Y * Z < 0) qpi = sub_rn(qpi, pyz2);
        const R eu = mul_rn(R(3), cu);
        const R p = add_rn(eu, mul_rn(R(0.5), fma_rn(eu, eu, -uv)));
        const R feq0 = mul_rn(w, add_rn(R(1), p));
        const R fneq = mul_rn(mul_rn(keep_f, w), qpi);
        const R force = mul_rn(mul_rn(kf, sub_rn(R(Y), m.uy)), feq0);
        fr[K] = add_rn(add_rn(mul_rn(w, add_rn(m.rho, p)), fneq), force);
        gr[K] = fma_rn(mul_rn(keep_g, w), cj, mul_rn(m.phi, feq0));
    });
}

// Correctly rounded a / b for a divisor b known in advance, from its correctly
// rounded reciprocal y = RN(1/b): q = RN(a y), r = a - b q (exact by FMA),
// result RN(q + r y).  Markstein's theorem (P. Markstein, IBM J. Res. Dev.
// 34(1), 1990; "IA-64 and Elementary Functions", 2000, Thm 8.10): if y is
// within half an ulp of 1/b and q within one ulp of a/b, the corrected
// quotient is the correctly rounded one.  Valid for finite quotients away
// from the subnormal range (all quotients here); the C ABI's
// lbm_selfcheck_division checks it against the hardware division on the GPU.
__device__ __forceinline__ double div_by(double a, double b, double y) {
    const double q = __dmul_rn(a, y);
    const double r = __fma_rn(-b, q, a);
    return __fma_rn(r, y, q);
}

// The same collision in FP64 as the reference binary computes it: the
// operations of src/collision.cu:19-33 and :65-72 in their order, correctly
// rounded divisions by RT = 1/3, tau and tauc, and a fused multiply-add
// exactly where the reference build has one (u*u sums, eu*eu - uv, f - w*feq,
// g - w*phi*geq; not the force term).  Written with round-to-nearest
// intrinsics, which the compiler never re-fuses, so the results are bitwise
// the reference's.
__device__ __forceinline__ void collide_exact(double (&fr)[Q], double (&gr)[Q], const Moments<double> &m,
                                              double tau, double tauc, double rcp_tau, double rcp_tauc,
                                              double rcp_rt, double force_fac, double gb, double t0) {
    const double RT = 1.0 / 3.0;
    const double uv = div_by(__fma_rn(m.uz, m.uz, __fma_rn(m.ux, m.ux, __dmul_rn(m.uy, m.uy))), RT, rcp_rt);
    const double fy = __dmul_rn(gb, __dsub_rn(m.phi, t0));
    const double kf = __dmul_rn(force_fac, fy);
    // ((1 - 1/(2 tau)) F_y (c_y - u_y)) / RT takes one of three values
    const double fc_m = div_by(__dmul_rn(kf, __dsub_rn(-1.0, m.uy)), RT, rcp_rt);
    const double fc_0 = div_by(__dmul_rn(kf, __dsub_rn(0.0, m.uy)), RT, rcp_rt);
    const double fc_p = div_by(__dmul_rn(kf, __dsub_rn(1.0, m.uy)), RT, rcp_rt);
    Unroll<0, Q>::run([&](auto kk) {
        constexpr int K = decltype(kk)::value;
        constexpr double w = wd(K);
        double cu = 0.0;   // (c.u), summed x, y, z as the reference does; c*u is exact
        if (cx(K) > 0) cu = __dadd_rn(cu, m.ux);
        if (cx(K) < 0) cu = __dsub_rn(cu, m.ux);
        if (cy(K) > 0) cu = __dadd_rn(cu, m.uy);
        if (cy(K) < 0) cu = __dsub_rn(cu, m.uy);
        if (cz(K) > 0) cu = __dadd_rn(cu, m.uz);
        if (cz(K) < 0) cu = __dsub_rn(cu, m.uz);
        const double eu = div_by(cu, RT, rcp_rt);
        const double hq = __dmul_rn(0.5, __fma_rn(eu, eu, -uv));
        const double feq_in = __dadd_rn(__dadd_rn(m.rho, eu), hq);
        const double inner0 = __dadd_rn(__dadd_rn(1.0, eu), hq);
        const double feq0 = __dmul_rn(w, inner0);
        const double fc = cy(K) < 0 ? fc_m : cy(K) > 0 ? fc_p : fc_0;
        const double fo = fr[K];
        double fch = -div_by(__fma_rn(-w, feq_in, fo), tau, rcp_tau);
        fch = __dadd_rn(fch, __dmul_rn(fc, feq0));
        fr[K] = __dadd_rn(fo, fch);
        const double go = gr[K];
        const double gch = -div_by(__fma_rn(-__dmul_rn(w, m.phi), inner0, go), tauc, rcp_tauc);
        gr[K] = __dadd_rn(go, gch);
    });
}

template <class S, int COLL = LBM_COLLISION_BGK, class A>
__device__ __forceinline__ void collide(typename Codec<S>::R (&fr)[Q], typename Codec<S>::R (&gr)[Q],
                                        const Moments<typename Codec<S>::R> &m, const A &a) {
    if constexpr (COLL == LBM_COLLISION_REGULARIZED)
        collide_reg(fr, gr, m, a.omega_f, a.omega_g, a.force_fac, a.gb, a.t0);
    else if constexpr (std::is_same<typename Codec<S>::R, double>::value)
        collide_exact(fr, gr, m, a.tau, a.tauc, a.rcp_tau, a.rcp_tauc, a.rcp_rt, a.force_fac, a.gb, a.t0);
    else
        collide_fast(fr, gr, m, a.omega_f, a.omega_g, a.force_fac, a.gb, a.t0);
}

// Anti-bounce-back value of an outgoing population gv at a plate of
// temperature tw: -gv + 2 w tw (1 + rho), src/streaming.cu:207-227 (the
// product fused into the sum in FP64, as the reference build does).
template <int I, class R>
__device__ __forceinline__ R abb(R gv, R tw, R rho) {
    if constexpr (std::is_same<R, double>::value)
        return __fma_rn(__dmul_rn(__dmul_rn(2.0, wd(I)), tw), __dadd_rn(1.0, rho), -gv);
    else
        return -gv + R(2) * R(wd(I)) * tw * (R(1) + rho);
}

// Write the post-collision populations of node g to where the next step
// reads them.  rho is the node's pre-collision density (for anti-bounce-back).
template <class S, bool SWAPPED, bool PERIODIC, int INTERIOR = kNoneInside, class A>
__device__ __forceinline__ void scatter(const A &a, const Node &g, const typename Codec<S>::R (&fr)[Q],
                                        const typename Codec<S>::R (&gr)[Q], typename Codec<S>::R rho) {
    using C = Codec<S>;
    using R = typename C::R;
    float s0 = 0.f;
    if constexpr (elem_stride<S>() == 2) s0 = shift0(a, g);
    Unroll<0, Q>::run([&](auto ii) {
        constexpr int I = decltype(ii)::value;
        constexpr int DX = cx(I), DY = cy(I), DZ = cz(I);
        R fv = fr[I];
        R gv = gr[I];
        const bool out_y = INTERIOR == kNoneInside && ((DY < 0 && !g.vym) || (DY > 0 && !g.vyp));
        const bool out_z = !PERIODIC && INTERIOR == kNoneInside && ((DZ < 0 && !g.vzm) || (DZ > 0 && !g.vzp));
        if (DY != 0 && out_y && !out_z) gv = abb<I>(gv, DY < 0 ? a.t_hot : a.t_cold, rho);
        if constexpr (elem_stride<S>() == 2) {   // (f, g) pairs: f/w and g/w - T_c at the location, packed
            // the location's T_c is s0 - write_shift_delta (it is s0 at the node itself)
            const float sl = s0 - write_shift_delta<SWAPPED, I, INTERIOR>(a, g);
            const auto v = Pack16<S>::pack(fv * (float)winv(I), fmaf(gv, (float)winv(I), -sl));
            if (SWAPPED && inside_t<INTERIOR, DX, DY, DZ>(g))
                a.st2(I, (int32_t)g.n + disp<DX, DY, DZ>(g)) = v;
            else
                a.st2(opp(I), g.n) = v;
        } else {
            // to the neighbour x + c_I (swapped layout, inside) or back to
            // the node itself, the address chosen by a select (see load_pop)
            const bool in = SWAPPED && inside_t<INTERIOR, DX, DY, DZ>(g);
            const int32_t j = (int32_t)g.n + disp<DX, DY, DZ>(g);
            *(in ? &a.st(0, I, j) : &a.st(0, opp(I), g.n)) = C::template f_out<I>(fv, a.t0);
            *(in ? &a.st(1, I, j) : &a.st(1, opp(I), g.n)) = C::template g_out<I>(gv, a.t0);
        }
    });
}

// Resident 128-thread blocks per SM the register allocation is sized for:
// 3 (<= 168 registers) for FP64, which holds 54 doubles across the
// collision (B200, 256^3: 6.7, 7.4 and 6.6 GLUPS at 2, 3 and 4 blocks, the
// last spilling); 4 (<= 128) for FP32 and 16-bit storage (256^3 FP16S with
// interleaved pairs: 21.7 GLUPS at 4 blocks, 14.2 at 5 and 14.6 at 6, where
// the update spills).
template <class S> struct StepOccupancy {
    static constexpr int value = sizeof(S) == 8 ? 3 : 4;
};
// Threads per block of step_kernel: FP32 steps in blocks of two warps (a
// block holds its SM slot until its slowest warp is done, and two-warp
// blocks waste less of it: B200, 256^3, natural layout -1.8%, closed-box
// swapped -3.6%); FP64 measured 3% slower so and keeps four, as does 16-bit
// storage with the regularised collision (not measured).  The register
// budget is the same: StepOccupancy x 128 threads per SM.
template <class S> constexpr int node_threads() { return std::is_same<S, float>::value ? 64 : 128; }

// The whole update of one node: gather, moments, collision, carried
// temperature, scatter.
// ---- observables of a node's moments --------------------------------------
//
// FP64 sums of
//   0 uy*phi  1 |u|^2  2 ux  3 uy  4 uz  5 phi
//   6..8  phi on the planes iy = 0, 1, 2
//   9..11 phi on the planes iy = LY-1, LY-2, LY-3
//   12 number of nodes with a non-finite moment
// (src/output.cu:199-256 and :24-34 reduce the same fields on the host).
constexpr int kObsTerms = 13;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <class R>
__device__ __forceinline__ void add_obs_terms(double (&acc)[kObsTerms], const Moments<R> &m, int iy, int ly) {
    const double ux = m.ux, uy = m.uy, uz = m.uz, phi = m.phi;
    acc[0] += uy * phi;
    acc[1] += ux * ux + uy * uy + uz * uz;
    acc[2] += ux;
    acc[3] += uy;
    acc[4] += uz;
    acc[5] += phi;
    if (iy == 0) acc[6] += phi;
    if (iy == 1) acc[7] += phi;
    if (iy == 2) acc[8] += phi;
    if (iy == ly - 1) acc[9] += phi;
    if (iy == ly - 2) acc[10] += phi;
    if (iy == ly - 3) acc[11] += phi;
    if (!isfinite(ux) || !isfinite(uy) || !isfinite(uz) || !isfinite(phi) || !isfinite((double)m.rho))
        acc[12] += 1.0;
}

// The warp's sums of the kObsTerms terms of its nodes into row[0 ..
// kObsTerms); all 32 lanes call it, `valid` false for lanes without a node.
// Each lane brings its node's six dense terms (0-5) and plane; the six are
// summed by butterflies; the plane terms are the warp's phi sum when all its
// nodes lie in one plane (rows of a multiple of 32 nodes), else butterflies
// too; the non-finite count is a ballot.  One row per warp and no block
// barrier: a warp that finishes its nodes early leaves at once instead of
// waiting for the block's slowest warp (in a closed box, the warps holding
// an x-wall node take the longer update).
__device__ __forceinline__ void warp_obs_row(const double (&d)[6], int iy, bool valid, bool bad, int ly,
                                             double *__restrict__ row) {
    const int lane = threadIdx.x & 31;
    double w[kObsTerms];
#pragma unroll
    for (int k = 0; k < 6; k++) w[k] = warp_sum(d[k]);
    const int iy0 = __shfl_sync(0xffffffffu, iy, 0);   // lane 0 holds a node if any lane does
    const int planes[6] = {0, 1, 2, ly - 1, ly - 2, ly - 3};
    if (__all_sync(0xffffffffu, !valid || iy == iy0)) {
#pragma unroll
        for (int k = 0; k < 6; k++) w[6 + k] = iy0 == planes[k] ? w[5] : 0.0;
    } else {
#pragma unroll
        for (int k = 0; k < 6; k++) w[6 + k] = warp_sum(valid && iy == planes[k] ? d[5] : 0.0);
    }
    w[12] = (double)__popc(__ballot_sync(0xffffffffu, valid && bad));
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < kObsTerms; k++) row[k] = w[k];
    }
}

// The moments a node update starts from (the observables of the state the
// step reads) and the node's plane.
template <class R> struct NodeOut {
    Moments<R> m;
    int32_t iy;
};

// ---- 16-bit storage: the collision in the stored, normalised variables ----
//
// FP16S / BF16S rows hold (fh_i, gh_i) pairs, fh_i = f_i / w_i and
// gh_i = g_i / w_i - T_c (T_c the conduction profile at the location, see
// shift0), one 32-bit word per population and node.  The
// update below works on those directly (FP32 arithmetic): the moments sum
// them per weight class and weight the four class sums, and the BGK steps in
// normalised form,
//   fh*_i = fh_i - (fh_i - (rho + p_i)) / tau + 3 (1 - 1/(2 tau)) F_y (c_iy - u_y) (1 + p_i)
//   gh*_i = gh_i - (gh_i + t0 - phi (1 + p_i)) / tau_c,
// p_i = 3 c_i.u + 4.5 (c_i.u)^2 - 1.5 u^2, need no weight on load or store.
// Opposite directions share c.u and the quadratic part of p.  The same
// update as collide_fast, with fewer instructions per node.

template <class S, bool SWAPPED, bool PERIODIC, int INTERIOR, class A>
__device__ __forceinline__ void gather_norm(const A &a, const Node &g, float2 (&fg)[Q]) {
    Unroll<0, Q>::run([&](auto kk) {
        constexpr int K = decltype(kk)::value;
        fg[K] = Pack16<S>::unpack(load_pair<S, SWAPPED, K, INTERIOR>(a, g));
        // relative to the node's T_c; on interior rows of a periodic box in
        // the swapped layout the read and write re-referencing is folded
        // into the collision (collide_norm's `fold`), as the moments do not
        // see it (the deltas of each weight class sum to zero); a closed
        // box's x walls keep some populations in the node's own plane, so
        // there each delta is applied
        if constexpr (!(SWAPPED && all_inside<INTERIOR, PERIODIC>())) fg[K].y += read_shift_delta<SWAPPED, K, INTERIOR>(a, g);
    });
}

// fg[i] = (fh_i, gh_i); gh here is g/w - s0 (s0 the node's conduction-profile temperature); t0 is
// the mean temperature of the force term.
__device__ __forceinline__ Moments<float> moments_norm(const float2 (&fg)[Q], float phip, float gbeta, float t0,
                                                       float s0) {
    float2 rt[4] = {};   // (sum fh, sum gh) per weight class, paired
    float x[4] = {0.f, 0.f, 0.f, 0.f}, y[4] = {0.f, 0.f, 0.f, 0.f}, z[4] = {0.f, 0.f, 0.f, 0.f};
    Unroll<0, Q>::run([&](auto kk) {
        constexpr int K = decltype(kk)::value;
        constexpr int C = wclass(K);
        rt[C] = add2(rt[C], fg[K]);
        if (cx(K) > 0) x[C] += fg[K].x;
        if (cx(K) < 0) x[C] -= fg[K].x;
        if (cy(K) > 0) y[C] += fg[K].x;
        if (cy(K) < 0) y[C] -= fg[K].x;
        if (cz(K) > 0) z[C] += fg[K].x;
        if (cz(K) < 0) z[C] -= fg[K].x;
    });
    const float w0 = (float)wd(0), w1 = (float)wd(1), w2 = (float)wd(7), w3 = (float)wd(19);
    Moments<float> m;
    const float2 s = fma2(splat(w3), rt[3], fma2(splat(w2), rt[2], fma2(splat(w1), rt[1], mul2(splat(w0), rt[0]))));
    m.rho = s.x;
    m.ux = fmaf(w3, x[3], fmaf(w2, x[2], w1 * x[1]));
    const float jy = fmaf(w3, y[3], fmaf(w2, y[2], w1 * y[1]));
    m.uz = fmaf(w3, z[3], fmaf(w2, z[2], w1 * z[1]));
    m.phi = s.y + s0;   // sum w_i (gh_i + s0)
    m.uy = jy + 0.5f * (gbeta * (phip - t0));
    return m;
}

// Both relaxations as affine maps of the old value, with per-node
// coefficients (k = kf (c_y - u_y) takes three values, one per c_y):
//   fh* = (1 - om_f) fh + (om_f rho + k) + (om_f + k) p
//   gh* = (1 - om_g) gh + om_g (phi - s0) + om_g phi p
// and p_I, p_J = (q +/- 2 eu) / 2 with q = eu^2 - 3 u^2 for a pair of
// opposite directions: two multiply-adds per population and three per pair.
// (gh = g/w - s0; t0 enters only the buoyancy force.)  fold: the plane
// spacing of the conduction profile when gh holds raw stored values that
// were read from, and go to, the planes y - c_y and y + c_y (interior rows
// of a periodic box, swapped layout): ag (v + c_y fold) + ... + c_y fold = ag v + ... +
// (ag + 1) c_y fold, one more coefficient per c_y; else 0.
__device__ __forceinline__ void collide_norm(float2 (&fg)[Q], const Moments<float> &m, float om_f, float om_g,
                                             float force_fac, float gbeta, float t0, float s0, float fold) {
    const float ux3 = 3.f * m.ux, uy3 = 3.f * m.uy, uz3 = 3.f * m.uz;
    const float uv = 3.f * (m.ux * m.ux + m.uy * m.uy + m.uz * m.uz);
    const float kf = 3.f * force_fac * (gbeta * (m.phi - t0));
    const float k_m = kf * (-1.f - m.uy), k_0 = kf * (-m.uy), k_p = kf * (1.f - m.uy);
    const float af = 1.f - om_f, orho = om_f * m.rho;
    const float c0[3] = {orho + k_m, orho + k_0, orho + k_p};    // indexed by c_y + 1
    const float c1[3] = {om_f + k_m, om_f + k_0, om_f + k_p};
    const float ag = 1.f - om_g, d1 = om_g * m.phi, d0 = om_g * (m.phi - s0);
    const float df = (ag + 1.f) * fold;
    const float d0c[3] = {d0 - df, d0, d0 + df};                    // indexed by c_y + 1
    // (fh, gh) <- (af fh + c1 p + c0, ag gh + d1 p + d0c): both at once
    const float2 a2 = make_float2(af, ag);
    auto relax = [&](float2 &v, float p, int cy1) {
        v = fma2(a2, v, fma2(make_float2(c1[cy1], d1), splat(p), make_float2(c0[cy1], d0c[cy1])));
    };
    relax(fg[0], -0.5f * uv, 1);
    Unroll<1, Q>::run([&](auto ii) {
        constexpr int I = decltype(ii)::value;
        constexpr int J = opp(I);
        if constexpr (I < J) {
            float eu = 0.f;
            if (cx(I) > 0) eu += ux3;
            if (cx(I) < 0) eu -= ux3;
            if (cy(I) > 0) eu += uy3;
            if (cy(I) < 0) eu -= uy3;
            if (cz(I) > 0) eu += uz3;
            if (cz(I) < 0) eu -= uz3;
            const float q = fmaf(eu, eu, -uv);
            relax(fg[I], fmaf(0.5f, q, eu), cy(I) + 1);
            relax(fg[J], fmaf(0.5f, q, -eu), cy(J) + 1);
        }
    });
}

// scatter() for the normalised variables: anti-bounce-back in normalised
// form, gh' = 2 T_wall (1 + rho) - gh* - 2 t0, no weights on store, and one
// 32-bit store of the packed (f, g) pair per population.
template <class S, bool SWAPPED, bool PERIODIC, int INTERIOR, class A>
__device__ __forceinline__ void scatter_norm(const A &a, const Node &g, const float2 (&fg)[Q], float rho, float s0) {
    Unroll<0, Q>::run([&](auto ii) {
        constexpr int I = decltype(ii)::value;
        constexpr int DX = cx(I), DY = cy(I), DZ = cz(I);
        float gv = fg[I].y;
        const bool out_y = INTERIOR == kNoneInside && ((DY < 0 && !g.vym) || (DY > 0 && !g.vyp));
        const bool out_z = !PERIODIC && INTERIOR == kNoneInside && ((DZ < 0 && !g.vzm) || (DZ > 0 && !g.vzp));
        if (DY != 0 && out_y && !out_z) gv = 2.f * (DY < 0 ? a.t_hot : a.t_cold) * (1.f + rho) - gv - 2.f * s0;
        // relative to T_c at the location written (folded into the
        // collision on interior rows of a periodic box's swapped layout)
        if constexpr (!(SWAPPED && all_inside<INTERIOR, PERIODIC>())) gv += write_shift_delta<SWAPPED, I, INTERIOR>(a, g);
        const typename Pack16<S>::T v = Pack16<S>::pack(fg[I].x, gv);
        if (SWAPPED && inside_t<INTERIOR, DX, DY, DZ>(g))
            a.st2(I, (int32_t)g.n + disp<DX, DY, DZ>(g)) = v;
        else
            a.st2(opp(I), g.n) = v;
    });
}

template <class S, bool SWAPPED, bool PERIODIC, class A>
__device__ __forceinline__ NodeOut<float> update_node_norm(const A &a, uint32_t n) {
    const Node g = make_node<PERIODIC>(a, n);
    float2 fg[Q];
    const int path = node_path<PERIODIC, SWAPPED>(g);
    if (path == kRowInside)
        gather_norm<S, SWAPPED, PERIODIC, kRowInside>(a, g, fg);
    else if (SWAPPED && !PERIODIC && path == kAllInside)
        gather_norm<S, SWAPPED, PERIODIC, PERIODIC ? kRowInside : kAllInside>(a, g, fg);
    else
        gather_norm<S, SWAPPED, PERIODIC, kNoneInside>(a, g, fg);
    const float s0 = shift0(a, g);
    Moments<float> m = moments_norm(fg, a.phip[n], a.gb, a.t0, s0);
    if (a.use_phi_fix) m.phi = a.phi_fix;
    const bool fold = SWAPPED && (path == kAllInside || (PERIODIC && path == kRowInside));
    collide_norm(fg, m, a.omega_f, a.omega_g, a.force_fac, a.gb, a.t0, s0, fold ? (float)a.t_dy : 0.f);
    a.phip[n] = m.phi;
    if (path == kRowInside)
        scatter_norm<S, SWAPPED, PERIODIC, kRowInside>(a, g, fg, m.rho, s0);
    else if (SWAPPED && !PERIODIC && path == kAllInside)
        scatter_norm<S, SWAPPED, PERIODIC, PERIODIC ? kRowInside : kAllInside>(a, g, fg, m.rho, s0);
    else
        scatter_norm<S, SWAPPED, PERIODIC, kNoneInside>(a, g, fg, m.rho, s0);
    return {m, g.iy};
}

// ---- 16-bit storage, BGK: one node's update split over two warps ----------
//
// The one-node update is latency-bound: a warp has its loads outstanding
// only before its long update.  Here two warps share 32 nodes: half 0 loads,
// relaxes and stores the rest population and the opposite pairs (1,3) (2,4)
// (5,6) (7,9) (19,25) (20,26), half 1 the other seven pairs.  Each sums the
// moments of its populations; the two exchange the five partial sums through
// shared memory under a two-warp barrier and add them (addition commutes
// exactly, so both hold the same moments).  A thread holds 13-14 pairs
// instead of 27, so twice the warps are resident, and each warp's update
// between its load phases is half as long.  The halves are chosen by warp
// index, so no warp diverges.

__host__ __device__ constexpr int pair_rep(int k) { return k < opp(k) ? k : opp(k); }
// the half of the split update that owns population k
__host__ __device__ constexpr int half_of(int k) {
    return (k == 0 || pair_rep(k) == 1 || pair_rep(k) == 2 || pair_rep(k) == 5 || pair_rep(k) == 7 ||
            pair_rep(k) == 19 || pair_rep(k) == 20)
               ? 0
               : 1;
}

// Every population in exactly one half, opposite pairs together (the
// in-place update of a pair's two locations stays within one warp), 13 and
// 14 populations.
__host__ __device__ constexpr bool split_halves_ok() {
    int n0 = 0;
    for (int k = 0; k < Q; k++) {
        if (half_of(k) != 0 && half_of(k) != 1) return false;
        if (half_of(k) != half_of(opp(k))) return false;
        n0 += half_of(k) == 0;
    }
    return n0 == 13 && half_of(0) == 0;
}
static_assert(split_halves_ok(), "split update: bad population halves");

template <int H, class S, bool SWAPPED, bool PERIODIC, int INTERIOR, class A>
__device__ __forceinline__ void gather_half(const A &a, const Node &g, float2 (&fg)[Q]) {
    Unroll<0, Q>::run([&](auto kk) {
        constexpr int K = decltype(kk)::value;
        if constexpr (half_of(K) == H) {
            fg[K] = Pack16<S>::unpack(load_pair<S, SWAPPED, K, INTERIOR>(a, g));
            if constexpr (!(SWAPPED && all_inside<INTERIOR, PERIODIC>())) fg[K].y += read_shift_delta<SWAPPED, K, INTERIOR>(a, g);
        }
    });
}

// The half's share of rho, j_x, j_y, j_z and sum w_i gh_i (as moments_norm);
// the (rho, phi) class sums and their weighting as paired FP32 operations
template <int H> __device__ __forceinline__ void partial_moments(const float2 (&fg)[Q], float (&p)[5]) {
    float2 rt[4] = {};   // (sum fh, sum gh) per weight class
    float x[4] = {0.f, 0.f, 0.f, 0.f}, y[4] = {0.f, 0.f, 0.f, 0.f}, z[4] = {0.f, 0.f, 0.f, 0.f};
    Unroll<0, Q>::run([&](auto kk) {
        constexpr int K = decltype(kk)::value;
        if constexpr (half_of(K) == H) {
            constexpr int C = wclass(K);
            rt[C] = add2(rt[C], fg[K]);
            if (cx(K) > 0) x[C] += fg[K].x;
            if (cx(K) < 0) x[C] -= fg[K].x;
            if (cy(K) > 0) y[C] += fg[K].x;
            if (cy(K) < 0) y[C] -= fg[K].x;
            if (cz(K) > 0) z[C] += fg[K].x;
            if (cz(K) < 0) z[C] -= fg[K].x;
        }
    });
    const float w0 = (float)wd(0), w1 = (float)wd(1), w2 = (float)wd(7), w3 = (float)wd(19);
    const float2 s = fma2(splat(w3), rt[3], fma2(splat(w2), rt[2], fma2(splat(w1), rt[1], mul2(splat(w0), rt[0]))));
    p[0] = s.x;
    p[1] = fmaf(w3, x[3], fmaf(w2, x[2], w1 * x[1]));
    p[2] = fmaf(w3, y[3], fmaf(w2, y[2], w1 * y[1]));
    p[3] = fmaf(w3, z[3], fmaf(w2, z[2], w1 * z[1]));
    p[4] = s.y;
}

// collide_norm for the half's populations
template <int H>
__device__ __forceinline__ void collide_half(float2 (&fg)[Q], const Moments<float> &m, float om_f, float om_g,
                                             float force_fac, float gbeta, float t0, float s0, float fold) {
    const float ux3 = 3.f * m.ux, uy3 = 3.f * m.uy, uz3 = 3.f * m.uz;
    const float uv = 3.f * (m.ux * m.ux + m.uy * m.uy + m.uz * m.uz);
    const float kf = 3.f * force_fac * (gbeta * (m.phi - t0));
    const float k_m = kf * (-1.f - m.uy), k_0 = kf * (-m.uy), k_p = kf * (1.f - m.uy);
    const float af = 1.f - om_f, orho = om_f * m.rho;
    const float c0[3] = {orho + k_m, orho + k_0, orho + k_p};
    const float c1[3] = {om_f + k_m, om_f + k_0, om_f + k_p};
    const float ag = 1.f - om_g, d1 = om_g * m.phi, d0 = om_g * (m.phi - s0);
    const float df = (ag + 1.f) * fold;
    const float d0c[3] = {d0 - df, d0, d0 + df};
    // (fh, gh) <- (af fh + c1 p + c0, ag gh + d1 p + d0c): both at once
    const float2 a2 = make_float2(af, ag);
    auto relax = [&](float2 &v, float p, int cy1) {
        v = fma2(a2, v, fma2(make_float2(c1[cy1], d1), splat(p), make_float2(c0[cy1], d0c[cy1])));
    };
    if constexpr (H == 0) relax(fg[0], -0.5f * uv, 1);
    Unroll<1, Q>::run([&](auto ii) {
        constexpr int I = decltype(ii)::value;
        constexpr int J = opp(I);
        if constexpr (I < J && half_of(I) == H) {
            float eu = 0.f;
            if (cx(I) > 0) eu += ux3;
            if (cx(I) < 0) eu -= ux3;
            if (cy(I) > 0) eu += uy3;
            if (cy(I) < 0) eu -= uy3;
            if (cz(I) > 0) eu += uz3;
            if (cz(I) < 0) eu -= uz3;
            const float q = fmaf(eu, eu, -uv);
            relax(fg[I], fmaf(0.5f, q, eu), cy(I) + 1);
            relax(fg[J], fmaf(0.5f, q, -eu), cy(J) + 1);
        }
    });
}

// scatter_norm for the half's populations
template <int H, class S, bool SWAPPED, bool PERIODIC, int INTERIOR, class A>
__device__ __forceinline__ void scatter_half(const A &a, const Node &g, const float2 (&fg)[Q], float rho, float s0) {
    Unroll<0, Q>::run([&](auto ii) {
        constexpr int I = decltype(ii)::value;
        if constexpr (half_of(I) == H) {
            constexpr int DX = cx(I), DY = cy(I), DZ = cz(I);
            float gv = fg[I].y;
            const bool out_y = INTERIOR == kNoneInside && ((DY < 0 && !g.vym) || (DY > 0 && !g.vyp));
            const bool out_z = !PERIODIC && INTERIOR == kNoneInside && ((DZ < 0 && !g.vzm) || (DZ > 0 && !g.vzp));
            if (DY != 0 && out_y && !out_z) gv = 2.f * (DY < 0 ? a.t_hot : a.t_cold) * (1.f + rho) - gv - 2.f * s0;
            if constexpr (!(SWAPPED && all_inside<INTERIOR, PERIODIC>())) gv += write_shift_delta<SWAPPED, I, INTERIOR>(a, g);
            const typename Pack16<S>::T v = Pack16<S>::pack(fg[I].x, gv);
            if (SWAPPED && inside_t<INTERIOR, DX, DY, DZ>(g))
                a.st2(I, (int32_t)g.n + disp<DX, DY, DZ>(g)) = v;
            else
                a.st2(opp(I), g.n) = v;
        }
    });
}

// Waits until both warps of warp pair `pair` (0 or 1; 64 threads) arrive,
// on named barrier 1 + pair (immediate ids, so the block reserves three
// barriers); the non-aligned form, so lanes need not be converged.
__device__ __forceinline__ void pair_barrier(int pair) {
    if (pair == 0)
        asm volatile("barrier.sync 1, 64;\n" ::: "memory");
    else
        asm volatile("barrier.sync 2, 64;\n" ::: "memory");
}

// Receives a node's moments as soon as a node update (update_node,
// split_update) has formed them, before the collision and the scatter.
struct NoMomentSink {
    template <class R> __device__ __forceinline__ void operator()(const Moments<R> &) const {}
};

// Parks a node's moments (ux, uy, uz, phi, rho) in shared memory, STRIDE
// elements apart, so a kernel that reduces them after the update does not
// hold them in registers through the collision and the scatter (in the FP64
// kernel, at its register limit, that cost a third of the swapped-layout
// step in a closed box).  T holds the moments exactly (T = double, or float
// for float moments).  Volatile, so the compiler does not forward the stores
// to the loads.
template <class T, int STRIDE> struct SharedMomentSink {
    volatile T *p;
    template <class R> __device__ __forceinline__ void operator()(const Moments<R> &m) const {
        static_assert(sizeof(T) >= sizeof(R), "the parked moments must hold the update's exactly");
        p[0] = (T)m.ux;
        p[STRIDE] = (T)m.uy;
        p[2 * STRIDE] = (T)m.uz;
        p[3 * STRIDE] = (T)m.phi;
        p[4 * STRIDE] = (T)m.rho;
    }
};

// Half H of the update of node n (valid: n is a node); xch is the warp
// pair's exchange area [half][moment][lane].  Both warps of a pair call it
// once, valid or not, and pass the barrier once.
// Returns the node's moments (those of the state it read) and plane; they
// are meaningful for valid nodes only.
template <int H, class S, bool SWAPPED, bool PERIODIC, class A, class Sink = NoMomentSink>
__device__ __forceinline__ NodeOut<float> split_update(const A &a, uint32_t n, bool valid, float (&xch)[2][5][32],
                                                       int lane, int pair, const Sink &sink = Sink()) {
    float2 fg[Q];
    float p[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    Node g{};
    int path = kNoneInside;
    float phip = 0.f;
    if (valid) {
        phip = a.phip[n];   // before the barrier: half 0 overwrites it after
        g = make_node<PERIODIC>(a, n);
        path = node_path<PERIODIC, SWAPPED>(g);
        if (path == kRowInside)
            gather_half<H, S, SWAPPED, PERIODIC, kRowInside>(a, g, fg);
        else if (SWAPPED && !PERIODIC && path == kAllInside)
            gather_half<H, S, SWAPPED, PERIODIC, PERIODIC ? kRowInside : kAllInside>(a, g, fg);
        else
            gather_half<H, S, SWAPPED, PERIODIC, kNoneInside>(a, g, fg);
        partial_moments<H>(fg, p);
    }
#pragma unroll
    for (int i = 0; i < 5; i++) xch[H][i][lane] = p[i];
    pair_barrier(pair);
    if (!valid) return {};
    float tot[5];
#pragma unroll
    for (int i = 0; i < 5; i++) tot[i] = p[i] + xch[1 - H][i][lane];
    const float s0 = shift0(a, g);
    Moments<float> m;
    m.rho = tot[0];
    m.ux = tot[1];
    m.uy = __fadd_rn(tot[2], __fmul_rn(0.5f, __fmul_rn(a.gb, __fsub_rn(phip, a.t0))));   // as split_moments
    m.uz = tot[3];
    m.phi = tot[4] + s0;
    if (a.use_phi_fix) m.phi = a.phi_fix;
    sink(m);
    const bool fold = SWAPPED && (path == kAllInside || (PERIODIC && path == kRowInside));
    collide_half<H>(fg, m, a.omega_f, a.omega_g, a.force_fac, a.gb, a.t0, s0, fold ? (float)a.t_dy : 0.f);
    if (H == 0) a.phip[n] = m.phi;
    if (path == kRowInside)
        scatter_half<H, S, SWAPPED, PERIODIC, kRowInside>(a, g, fg, m.rho, s0);
    else if (SWAPPED && !PERIODIC && path == kAllInside)
        scatter_half<H, S, SWAPPED, PERIODIC, PERIODIC ? kRowInside : kAllInside>(a, g, fg, m.rho, s0);
    else
        scatter_half<H, S, SWAPPED, PERIODIC, kNoneInside>(a, g, fg, m.rho, s0);
    return {m, g.iy};
}

// The moments of node g exactly as step16_split_kernel's two halves form
// them (the same loads on the same path, the same partial sums, added in the
// same order), so observables reduced from them match those the kernel
// reduces when it steps (the observables of its OBS variant).
template <class S, bool SWAPPED, bool PERIODIC, class A>
__device__ __forceinline__ Moments<float> split_moments(const A &a, const Node &g) {
    float2 fg[Q];
    float p0[5], p1[5];
    const int path = node_path<PERIODIC, SWAPPED>(g);
    if (path == kRowInside) {
        gather_half<0, S, SWAPPED, PERIODIC, kRowInside>(a, g, fg);
        gather_half<1, S, SWAPPED, PERIODIC, kRowInside>(a, g, fg);
    } else if (SWAPPED && !PERIODIC && path == kAllInside) {
        gather_half<0, S, SWAPPED, PERIODIC, PERIODIC ? kRowInside : kAllInside>(a, g, fg);
        gather_half<1, S, SWAPPED, PERIODIC, PERIODIC ? kRowInside : kAllInside>(a, g, fg);
    } else {
        gather_half<0, S, SWAPPED, PERIODIC, kNoneInside>(a, g, fg);
        gather_half<1, S, SWAPPED, PERIODIC, kNoneInside>(a, g, fg);
    }
    partial_moments<0>(fg, p0);
    partial_moments<1>(fg, p1);
    Moments<float> m;
    m.rho = p0[0] + p1[0];
    m.ux = p0[1] + p1[1];
    m.uy = __fadd_rn(p0[2] + p1[2], __fmul_rn(0.5f, __fmul_rn(a.gb, __fsub_rn((float)a.phip[g.n], a.t0))));
    m.uz = p0[3] + p1[3];
    m.phi = (p0[4] + p1[4]) + shift0(a, g);
    if (a.use_phi_fix) m.phi = a.phi_fix;
    return m;
}

template <class S, bool SWAPPED, bool PERIODIC, int COLL = LBM_COLLISION_BGK, class A, class Sink = NoMomentSink>
__device__ __forceinline__ NodeOut<typename Codec<S>::R> update_node(const A &a, uint32_t n,
                                                                     const Sink &sink = Sink()) {
    if constexpr (sizeof(S) == 2 && COLL == LBM_COLLISION_BGK) {
        const auto o = update_node_norm<S, SWAPPED, PERIODIC>(a, n);
        sink(o.m);
        return o;
    }
    using R = typename Codec<S>::R;
    const Node g = make_node<PERIODIC>(a, n);
    R fr[Q], gr[Q];
    // Rows away from the plates (and, in a closed box, from the z walls)
    // need no y or z boundary tests, a closed box's warps with no x-wall
    // node none at all, and in the swapped layout (the one whose accesses
    // depend on them) the warps at one x wall test that side only; the
    // path is uniform over a warp whenever LX is a multiple of 32.
    constexpr bool kOneWall = SWAPPED && !PERIODIC;
    const int path = kOneWall ? node_path_x<PERIODIC>(g) : node_path<PERIODIC, SWAPPED>(g);
    if (!kOneWall && path == kRowInside)
        gather<S, SWAPPED, kRowInside>(a, g, fr, gr);
    else if (SWAPPED && !PERIODIC && path == kAllInside)
        gather<S, SWAPPED, PERIODIC ? kRowInside : kAllInside>(a, g, fr, gr);
    else if (kOneWall && path == kRowLoWall)
        gather<S, SWAPPED, kOneWall ? kRowLoWall : kRowInside>(a, g, fr, gr);
    else if (kOneWall && path == kRowHiWall)
        gather<S, SWAPPED, kOneWall ? kRowHiWall : kRowInside>(a, g, fr, gr);
    else
        gather<S, SWAPPED, kNoneInside>(a, g, fr, gr);
    const Moments<R> m = node_moments<S>(a, fr, gr, n);
    sink(m);
    collide<S, COLL>(fr, gr, m, a);
    a.phip[n] = (typename Codec<S>::P)m.phi;
    if (!kOneWall && path == kRowInside)
        scatter<S, SWAPPED, PERIODIC, kRowInside>(a, g, fr, gr, m.rho);
    else if (SWAPPED && !PERIODIC && path == kAllInside)
        scatter<S, SWAPPED, PERIODIC, PERIODIC ? kRowInside : kAllInside>(a, g, fr, gr, m.rho);
    else if (kOneWall && path == kRowLoWall)
        scatter<S, SWAPPED, PERIODIC, kOneWall ? kRowLoWall : kRowInside>(a, g, fr, gr, m.rho);
    else if (kOneWall && path == kRowHiWall)
        scatter<S, SWAPPED, PERIODIC, kOneWall ? kRowHiWall : kRowInside>(a, g, fr, gr, m.rho);
    else
        scatter<S, SWAPPED, PERIODIC, kNoneInside>(a, g, fr, gr, m.rho);
    return {m, g.iy};
}

// One time step.  With OBS, the kernel also reduces the observables of the
// state it reads — the moments every node update computes anyway — into one
// row of kObsTerms FP64 sums per warp (a.obs_rows, row W b + w for warp w of
// block b, W = node_threads / 32), at no extra read of the populations.
template <class S, bool SWAPPED, bool PERIODIC, int COLL, bool OBS = false>
__global__ void __launch_bounds__(128, StepOccupancy<S>::value) step_kernel(const StepArgs<S> a) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if constexpr (!OBS) {
        if (n >= a.nodes) return;
        update_node<S, SWAPPED, PERIODIC, COLL>(a, n);
    } else {
        __shared__ double parked[5][128];   // ux, uy, uz, phi, rho per thread
        // the terms of add_obs_terms: uy*phi, |u|^2, ux, uy, uz, phi
        double d[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        int iy = 0;
        bool bad = false;
        const bool valid = n < a.nodes;
        if (valid) {
            volatile double *mine = &parked[0][threadIdx.x];
            iy = update_node<S, SWAPPED, PERIODIC, COLL>(a, n, SharedMomentSink<double, 128>{mine}).iy;
            const double ux = mine[0], uy = mine[128], uz = mine[256], phi = mine[384], rho = mine[512];
            d[0] = uy * phi;
            d[1] = ux * ux + uy * uy + uz * uz;
            d[2] = ux;
            d[3] = uy;
            d[4] = uz;
            d[5] = phi;
            bad = !isfinite(ux) || !isfinite(uy) || !isfinite(uz) || !isfinite(phi) || !isfinite(rho);
        }
        const size_t warp_row = (size_t)blockIdx.x * (node_threads<S>() / 32) + (threadIdx.x >> 5);
        warp_obs_row(d, iy, valid, bad, a.ly, a.obs_rows + warp_row * kObsTerms);
    }
}

// 16-bit storage, BGK: block b updates nodes [64 b, 64 b + 64); warps 2p
// and 2p + 1 share nodes 64 b + 32 p + lane (split_update).  8 blocks of
// 128 threads per SM (64 registers, no spills): B200, 256^3, 24.6 GLUPS
// FP16S and 23.7 BF16S, against 20.7 and 21.3 for the one-thread-per-node
// kernel at 4 blocks.
//
// With OBS, the kernel also reduces the observables of the state it reads
// into one row of kObsTerms FP64 sums per warp pair (a.obs_rows, row 2 b + p
// for pair p of block b): half 0 parks its 32 nodes' moments in shared memory
// when it forms them and reduces them after its update; half 1 leaves when
// its update is done.  (Splitting the reduction between the halves measured
// slower: both then form the terms.)
constexpr int kSplitBlocks = 8;
template <class S, bool SWAPPED, bool PERIODIC, bool OBS = false>
__global__ void __launch_bounds__(128, kSplitBlocks) step16_split_kernel(const StepArgs<S> a) {
    __shared__ float xch[2][2][5][32];   // [warp pair][half][moment][lane]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pair = warp >> 1;
    const uint32_t n = blockIdx.x * 64u + (uint32_t)(pair * 32 + lane);
    const bool valid = n < a.nodes;
    if constexpr (!OBS) {
        if ((warp & 1) == 0)
            split_update<0, S, SWAPPED, PERIODIC>(a, n, valid, xch[pair], lane, pair);
        else
            split_update<1, S, SWAPPED, PERIODIC>(a, n, valid, xch[pair], lane, pair);
    } else {
        __shared__ float parked[2][5][32];   // [warp pair][ux, uy, uz, phi, rho][lane]
        if (warp & 1) {
            split_update<1, S, SWAPPED, PERIODIC>(a, n, valid, xch[pair], lane, pair);
            return;
        }
        volatile float *mine = &parked[pair][0][lane];
        const int iy = split_update<0, S, SWAPPED, PERIODIC>(a, n, valid, xch[pair], lane, pair,
                                                             SharedMomentSink<float, 32>{mine}).iy;
        double d[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        bool bad = false;
        if (valid) {
            const double ux = mine[0], uy = mine[32], uz = mine[64], phi = mine[96], rho = mine[128];
            d[0] = uy * phi;
            d[1] = ux * ux + uy * uy + uz * uz;
            d[2] = ux;
            d[3] = uy;
            d[4] = uz;
            d[5] = phi;
            bad = !isfinite(ux) || !isfinite(uy) || !isfinite(uz) || !isfinite(phi) || !isfinite(rho);
        }
        warp_obs_row(d, iy, valid, bad, a.ly, a.obs_rows + ((size_t)blockIdx.x * 2 + pair) * kObsTerms);
    }
}

}  // namespace lbm
