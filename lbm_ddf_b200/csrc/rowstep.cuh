// rowstep.cuh — the fused step with whole x-rows staged through shared memory
// by bulk asynchronous copies (TMA, untiled, each into its own CTA).
//
// Same update as step_kernel (step.cuh), same AA layouts, same results; only
// the data movement differs.  One block owns one x-row of the grid (LX
// nodes, one per thread).  For each of the 54 populations it needs, one
// thread issues a single bulk copy of a whole row of LX values into shared
// memory, so the loads in flight no longer depend on how many registers the
// threads can spare, and every access to HBM is a contiguous, aligned row.
//
//   natural layout: population k of the row is row k of the row itself;
//   swapped layout: population k comes from slot opp(k) of row
//     (y - c_ky, z - c_kz), shifted by c_kx along x, or, when that row is
//     beyond a plate, from slot k of the row itself (bounce-back); the x
//     shift (periodic) is applied when reading shared memory.
//
// Outputs are assembled in shared memory as whole rows and written with bulk
// stores: in the natural layout row I goes to slot opp(I) of the row itself;
// in the swapped layout to slot I of row (y + c_Iy, z + c_Iz), shifted by
// c_Ix, or, beyond a plate, to slot opp(I) of the row itself with the
// anti-bounce-back transform for g.  With periodic sides every (slot, row)
// of the grid is written by exactly one block, so whole-row stores are
// race-free; closed boxes (x walls) use step_kernel instead.
//
// Eligibility (checked on the host): periodic sides, 32 <= LX <= 256 and
// LX * sizeof(S) a multiple of 16 bytes.
#pragma once

#include "bulk.cuh"
#include "step.cuh"

namespace lbm {

constexpr uint32_t kRowMaxPolls = 1u << 22;          // bounds on each shared-memory barrier wait:
constexpr uint64_t kRowMaxNs = 1000000000ull;         // polls and 1 s of the global timer

template <class S> struct RowOccupancy { static constexpr int value = sizeof(S) == 8 ? 1 : 2; };

// Shared-memory rows are PITCH elements apart (PITCH >= LX, one of 64, 128,
// 256), a compile-time constant, so every shared access is a fixed offset
// from one of three per-thread bases (x - 1, x, x + 1 with periodic wrap).
template <class S> __host__ __device__ constexpr size_t row_smem_bytes(int pitch) {
    return (size_t)2 * Q * (size_t)pitch * sizeof(S) + 16;
}

template <class S, bool SWAPPED, int PITCH>
// extra_tx: bytes announced on the barrier beyond those the copies bring,
// 0 except in the test of the bounded wait (lbm_debug_row_wait_extra_bytes):
// the copies then all land but the phase never completes, and the wait runs
// out as it would if a copy never arrived.
__global__ void __launch_bounds__(256, RowOccupancy<S>::value) row_step_kernel(const StepArgs<S> a, int *err,
                                                                             uint32_t extra_tx) {
    using C = Codec<S>;
    using R = typename C::R;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int lx = a.lx;
    S *sm = reinterpret_cast<S *>(smem_raw);                      // rows 0..26 f, 27..53 g
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + (size_t)2 * Q * PITCH * sizeof(S));
    const uint32_t row = blockIdx.x;                               // z*LY + y
    const uint32_t z = a.div_ly.div(row);
    const int y = (int)(row - z * (uint32_t)a.ly);
    const uint32_t bytes = (uint32_t)lx * sizeof(S);
    const int x = threadIdx.x;

    // source / destination row of a displacement (dy, dz), z periodic
    auto row_of = [&](int dy, int dz) -> uint32_t {
        int zz = (int)z + dz;
        zz = zz < 0 ? zz + a.lz : zz >= a.lz ? zz - a.lz : zz;
        return (uint32_t)zz * (uint32_t)a.ly + (uint32_t)(y + dy);
    };

    if (x == 0) {
        bulk::mbar_init(bar, 1);
        bulk::fence_mbar_init();
    }
    __syncthreads();
    if (x == 0) {
        bulk::mbar_expect_tx(bar, 2u * Q * bytes + extra_tx);
        Unroll<0, Q>::run([&](auto kk) {
            constexpr int K = decltype(kk)::value;
            const S *fsrc;
            const S *gsrc;
            if (!SWAPPED) {
                fsrc = a.fl[K] + (size_t)row * lx;
                gsrc = a.gl[K] + (size_t)row * lx;
            } else {
                const int sy = y - cy(K);
                if (sy >= 0 && sy < a.ly) {
                    const uint32_t srow = row_of(-cy(K), -cz(K));
                    fsrc = a.fl[opp(K)] + (size_t)srow * lx;
                    gsrc = a.gl[opp(K)] + (size_t)srow * lx;
                } else {
                    fsrc = a.fl[K] + (size_t)row * lx;
                    gsrc = a.gl[K] + (size_t)row * lx;
                }
            }
            bulk::load_row(sm + K * PITCH, fsrc, bytes, bar);
            bulk::load_row(sm + (Q + K) * PITCH, gsrc, bytes, bar);
        });
    }
    const uint32_t n = row * (uint32_t)lx + (uint32_t)x;
    const R pp = (R)a.phip[n];
    const bool ok = bulk::mbar_wait(bar, 0, kRowMaxPolls, kRowMaxNs);
    if (!ok) {
        atomicOr(err, 1);
        // copies still on their way land in this block's shared memory: give
        // them one more bounded wait before the block leaves it
        (void)bulk::mbar_wait(bar, 0, kRowMaxPolls, kRowMaxNs);
    }
    if (!__syncthreads_and(ok)) return;   // the whole block leaves together

    const int xm = x == 0 ? lx - 1 : x - 1;
    const int xp = x == lx - 1 ? 0 : x + 1;
    const S *s0 = sm + x, *sm1 = sm + xm, *sp1 = sm + xp;
    const bool y_lo = y > 0, y_hi = y < a.ly - 1;    // rows y-1 / y+1 exist
    R fr[Q], gr[Q];
    Unroll<0, Q>::run([&](auto kk) {
        constexpr int K = decltype(kk)::value;
        const S *b = s0;
        if (SWAPPED) {
            const bool in = cy(K) > 0 ? y_lo : cy(K) < 0 ? y_hi : true;
            if (in) b = cx(K) > 0 ? sm1 : cx(K) < 0 ? sp1 : s0;
        }
        fr[K] = C::template f_in<K>(b[K * PITCH], a.t0);
        gr[K] = C::template g_in<K>(b[(Q + K) * PITCH], a.t0);
    });
    Moments<R> m = moments(fr, gr, pp, a.gb, a.t0);
    if (a.use_phi_fix) m.phi = a.phi_fix;
    collide<S>(fr, gr, m, a);
    a.phip[n] = (typename C::P)m.phi;

    if (SWAPPED) __syncthreads();   // every thread has read its inputs before rows are overwritten
    Unroll<0, Q>::run([&](auto ii) {
        constexpr int I = decltype(ii)::value;
        const bool out_y = cy(I) < 0 ? !y_lo : cy(I) > 0 ? !y_hi : false;
        R gv = gr[I];
        if (cy(I) != 0 && out_y) gv = abb<I>(gv, cy(I) < 0 ? a.t_hot : a.t_cold, m.rho);
        S *b = sm + x;
        if (SWAPPED && !out_y) b = cx(I) > 0 ? sm + xp : cx(I) < 0 ? sm + xm : sm + x;
        b[I * PITCH] = C::template f_out<I>(fr[I], a.t0);
        b[(Q + I) * PITCH] = C::template g_out<I>(gv, a.t0);
    });
    bulk::fence_proxy_async();
    __syncthreads();
    if (x == 0) {
        Unroll<0, Q>::run([&](auto ii) {
            constexpr int I = decltype(ii)::value;
            S *fdst;
            S *gdst;
            const int dy = y + cy(I);
            if (SWAPPED && dy >= 0 && dy < a.ly) {
                const uint32_t drow = row_of(cy(I), cz(I));
                fdst = a.fs[I] + (size_t)drow * lx;
                gdst = a.gs[I] + (size_t)drow * lx;
            } else {
                fdst = a.fs[opp(I)] + (size_t)row * lx;
                gdst = a.gs[opp(I)] + (size_t)row * lx;
            }
            bulk::store_row(fdst, sm + I * PITCH, bytes);
            bulk::store_row(gdst, sm + (Q + I) * PITCH, bytes);
        });
        bulk::store_commit();
        bulk::store_wait_read();
    }
}

}  // namespace lbm
