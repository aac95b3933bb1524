// lattice.cuh — D3Q27 lattice, integer helpers and population storage codecs.
//
// The velocity set and its order are those of the reference
// (Summer536/LBM_DDF src/initial.cu:71-73); the weights are those of
// src/initial.cu:77-83.  Population order has to match the reference because
// the C ABI exchanges states in the reference's restart layout.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <type_traits>

namespace lbm {

constexpr int Q = 27;

__host__ __device__ constexpr int cx(int i) {
    const int t[Q] = {0, 1, 0, -1, 0, 0, 0, 1, -1, -1, 1, 1, 0, -1,
                      0, 1, 0, -1, 0, 1, -1, -1, 1, 1, -1, -1, 1};
    return t[i];
}
__host__ __device__ constexpr int cy(int i) {
    const int t[Q] = {0, 0, 1, 0, -1, 0, 0, 1, 1, -1, -1, 0, 1, 0,
                      -1, 0, 1, 0, -1, 1, 1, -1, -1, 1, 1, -1, -1};
    return t[i];
}
__host__ __device__ constexpr int cz(int i) {
    const int t[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, 1,
                      1, -1, -1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1};
    return t[i];
}
// index of the population travelling the opposite way
__host__ __device__ constexpr int opp(int i) {
    const int t[Q] = {0, 3, 4, 1, 2, 6, 5, 9, 10, 7, 8, 17, 18, 15,
                      16, 13, 14, 11, 12, 25, 26, 23, 24, 21, 22, 19, 20};
    return t[i];
}
// weight class: 0 rest, 1 face (|c|=1), 2 edge (|c|^2=2), 3 corner (|c|^2=3)
__host__ __device__ constexpr int wclass(int i) { return i == 0 ? 0 : i <= 6 ? 1 : i <= 18 ? 2 : 3; }
__host__ __device__ constexpr double wd(int i) {
    return wclass(i) == 0 ? 8.0 / 27.0 : wclass(i) == 1 ? 2.0 / 27.0 : wclass(i) == 2 ? 1.0 / 54.0 : 1.0 / 216.0;
}
// 1/w_i; these four values are exact in binary
__host__ __device__ constexpr double winv(int i) {
    return wclass(i) == 0 ? 3.375 : wclass(i) == 1 ? 13.5 : wclass(i) == 2 ? 54.0 : 216.0;
}

// Unsigned division by a runtime constant d (1 <= d < 2^31) for dividends
// n < 2^31, by a multiply-high and shift (Granlund & Montgomery, PLDI 1994):
// with l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1,
// n / d = (umulhi(n, m) + n) >> l.
struct FastDiv {
    uint32_t d, m, l;
    FastDiv() = default;
    __host__ explicit FastDiv(uint32_t div) : d(div) {
        l = 0;
        while ((1ull << l) < div) ++l;
        m = (uint32_t)((((1ull << 32) * ((1ull << l) - div)) / div) + 1);
    }
    __device__ __forceinline__ uint32_t div(uint32_t n) const {
        return (__umulhi(n, m) + n) >> l;
    }
};

// Population codecs.  R is the arithmetic type; S the stored type.
//   F64, F32: populations stored as they are.
//   F16S, BF16S: the shifted, normalised values f_i / w_i and g_i / w_i - t0,
//   which lie in about [-1, 1] where 16-bit formats keep their relative
//   precision (f is already a deviation: its rest equilibrium is 0 because
//   rho is a density deviation, src/collision.cu:30).
template <class S> struct Codec;

template <> struct Codec<double> {
    using R = double;
    using P = double;  // carried previous-step temperature
    template <int I> __device__ __forceinline__ static R f_in(double s, R) { return s; }
    template <int I> __device__ __forceinline__ static R g_in(double s, R) { return s; }
    template <int I> __device__ __forceinline__ static double f_out(R v, R) { return v; }
    template <int I> __device__ __forceinline__ static double g_out(R v, R) { return v; }
};

template <> struct Codec<float> {
    using R = float;
    using P = float;
    template <int I> __device__ __forceinline__ static R f_in(float s, R) { return s; }
    template <int I> __device__ __forceinline__ static R g_in(float s, R) { return s; }
    template <int I> __device__ __forceinline__ static float f_out(R v, R) { return v; }
    template <int I> __device__ __forceinline__ static float g_out(R v, R) { return v; }
};

template <> struct Codec<__half> {
    using R = float;
    using P = float;
    template <int I> __device__ __forceinline__ static R f_in(__half s, R) { return (float)wd(I) * __half2float(s); }
    template <int I> __device__ __forceinline__ static R g_in(__half s, R t0) { return (float)wd(I) * (__half2float(s) + t0); }
    template <int I> __device__ __forceinline__ static __half f_out(R v, R) { return __float2half_rn(v * (float)winv(I)); }
    template <int I> __device__ __forceinline__ static __half g_out(R v, R t0) { return __float2half_rn(fmaf(v, (float)winv(I), -t0)); }
};

template <> struct Codec<__nv_bfloat16> {
    using R = float;
    using P = float;
    template <int I> __device__ __forceinline__ static R f_in(__nv_bfloat16 s, R) { return (float)wd(I) * __bfloat162float(s); }
    template <int I> __device__ __forceinline__ static R g_in(__nv_bfloat16 s, R t0) { return (float)wd(I) * (__bfloat162float(s) + t0); }
    template <int I> __device__ __forceinline__ static __nv_bfloat16 f_out(R v, R) { return __float2bfloat16_rn(v * (float)winv(I)); }
    template <int I> __device__ __forceinline__ static __nv_bfloat16 g_out(R v, R t0) { return __float2bfloat16_rn(fmaf(v, (float)winv(I), -t0)); }
};

// 16-bit storage interleaves the two distributions: element 2j of row k is
// f_k at node j and element 2j + 1 is g_k there, so one 32-bit access moves
// both (f_k and g_k always travel to the same slot of the same node).  FP32
// and FP64 keep separate f and g arrays.
template <class S> __host__ __device__ constexpr int elem_stride() { return sizeof(S) == 2 ? 2 : 1; }

// the packed (f_k, g_k) pair of 16-bit storage and its conversions
template <class S> struct Pack16;
template <> struct Pack16<__half> {
    using T = __half2;
    __device__ __forceinline__ static float2 unpack(T v) { return __half22float2(v); }
    __device__ __forceinline__ static T pack(float f, float g) { return __floats2half2_rn(f, g); }
};
template <> struct Pack16<__nv_bfloat16> {
    using T = __nv_bfloat162;
    __device__ __forceinline__ static float2 unpack(T v) { return __bfloat1622float2(v); }
    __device__ __forceinline__ static T pack(float f, float g) { return __floats2bfloat162_rn(f, g); }
};

// compile-time loop: calls fn(std::integral_constant<int, I>) for I = 0..N-1
template <int I, int N> struct Unroll {
    template <class Fn> __device__ __forceinline__ static void run(Fn &&fn) {
        fn(std::integral_constant<int, I>{});
        Unroll<I + 1, N>::run(fn);
    }
};
template <int N> struct Unroll<N, N> {
    template <class Fn> __device__ __forceinline__ static void run(Fn &&) {}
};

}  // namespace lbm
