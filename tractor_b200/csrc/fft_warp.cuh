// Shared-memory Stockham FFT for power-of-two lengths 32..256, executed by a
// group of N/8 threads of one warp, each holding 8 complex values.
//
// Pass with radix R and current sub-transform length L (L = 1 at the start):
// for every group j in [0, N/R) with k = j mod L,
//     y[(j-k) R + k + q L] = sum_m x[j + m N/R] W_{LR}^{s m k} W_R^{s m q},
// with W_M = exp(2 pi i / M) and s = +1 (inverse, unnormalised) or -1.
// Intermediate arrays live in a per-group exchange buffer of float2 (one pad
// element per 16, which keeps every access conflict-free except one 2-way
// pattern in the second pass).  The first pass takes its inputs from
// registers: thread t holds x[t + m N/8], m = 0..7.
#pragma once
#include "tb_common.cuh"

namespace tb {

template <int N> struct FftPlan;
template <> struct FftPlan<256> { static constexpr int R2 = 8, R3 = 4, passes = 3; };
template <> struct FftPlan<128> { static constexpr int R2 = 4, R3 = 4, passes = 3; };
template <> struct FftPlan<64>  { static constexpr int R2 = 8, R3 = 1, passes = 2; };
template <> struct FftPlan<32>  { static constexpr int R2 = 4, R3 = 1, passes = 2; };

// float2 elements of one group's exchange buffer.
template <int N> __host__ __device__ constexpr int fft_xbuf_elems() { return N + N / 16; }

__device__ __forceinline__ int xpad(int i) { return i + (i >> 4); }

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// s * i * a
template <int S> __device__ __forceinline__ float2 mul_si(float2 a) {
    return S > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <int S> __device__ __forceinline__ void dft4(float2* a) {
    const float2 s02 = make_float2(a[0].x + a[2].x, a[0].y + a[2].y);
    const float2 d02 = make_float2(a[0].x - a[2].x, a[0].y - a[2].y);
    const float2 s13 = make_float2(a[1].x + a[3].x, a[1].y + a[3].y);
    const float2 d13 = mul_si<S>(make_float2(a[1].x - a[3].x, a[1].y - a[3].y));
    a[0] = make_float2(s02.x + s13.x, s02.y + s13.y);
    a[2] = make_float2(s02.x - s13.x, s02.y - s13.y);
    a[1] = make_float2(d02.x + d13.x, d02.y + d13.y);
    a[3] = make_float2(d02.x - d13.x, d02.y - d13.y);
}

template <int S> __device__ __forceinline__ void dft8(float2* a) {
    float2 e[4] = {a[0], a[2], a[4], a[6]};
    float2 o[4] = {a[1], a[3], a[5], a[7]};
    dft4<S>(e);
    dft4<S>(o);
    const float r = 0.70710678118654752f;
    // o[q] *= exp(s i pi q / 4)
    o[1] = make_float2(r * (o[1].x - S * o[1].y), r * (o[1].y + S * o[1].x));
    o[2] = mul_si<S>(o[2]);
    o[3] = make_float2(r * (-o[3].x - S * o[3].y), r * (-o[3].y + S * o[3].x));
#pragma unroll
    for (int q = 0; q < 4; q++) {
        a[q] = make_float2(e[q].x + o[q].x, e[q].y + o[q].y);
        a[q + 4] = make_float2(e[q].x - o[q].x, e[q].y - o[q].y);
    }
}

template <int R, int S> __device__ __forceinline__ void dftR(float2* a) {
    if constexpr (R == 8) dft8<S>(a); else dft4<S>(a);
}

// Twiddle W_N^(s e) from a table of exp(2 pi i e / N), e in [0, N).
template <int N, int S> __device__ __forceinline__ float2 twid(const float2* tw, int e) {
    const float2 w = tw[e & (N - 1)];
    return S > 0 ? w : make_float2(w.x, -w.y);
}

// Runs the whole transform.  `v` holds the first-pass inputs of thread t
// (v[m] = x[t + m N/8]).  `store(idx, value)` receives every output in natural
// order exactly once (8 calls per thread).  `xb` is the group's exchange
// buffer.  All threads of the warp must call this together.
template <int N, int S, class Store>
__device__ __forceinline__ void fft_run(float2* v, int t, float2* xb, const float2* tw,
                                        Store store) {
    using P = FftPlan<N>;
    constexpr int R2 = P::R2, R3 = P::R3;
    // pass 1: radix 8, L = 1, group j = t
    dftR<8, S>(v);
    if constexpr (P::passes == 1) {
#pragma unroll
        for (int q = 0; q < 8; q++) store(8 * t + q, v[q]);
        return;
    }
#pragma unroll
    for (int q = 0; q < 8; q++) xb[xpad(8 * t + q)] = v[q];
    __syncwarp();
    // pass 2: radix R2, L = 8
    {
        constexpr int L = 8, G = 8 / R2, NR = N / R2;
        float2 a[8];
#pragma unroll
        for (int g = 0; g < G; g++) {
            const int j = t + (N / 8) * g;
#pragma unroll
            for (int m = 0; m < R2; m++) a[g * R2 + m] = xb[xpad(j + m * NR)];
        }
        __syncwarp();
#pragma unroll
        for (int g = 0; g < G; g++) {
            const int j = t + (N / 8) * g, k = j % L;
            float2* b = a + g * R2;
#pragma unroll
            for (int m = 1; m < R2; m++) b[m] = cmul(b[m], twid<N, S>(tw, m * k * (N / (L * R2))));
            dftR<R2, S>(b);
#pragma unroll
            for (int q = 0; q < R2; q++) {
                const int oi = (j - k) * R2 + k + q * L;
                if constexpr (P::passes == 2) store(oi, b[q]);
                else xb[xpad(oi)] = b[q];
            }
        }
        if constexpr (P::passes == 2) return;
        __syncwarp();
    }
    // pass 3: radix R3, L = 8 R2
    {
        constexpr int L = 8 * R2, G = 8 / R3, NR = N / R3;
        float2 a[8];
#pragma unroll
        for (int g = 0; g < G; g++) {
            const int j = t + (N / 8) * g;
#pragma unroll
            for (int m = 0; m < R3; m++) a[g * R3 + m] = xb[xpad(j + m * NR)];
        }
        __syncwarp();
#pragma unroll
        for (int g = 0; g < G; g++) {
            const int j = t + (N / 8) * g, k = j % L;
            float2* b = a + g * R3;
#pragma unroll
            for (int m = 1; m < R3; m++) b[m] = cmul(b[m], twid<N, S>(tw, m * k * (N / (L * R3))));
            dftR<R3, S>(b);
#pragma unroll
            for (int q = 0; q < R3; q++) store((j - k) * R3 + k + q * L, b[q]);
        }
    }
}

// exp(2 pi i e / N) table, built once per CTA in FP64.
template <int N> __device__ void build_twiddles(float2* tw) {
    for (int e = threadIdx.x; e < N; e += blockDim.x) {
        double s, c;
        sincospi(2.0 * e / N, &s, &c);
        tw[e] = make_float2((float)c, (float)s);
    }
}

}  // namespace tb
