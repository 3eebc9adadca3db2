// 256-point FFT by 16 threads (a half warp), 16 complex values per thread:
// a radix-16 x 16 Stockham transform with a single shared-memory exchange.
//
// Pass 1 (L = 1): thread t holds x[t + 16 m], m = 0..15, and computes the
// 16-point DFT y[16 t + q] = sum_m x[t + 16 m] W_16^{s m q}.
// Pass 2 (L = 16): thread t reads y[t + 16 m], applies the twiddles
// W_256^{s m t} and computes X[t + 16 q] = sum_m y'[t + 16 m] W_16^{s m q}.
// W_M = exp(2 pi i / M), s = +1 (inverse, unnormalised) or -1.
//
// Against the radix-8/8/4 schedule of fft_warp.cuh this halves the shared-
// memory traffic of the exchanges (which bound that transform), and two
// transforms run side by side in one warp.  The exchange buffer of a half
// warp holds 256 + 16 float2 (one pad element per 16, so the transposing
// writes and the reads are both conflict-free).
#pragma once
#include "fft_warp.cuh"

namespace tb {

constexpr int kR16Xbuf = 256 + 16;   // float2 per half-warp exchange buffer

__device__ __forceinline__ int r16pad(int i) { return i + (i >> 4); }

// In-place 16-point DFT with natural-order output, as 4 x 4: DFTs of length 4
// over the stride-4 subsequences, the internal twiddles W_16^{s n2 k1}, then
// DFTs of length 4 across them.
template <int S> __device__ __forceinline__ void dft16(float2* a) {
    constexpr float C1 = 0.92387953251128674f, S1 = 0.38268343236508978f;
    constexpr float R = 0.70710678118654752f;
    float2 y[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) {
        float2 b[4] = {a[n2], a[4 + n2], a[8 + n2], a[12 + n2]};
        dft4<S>(b);
#pragma unroll
        for (int k1 = 0; k1 < 4; k1++) y[n2][k1] = b[k1];
    }
    // W_16^{s e} for e = n2 k1: 1, 2, 3 (n2 = 1), 2, 4, 6 (n2 = 2), 3, 6, 9 (n2 = 3)
    const float2 w1 = make_float2(C1, S * S1), w2 = make_float2(R, S * R);
    const float2 w3 = make_float2(S1, S * C1), w6 = make_float2(-R, S * R);
    const float2 w9 = make_float2(-C1, -S * S1);
    y[1][1] = cmul(y[1][1], w1);
    y[1][2] = cmul(y[1][2], w2);
    y[1][3] = cmul(y[1][3], w3);
    y[2][1] = cmul(y[2][1], w2);
    y[2][2] = mul_si<S>(y[2][2]);
    y[2][3] = cmul(y[2][3], w6);
    y[3][1] = cmul(y[3][1], w3);
    y[3][2] = cmul(y[3][2], w6);
    y[3][3] = cmul(y[3][3], w9);
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) {
        float2 c[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
        dft4<S>(c);
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++) a[k1 + 4 * k2] = c[k2];
    }
}

// Runs one 256-point transform on the 16 threads of a half warp (t = lane
// within the half).  `v[m]` = x[t + 16 m] on entry.  `store(idx, value)`
// receives the outputs X[t + 16 q], q = 0..15 (16 calls per thread).  `xb` is
// the half warp's exchange buffer (kR16Xbuf float2), `tw16` the pass-2
// twiddles laid out by thread: tw16[16 m + t] = exp(2 pi i m t / 256)
// (build_r16_twiddles), so a half warp's loads of one m are conflict-free.
// Both halves of the warp must call this together.
template <int S, class Store>
__device__ __forceinline__ void fft256_r16(float2* v, int t, float2* xb, const float2* tw16,
                                           Store store) {
    dft16<S>(v);
#pragma unroll
    for (int q = 0; q < 16; q++) xb[r16pad(16 * t + q)] = v[q];
    __syncwarp();
#pragma unroll
    for (int m = 0; m < 16; m++) v[m] = xb[r16pad(t + 16 * m)];
    __syncwarp();
#pragma unroll
    for (int m = 1; m < 16; m++) {
        const float2 w = tw16[16 * m + t];
        v[m] = cmul(v[m], S > 0 ? w : make_float2(w.x, -w.y));
    }
    dft16<S>(v);
#pragma unroll
    for (int q = 0; q < 16; q++) store(t + 16 * q, v[q]);
}

// tw16[16 m + t] = exp(2 pi i m t / 256), m, t = 0..15, built once per CTA in
// FP64.
__device__ inline void build_r16_twiddles(float2* tw16) {
    for (int e = threadIdx.x; e < 256; e += blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)((e >> 4) * (e & 15)) / 256.0, &s, &c);
        tw16[e] = make_float2((float)c, (float)s);
    }
}

}  // namespace tb
