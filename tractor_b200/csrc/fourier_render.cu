// K3: fused pixelized-PSF galaxy renderer (sm_100a).
//
// One CTA renders one item (galaxy) at a time, persistent over items taken
// from a global counter, entirely in shared memory.  Two variants, chosen per
// item:
//
// Spectral-Lanczos path (the output window keeps >= 3 pixels from the edges
// of the sz x sz FFT box in every shifted direction, or there is no shift).
// The reference's Lanczos-3 correlation with zero edges then equals a
// circular correlation, i.e. a product of the spectrum with the taps'
// frequency responses Hx(v) Hy(w), so no spatial pass is needed:
//   1. column pass: per rfft column v, a thread group evaluates the
//      zero-mean mixture spectrum sum_k amp_k exp2(e_k(v, w)) for all sz rows
//      w (one SFU ex2 per element and component), multiplies by the PSF
//      spectrum column (column-major, coalesced) and by Hy(w), and runs an
//      inverse complex FFT along w, keeping only the output window's rows.
//      The DC and Nyquist columns keep only the real part of their
//      transform, as irfftn does.
//   2. row pass: pairs of kept rows, times Hx(v), packed as H1 + i H2 with
//      their Hermitian extension; one inverse complex FFT along v yields both
//      real rows, written straight to the output (integer shift and crop),
//      scaled by scale / sz^2 (irfftn's normalisation).
// Spatial path (windows near the box edge): as above without Hx / Hy, all
// columns transformed separately, 3 halo rows / columns kept, then Lanczos-3
// along x in place and along y with the reference's zero edges.
//
// This is ProfileGalaxy._realGetUnitFluxModelPatch's FFT branch with a
// ModelMask (tractor/galaxy.py:336-519) for a non-hybrid PixelizedPSF.
// Windows taller than the row buffer are processed in row chunks (the column
// pass is repeated per chunk).
#include "fft16.cuh"
#include "galaxy_geom.cuh"

namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxK = 128;
constexpr int kXbufPerWarp = 272;                  // float2, any N in [32, 256]
// the persistent kernel's exchange buffers: two half-warp radix-16
// transforms per warp at N = 256, one radix-8/8/4 transform below
constexpr int kXbufPersist = 2 * tb::kR16Xbuf;
static_assert(kXbufPersist >= kXbufPerWarp, "exchange buffer covers every N");
constexpr int kRmax256 = 134;                      // kept rows at sz = 256

__host__ __device__ constexpr int s1_bytes(int N, int rmax) { return rmax * (N / 2 + 1) * 8; }

constexpr int kS1Bytes = s1_bytes(256, kRmax256) > s1_bytes(128, 128) ? s1_bytes(256, kRmax256)
                                                                       : s1_bytes(128, 128);
constexpr int kSmemBytes = 256 * 8               /* twiddles */
                           + 2 * kMaxK * 16       /* components, derivative prefactors */
                           + 16 * 4               /* taps */
                           + (129 + 256) * 8      /* Hx, Hy */
                           + kWarps * kXbufPersist * 8 + kS1Bytes + 2 * 256 * 4
                           + 256 * 8 /* radix-16 twiddles */;

struct Shared {
    float2* tw;
    float4* comp;   // (amp, ca, cb, cd): exponent = ca v^2 + cb v w + cd w^2 (log2 units)
    float4* dcomp;  // derivative items: prefactor (da, ba, bb, bc) = da + ba v^2 + bb v w + bc w^2
    float* taps;    // fx[0..6], fy[0..6]
    float2* hx;     // frequency response of the x taps, v = 0..N/2
    float2* hy;     // frequency response of the y taps, row index j = 0..N-1
    float2* xbuf;
    float2* s1;
    float* gsp;     // N = 256: mixture spectrum of the DC and Nyquist columns, all rows
    float2* tw16;   // N = 256: the radix-16 pass-2 twiddles by thread (build_r16_twiddles)
};

// The 7 Lanczos-3 taps of a sub-pixel shift dx (lanczos_shift_3f's kernel
// L(p) = 3 sin(p) sin(p/3) / p^2, p = pi (i - 3 + dx), normalised to unit
// sum; dx = 0 is the identity) or, with `deriv`, their derivative d/d dx by
// the quotient rule (at dx = 0 the limit from dx > 0: support 0..5).  One
// warp: lane i < 7 evaluates tap i, the sums over the taps by shuffles.
// Called by all 32 lanes.
__device__ void taps_warp(double dx, bool deriv, float* f) {
    const int i = threadIdx.x & 31;
    double L = 0.0, D = 0.0;
    bool on;
    if (!deriv && dx == 0.0) {
        if (i < 7) f[i] = i == 3 ? 1.f : 0.f;
        return;
    }
    if (deriv) on = i >= (dx >= 0.0 ? 0 : 1) && i < (dx >= 0.0 ? 6 : 7);
    else on = i >= (dx > 0.0 ? 0 : 1) && i < (dx > 0.0 ? 6 : 7);
    if (on) {
        // sin / cos of pi t by sincospi (no argument reduction)
        const double t = i - 3.0 + dx;
        const double p = TB_PI * t;
        if (p == 0.0) {
            L = 1.0;
        } else {
            double sp, cp, s3, c3;
            sincospi(t, &sp, &cp);
            sincospi(t / 3.0, &s3, &c3);
            L = 3.0 * sp * s3 / (p * p);
            if (deriv)
                D = TB_PI * 3.0 * (cp * s3 / (p * p) + sp * c3 / (3.0 * p * p) -
                                   2.0 * sp * s3 / (p * p * p));
        }
    }
    double S = L, Sd = D;
    for (int o = 16; o > 0; o >>= 1) {
        S += __shfl_xor_sync(0xffffffffu, S, o);
        Sd += __shfl_xor_sync(0xffffffffu, Sd, o);
    }
    if (i < 7) f[i] = on ? (float)(deriv ? (D - L / S * Sd) / S : L / S) : 0.f;
}

// Mixture spectrum at (v, w) for the R rows of one thread: acc[m] =
// sum_k amp_k exp2(ca v^2 + cb v w_m + cd w_m^2).
template <int R>
__device__ __forceinline__ void spectrum_rows(const float4* comp, int K, float vf, const float* wf,
                                          float* acc) {
#pragma unroll
    for (int m = 0; m < R; m++) acc[m] = 0.f;
    for (int k = 0; k < K; k++) {
        const float4 c = comp[k];
        const float al = c.y * vf * vf, be = c.z * vf;
#pragma unroll
        for (int m = 0; m < R; m++) {
            const float e = fmaf(wf[m], fmaf(c.w, wf[m], be), al);
            acc[m] = fmaf(c.x, tb::ex2(e), acc[m]);
        }
    }
}

// Derivative spectrum: acc[m] = sum_k (da_k + ba_k v^2 + bb_k v w_m + bc_k w_m^2)
// * amp-less exp2(...) -- d/dtheta [a exp(-2 pi^2 f^T C f)] for a parameter
// theta that moves a and C.
template <int R>
__device__ __forceinline__ void dspectrum_rows(const float4* comp, const float4* dcomp, int K,
                                           float vf, const float* wf, float* acc) {
#pragma unroll
    for (int m = 0; m < R; m++) acc[m] = 0.f;
    for (int k = 0; k < K; k++) {
        const float4 c = comp[k];
        const float4 d = dcomp[k];
        const float al = c.y * vf * vf, be = c.z * vf;
        const float d0 = fmaf(d.y * vf, vf, d.x), d1 = d.z * vf;
#pragma unroll
        for (int m = 0; m < R; m++) {
            const float e = fmaf(wf[m], fmaf(c.w, wf[m], be), al);
            const float pre = fmaf(wf[m], fmaf(d.w, wf[m], d1), d0);
            acc[m] = fmaf(pre, tb::ex2(e), acc[m]);
        }
    }
}

// Difference spectrum (TB_FFT_DIFF): acc[m] = sum_k exp2(e_k) (a'_k
// expm1(de_k) + (a'_k - a_k)), de_k = dca v^2 + dcb v w + dcd w^2 the
// exponent change in natural-log units; dcomp = (a'_k - a_k, dca, dcb, dcd).
template <int R>
__device__ __forceinline__ void diffspectrum_rows(const float4* comp, const float4* dcomp, int K,
                                              float vf, const float* wf, float* acc) {
#pragma unroll
    for (int m = 0; m < R; m++) acc[m] = 0.f;
    for (int k = 0; k < K; k++) {
        const float4 c = comp[k];
        const float4 d = dcomp[k];
        const float al = c.y * vf * vf, be = c.z * vf;
        const float d0 = d.y * vf * vf, d1 = d.z * vf;
        const float a2 = c.x + d.x;
#pragma unroll
        for (int m = 0; m < R; m++) {
            const float e = fmaf(wf[m], fmaf(c.w, wf[m], be), al);
            const float de = fmaf(wf[m], fmaf(d.w, wf[m], d1), d0);
            const float pre = fmaf(a2, expm1f(de), d.x);
            acc[m] = fmaf(pre, tb::ex2(e), acc[m]);
        }
    }
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) { return tb::cmul(a, b); }

// Zero-fills (STORE mode) the output pixels outside the window
// [gr0, gr1) x [gc0, gc1) of G coordinates.
__device__ void zero_outside(float* O, int64_t ldo, int mw, int mh, int sx, int sy, int gr0,
                             int gr1, int gc0, int gc1, bool empty) {
    // nothing to do when the window covers the whole mask
    if (!empty && gr0 + sy <= 0 && gr1 + sy >= mh && gc0 + sx <= 0 && gc1 + sx >= mw) return;
    for (int i = threadIdx.x; i < mh * mw; i += kThreads) {
        const int r = i / mw - sy, c = i % mw - sx;
        if (empty || r < gr0 || r >= gr1 || c < gc0 || c >= gc1)
            O[(int64_t)(i / mw) * ldo + i % mw] = 0.f;
    }
}

// Writes one output pixel; in TB_FFT_DOT mode `o` points into the upstream
// gradient and the pixel's contribution to the item's dot product is
// accumulated instead.
template <bool kDeriv>
__device__ __forceinline__ void put(float* o, float v, int mode, float& dot) {
    if (kDeriv && mode == TB_FFT_DOT) dot = fmaf(*o, v, dot);
    else if (mode == TB_MOG_ATOMIC) atomicAdd(o, v);
    else if (mode == TB_MOG_ACCUM) *o += v;
    else *o = v;
}

// ---------------------------------------------------------------------------
// N = 256: radix-16 transforms (tb::fft256_r16), one per half warp, so each
// warp runs two side by side.  Thread t of a half holds rows (column pass)
// or columns (row pass) t + 16 m, m = 0..15.
// ---------------------------------------------------------------------------
template <bool kDeriv, int R>
__device__ __forceinline__ void col_spectrum(const tb_fft_item& it, int K, const Shared& sh,
                                             float vf, const float* wf, float* acc) {
    if (kDeriv && it.dmode == TB_FFT_DSPEC) dspectrum_rows<R>(sh.comp, sh.dcomp, K, vf, wf, acc);
    else if (kDeriv && it.dmode == TB_FFT_DIFF)
        diffspectrum_rows<R>(sh.comp, sh.dcomp, K, vf, wf, acc);
    else spectrum_rows<R>(sh.comp, K, vf, wf, acc);
}

// Column pass: the 127 interior rfft columns and one transform carrying both
// the DC and the Nyquist column, 128 transforms over the 32 half warps (four
// per warp).  irfftn keeps the real parts of the DC and Nyquist columns'
// transforms along w, which are the transforms of their Hermitian parts
// Xh(w) = (X(w) + conj X(-w)) / 2 (row -w = row (N - j) mod N); those are
// real, so Z = Xh_0 + i Xh_N gives both in one complex transform (real part
// -> DC, imaginary part -> Nyquist).  The mixture spectrum of those two
// columns is evaluated first by the whole block (one row per thread), so
// every half warp evaluates at most one column.  With kHy every column is
// multiplied by the y taps' frequency response.  Rows [rlo, rhi) of every
// column go to S1 (row-major, N/2 + 1 columns).  Called by the whole block.
template <bool kDeriv, bool kHy>
__device__ void colpass256(const tb_fft_item& it, int K, const float* __restrict__ spec,
                           const Shared& sh, int rlo, int rhi) {
    constexpr int N = 256, NH = 129;
    static_assert(kThreads == 2 * N, "one thread per row of the DC and Nyquist columns");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int half = lane >> 4, t = lane & 15;
    float2* xb = sh.xbuf + warp * kXbufPersist + half * tb::kR16Xbuf;
    const float2* P = reinterpret_cast<const float2*>(spec);
    {
        const int j = threadIdx.x & (N - 1);
        const float w1 = (float)(j < N / 2 ? j : j - N) / (float)N;
        float g;
        col_spectrum<kDeriv, 1>(it, K, sh, threadIdx.x < N ? 0.f : 0.5f, &w1, &g);
        sh.gsp[threadIdx.x] = g;
    }
    __syncthreads();
    float wf[16];
#pragma unroll
    for (int m = 0; m < 16; m++) {
        const int j = t + 16 * m;
        wf[m] = (float)(j < N / 2 ? j : j - N) / (float)N;
    }
    for (int s0 = 2 * warp; s0 < 128; s0 += 2 * kWarps) {
        const int slot = s0 + half;          // 0: DC + Nyquist, else the column v = slot
        float2 x[16];
        if (slot != 0) {
            // the PSF spectrum's loads go out before the mixture spectrum is evaluated
            const float2* Pc = P + (int64_t)slot * N;
#pragma unroll
            for (int m = 0; m < 16; m++) x[m] = __ldg(Pc + t + 16 * m);
            float acc[16];
            col_spectrum<kDeriv, 16>(it, K, sh, (float)slot / (float)N, wf, acc);
#pragma unroll
            for (int m = 0; m < 16; m++) {
                const float2 z = make_float2(acc[m] * x[m].x, acc[m] * x[m].y);
                x[m] = kHy ? cmulf(z, sh.hy[t + 16 * m]) : z;
            }
        } else {
            const float2* Pn = P + (int64_t)(N / 2) * N;
#pragma unroll
            for (int m = 0; m < 16; m++) {
                const int j = t + 16 * m, jn = (N - j) & (N - 1);
                float2 a = __ldg(P + j), b = __ldg(P + jn);
                float2 an = __ldg(Pn + j), bn = __ldg(Pn + jn);
                if (kHy) {
                    const float2 hj = sh.hy[j], hn = sh.hy[jn];
                    a = cmulf(a, hj);
                    b = cmulf(b, hn);
                    an = cmulf(an, hj);
                    bn = cmulf(bn, hn);
                }
                const float g0 = sh.gsp[j], g0n = sh.gsp[jn];
                const float gN = sh.gsp[N + j], gNn = sh.gsp[N + jn];
                // Xh_0 = (G0(w) a + G0(-w) conj b) / 2, Xh_N likewise; Z = Xh_0 + i Xh_N
                const float2 h0 = make_float2(0.5f * (g0 * a.x + g0n * b.x),
                                              0.5f * (g0 * a.y - g0n * b.y));
                const float2 hN = make_float2(0.5f * (gN * an.x + gNn * bn.x),
                                              0.5f * (gN * an.y - gNn * bn.y));
                x[m] = make_float2(h0.x - hN.y, h0.y + hN.x);
            }
        }
        tb::fft256_r16<+1>(x, t, xb, sh.tw16, [&](int row, float2 z) {
            if (row >= rlo && row < rhi) {
                float2* r = sh.s1 + (row - rlo) * NH;
                if (slot != 0) {
                    r[slot] = z;
                } else {
                    r[0] = make_float2(z.x, 0.f);
                    r[N / 2] = make_float2(z.y, 0.f);
                }
            }
        });
        __syncwarp();
    }
}

// Row pass: pairs of S1 rows (times Hx with kHx), packed as H1 + i H2 with
// their Hermitian extension, two pairs per warp; one inverse transform gives
// both real rows.  kToS1: the rows' columns [c0, c1) go back into the rows'
// own S1 storage (as floats, for the spatial Lanczos pass); otherwise the
// columns [gc0, gc1) go to the output (oa / ob rows) through put().
template <bool kDeriv, bool kHx, bool kToS1>
__device__ void rowpass256(const tb_fft_item& it, const Shared& sh, int nrows, float* O,
                           int64_t ldo, int row0, int sx, int c0, int c1, float osc, float& dot) {
    constexpr int N = 256, NH = 129;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int half = lane >> 4, t = lane & 15;
    float2* xb = sh.xbuf + warp * kXbufPersist + half * tb::kR16Xbuf;
    const int npairs = (nrows + 1) / 2;
    for (int p0 = 2 * warp; p0 < npairs; p0 += 2 * kWarps) {
        const bool act = p0 + half < npairs;
        const int p = act ? p0 + half : npairs - 1;
        const int ia = 2 * p, ib = 2 * p + 1;
        const bool hasb = ib < nrows;
        const float2* H1 = sh.s1 + ia * NH;
        const float2* H2 = sh.s1 + (hasb ? ib : ia) * NH;
        float2 x[16];
#pragma unroll
        for (int m = 0; m < 16; m++) {
            const int n = t + 16 * m;
            const int q = n <= N / 2 ? n : N - n;
            float2 h1 = H1[q];
            float2 h2 = hasb ? H2[q] : make_float2(0.f, 0.f);
            if (kHx) {
                const float2 hx = sh.hx[q];
                h1 = cmulf(h1, hx);
                h2 = cmulf(h2, hx);
            }
            if (q == 0 || q == N / 2) {
                h1.y = 0.f;
                h2.y = 0.f;
            }
            x[m] = n <= N / 2 ? make_float2(h1.x - h2.y, h1.y + h2.x)
                              : make_float2(h1.x + h2.y, h2.x - h1.y);
        }
        if (kToS1) {
            float* rowA = reinterpret_cast<float*>(sh.s1 + ia * NH);
            float* rowB = reinterpret_cast<float*>(sh.s1 + ib * NH);
            tb::fft256_r16<+1>(x, t, xb, sh.tw16, [&](int col, float2 z) {
                if (act && col >= c0 && col < c1) {
                    rowA[col - c0] = z.x;
                    if (hasb) rowB[col - c0] = z.y;
                }
            });
        } else {
            float* oa = O + (int64_t)(row0 + ia) * ldo + sx;
            float* ob = O + (int64_t)(row0 + ib) * ldo + sx;
            tb::fft256_r16<+1>(x, t, xb, sh.tw16, [&](int col, float2 z) {
                if (act && col >= c0 && col < c1) {
                    put<kDeriv>(oa + col, z.x * osc, it.mode, dot);
                    if (hasb) put<kDeriv>(ob + col, z.y * osc, it.mode, dot);
                }
            });
        }
        __syncwarp();
    }
}

template <int N, bool kDeriv>
__device__ void render_item_spectral(const tb_fft_item& it, int K, const float* __restrict__ spec,
                                     float* __restrict__ out, const Shared& sh, int rcap,
                                     float& dot) {
    constexpr int NH = N / 2 + 1;
    constexpr int T = N / 8;            // threads per FFT
    constexpr int GPW = 32 / T;         // FFT groups per warp
    constexpr int XB = tb::fft_xbuf_elems<N>();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = lane % T;
    const int ngroups = kWarps * GPW;
    float2* xb = sh.xbuf + warp * kXbufPersist + (lane / T) * XB;

    const int mw = it.mw, mh = it.mh, sx = it.sx, sy = it.sy;
    const float osc = it.scale / (float)(N * N);
    float* O = out + it.out_off;
    const int64_t ldo = it.ldo > 0 ? it.ldo : mw;
    const int gr0 = max(0, -sy), gr1 = min(N, mh - sy);
    const int gc0 = max(0, -sx), gc1 = min(N, mw - sx);

    // frequency responses of the taps: H(f) = sum_k tap_k exp(2 pi i f (k-3) / N)
    for (int f = threadIdx.x; f < NH + N; f += kThreads) {
        const bool isx = f < NH;
        const int fr = isx ? f : f - NH;
        const float* tp = isx ? sh.taps : sh.taps + 7;
        float2 h = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < 7; k++) {
            const float2 w = sh.tw[(fr * (k - 3)) & (N - 1)];
            h.x = fmaf(tp[k], w.x, h.x);
            h.y = fmaf(tp[k], w.y, h.y);
        }
        if (isx) sh.hx[fr] = h; else sh.hy[fr] = h;
    }
    __syncthreads();

    if constexpr (N == 256) {
        for (int a = gr0; a < gr1; a += rcap) {
            const int rlo = a, rhi = min(gr1, a + rcap);
            colpass256<kDeriv, true>(it, K, spec, sh, rlo, rhi);
            __syncthreads();
            rowpass256<kDeriv, true, false>(it, sh, rhi - rlo, O, ldo, rlo + sy, sx, gc0, gc1, osc,
                                            dot);
            __syncthreads();
        }
    } else {
        for (int a = gr0; a < gr1; a += rcap) {
            const int rlo = a, rhi = min(gr1, a + rcap);
            const int nrows = rhi - rlo;

            // ---- 1. column pass: N/2 + 1 column FFTs, times Hy ----
            for (int v0 = warp * GPW; v0 < NH; v0 += ngroups) {
                const bool act = v0 + lane / T < NH;
                const int v = act ? v0 + lane / T : NH - 1;
                float wf[8], acc[8];
#pragma unroll
                for (int m = 0; m < 8; m++) {
                    const int j = t + m * T;
                    wf[m] = (float)(j < N / 2 ? j : j - N) / (float)N;
                }
                if (kDeriv && it.dmode == TB_FFT_DSPEC)
                    dspectrum_rows<8>(sh.comp, sh.dcomp, K, (float)v / (float)N, wf, acc);
                else if (kDeriv && it.dmode == TB_FFT_DIFF)
                    diffspectrum_rows<8>(sh.comp, sh.dcomp, K, (float)v / (float)N, wf, acc);
                else
                    spectrum_rows<8>(sh.comp, K, (float)v / (float)N, wf, acc);
                float2 x[8];
                const float2* P = reinterpret_cast<const float2*>(spec) + (int64_t)v * N;
#pragma unroll
                for (int m = 0; m < 8; m++) {
                    const int j = t + m * T;
                    const float2 p = __ldg(P + j);
                    x[m] = cmulf(make_float2(acc[m] * p.x, acc[m] * p.y), sh.hy[j]);
                }
                // irfftn drops the imaginary parts of the DC and Nyquist columns
                // after the transform along y.
                const bool realcol = v == 0 || v == N / 2;
                float2* S1 = sh.s1;
                tb::fft_run<N, +1>(x, t, xb, sh.tw, [&](int row, float2 z) {
                    if (act && row >= rlo && row < rhi)
                        S1[(row - rlo) * NH + v] = realcol ? make_float2(z.x, 0.f) : z;
                });
                __syncwarp();
            }
            __syncthreads();

            // ---- 2. row pass: two real rows per complex FFT, straight to the output ----
            const int npairs = (nrows + 1) / 2;
            for (int p0 = warp * GPW; p0 < npairs; p0 += ngroups) {
                const bool act = p0 + lane / T < npairs;
                const int p = act ? p0 + lane / T : npairs - 1;
                const int ia = 2 * p, ib = 2 * p + 1;
                const bool hasb = ib < nrows;
                const float2* H1 = sh.s1 + ia * NH;
                const float2* H2 = sh.s1 + (hasb ? ib : ia) * NH;
                float2 x[8];
#pragma unroll
                for (int m = 0; m < 8; m++) {
                    const int n = t + m * T;
                    const int q = n <= N / 2 ? n : N - n;
                    const float2 hx = sh.hx[q];
                    const float2 h1 = cmulf(H1[q], hx);
                    const float2 h2 = hasb ? cmulf(H2[q], hx) : make_float2(0.f, 0.f);
                    x[m] = n <= N / 2 ? make_float2(h1.x - h2.y, h1.y + h2.x)
                                      : make_float2(h1.x + h2.y, h2.x - h1.y);
                }
                float* oa = O + (int64_t)(rlo + ia + sy) * ldo + sx;
                float* ob = O + (int64_t)(rlo + ib + sy) * ldo + sx;
                tb::fft_run<N, +1>(x, t, xb, sh.tw, [&](int col, float2 z) {
                    if (act && col >= gc0 && col < gc1) {
                        put<kDeriv>(oa + col, z.x * osc, it.mode, dot);
                        if (hasb) put<kDeriv>(ob + col, z.y * osc, it.mode, dot);
                    }
                });
                __syncwarp();
            }
            __syncthreads();
        }
    }
}

template <int N, bool kDeriv>
__device__ void render_item_spatial(const tb_fft_item& it, int K, const float* __restrict__ spec,
                                    float* __restrict__ out, const Shared& sh, int rmax,
                                    float& dot) {
    constexpr int NH = N / 2 + 1;
    constexpr int T = N / 8;
    constexpr int GPW = 32 / T;
    constexpr int XB = tb::fft_xbuf_elems<N>();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = lane % T;
    const int ngroups = kWarps * GPW;
    float2* xb = sh.xbuf + warp * kXbufPersist + (lane / T) * XB;

    const int mw = it.mw, mh = it.mh, sx = it.sx, sy = it.sy;
    const float osc = it.scale / (float)(N * N);
    float* O = out + it.out_off;
    const int64_t ldo = it.ldo > 0 ? it.ldo : mw;
    const int gr0 = max(0, -sy), gr1 = min(N, mh - sy);
    const int gc0 = max(0, -sx), gc1 = min(N, mw - sx);
    const int c0 = max(0, gc0 - 3), c1 = min(N, gc1 + 3);
    const int chunk = rmax - 6;
    const float* fx = sh.taps;
    const float* fy = sh.taps + 7;

    for (int a = gr0; a < gr1; a += chunk) {
        const int b = min(gr1, a + chunk);
        const int rlo = max(0, a - 3), rhi = min(N, b + 3);
        const int nrows = rhi - rlo;

        // ---- 1. column pass (all N/2 + 1 columns) ----
        if constexpr (N == 256) {
            colpass256<kDeriv, false>(it, K, spec, sh, rlo, rhi);
        } else
        for (int v0 = warp * GPW; v0 < NH; v0 += ngroups) {
            const bool act = v0 + lane / T < NH;
            const int v = act ? v0 + lane / T : NH - 1;
            float wf[8], acc[8];
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const int j = t + m * T;
                wf[m] = (float)(j < N / 2 ? j : j - N) / (float)N;
            }
            if (kDeriv && it.dmode == TB_FFT_DSPEC)
                dspectrum_rows<8>(sh.comp, sh.dcomp, K, (float)v / (float)N, wf, acc);
            else if (kDeriv && it.dmode == TB_FFT_DIFF)
                diffspectrum_rows<8>(sh.comp, sh.dcomp, K, (float)v / (float)N, wf, acc);
            else
                spectrum_rows<8>(sh.comp, K, (float)v / (float)N, wf, acc);
            float2 x[8];
            const float2* P = reinterpret_cast<const float2*>(spec) + (int64_t)v * N;
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const float2 p = __ldg(P + t + m * T);
                x[m] = make_float2(acc[m] * p.x, acc[m] * p.y);
            }
            float2* S1 = sh.s1;
            tb::fft_run<N, +1>(x, t, xb, sh.tw, [&](int row, float2 z) {
                if (act && row >= rlo && row < rhi) S1[(row - rlo) * NH + v] = z;
            });
            __syncwarp();
        }
        __syncthreads();

        // ---- 2. row pass (two real rows per complex FFT) ----
        const int npairs = (nrows + 1) / 2;
        if constexpr (N == 256) {
            rowpass256<kDeriv, false, true>(it, sh, nrows, nullptr, 0, 0, 0, c0, c1, 0.f, dot);
        } else
        for (int p0 = warp * GPW; p0 < npairs; p0 += ngroups) {
            const bool act = p0 + lane / T < npairs;
            const int p = act ? p0 + lane / T : npairs - 1;
            const int ia = 2 * p, ib = 2 * p + 1;
            const bool hasb = ib < nrows;
            const float2* H1 = sh.s1 + ia * NH;
            const float2* H2 = sh.s1 + (hasb ? ib : ia) * NH;
            float2 x[8];
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const int n = t + m * T;
                const int q = n <= N / 2 ? n : N - n;
                float2 h1 = H1[q];
                float2 h2 = hasb ? H2[q] : make_float2(0.f, 0.f);
                if (q == 0 || q == N / 2) { h1.y = 0.f; h2.y = 0.f; }
                x[m] = n <= N / 2 ? make_float2(h1.x - h2.y, h1.y + h2.x)
                                  : make_float2(h1.x + h2.y, h2.x - h1.y);
            }
            float* rowA = reinterpret_cast<float*>(sh.s1 + ia * NH);
            float* rowB = reinterpret_cast<float*>(sh.s1 + ib * NH);
            tb::fft_run<N, +1>(x, t, xb, sh.tw, [&](int col, float2 z) {
                if (act && col >= c0 && col < c1) {
                    rowA[col - c0] = z.x;
                    if (hasb) rowB[col - c0] = z.y;
                }
            });
            __syncwarp();
        }
        __syncthreads();

        // ---- 3a. Lanczos along x, in place per row (columns [gc0, gc1)) ----
        const int ncol = gc1 - gc0;
        for (int r = warp; r < nrows; r += kWarps) {
            float* row = reinterpret_cast<float*>(sh.s1 + r * NH);
            float res[8];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int cc = lane + 32 * i;
                float acc = 0.f;
                if (cc < ncol) {
                    const int c = gc0 + cc;
#pragma unroll
                    for (int k = 0; k < 7; k++) {
                        const int xsrc = c - 3 + k;
                        const float g = (xsrc >= c0 && xsrc < c1) ? row[xsrc - c0] : 0.f;
                        acc = fmaf(fx[k], g, acc);
                    }
                }
                res[i] = acc;
            }
            __syncwarp();
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int cc = lane + 32 * i;
                if (cc < ncol) row[cc] = res[i];
            }
        }
        __syncthreads();

        // ---- 3b. Lanczos along y, shift, crop, write ----
        const int orows = b - a;
        for (int idx = threadIdx.x; idx < orows * ncol; idx += kThreads) {
            const int r = a + idx / ncol;
            const int c = gc0 + idx % ncol;
            float val = 0.f;
#pragma unroll
            for (int k = 0; k < 7; k++) {
                const int rr = r - 3 + k;
                if (rr >= rlo && rr < rhi) {
                    const float* row = reinterpret_cast<const float*>(sh.s1 + (rr - rlo) * NH);
                    val = fmaf(fy[k], row[c - gc0], val);
                }
            }
            put<kDeriv>(O + (int64_t)(r + sy) * ldo + (c + sx), val * osc, it.mode, dot);
        }
        __syncthreads();
    }
}

template <int N, bool kDeriv>
__device__ void render_item(const tb_fft_item& it, int K, const float* __restrict__ spec,
                            float* __restrict__ out, const Shared& sh, float& dot) {
    const int mw = it.mw, mh = it.mh, sx = it.sx, sy = it.sy;
    const int gr0 = max(0, -sy), gr1 = min(N, mh - sy);
    const int gc0 = max(0, -sx), gc1 = min(N, mw - sx);
    const bool empty = gr0 >= gr1 || gc0 >= gc1;
    const bool accum = it.mode == TB_MOG_ACCUM || it.mode == TB_MOG_ATOMIC || it.mode == TB_FFT_DOT;
    if (!accum)
        zero_outside(out + it.out_off, it.ldo > 0 ? it.ldo : mw, mw, mh, sx, sy, gr0, gr1, gc0,
                     gc1, empty);
    if (empty) return;
    // Zero-edged Lanczos = circular correlation when no tap leaves the box
    // (no shift: the identity taps; a tap derivative is never the identity).
    const bool xin = (it.mux == 0.0 && it.dmode != TB_FFT_DX) || (gc0 >= 3 && gc1 <= N - 3);
    const bool yin = (it.muy == 0.0 && it.dmode != TB_FFT_DY) || (gr0 >= 3 && gr1 <= N - 3);
    const int rcap = N == 256 ? kRmax256 : N;
    if (xin && yin) render_item_spectral<N, kDeriv>(it, K, spec, out, sh, rcap, dot);
    else render_item_spatial<N, kDeriv>(it, K, spec, out, sh, N == 256 ? kRmax256 : N + 6, dot);
}

// Shared-memory carve-up of the persistent kernels.
__device__ __forceinline__ Shared carve_shared(unsigned char* smem_raw) {
    Shared sh;
    unsigned char* p = smem_raw;
    sh.tw = reinterpret_cast<float2*>(p);
    p += 256 * 8;
    sh.comp = reinterpret_cast<float4*>(p);
    p += kMaxK * 16;
    sh.dcomp = reinterpret_cast<float4*>(p);
    p += kMaxK * 16;
    sh.taps = reinterpret_cast<float*>(p);
    p += 16 * 4;
    sh.hx = reinterpret_cast<float2*>(p);
    p += 129 * 8;
    sh.hy = reinterpret_cast<float2*>(p);
    p += 256 * 8;
    sh.xbuf = reinterpret_cast<float2*>(p);
    p += kWarps * kXbufPersist * 8;
    sh.s1 = reinterpret_cast<float2*>(p);
    p += kS1Bytes;
    sh.gsp = reinterpret_cast<float*>(p);
    p += 2 * 256 * 4;
    sh.tw16 = reinterpret_cast<float2*>(p);
    return sh;
}

// The rest of one item once its components (and derivative coefficients)
// are in shared memory: taps, twiddles for its FFT size, the render, and
// for TB_FFT_DOT the item's dot product.  Called by the whole block.
template <bool kDeriv>
__device__ void render_staged_item(const tb_fft_item& it, int K,
                                   const float* __restrict__ psf_spec, float* __restrict__ out,
                                   double* __restrict__ dots, Shared& sh, int& cur_n) {
    const int N = it.sz;
    if (threadIdx.x >= 32 && threadIdx.x < 64)
        taps_warp(it.mux, kDeriv && it.dmode == TB_FFT_DX, sh.taps);
    if (threadIdx.x >= 64 && threadIdx.x < 96)
        taps_warp(it.muy, kDeriv && it.dmode == TB_FFT_DY, sh.taps + 7);
    __syncthreads();
    if (cur_n != N) {
        __syncthreads();
        switch (N) {
            case 256:
                tb::build_twiddles<256>(sh.tw);
                tb::build_r16_twiddles(sh.tw16);
                break;
            case 128: tb::build_twiddles<128>(sh.tw); break;
            case 64: tb::build_twiddles<64>(sh.tw); break;
            default: tb::build_twiddles<32>(sh.tw); break;
        }
        __syncthreads();
        if (threadIdx.x == 0) cur_n = N;
    }
    __syncthreads();
    const float* spec = psf_spec + it.spec_off;
    float dot = 0.f;
    switch (N) {
        case 256: render_item<256, kDeriv>(it, K, spec, out, sh, dot); break;
        case 128: render_item<128, kDeriv>(it, K, spec, out, sh, dot); break;
        case 64: render_item<64, kDeriv>(it, K, spec, out, sh, dot); break;
        default: render_item<32, kDeriv>(it, K, spec, out, sh, dot); break;
    }
    if (kDeriv && it.mode == TB_FFT_DOT) {
        // fixed-order block reduction of the item's dot product
        __shared__ double red[kWarps];
        double dd = (double)dot;
        for (int o = 16; o > 0; o >>= 1) dd += __shfl_xor_sync(0xffffffffu, dd, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dd;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s2 = 0.0;
            for (int w = 0; w < kWarps; w++) s2 += red[w];
            dots[it.dot_off] = s2;
        }
        __syncthreads();
    }
}

template <bool kDeriv>
__global__ void __launch_bounds__(kThreads, 1)
fourier_render_kernel(const tb_fft_item* __restrict__ items, int n_items,
                      const double* __restrict__ amp, const double* __restrict__ var,
                      const double* __restrict__ dcoef, const float* __restrict__ psf_spec,
                      float* __restrict__ out, double* __restrict__ dots, int32_t* counter,
                      tb_status* st, const int32_t* __restrict__ list = nullptr,
                      const int32_t* __restrict__ list_count = nullptr) {
    // `list` (optional): render only items list[0 .. *list_count)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Shared sh = carve_shared(smem_raw);
    __shared__ int64_t slot;
    __shared__ int cur_n;
    if (threadIdx.x == 0) cur_n = 0;

    const int64_t n_units = list ? (int64_t)*list_count : (int64_t)n_items;
    for (;;) {
        const int64_t uu = tb::next_unit(counter, &slot);
        if (uu >= n_units) break;
        const int64_t u = list ? (int64_t)list[uu] : uu;
        const tb_fft_item& it = items[u];
        const int N = it.sz, K = it.K;
        const bool okN = N == 32 || N == 64 || N == 128 || N == 256;
        const bool okD = kDeriv ? (it.dmode >= TB_FFT_VALUE && it.dmode <= TB_FFT_DIFF &&
                                   ((it.dmode != TB_FFT_DSPEC && it.dmode != TB_FFT_DIFF) ||
                                    dcoef != nullptr) &&
                                   (it.mode != TB_FFT_DOT || dots != nullptr))
                                : (it.dmode == TB_FFT_VALUE && it.mode != TB_FFT_DOT);
        if (!okN || !okD || K < 0 || K > kMaxK || it.mw <= 0 || it.mh <= 0 ||
            !(fabs(it.mux) <= 0.5) || !(fabs(it.muy) <= 0.5)) {
            if (threadIdx.x == 0) tb::report(st, TB_STATUS_BAD_ITEM, (int)u, N);
            continue;
        }
        // components (FP64 -> FP32 exponent coefficients in log2 units)
        const double c2 = -2.0 * TB_PI * TB_PI * TB_LOG2E;
        for (int k = threadIdx.x; k < K; k += kThreads) {
            const int c = it.c0 + k;
            const double a = var[4 * c], bb = var[4 * c + 1], d = var[4 * c + 3];
            sh.comp[k] = make_float4((float)amp[c], (float)(c2 * a), (float)(c2 * 2.0 * bb),
                                     (float)(c2 * d));
            if (kDeriv && it.dmode == TB_FFT_DSPEC) {
                // d/dtheta [a exp(-2 pi^2 f^T C f)] = (da - 2 pi^2 a f^T dC f) exp(...)
                const double* dc = dcoef + 4 * ((int64_t)it.dc0 + k);
                const double m2 = -2.0 * TB_PI * TB_PI * amp[c];
                sh.dcomp[k] = make_float4((float)dc[0], (float)(m2 * dc[1]),
                                          (float)(m2 * 2.0 * dc[2]), (float)(m2 * dc[3]));
            }
            if (kDeriv && it.dmode == TB_FFT_DIFF) {
                // (a' - a, exponent change -2 pi^2 f^T (C' - C) f in natural-log units)
                const double* dc = dcoef + 4 * ((int64_t)it.dc0 + k);
                const double n2 = -2.0 * TB_PI * TB_PI;
                sh.dcomp[k] = make_float4((float)dc[0], (float)(n2 * dc[1]),
                                          (float)(n2 * 2.0 * dc[2]), (float)(n2 * dc[3]));
            }
        }
        render_staged_item<kDeriv>(it, K, psf_spec, out, dots, sh, cur_n);
    }
}

// Fused preparation and render (tb_galaxy_fft_render): the persistent
// kernel taking galaxy source records instead of prepared items.  For each
// source warp 0 does the prep kernel's work (tb::prep_galaxy_warp: profile,
// shape, geometry) straight into shared memory -- the FP32 exponent
// coefficients from the same FP64 products the two-launch path writes and
// reads back, so both paths render the same item bit for bit -- then the
// block renders it.  One launch per batch instead of two, and no component
// tables in global memory.
__global__ void __launch_bounds__(kThreads, 1)
galaxy_fft_render_kernel(const tb_galaxy_src* __restrict__ srcs, int n, tb_fft_image img,
                         tb_profile_tables T, const float* __restrict__ psf_spec,
                         float* __restrict__ out, tb_fft_item* __restrict__ items,
                         int32_t* __restrict__ flags, int32_t* counter) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Shared sh = carve_shared(smem_raw);
    __shared__ int64_t slot;
    __shared__ int cur_n;
    __shared__ tb_fft_item item;
    if (threadIdx.x == 0) cur_n = 0;
    for (;;) {
        const int64_t u = tb::next_unit(counter, &slot);
        if (u >= n) break;
        if (threadIdx.x < 32) {
            const int lane = threadIdx.x;
            const tb_galaxy_src s = srcs[u];
            double a, v, M[3];
            int rank, flag;
            tb_fft_item it;
            const int K = tb::prep_galaxy_warp(s, img, T, lane, a, v, rank, M, flag, it);
            if (flag == 0 && lane < K) {
                const double c2 = -2.0 * TB_PI * TB_PI * TB_LOG2E;
                sh.comp[rank] = make_float4((float)a, (float)(c2 * (v * M[0])),
                                            (float)(c2 * 2.0 * (v * M[1])),
                                            (float)(c2 * (v * M[2])));
            }
            if (lane == 0) {
                item = it;
                if (items) items[u] = it;
                flags[u] = flag;
            }
        }
        __syncthreads();
        render_staged_item<false>(item, item.K, psf_spec, out, nullptr, sh, cur_n);
    }
}

// ---------------------------------------------------------------------------
// Split spectral path (tb_fourier_render_split): a column kernel and a row
// kernel joined by an L2-resident scratch, for every item whose Lanczos-3
// shift is a spectral product (render_item's xin && yin) and whose output is
// written or added (not TB_FFT_DOT).  Work units are small -- 16 rfft
// columns or 16 kept rows of one item -- so every SM runs several CTAs of
// 8 warps and the units of 256 galaxies spread evenly over the SMs; the
// persistent kernel above holds one galaxy per SM and needs the whole
// sz x (sz/2+1) transpose in its 180 KB of shared memory.
//
// Scratch: per item, column-major over the N/2 + 1 rfft columns, the kept
// rows [gr0, gr1) of each column transform: S1[v * (gr1 - gr0) + (row -
// gr0)] (the DC and Nyquist columns' real parts only, as irfftn).
// Items that are not eligible are appended to a list for the persistent
// kernel (third launch).
// ---------------------------------------------------------------------------
// CTAs per SM the column and row kernels are compiled for (their register
// budget: 3 -> 80, 4 -> 64 registers per thread)
#ifndef TB_SPLIT_COL_MINB
#define TB_SPLIT_COL_MINB 3
#endif
#ifndef TB_SPLIT_ROW_MINB
#define TB_SPLIT_ROW_MINB 4
#endif
constexpr int kSplitThreads = 256;
constexpr int kSplitWarps = kSplitThreads / 32;
constexpr int kColBlock = 16;                 // rfft columns per column unit
constexpr int kColUnits = (128 + 1 + kColBlock - 1) / kColBlock;   // per item at N = 256
constexpr int kRowBlock = 16;                 // kept rows per row unit
constexpr int kRowUnits = 256 / kRowBlock;
constexpr int64_t kS1PerItem = 256 * 129;     // float2 per item (N x (N/2+1) at N = 256)

struct SplitWs {
    int32_t col_counter, row_counter, fb_counter, fb_count;
    int32_t pad[60];
};

__device__ __forceinline__ bool split_eligible(const tb_fft_item& it) {
    const int N = it.sz;
    const int gr0 = max(0, -it.sy), gr1 = min(N, it.mh - it.sy);
    const int gc0 = max(0, -it.sx), gc1 = min(N, it.mw - it.sx);
    const bool xin = (it.mux == 0.0 && it.dmode != TB_FFT_DX) || (gc0 >= 3 && gc1 <= N - 3);
    const bool yin = (it.muy == 0.0 && it.dmode != TB_FFT_DY) || (gr0 >= 3 && gr1 <= N - 3);
    return xin && yin && it.mode != TB_FFT_DOT;
}

__device__ __forceinline__ bool item_ok(const tb_fft_item& it, const double* dcoef) {
    const int N = it.sz;
    return (N == 32 || N == 64 || N == 128 || N == 256) && it.dmode >= TB_FFT_VALUE &&
           it.dmode <= TB_FFT_DIFF &&
           ((it.dmode != TB_FFT_DSPEC && it.dmode != TB_FFT_DIFF) || dcoef != nullptr) &&
           it.K >= 0 && it.K <= kMaxK && it.mw > 0 && it.mh > 0 && fabs(it.mux) <= 0.5 &&
           fabs(it.muy) <= 0.5;
}

struct SplitColShared {
    float2 tw[256];
    float4 comp[kMaxK];
    float4 dcomp[kMaxK];
    float taps[8];
    float2 hy[256];
    float2 xbuf[kSplitWarps * kXbufPerWarp];
    int cur_n;
    int64_t slot;
};

__device__ void stage_components(const tb_fft_item& it, const double* __restrict__ amp,
                                 const double* __restrict__ var, const double* __restrict__ dcoef,
                                 float4* comp, float4* dcomp) {
    const double c2 = -2.0 * TB_PI * TB_PI * TB_LOG2E;
    for (int k = threadIdx.x; k < it.K; k += kSplitThreads) {
        const int c = it.c0 + k;
        const double a = var[4 * c], bb = var[4 * c + 1], d = var[4 * c + 3];
        comp[k] = make_float4((float)amp[c], (float)(c2 * a), (float)(c2 * 2.0 * bb),
                              (float)(c2 * d));
        if (it.dmode == TB_FFT_DSPEC) {
            const double* dc = dcoef + 4 * ((int64_t)it.dc0 + k);
            const double m2 = -2.0 * TB_PI * TB_PI * amp[c];
            dcomp[k] = make_float4((float)dc[0], (float)(m2 * dc[1]), (float)(m2 * 2.0 * dc[2]),
                                   (float)(m2 * dc[3]));
        } else if (it.dmode == TB_FFT_DIFF) {
            const double* dc = dcoef + 4 * ((int64_t)it.dc0 + k);
            const double n2 = -2.0 * TB_PI * TB_PI;
            dcomp[k] = make_float4((float)dc[0], (float)(n2 * dc[1]), (float)(n2 * 2.0 * dc[2]),
                                   (float)(n2 * dc[3]));
        }
    }
}

// Spectrum of column v for the 8 rows of one thread, by item mode.
__device__ __forceinline__ void spectrum_any(const tb_fft_item& it, const float4* comp,
                                             const float4* dcomp, float vf, const float* wf,
                                             float* acc) {
    if (it.dmode == TB_FFT_DSPEC) dspectrum_rows<8>(comp, dcomp, it.K, vf, wf, acc);
    else if (it.dmode == TB_FFT_DIFF) diffspectrum_rows<8>(comp, dcomp, it.K, vf, wf, acc);
    else spectrum_rows<8>(comp, it.K, vf, wf, acc);
}

// Frequency response of the 7 Lanczos-3 taps at frequency index fr of an
// N-point transform: sum_k taps[k] exp(2 pi i fr (k - 3) / N), from the
// twiddle table.
__device__ __forceinline__ float2 taps_response(const float* taps, const float2* tw, int fr,
                                                int N) {
    float2 r = make_float2(0.f, 0.f);
#pragma unroll
    for (int k = 0; k < 7; k++) {
        const float2 w = tw[(fr * (k - 3)) & (N - 1)];
        r.x = fmaf(taps[k], w.x, r.x);
        r.y = fmaf(taps[k], w.y, r.y);
    }
    return r;
}

template <int N>
__device__ void split_col_unit(const tb_fft_item& it, int cb, const float* __restrict__ spec,
                               float2* __restrict__ s1, SplitColShared& sh) {
    constexpr int NH = N / 2 + 1;         // rfft columns
    constexpr int T = N / 8;
    constexpr int GPW = 32 / T;
    constexpr int XB = tb::fft_xbuf_elems<N>();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = lane % T;
    float2* xb = sh.xbuf + warp * kXbufPerWarp + (lane / T) * XB;
    const int gr0 = max(0, -it.sy), gr1 = min(N, it.mh - it.sy);
    const int nr = gr1 - gr0;
    const int cend = min(NH, (cb + 1) * kColBlock);
    float wf[8];
#pragma unroll
    for (int m = 0; m < 8; m++) {
        const int j = t + m * T;
        wf[m] = (float)(j < N / 2 ? j : j - N) / (float)N;
    }
    for (int c0 = cb * kColBlock + warp * GPW; c0 < cend; c0 += kSplitWarps * GPW) {
        const bool act = c0 + lane / T < cend;
        const int c = act ? c0 + lane / T : cend - 1;
        float2 x[8];
        float acc[8];
        spectrum_any(it, sh.comp, sh.dcomp, (float)c / (float)N, wf, acc);
        const float2* P = reinterpret_cast<const float2*>(spec) + (int64_t)c * N;
#pragma unroll
        for (int m = 0; m < 8; m++) {
            const int j = t + m * T;
            const float2 p = __ldg(P + j);
            x[m] = cmulf(make_float2(acc[m] * p.x, acc[m] * p.y), sh.hy[j]);
        }
        // irfftn keeps only the real parts of the DC and Nyquist columns'
        // transforms (the Nyquist column of the mixture spectrum is not
        // Hermitian in w, so the two cannot share one complex transform)
        const bool realcol = c == 0 || c == N / 2;
        float2* col = s1 + (int64_t)c * nr;
        tb::fft_run<N, +1>(x, t, xb, sh.tw, [&](int row, float2 z) {
            if (act && row >= gr0 && row < gr1) col[row - gr0] = realcol ? make_float2(z.x, 0.f) : z;
        });
        __syncwarp();
    }
}

__global__ void __launch_bounds__(kSplitThreads, TB_SPLIT_COL_MINB)
fourier_split_col_kernel(const tb_fft_item* __restrict__ items, int i0, int n_items,
                         const double* __restrict__ amp, const double* __restrict__ var,
                         const double* __restrict__ dcoef, const float* __restrict__ psf_spec,
                         float* __restrict__ out, SplitWs* ws, int32_t* fb_list,
                         float2* __restrict__ s1_all, tb_status* st) {
    __shared__ SplitColShared sh;
    if (threadIdx.x == 0) sh.cur_n = 0;
    const int64_t n_units = (int64_t)n_items * kColUnits;
    for (;;) {
        const int64_t u = tb::next_unit(&ws->col_counter, &sh.slot);
        if (u >= n_units) break;
        const int li = (int)(u / kColUnits), cb = (int)(u % kColUnits);
        const int ii = i0 + li;
        const tb_fft_item& it = items[ii];
        const int N = it.sz;
        if (cb == 0) {
            if (!item_ok(it, dcoef)) {
                if (threadIdx.x == 0) tb::report(st, TB_STATUS_BAD_ITEM, ii, N);
                continue;
            }
            if (!split_eligible(it)) {
                if (threadIdx.x == 0) fb_list[atomicAdd(&ws->fb_count, 1)] = ii;
                continue;
            }
            // STORE: the mask's pixels outside the transform window are zero
            const int gr0 = max(0, -it.sy), gr1 = min(N, it.mh - it.sy);
            const int gc0 = max(0, -it.sx), gc1 = min(N, it.mw - it.sx);
            if (it.mode == TB_MOG_STORE)
                zero_outside(out + it.out_off, it.ldo > 0 ? it.ldo : it.mw, it.mw, it.mh, it.sx,
                             it.sy, gr0, gr1, gc0, gc1, gr0 >= gr1 || gc0 >= gc1);
        } else if (!item_ok(it, dcoef) || !split_eligible(it)) {
            continue;
        }
        if (cb * kColBlock > N / 2) continue;
        {
            const int gr0 = max(0, -it.sy), gr1 = min(N, it.mh - it.sy);
            const int gc0 = max(0, -it.sx), gc1 = min(N, it.mw - it.sx);
            if (gr0 >= gr1 || gc0 >= gc1) continue;
        }
        // stage: components, y taps and their frequency response, twiddles
        stage_components(it, amp, var, dcoef, sh.comp, sh.dcomp);
        if (threadIdx.x < 32) taps_warp(it.muy, it.dmode == TB_FFT_DY, sh.taps);
        if (sh.cur_n != N) {
            __syncthreads();
            switch (N) {
                case 256: tb::build_twiddles<256>(sh.tw); break;
                case 128: tb::build_twiddles<128>(sh.tw); break;
                case 64: tb::build_twiddles<64>(sh.tw); break;
                default: tb::build_twiddles<32>(sh.tw); break;
            }
            if (threadIdx.x == 0) sh.cur_n = N;
        }
        __syncthreads();
        for (int j = threadIdx.x; j < N; j += kSplitThreads)
            sh.hy[j] = taps_response(sh.taps, sh.tw, j, N);
        __syncthreads();
        float2* s1 = s1_all + (int64_t)li * kS1PerItem;
        const float* spec = psf_spec + it.spec_off;
        switch (N) {
            case 256: split_col_unit<256>(it, cb, spec, s1, sh); break;
            case 128: split_col_unit<128>(it, cb, spec, s1, sh); break;
            case 64: split_col_unit<64>(it, cb, spec, s1, sh); break;
            default: split_col_unit<32>(it, cb, spec, s1, sh); break;
        }
    }
}

struct SplitRowShared {
    float2 tw[256];
    float taps[8];
    float2 hx[129];
    float2 xbuf[kSplitWarps * kXbufPerWarp];
    float2 rows[kRowBlock * 129];     // [r][v], the N/2 + 1 rfft columns
    int cur_n;
    int64_t slot;
};

template <int N>
__device__ void split_row_unit(const tb_fft_item& it, int rb, const float2* __restrict__ s1,
                               float* __restrict__ out, SplitRowShared& sh) {
    constexpr int NH = N / 2 + 1;
    constexpr int T = N / 8;
    constexpr int GPW = 32 / T;
    constexpr int XB = tb::fft_xbuf_elems<N>();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = lane % T;
    float2* xb = sh.xbuf + warp * kXbufPerWarp + (lane / T) * XB;
    const int gr0 = max(0, -it.sy), gr1 = min(N, it.mh - it.sy);
    const int gc0 = max(0, -it.sx), gc1 = min(N, it.mw - it.sx);
    const int nr = gr1 - gr0;
    const int r0 = rb * kRowBlock;
    const int nrows = min(kRowBlock, nr - r0);
    // this unit's rows of every rfft column, transposed into shared memory
    // by asynchronous 8-byte copies (all of a thread's copies in flight at
    // once, no registers held); rows >= nrows are not read below
    constexpr int kLd = (NH * kRowBlock + kSplitThreads - 1) / kSplitThreads;
#pragma unroll
    for (int q = 0; q < kLd; q++) {
        const int e = threadIdx.x + q * kSplitThreads;
        const int c = e / kRowBlock, r = e % kRowBlock;
        if (e < NH * kRowBlock && r < nrows) {
            const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&sh.rows[r * 129 + c]);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst),
                         "l"(s1 + (int64_t)c * nr + r0 + r) : "memory");
        }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    const float osc = it.scale / (float)(N * N);
    float* O = out + it.out_off;
    const int64_t ldo = it.ldo > 0 ? it.ldo : it.mw;
    const int npairs = (nrows + 1) / 2;
    for (int p0 = warp * GPW; p0 < npairs; p0 += kSplitWarps * GPW) {
        const bool act = p0 + lane / T < npairs;
        const int p = act ? p0 + lane / T : npairs - 1;
        const int ia = 2 * p, ib = 2 * p + 1;
        const bool hasb = ib < nrows;
        const float2* H1 = sh.rows + ia * 129;
        const float2* H2 = sh.rows + (hasb ? ib : ia) * 129;
        float2 x[8];
#pragma unroll
        for (int m = 0; m < 8; m++) {
            const int n = t + m * T;
            const int q = n <= N / 2 ? n : N - n;
            const float2 g1 = H1[q], g2 = H2[q];
            const float2 hx = sh.hx[q];
            const float2 h1 = cmulf(g1, hx);
            const float2 h2 = hasb ? cmulf(g2, hx) : make_float2(0.f, 0.f);
            x[m] = n <= N / 2 ? make_float2(h1.x - h2.y, h1.y + h2.x)
                              : make_float2(h1.x + h2.y, h2.x - h1.y);
        }
        float* oa = O + (int64_t)(gr0 + r0 + ia + it.sy) * ldo + it.sx;
        float* ob = O + (int64_t)(gr0 + r0 + ib + it.sy) * ldo + it.sx;
        float dummy = 0.f;
        tb::fft_run<N, +1>(x, t, xb, sh.tw, [&](int col, float2 z) {
            if (act && col >= gc0 && col < gc1) {
                put<false>(oa + col, z.x * osc, it.mode, dummy);
                if (hasb) put<false>(ob + col, z.y * osc, it.mode, dummy);
            }
        });
        __syncwarp();
    }
}

__global__ void __launch_bounds__(kSplitThreads, TB_SPLIT_ROW_MINB)
fourier_split_row_kernel(const tb_fft_item* __restrict__ items, int i0, int n_items,
                         const double* __restrict__ dcoef, float* __restrict__ out, SplitWs* ws,
                         const float2* __restrict__ s1_all) {
    __shared__ SplitRowShared sh;
    if (threadIdx.x == 0) sh.cur_n = 0;
    const int64_t n_units = (int64_t)n_items * kRowUnits;
    for (;;) {
        const int64_t u = tb::next_unit(&ws->row_counter, &sh.slot);
        if (u >= n_units) break;
        const int li = (int)(u / kRowUnits), rb = (int)(u % kRowUnits);
        const tb_fft_item& it = items[i0 + li];
        if (!item_ok(it, dcoef) || !split_eligible(it)) continue;
        const int N = it.sz;
        const int gr0 = max(0, -it.sy), gr1 = min(N, it.mh - it.sy);
        const int gc0 = max(0, -it.sx), gc1 = min(N, it.mw - it.sx);
        if (gr0 >= gr1 || gc0 >= gc1 || rb * kRowBlock >= gr1 - gr0) continue;
        if (threadIdx.x < 32) taps_warp(it.mux, it.dmode == TB_FFT_DX, sh.taps);
        if (sh.cur_n != N) {
            __syncthreads();
            switch (N) {
                case 256: tb::build_twiddles<256>(sh.tw); break;
                case 128: tb::build_twiddles<128>(sh.tw); break;
                case 64: tb::build_twiddles<64>(sh.tw); break;
                default: tb::build_twiddles<32>(sh.tw); break;
            }
            if (threadIdx.x == 0) sh.cur_n = N;
        }
        __syncthreads();
        // the x taps' frequency response
        for (int f = threadIdx.x; f <= N / 2; f += kSplitThreads)
            sh.hx[f] = taps_response(sh.taps, sh.tw, f, N);
        __syncthreads();
        const float2* s1 = s1_all + (int64_t)li * kS1PerItem;
        switch (N) {
            case 256: split_row_unit<256>(it, rb, s1, out, sh); break;
            case 128: split_row_unit<128>(it, rb, s1, out, sh); break;
            case 64: split_row_unit<64>(it, rb, s1, out, sh); break;
            default: split_row_unit<32>(it, rb, s1, out, sh); break;
        }
    }
}

}  // namespace

static int launch_fourier(const tb_fft_item* items, int32_t n_items, const double* comp_amp,
                          const double* comp_var, const double* comp_dcoef, const float* psf_spec,
                          float* out, double* dots, int32_t* work_counter, tb_status* status,
                          void* stream) {
    if (n_items < 0) return TB_ERR_ARG;
    if (n_items == 0) return TB_OK;
    if (!items || !comp_amp || !comp_var || !psf_spec || !out || !work_counter) return TB_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const bool deriv = comp_dcoef != nullptr || dots != nullptr;
    if (cudaFuncSetAttribute(deriv ? fourier_render_kernel<true> : fourier_render_kernel<false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes) != cudaSuccess)
        return TB_ERR_LAUNCH;
    if (cudaMemsetAsync(work_counter, 0, sizeof(int32_t), s) != cudaSuccess) return TB_ERR_LAUNCH;
    if (status && cudaMemsetAsync(status, 0, sizeof(tb_status), s) != cudaSuccess)
        return TB_ERR_LAUNCH;
    const int grid = n_items < tb::num_sms() ? n_items : tb::num_sms();
    if (deriv)
        fourier_render_kernel<true><<<grid, kThreads, kSmemBytes, s>>>(
            items, n_items, comp_amp, comp_var, comp_dcoef, psf_spec, out, dots, work_counter,
            status);
    else
        fourier_render_kernel<false><<<grid, kThreads, kSmemBytes, s>>>(
            items, n_items, comp_amp, comp_var, nullptr, psf_spec, out, nullptr, work_counter,
            status);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

extern "C" int tb_fourier_render(const tb_fft_item* items, int32_t n_items,
                                 const double* comp_amp, const double* comp_var,
                                 const float* psf_spec, float* out, int32_t* work_counter,
                                 tb_status* status, void* stream) {
    return launch_fourier(items, n_items, comp_amp, comp_var, nullptr, psf_spec, out, nullptr,
                          work_counter, status, stream);
}

extern "C" int tb_fourier_render_deriv(const tb_fft_item* items, int32_t n_items,
                                       const double* comp_amp, const double* comp_var,
                                       const double* comp_dcoef, const float* psf_spec,
                                       float* out, double* dots, int32_t* work_counter,
                                       tb_status* status, void* stream) {
    return launch_fourier(items, n_items, comp_amp, comp_var, comp_dcoef, psf_spec, out, dots,
                          work_counter, status, stream);
}

extern "C" int tb_galaxy_fft_render(const tb_galaxy_src* srcs, int32_t n,
                                    const tb_fft_image* image, const tb_profile_tables* tables,
                                    const float* psf_spec, float* out, tb_fft_item* items,
                                    int32_t* flags, int32_t* work_counter, tb_status* status,
                                    void* stream) {
    if (n < 0) return TB_ERR_ARG;
    if (n == 0) return TB_OK;
    if (!srcs || !image || !tables || !psf_spec || !out || !flags || !work_counter)
        return TB_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaFuncSetAttribute(galaxy_fft_render_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kSmemBytes) != cudaSuccess)
        return TB_ERR_LAUNCH;
    if (cudaMemsetAsync(work_counter, 0, sizeof(int32_t), s) != cudaSuccess) return TB_ERR_LAUNCH;
    if (status && cudaMemsetAsync(status, 0, sizeof(tb_status), s) != cudaSuccess)
        return TB_ERR_LAUNCH;
    const int grid = n < tb::num_sms() ? n : tb::num_sms();
    galaxy_fft_render_kernel<<<grid, kThreads, kSmemBytes, s>>>(srcs, n, *image, *tables, psf_spec,
                                                                out, items, flags, work_counter);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

namespace {
constexpr int kSplitChunk = 256;      // items per column/row launch pair (scratch bound)

int64_t split_list_bytes(int32_t n_items) { return ((int64_t)n_items * 4 + 255) / 256 * 256; }

int split_grid(const void* fn) {
    static int cached[2] = {0, 0};
    const int which = fn == (const void*)fourier_split_col_kernel ? 0 : 1;
    if (cached[which] == 0) {
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kSplitThreads, 0) !=
                cudaSuccess || per_sm < 1)
            per_sm = 1;
        cached[which] = per_sm;
    }
    return tb::num_sms() * cached[which];
}
}  // namespace

extern "C" int tb_fourier_workspace(int32_t n_items, int64_t* bytes) {
    if (n_items < 0 || !bytes) return TB_ERR_ARG;
    const int64_t chunk = n_items < kSplitChunk ? n_items : kSplitChunk;
    *bytes = (int64_t)sizeof(SplitWs) + split_list_bytes(n_items) +
             chunk * kS1PerItem * (int64_t)sizeof(float2);
    return TB_OK;
}

extern "C" int tb_fourier_render_split(const tb_fft_item* items, int32_t n_items,
                                       const double* comp_amp, const double* comp_var,
                                       const double* comp_dcoef, const float* psf_spec,
                                       float* out, double* dots, void* workspace,
                                       int64_t workspace_bytes, tb_status* status,
                                       void* stream) {
    if (n_items < 0) return TB_ERR_ARG;
    if (n_items == 0) return TB_OK;
    if (!items || !comp_amp || !comp_var || !psf_spec || !out || !workspace) return TB_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0) return TB_ERR_ARG;
    int64_t need = 0;
    tb_fourier_workspace(n_items, &need);
    if (workspace_bytes < need) return TB_ERR_SIZE;
    cudaStream_t s = (cudaStream_t)stream;
    SplitWs* ws = static_cast<SplitWs*>(workspace);
    int32_t* fb_list = reinterpret_cast<int32_t*>(static_cast<char*>(workspace) + sizeof(SplitWs));
    float2* s1 = reinterpret_cast<float2*>(static_cast<char*>(workspace) + sizeof(SplitWs) +
                                           split_list_bytes(n_items));
    if (cudaMemsetAsync(ws, 0, sizeof(SplitWs), s) != cudaSuccess) return TB_ERR_LAUNCH;
    if (status && cudaMemsetAsync(status, 0, sizeof(tb_status), s) != cudaSuccess)
        return TB_ERR_LAUNCH;
    const int gcol = split_grid((const void*)fourier_split_col_kernel);
    const int grow = split_grid((const void*)fourier_split_row_kernel);
    for (int32_t i0 = 0; i0 < n_items; i0 += kSplitChunk) {
        const int32_t n = n_items - i0 < kSplitChunk ? n_items - i0 : kSplitChunk;
        if (i0 > 0 && cudaMemsetAsync(ws, 0, 2 * sizeof(int32_t), s) != cudaSuccess)
            return TB_ERR_LAUNCH;
        const int64_t cu = (int64_t)n * kColUnits, ru = (int64_t)n * kRowUnits;
        fourier_split_col_kernel<<<(int)(cu < gcol ? cu : gcol), kSplitThreads, 0, s>>>(
            items, i0, n, comp_amp, comp_var, comp_dcoef, psf_spec, out, ws, fb_list, s1,
            status);
        fourier_split_row_kernel<<<(int)(ru < grow ? ru : grow), kSplitThreads, 0, s>>>(
            items, i0, n, comp_dcoef, out, ws, s1);
    }
    // items outside the split path (Lanczos-3 reaching the box edge, TB_FFT_DOT)
    const bool deriv = comp_dcoef != nullptr || dots != nullptr;
    if (cudaFuncSetAttribute(deriv ? fourier_render_kernel<true> : fourier_render_kernel<false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes) != cudaSuccess)
        return TB_ERR_LAUNCH;
    const int gfb = tb::num_sms() < n_items ? tb::num_sms() : n_items;
    if (deriv)
        fourier_render_kernel<true><<<gfb, kThreads, kSmemBytes, s>>>(
            items, n_items, comp_amp, comp_var, comp_dcoef, psf_spec, out, dots, &ws->fb_counter,
            status, fb_list, &ws->fb_count);
    else
        fourier_render_kernel<false><<<gfb, kThreads, kSmemBytes, s>>>(
            items, n_items, comp_amp, comp_var, nullptr, psf_spec, out, nullptr, &ws->fb_counter,
            status, fb_list, &ws->fb_count);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

// ---------------------------------------------------------------------------
// PSF spectra: forward rfft2 of zero-padded PSF images, stored column-major
// (element (row j, column v) at v * sz + j) so the column pass above reads
// contiguous memory.
// ---------------------------------------------------------------------------
namespace {

constexpr int kSpecThreads = 256;

template <int N>
__device__ void spec_rows(const float* __restrict__ pad, float* __restrict__ spec, int img,
                          float2* xbuf, const float2* tw) {
    constexpr int T = N / 8, GPW = 32 / T, XB = tb::fft_xbuf_elems<N>();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = lane % T;
    float2* xb = xbuf + warp * kXbufPerWarp + (lane / T) * XB;
    const int nwarps = kSpecThreads / 32;
    const float* I = pad + (int64_t)img * N * N;
    float2* S = reinterpret_cast<float2*>(spec) + (int64_t)img * N * (N / 2 + 1);
    for (int y0 = blockIdx.x * nwarps * GPW + warp * GPW; y0 < N; y0 += gridDim.x * nwarps * GPW) {
        const int y = y0 + lane / T;   // N rows, groups never run past the end
        float2 x[8];
#pragma unroll
        for (int m = 0; m < 8; m++) x[m] = make_float2(I[(int64_t)y * N + t + m * T], 0.f);
        tb::fft_run<N, -1>(x, t, xb, tw, [&](int k, float2 z) {
            if (k <= N / 2) S[(int64_t)k * N + y] = z;
        });
        __syncwarp();
    }
}

template <int N>
__device__ void spec_cols(float* __restrict__ spec, int img, float2* xbuf, const float2* tw) {
    constexpr int T = N / 8, GPW = 32 / T, XB = tb::fft_xbuf_elems<N>(), NH = N / 2 + 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = lane % T;
    float2* xb = xbuf + warp * kXbufPerWarp + (lane / T) * XB;
    const int nwarps = kSpecThreads / 32;
    float2* S = reinterpret_cast<float2*>(spec) + (int64_t)img * N * NH;
    for (int v0 = blockIdx.x * nwarps * GPW + warp * GPW; v0 < NH; v0 += gridDim.x * nwarps * GPW) {
        const bool act = v0 + lane / T < NH;
        const int v = act ? v0 + lane / T : NH - 1;
        float2 x[8];
#pragma unroll
        for (int m = 0; m < 8; m++) x[m] = S[(int64_t)v * N + t + m * T];
        __syncwarp();
        tb::fft_run<N, -1>(x, t, xb, tw, [&](int j, float2 z) {
            if (act) S[(int64_t)v * N + j] = z;
        });
        __syncwarp();
    }
}

template <int N>
__global__ void __launch_bounds__(kSpecThreads) spec_kernel(const float* pad, float* spec, int pass) {
    __shared__ float2 tw[N];
    __shared__ float2 xbuf[(kSpecThreads / 32) * kXbufPerWarp];
    tb::build_twiddles<N>(tw);
    __syncthreads();
    if (pass == 0) spec_rows<N>(pad, spec, blockIdx.y, xbuf, tw);
    else spec_cols<N>(spec, blockIdx.y, xbuf, tw);
}

__global__ void spec_normalize_kernel(float* spec, int N) {
    const int img = blockIdx.y;
    float2* S = reinterpret_cast<float2*>(spec) + (int64_t)img * N * (N / 2 + 1);
    const float2 p00 = S[0];
    const float n = sqrtf(p00.x * p00.x + p00.y * p00.y);
    __syncthreads();
    if (n == 0.f) return;
    const int total = N * (N / 2 + 1);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        if (i == 0) continue;
        float2 z = S[i];
        S[i] = make_float2(z.x / n, z.y / n);
    }
}

__global__ void spec_normalize_dc_kernel(float* spec, int N) {
    float2* S = reinterpret_cast<float2*>(spec) + (int64_t)blockIdx.x * N * (N / 2 + 1);
    const float2 p00 = S[0];
    const float n = sqrtf(p00.x * p00.x + p00.y * p00.y);
    if (threadIdx.x == 0 && n != 0.f) S[0] = make_float2(p00.x / n, p00.y / n);
}

template <int N>
int launch_spec(const float* pad, float* spec, int n, cudaStream_t s) {
    constexpr int GPW = 32 / (N / 8);
    const int lines_per_cta = (kSpecThreads / 32) * GPW;
    dim3 g0((N + lines_per_cta - 1) / lines_per_cta, n);
    spec_kernel<N><<<g0, kSpecThreads, 0, s>>>(pad, spec, 0);
    dim3 g1((N / 2 + 1 + lines_per_cta - 1) / lines_per_cta, n);
    spec_kernel<N><<<g1, kSpecThreads, 0, s>>>(pad, spec, 1);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

}  // namespace

extern "C" int tb_psf_spectrum(const float* pad, float* spec, int32_t n, int32_t sz,
                               int32_t normalize, void* stream) {
    if (n < 0) return TB_ERR_ARG;
    if (n == 0) return TB_OK;
    if (!pad || !spec) return TB_ERR_ARG;
    if (n > 65535) return TB_ERR_SIZE;
    cudaStream_t s = (cudaStream_t)stream;
    int r;
    switch (sz) {
        case 32: r = launch_spec<32>(pad, spec, n, s); break;
        case 64: r = launch_spec<64>(pad, spec, n, s); break;
        case 128: r = launch_spec<128>(pad, spec, n, s); break;
        case 256: r = launch_spec<256>(pad, spec, n, s); break;
        default: return TB_ERR_SIZE;
    }
    if (r != TB_OK || !normalize) return r;
    // Divide every element by |P[0,0]| (the DC element last, after all blocks
    // have read it).
    dim3 g(64, n);
    spec_normalize_kernel<<<g, 256, 0, s>>>(spec, sz);
    spec_normalize_dc_kernel<<<n, 32, 0, s>>>(spec, sz);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}
