// Batched blob fitting (sm_100a): Levenberg-Marquardt on many independent
// blobs at once, each blob a few galaxies seen in several bands.  It is the
// batched form of Tractor.optimize / optimize_loop with LsqrOptimizer
// (tractor/lsqr_optimizer.py:280-326) over getDerivs + getChiImage
// (tractor/engine.py:279-339, 455-473), with ConstrainedOptimizer's bounds and
// maximum steps (tractor/constrained_optimizer.py:12-159).
//
// One iteration = three launches:
//   tb_fit_prep  one warp per source: the profile mixture (exp / deV /
//                Sersic) and its derivative with respect to the Sersic index,
//                the pixel-space shape factor M = T T^T and its derivatives
//                with respect to (log r_e, ee1, ee2) -- FP64 central
//                differences of the exact FP64 maps (sersic.py:288-342,
//                ellipses.py:165-263);
//   tb_fit_pass  one CTA per (blob, band) image, 32 x 8 pixel tiles: the
//                model (every source's PSF-convolved mixture, as
//                galaxy.py:307-326) and the analytic derivative columns
//                (position, flux, shape, index), weighted by inverr, staged
//                in shared memory; per tile A^T A, A^T r and r^T r added into
//                buffers the CTA owns (no atomics);
//   tb_fit_step  one CTA per blob: sums the band partials, accepts or
//                rejects the trial parameters, solves the Marquardt-damped
//                normal equations by FP64 Cholesky with one refinement step,
//                limits the step (bounds, maximum steps) and writes the next
//                trial parameters.
#include "profile_eval.cuh"

namespace {

constexpr int kPrepThreads = 128;      // 4 sources per block
constexpr int kMaxGalK = 10;           // galaxy components of one source
constexpr int kThreads = 256;          // pass CTA = one 32 x 8 tile, one pixel per thread
constexpr int kTileW = 32;
constexpr int kTileH = 8;
constexpr int kCols = 7;               // columns per (source, band): x y flux logre ee1 ee2 n
constexpr int kG = 4;                  // sources per shared-memory column group
constexpr int kLd = kThreads + 1;      // padded column stride (floats)
constexpr double kHn = 1e-5;           // central-difference step in n
constexpr double kHs = 1e-6;           // central-difference step in shape parameters

constexpr int kCompStride = kMaxGalK * TB_FIT_MAX_PSF;   // component slots per (source, band)

// Per-source summary written by tb_fit_prep.
struct SrcTab {
    double flux[TB_FIT_MAX_BANDS];
    float M[3];                    // T T^T (xx, xy, yy)
    float dM[3][3];                // d(T T^T) / d(logre, ee1, ee2)
    int32_t K[TB_FIT_MAX_BANDS];   // components in each band (galaxy x PSF)
    int32_t ok;
    double M64[3];                 // the same in FP64 (refinement pass)
    double dM64[3][3];
};

// One PSF-convolved component of a (source, band), written by tb_fit_prep:
// value, position and shape-derivative coefficients, the 1/2 of dN/dC
// folded in.  The mean stays FP64 (absolute pixels); the pass makes it
// tile-relative.
// The shape derivative of component k is dC_k = v_k dM (dM per source), the
// index derivative dC_k = dv_k M: the pass accumulates per source the
// moments sum_k val_k v_k u u^T and sum_k val_k dv_k u u^T over components
// and applies dM / M once per source and pixel.
struct FitC {
    double mx, my;
    float qxx, qxy, qyy;      // exponent, log2 units
    float ixx, ixy, iyy;      // C^-1
    float s;                  // unit-flux amplitude a / (2 pi sqrt det)
    float sn;                 // d a / d n / (2 pi sqrt det)
    float fl;                 // exponent floor, log2 units
    float v, dv;              // the galaxy component's variance and d/dn
    float t[4];               // tr(C^-1 dM_j) (j < 3), tr(C^-1 M)
    int32_t pad[7];
};

// The same component in FP64 for the refinement pass (tb_fit_refine): the
// model and its derivative columns evaluated in FP64 at the end of a fit.
struct FitC64 {
    double mx, my;
    double i00, i01, i11;     // C^-1
    double s, sn;             // a / (2 pi sqrt det), d a / d n / (2 pi sqrt det)
    double v, dv;             // galaxy variance and d/dn
    double t[4];              // tr(C^-1 dM_j) (j < 3), tr(C^-1 M)
    double pad[3];
};

// One component staged for one pixel row y of a tile (origin (ox, oy)) by
// the warp that owns the row: its FP32 tile-relative mean x, the exponent
// along the row e(dx) = qxx dx^2 + bx dx + c0 (bx = qxy dy, c0 = qyy dy^2,
// dy = y - my), C^-1 u = (ixx dx + uxy, ixy dx + uyy) (uxy = ixy dy,
// uyy = iyy dy), and the per-component factors of FitC.
struct __align__(16) FitR {
    float mx, qxx, bx, c0;
    float s, fl, ixx, ixy;
    float uxy, uyy, sn, v;
    float dv, t0, t1, t2;
    float t3, pad[3];
};

// ---------------------------------------------------------------------------
// prep
// ---------------------------------------------------------------------------

__device__ void shape_M(const double* cd, double s0, double s1, double s2, double M[3]) {
    double G[4], re;
    tb::shape_basis(TB_SHAPE_ELLIPSE_ESOFT, s0, s1, s2, G, re);
    tb::pixel_factor(cd, G, M[0], M[1], M[2]);
}

__global__ void __launch_bounds__(kPrepThreads)
fit_prep_kernel(const tb_fit_source* __restrict__ srcs, int n, const double* __restrict__ params,
                int n_bands, const tb_fit_unit* __restrict__ units, int n_units,
                tb_profile_tables Tg, double cd0, double cd1, double cd2, double cd3,
                SrcTab* __restrict__ tab, FitC* __restrict__ comps,
                FitC64* __restrict__ comps64, const tb_fit_state* __restrict__ state) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const tb_profile_tables T = tb::stage_tables(Tg, smem_raw);
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * (kPrepThreads / 32) + (threadIdx.x >> 5);
    if (i >= n) return;
    const tb_fit_source s = srcs[i];
    // a converged or stopped blob's tables stay as they are (nothing reads them)
    if (state && s.blob >= 0 && (int64_t)(s.blob + 1) * n_bands <= n_units &&
        state[s.blob].status != 0)
        return;
    const double* p = params + (int64_t)i * TB_FIT_NPAR;
    const double cd[4] = {cd0, cd1, cd2, cd3};
    int ok = s.blob >= 0 && (int64_t)(s.blob + 1) * n_bands <= n_units;
    double a = 0.0, v = 0.0, da = 0.0, dv = 0.0;
    int K = 0;
    if (s.profile == TB_PROFILE_SERSIC) {
        double nn = p[8];
        const double lowest = T.range_lohi[0], highest = T.range_lohi[2 * T.n_ranges - 1];
        int r = -1;
        bool clamped = false;
        if (nn <= lowest) { r = 0; nn = lowest; clamped = true; }
        else if (nn >= highest) { r = T.n_ranges - 1; nn = highest; clamped = true; }
        else {
            for (int q = 0; q < T.n_ranges; q++)
                if (T.range_lohi[2 * q] <= nn && nn < T.range_lohi[2 * q + 1]) { r = q; break; }
        }
        if (r < 0 || T.range_info[4 * r] + 1 > kMaxGalK) {
            ok = 0;
        } else {
            const bool core = nn > 1.0;
            K = tb::sersic_fixed(T, r, nn, core, lane, a, v);
            if (!clamped) {
                double ap, vp, am, vm;
                tb::sersic_fixed(T, r, nn + kHn, core, lane, ap, vp);
                tb::sersic_fixed(T, r, nn - kHn, core, lane, am, vm);
                da = (ap - am) / (2.0 * kHn);
                dv = (vp - vm) / (2.0 * kHn);
            }
            // components sorted by variance (sersic.py:338-341); the sort is
            // a permutation of lanes, kept fixed for the derivative
            const int rank = tb::variance_rank(v, K, lane);
            double a2 = 0.0, v2 = 0.0, da2 = 0.0, dv2 = 0.0;
            for (int j = 0; j < K; j++) {
                const int rj = __shfl_sync(0xffffffffu, rank, j);
                const double aj = __shfl_sync(0xffffffffu, a, j);
                const double vj = __shfl_sync(0xffffffffu, v, j);
                const double daj = __shfl_sync(0xffffffffu, da, j);
                const double dvj = __shfl_sync(0xffffffffu, dv, j);
                if (rj == lane) { a2 = aj; v2 = vj; da2 = daj; dv2 = dvj; }
            }
            a = a2; v = v2; da = da2; dv = dv2;
        }
    } else if (s.profile == TB_PROFILE_EXP || s.profile == TB_PROFILE_DEV) {
        K = tb::warp_profile(T, s.profile, 0.0, lane, kMaxGalK, a, v);
        if (K < 0) { ok = 0; K = 0; }
    } else if (s.profile == TB_PROFILE_POINT) {
        K = 1;
        a = lane == 0 ? 1.0 : 0.0;
    } else {
        ok = 0;
    }
    // shape factor and its derivatives (every lane, redundantly)
    double M[3] = {0.0, 0.0, 0.0};
    double dM[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    if (s.profile != TB_PROFILE_POINT) {
        const double* sh = p + 5;
        shape_M(cd, sh[0], sh[1], sh[2], M);
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double hp[3] = {sh[0], sh[1], sh[2]}, hm[3] = {sh[0], sh[1], sh[2]};
            hp[j] += kHs;
            hm[j] -= kHs;
            double Mp[3], Mm[3];
            shape_M(cd, hp[0], hp[1], hp[2], Mp);
            shape_M(cd, hm[0], hm[1], hm[2], Mm);
#pragma unroll
            for (int q = 0; q < 3; q++) dM[j][q] = (Mp[q] - Mm[q]) / (2.0 * kHs);
        }
    }
    bool fin = isfinite(p[0]) && isfinite(p[1]);
    for (int q = 0; q < 3; q++) fin = fin && isfinite(M[q]);
    ok = ok && fin;
    // components per band: PSF component p (outer) x galaxy component gi
    // (inner), mixture_profiles.py:158-172
    int Kb[TB_FIT_MAX_BANDS] = {0, 0, 0};
    for (int bd = 0; bd < n_bands; bd++) {
        const tb_fit_unit* u = ok ? units + (int64_t)s.blob * n_bands + bd : units;
        const int Kp = u->psf_K;
        if (Kp < 1 || Kp > TB_FIT_MAX_PSF) ok = 0;
        const int Kt = ok ? K * Kp : 0;
        Kb[bd] = Kt;
        for (int k0 = 0; k0 < kCompStride; k0 += 32) {
            const int k = k0 + lane;
            const int gi = (Kt > 0 && k < Kt) ? k % K : 0;
            const int pp = (Kt > 0 && k < Kt) ? k / K : 0;
            const double ag = __shfl_sync(0xffffffffu, a, gi);
            const double vg = __shfl_sync(0xffffffffu, v, gi);
            const double dag = __shfl_sync(0xffffffffu, da, gi);
            const double dvg = __shfl_sync(0xffffffffu, dv, gi);
            if (k >= Kt) continue;
            const double C00 = vg * M[0] + u->psf_var[4 * pp];
            const double C01 = vg * M[1] + 0.5 * (u->psf_var[4 * pp + 1] + u->psf_var[4 * pp + 2]);
            const double C11 = vg * M[2] + u->psf_var[4 * pp + 3];
            const double det = C00 * C11 - C01 * C01;
            const double i00 = C11 / det, i01 = -C01 / det, i11 = C00 / det;
            const double norm = 1.0 / (2.0 * TB_PI * sqrt(det));
            FitC c;
            c.mx = p[0] + u->psf_mean[2 * pp];
            c.my = p[1] + u->psf_mean[2 * pp + 1];
            c.qxx = (float)(-0.5 * TB_LOG2E * i00);
            c.qxy = (float)(-TB_LOG2E * i01);
            c.qyy = (float)(-0.5 * TB_LOG2E * i11);
            c.ixx = (float)i00;
            c.ixy = (float)i01;
            c.iyy = (float)i11;
            c.s = (float)(ag * u->psf_amp[pp] * norm);
            c.sn = (float)(dag * u->psf_amp[pp] * norm);
            c.fl = (float)(-50.0 * TB_LOG2E);
            c.v = (float)vg;
            c.dv = (float)dvg;
            // dC / d(logre, ee1, ee2) = v dM_j; dC / dn = dv M
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const double* d = j < 3 ? dM[j] : M;
                c.t[j] = (float)(i00 * d[0] + 2.0 * i01 * d[1] + i11 * d[2]);
            }
#pragma unroll
            for (int q = 0; q < 7; q++) c.pad[q] = 0;
            const bool good = det > 0.0 && isfinite(norm);
            if (!good) ok = 0;
            comps[((int64_t)i * n_bands + bd) * kCompStride + k] = c;
            FitC64 c6;
            c6.mx = c.mx;
            c6.my = c.my;
            c6.i00 = i00;
            c6.i01 = i01;
            c6.i11 = i11;
            c6.s = ag * u->psf_amp[pp] * norm;
            c6.sn = dag * u->psf_amp[pp] * norm;
            c6.v = vg;
            c6.dv = dvg;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const double* d = j < 3 ? dM[j] : M;
                c6.t[j] = i00 * d[0] + 2.0 * i01 * d[1] + i11 * d[2];
            }
            c6.pad[0] = c6.pad[1] = c6.pad[2] = 0.0;
            comps64[((int64_t)i * n_bands + bd) * kCompStride + k] = c6;
        }
    }
    ok = __all_sync(0xffffffffu, ok);
    if (lane == 0) {
        SrcTab t;
        for (int bd = 0; bd < TB_FIT_MAX_BANDS; bd++) {
            t.flux[bd] = bd < n_bands ? p[2 + bd] : 0.0;
            t.K[bd] = bd < n_bands ? Kb[bd] : 0;
        }
        t.ok = ok;
        for (int q = 0; q < 3; q++) {
            t.M[q] = (float)M[q];
            t.M64[q] = M[q];
            for (int j = 0; j < 3; j++) {
                t.dM[j][q] = (float)dM[j][q];
                t.dM64[j][q] = dM[j][q];
            }
        }
        tab[i] = t;
    }
}

// ---------------------------------------------------------------------------
// pass
// ---------------------------------------------------------------------------

// One source of the unit (its mask rectangle and shape factors in the
// unit's band), copied to shared memory once per unit.
struct UnitSrc {
    int32_t x0, y0, x1, y1;   // mask [x0, x1) x [y0, y1), image pixels; an empty mask is all 0
    float counts;             // flux in the unit's band
    int32_t K;                // components (galaxy x PSF) in the unit's band
    float M[3];               // T T^T (xx, xy, yy)
    float dM[3][3];           // its shape derivatives
};

struct PassSmem {
    float A[2][kG * kCols][kLd];            // two column groups (multi-source tiles)
    float hstage[kG * kCols][kG * kCols];   // a block of A^T A before its global update
    float gstage[kG * kCols];               // a group's A^T r before its global update
    FitR wc[kThreads / 32][kCompStride];    // each warp's components staged for its pixel row
    UnitSrc us[TB_FIT_MAX_SRC];
    float r[kThreads];
    float runred[kThreads / 32][36];
    double red[kThreads / 32];
    int64_t slot;
    int skip;
};

// Stages, by one warp, the components of one source (src_comps[0, K)) that
// reach pixels [x0, x1] (tile-relative, inclusive) of row y of the tile at
// (ox, oy) into wc[0 ..), in their order; returns how many.  Along a row
// the exponent is a concave quadratic in dx whose maximum over the segment
// is at its vertex clamped to the segment.  A component whose maximum
// stays below its floor (minus a margin of 1, far above FP32 rounding)
// contributes exactly zero to every pixel of the segment (E = 0, val = 0)
// and is left out, so the sums over the staged components are the same.
// Components with non-finite or non-concave coefficients are always staged.
// The row terms are computed as the per-pixel expressions would compute
// them, so every pixel's exponent and C^-1 u is bit-identical.
__device__ __forceinline__ int stage_row(FitR* wc, const FitC* __restrict__ src_comps, int K,
                                         int ox, int oy, int y, float x0, float x1) {
    const int lane = threadIdx.x & 31;
    int n = 0;
    __syncwarp();   // the warp's previous components are no longer read
    for (int k0 = 0; k0 < K; k0 += 32) {
        const int k = k0 + lane;
        bool keep = false;
        float mx = 0.f, dy = 0.f, bx = 0.f, c0 = 0.f;
        if (k < K) {
            const FitC& c = src_comps[k];
            mx = (float)(c.mx - (double)ox);
            dy = (float)y - (float)(c.my - (double)oy);
            bx = c.qxy * dy;
            c0 = c.qyy * dy * dy;
            const float qxx = c.qxx;
            const bool ok = isfinite(mx) && isfinite(bx) && isfinite(c0) && qxx < 0.f;
            float emax = 0.f;
            if (ok) {
                const float xs = fminf(fmaxf(mx - bx / (2.f * qxx), x0), x1);
                const float dx = xs - mx;
                emax = fmaf(dx, fmaf(qxx, dx, bx), c0);
            }
            keep = !ok || !(emax < c.fl - 1.f);
        }
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const FitC& c = src_comps[k];
            float4* f = reinterpret_cast<float4*>(wc + n + __popc(bal & ((1u << lane) - 1u)));
            f[0] = make_float4(mx, c.qxx, bx, c0);
            f[1] = make_float4(c.s, c.fl, c.ixx, c.ixy);
            f[2] = make_float4(c.ixy * dy, c.iyy * dy, c.sn, c.v);
            f[3] = make_float4(c.dv, c.t[0], c.t[1], c.t[2]);
            f[4] = make_float4(c.t[3], 0.f, 0.f, 0.f);
        }
        n += __popc(bal);
    }
    __syncwarp();   // staged components visible to the whole warp
    return n;
}

// One source at this thread's pixel (lane, warp) of the tile at (ox, oy):
// returns its model (counts x its PSF-convolved mixture, 0 outside its
// mask) and, with kDeriv, its 7 weighted derivative columns in J (0 outside
// the mask), d/dtheta = 1/2 (dM : sum v val u u^T - sum v val tr(C^-1 dM))
// for the shape and likewise (M, dv) for the index.  The warp stages the
// components that reach its row of the mask; a row outside the mask
// evaluates nothing.  No block barrier: each warp works on its own.
template <bool kDeriv>
__device__ __forceinline__ float eval_source(FitR* wc, const FitC* __restrict__ src_comps,
                                             const UnitSrc& U, int ox, int oy, float w,
                                             float* J) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int xa = max(U.x0 - ox, 0), xb = min(U.x1 - ox, kTileW);
    const bool row = warp >= U.y0 - oy && warp < U.y1 - oy && xa < xb;   // warp-uniform
    float m = 0.f, jx = 0.f, jy = 0.f, jn = 0.f;
    float axx = 0.f, axy = 0.f, ayy = 0.f, t0 = 0.f, t1 = 0.f, t2 = 0.f;
    float bxx = 0.f, bxy = 0.f, byy = 0.f, tn = 0.f;
    if (row) {
        const int K = stage_row(wc, src_comps, U.K, ox, oy, warp, (float)xa, (float)(xb - 1));
        const float xf = (float)lane;
#pragma unroll 2
        for (int g = 0; g < K; g++) {
            const FitR& c = wc[g];
            const float dx = xf - c.mx;
            const float e = fmaf(dx, fmaf(c.qxx, dx, c.bx), c.c0);
            const float E = (e >= c.fl) ? tb::ex2(e) : 0.f;
            const float val = c.s * E;
            m += val;
            if (kDeriv) {
                const float ux = fmaf(c.ixx, dx, c.uxy);
                const float uy = fmaf(c.ixy, dx, c.uyy);
                jx = fmaf(val, ux, jx);
                jy = fmaf(val, uy, jy);
                const float pxx = ux * ux, pxy = ux * uy, pyy = uy * uy;
                const float sv = val * c.v, wv = val * c.dv;
                axx = fmaf(sv, pxx, axx);
                axy = fmaf(sv, pxy, axy);
                ayy = fmaf(sv, pyy, ayy);
                t0 = fmaf(sv, c.t0, t0);
                t1 = fmaf(sv, c.t1, t1);
                t2 = fmaf(sv, c.t2, t2);
                bxx = fmaf(wv, pxx, bxx);
                bxy = fmaf(wv, pxy, bxy);
                byy = fmaf(wv, pyy, byy);
                tn = fmaf(wv, c.t3, tn);
                jn = fmaf(c.sn, E, jn);
            }
        }
    }
    const bool in = row && lane >= xa && lane < xb;
    const float cnt = U.counts;
    if (kDeriv) {
        const float cw = in ? cnt * w : 0.f;
        const float h = 0.5f * cw;
        J[0] = cw * jx;
        J[1] = cw * jy;
        J[2] = in ? w * m : 0.f;
        J[3] = h * (fmaf(U.dM[0][0], axx, fmaf(2.f * U.dM[0][1], axy, U.dM[0][2] * ayy)) - t0);
        J[4] = h * (fmaf(U.dM[1][0], axx, fmaf(2.f * U.dM[1][1], axy, U.dM[1][2] * ayy)) - t1);
        J[5] = h * (fmaf(U.dM[2][0], axx, fmaf(2.f * U.dM[2][1], axy, U.dM[2][2] * ayy)) - t2);
        J[6] = h * (fmaf(U.M[0], bxx, fmaf(2.f * U.M[1], bxy, U.M[2] * byy)) - tn) + cw * jn;
    }
    return in ? cnt * m : 0.f;
}

// Position of the (q+1)-th set bit of m (q < popc(m)).
__device__ __forceinline__ int nth_bit(unsigned m, int q) {
    for (int i = 0; i < q; i++) m &= m - 1u;
    return __ffs(m) - 1;
}

// Sources q0 .. q0 + nq - 1 of the tile's hit list (the set bits of `hit`,
// in source order) at this thread's pixel: returns their model; with
// kDeriv writes the 7 columns of source q at A[7 (q - q0) + c][thread].
// No block barrier inside.
template <bool kDeriv>
__device__ float eval_group(PassSmem& sm, const FitC* __restrict__ band_comps, int n_bands,
                            unsigned hit, int q0, int nq, int ox, int oy, float w,
                            float (*A)[kLd]) {
    const int tid = threadIdx.x, warp = tid >> 5;
    unsigned mm = hit;
    for (int i = 0; i < q0; i++) mm &= mm - 1u;
    float model = 0.f;
    for (int q = q0; q < q0 + nq; q++) {
        const int s = __ffs(mm) - 1;
        mm &= mm - 1u;
        float J[kCols];
        model += eval_source<kDeriv>(sm.wc[warp], band_comps + (int64_t)s * n_bands * kCompStride,
                                     sm.us[s], ox, oy, w, J);
        if (kDeriv) {
            float* col = &A[(q - q0) * kCols][tid];
#pragma unroll
            for (int c = 0; c < kCols; c++) col[c * kLd] = J[c];
        }
    }
    return model;
}

__device__ __forceinline__ int col_of(int src, int c, int band) {
    // parameter slots per source: x, y, flux[3], logre, ee1, ee2, n
    const int off = c < 2 ? c : (c == 2 ? 2 + band : c + 2);
    return src * TB_FIT_NPAR + off;
}

// Adds a single-source run's register accumulators (this thread's share of
// the 7 x 7 block's upper triangle and of A^T r) into the owned H / g:
// warp reductions, then a fixed-order sum over warps.
__device__ void flush_run(PassSmem& sm, float* hacc, float* gacc, int src, double* H, double* g,
                          int P, int band) {
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int v = 0; v < 35; v++) {
        float x = v < 28 ? hacc[v] : gacc[v - 28];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sm.runred[warp][v] = x;
    }
    __syncthreads();
    if (tid < 35) {
        double sum = 0.0;
        for (int w2 = 0; w2 < kThreads / 32; w2++) sum += (double)sm.runred[w2][tid];
        if (tid < 28) {
            // upper-triangle index tid -> (c, c'), row-major over c <= c'
            int c = 0, base = 0;
            while (base + (kCols - c) <= tid) { base += kCols - c; c++; }
            const int c2 = c + (tid - base);
            const int r = col_of(src, c, band), cc = col_of(src, c2, band);
            H[(int64_t)r * P + cc] += sum;
        } else {
            g[col_of(src, tid - 28, band)] += sum;
        }
    }
    __syncthreads();
}

// A_a^T A_b of the column groups in Aa (na sources) and Ab (nb sources)
// into hstage (upper triangle when diag) and, with grad, A_a^T r into
// gstage.  Tasks of 2 x 2 column pairs (or 2 gradient columns) go to the
// warps in turn; each task splits the tile's pixels over the lanes
// (conflict-free consecutive shared-memory reads), then reduces.
__device__ void stage_products(PassSmem& sm, float (*Aa)[kLd], int na, float (*Ab)[kLd], int nb,
                               bool diag, bool grad) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ca = na * kCols, cb = nb * kCols;
    const int ba = (ca + 1) / 2, bb = (cb + 1) / 2;
    const int nblk = diag ? ba * (ba + 1) / 2 : ba * bb;
    const int ntask = nblk + (grad ? ba : 0);
    for (int e = warp; e < ntask; e += kThreads / 32) {
        if (e < nblk) {
            int bi, bj;
            if (diag) {   // row-major over the upper triangle of 2 x 2 blocks
                int t = e;
                bi = 0;
                while (t >= ba - bi) { t -= ba - bi; bi++; }
                bj = bi + t;
            } else {
                bi = e / bb;
                bj = e % bb;
            }
            const int i = 2 * bi, j = 2 * bj;
            const int i1 = min(i + 1, ca - 1), j1 = min(j + 1, cb - 1);
            float s00 = 0.f, s01 = 0.f, s10 = 0.f, s11 = 0.f;
#pragma unroll
            for (int p = lane; p < kThreads; p += 32) {
                const float x0 = Aa[i][p], x1 = Aa[i1][p], y0 = Ab[j][p], y1 = Ab[j1][p];
                s00 = fmaf(x0, y0, s00);
                s01 = fmaf(x0, y1, s01);
                s10 = fmaf(x1, y0, s10);
                s11 = fmaf(x1, y1, s11);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                s00 += __shfl_xor_sync(0xffffffffu, s00, o);
                s01 += __shfl_xor_sync(0xffffffffu, s01, o);
                s10 += __shfl_xor_sync(0xffffffffu, s10, o);
                s11 += __shfl_xor_sync(0xffffffffu, s11, o);
            }
            if (lane < 4) {
                const int di = lane >> 1, dj = lane & 1;
                const int ii = i + di, jj = j + dj;
                if (ii < ca && jj < cb && !(diag && jj < ii))
                    sm.hstage[ii][jj] = di == 0 ? (dj == 0 ? s00 : s01) : (dj == 0 ? s10 : s11);
            }
        } else {
            const int i = 2 * (e - nblk), i1 = min(i + 1, ca - 1);
            float s0 = 0.f, s1 = 0.f;
#pragma unroll
            for (int p = lane; p < kThreads; p += 32) {
                const float rp = sm.r[p];
                s0 = fmaf(Aa[i][p], rp, s0);
                s1 = fmaf(Aa[i1][p], rp, s1);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                s0 += __shfl_xor_sync(0xffffffffu, s0, o);
                s1 += __shfl_xor_sync(0xffffffffu, s1, o);
            }
            if (lane == 0) sm.gstage[i] = s0;
            if (lane == 1 && i + 1 < ca) sm.gstage[i + 1] = s1;
        }
    }
}

// The staged products' global updates by all threads at once (each element
// of the owned H / g once: independent read-modify-writes).  Column c of
// group a belongs to hit source qa0 + c / 7 (likewise for b).
__device__ void apply_products(PassSmem& sm, unsigned hit, int qa0, int na, int qb0, int nb,
                               bool diag, bool grad, double* H, double* g, int P, int band) {
    const int ca = na * kCols, cb = nb * kCols;
    for (int e = threadIdx.x; e < ca * cb; e += kThreads) {
        const int ii = e / cb, jj = e % cb;
        if (diag && jj < ii) continue;
        const int ga = col_of(nth_bit(hit, qa0 + ii / kCols), ii % kCols, band);
        const int gb = col_of(nth_bit(hit, qb0 + jj / kCols), jj % kCols, band);
        // upper triangle in global parameter order
        const int r = min(ga, gb), c = max(ga, gb);
        H[(int64_t)r * P + c] += (double)sm.hstage[ii][jj];
    }
    if (grad)
        for (int c = threadIdx.x; c < ca; c += kThreads)
            g[col_of(nth_bit(hit, qa0 + c / kCols), c % kCols, band)] += (double)sm.gstage[c];
}

__global__ void __launch_bounds__(kThreads, 2)
fit_pass_kernel(const tb_fit_unit* __restrict__ units, const int32_t* __restrict__ order,
                int n_units, const tb_fit_blob* __restrict__ blobs,
                const tb_fit_source* __restrict__ srcs, const SrcTab* __restrict__ tab,
                const FitC* __restrict__ gcomps, const float* __restrict__ data,
                const float* __restrict__ inverr, double* __restrict__ hbuf,
                double* __restrict__ gbuf, double* __restrict__ chi2_part,
                const tb_fit_state* __restrict__ state, int n_bands,
                const int32_t* __restrict__ tiles, double* __restrict__ chi2_const, int mode,
                int32_t* counter, tb_status* st) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PassSmem& sm = *reinterpret_cast<PassSmem*>(smem_raw);
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    for (;;) {
        const int64_t oi = tb::next_unit(counter, &sm.slot);   // barriers on both sides
        if (oi >= n_units) break;
        const int ui = order[oi];
        if (ui < 0 || ui >= n_units) {
            if (tid == 0) tb::report(st, TB_STATUS_BAD_ITEM, (int)oi, ui);
            continue;
        }
        const tb_fit_unit& u = units[ui];
        const tb_fit_blob b = blobs[u.blob];
        if (mode == 0 && state[u.blob].status != 0) continue;   // converged or stopped
        const int P = b.P;
        const int nsrc = b.n_src;
        double* H = hbuf + b.h_off + (int64_t)u.slice * P * P;
        double* g = gbuf + b.g_off + (int64_t)u.slice * P;
        if (mode == 0) {
            for (int e = tid; e < P * P; e += kThreads) H[e] = 0.0;
            for (int e = tid; e < P; e += kThreads) g[e] = 0.0;
        }
        // checks, and the unit's sources into shared memory (lane = source)
        if (warp == 0) {
            const bool unit_bad = nsrc < 0 || nsrc > TB_FIT_MAX_SRC || P != nsrc * TB_FIT_NPAR ||
                                  u.psf_K < 1 || u.psf_K > TB_FIT_MAX_PSF || u.band < 0 ||
                                  u.band >= n_bands || u.slice < 0 || u.slice >= b.n_slices ||
                                  u.t0 < 0 || u.t1 < u.t0 || u.t1 > b.n_active;
            bool src_bad = false;
            if (!unit_bad && lane < nsrc) {
                const SrcTab& S = tab[b.src0 + lane];
                const int K = S.K[u.band];
                src_bad = !S.ok || K < 0 || K > kCompStride;
                const tb_fit_source fs = srcs[b.src0 + lane];
                const bool live = fs.w > 0 && fs.h > 0;
                UnitSrc U;
                U.x0 = live ? fs.x0 : 0;
                U.y0 = live ? fs.y0 : 0;
                U.x1 = live ? fs.x0 + fs.w : 0;
                U.y1 = live ? fs.y0 + fs.h : 0;
                U.counts = (float)S.flux[u.band];
                U.K = K;
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    U.M[q] = S.M[q];
#pragma unroll
                    for (int j = 0; j < 3; j++) U.dM[j][q] = S.dM[j][q];
                }
                sm.us[lane] = U;
            }
            const bool bad = unit_bad || __any_sync(0xffffffffu, src_bad);
            if (lane == 0) {
                sm.skip = bad;
                if (bad) tb::report(st, TB_STATUS_BAD_ITEM, ui, nsrc);
            }
        }
        __syncthreads();
        if (sm.skip) {
            if (tid == 0) {
                if (mode == 0) chi2_part[b.unit0 + u.slice] = INFINITY;
                else chi2_const[b.unit0 + u.slice] = INFINITY;
            }
            continue;
        }
        // the unit's band of source s: band_comps + s * n_bands * kCompStride
        const FitC* band_comps = gcomps + ((int64_t)b.src0 * n_bands + u.band) * kCompStride;
        double chi2 = 0.0;
        // mode 0: the unit's range of the tiles some source's mask reaches;
        // mode 1: the others (their chi^2 does not depend on the parameters),
        // covered by the unit that starts the range
        const int n_t = mode == 0 ? u.t1 - u.t0 : (u.t0 == 0 ? b.n_tiles - b.n_active : 0);
        const int32_t* tl = tiles + b.tile_off + (mode == 0 ? u.t0 : b.n_active);
        // this thread's pixel of tile t (0 outside the image)
        auto load_px = [&](int t, float& d, float& w) {
            d = 0.f;
            w = 0.f;
            if (t >= n_t) return;
            const int px = (tl[t] & 0x3ff) * kTileW + lane, py = ((tl[t] >> 10) & 0x3ff) * kTileH + warp;
            if (px < u.W && py < u.H) {
                const int64_t pix = u.pix_off + (int64_t)py * u.W + px;
                d = data[pix];
                w = inverr[pix];
            }
        };
        float d_next, w_next;
        load_px(0, d_next, w_next);
        // single-source runs: this thread's pixel contributions to the run's
        // 7 x 7 block (upper triangle) and gradient
        int run_src = -1;
        float hacc[28], gacc[7];
        for (int t = 0; t < n_t; t++) {
            const int ox = (tl[t] & 0x3ff) * kTileW, oy = ((tl[t] >> 10) & 0x3ff) * kTileH;
            const int single = mode == 0 ? ((tl[t] >> 20) & 0xff) - 1 : -1;
            const float d = d_next, w = w_next;
            load_px(t + 1, d_next, w_next);   // prefetch the next tile's pixel
            if (single != run_src) {
                if (run_src >= 0) flush_run(sm, hacc, gacc, run_src, H, g, P, u.band);
                run_src = single;
#pragma unroll
                for (int v = 0; v < 28; v++) hacc[v] = 0.f;
#pragma unroll
                for (int v = 0; v < 7; v++) gacc[v] = 0.f;
            }
            if (single >= 0 && single < nsrc) {
                // one source: every warp on its own row, no block barrier
                float J[kCols];
                const float model = eval_source<true>(
                    sm.wc[warp], band_comps + (int64_t)single * n_bands * kCompStride,
                    sm.us[single], ox, oy, w, J);
                const float rr = (d - model) * w;
                chi2 += (double)(rr * rr);
                int v = 0;
#pragma unroll
                for (int c = 0; c < kCols; c++) {
                    gacc[c] = fmaf(J[c], rr, gacc[c]);
#pragma unroll
                    for (int c2 = c; c2 < kCols; c2++, v++) hacc[v] = fmaf(J[c], J[c2], hacc[v]);
                }
                continue;
            }
            // sources whose mask meets this tile, in source order (every warp
            // finds the same set); mode 1 tiles meet none by construction
            bool meets = false;
            if (mode == 0 && lane < nsrc) {
                const UnitSrc& U = sm.us[lane];
                meets = U.x0 < ox + kTileW && U.x1 > ox && U.y0 < oy + kTileH && U.y1 > oy;
            }
            const unsigned hit = __ballot_sync(0xffffffffu, meets);
            const int R = __popc(hit);
            if (R == 0) {
                const float rr = d * w;
                chi2 += (double)(rr * rr);
                continue;
            }
            // Shared A, r, hstage and gstage are written only after the
            // previous multi-source tile's reads of them have passed a
            // barrier: A and r are read before its second barrier, hstage
            // and gstage after it and are written here only after this
            // tile's first barrier.
            const int ngroups = (R + kG - 1) / kG;
            float model = 0.f;
            if (ngroups == 1) {
                model = eval_group<true>(sm, band_comps, n_bands, hit, 0, R, ox, oy, w, sm.A[0]);
            } else {
                for (int q0 = 0; q0 < R; q0 += kG)
                    model += eval_group<false>(sm, band_comps, n_bands, hit, q0, min(kG, R - q0),
                                               ox, oy, w, sm.A[0]);
            }
            const float rr = (d - model) * w;
            chi2 += (double)(rr * rr);
            sm.r[tid] = rr;
            for (int ga = 0; ga < ngroups; ga++) {
                const int qa = ga * kG, na = min(kG, R - qa);
                if (ngroups > 1)
                    eval_group<true>(sm, band_comps, n_bands, hit, qa, na, ox, oy, w, sm.A[0]);
                __syncthreads();   // columns (and r) complete; earlier updates applied
                stage_products(sm, sm.A[0], na, sm.A[0], na, true, true);
                __syncthreads();
                apply_products(sm, hit, qa, na, qa, na, true, true, H, g, P, u.band);
                for (int gb = ga + 1; gb < ngroups; gb++) {
                    const int qb = gb * kG, nb = min(kG, R - qb);
                    eval_group<true>(sm, band_comps, n_bands, hit, qb, nb, ox, oy, w, sm.A[1]);
                    __syncthreads();
                    stage_products(sm, sm.A[0], na, sm.A[1], nb, false, false);
                    __syncthreads();
                    apply_products(sm, hit, qa, na, qb, nb, false, false, H, g, P, u.band);
                }
            }
        }
        if (run_src >= 0) flush_run(sm, hacc, gacc, run_src, H, g, P, u.band);
        // chi^2 of the unit: fixed-order block reduction
        for (int o = 16; o > 0; o >>= 1) chi2 += __shfl_xor_sync(0xffffffffu, chi2, o);
        if (lane == 0) sm.red[warp] = chi2;
        __syncthreads();
        if (tid == 0) {
            double s = 0.0;
            for (int w2 = 0; w2 < kThreads / 32; w2++) s += sm.red[w2];
            if (mode == 0) chi2_part[b.unit0 + u.slice] = s + chi2_const[b.unit0 + u.slice];
            else chi2_const[b.unit0 + u.slice] = s;
        }
    }
}

// ---------------------------------------------------------------------------
// step
// ---------------------------------------------------------------------------

constexpr int kStepThreads = 256;

__device__ double max_step(int off) {
    // PixPos [1, 1] (wcs.py:384), fluxes unlimited, EllipseESoft inherits
    // EllipseE's [1, 0.1, 0.1] (ellipses.py:48), SersicIndex 0.1 (sersic.py:352)
    switch (off) {
        case 0: case 1: case 5: return 1.0;
        case 6: case 7: case 8: return 0.1;
        default: return 0.0;   // none
    }
}

// ---------------------------------------------------------------------------
// refinement pass (tb_fit_refine): the normal equations of the running blobs
// in FP64 -- the model, the seven derivative columns of every source, the
// residuals, A^T A, A^T r and chi^2 -- written over the slices tb_fit_pass
// fills.  Near the optimum the gradient is a sum of terms that cancel, FP32
// chi^2 cannot verify gains below ~1e-4, and an FP32 A^T A (FP32 columns:
// the index column is a difference of nearly equal sums) is too inexact for
// the steps of an ill-conditioned blob to converge; the final iterations of
// a fit take all of them in FP64.  Same units, slices and layout as
// tb_fit_pass.
// ---------------------------------------------------------------------------
constexpr int kRefThreads = 256;       // one 32 x 8 tile, one pixel per thread
constexpr int kRefChunks = 8;          // 16-value chunks staged before a flush

struct RefSrc {
    int32_t x0, y0, x1, y1;
    int32_t K, profile;
    double counts;
    double M[3];
    double dM[3][3];
};

struct RefSmem {
    RefSrc us[TB_FIT_MAX_SRC];
    double red[kRefThreads / 32][kRefChunks * 16];
    int dst[kRefChunks * 16];   // >= 0: H index; <= -2: g index -dst - 2; -1: none
    int64_t slot;
    int skip;
};

// Sum over the warp of v[0 .. 16): afterwards lanes 2k and 2k + 1 hold the
// sum of v[k] (a reduce-scatter: 16 shuffles instead of 16 x 5).
__device__ __forceinline__ double warp_reduce_scatter16(double (&v)[16], int lane) {
    {
        const bool hi = lane & 16;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const double send = hi ? v[i] : v[i + 8];
            const double keep = hi ? v[i + 8] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
        }
    }
    {
        const bool hi = lane & 8;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const double send = hi ? v[i] : v[i + 4];
            const double keep = hi ? v[i + 4] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
        }
    }
    {
        const bool hi = lane & 4;
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const double send = hi ? v[i] : v[i + 2];
            const double keep = hi ? v[i + 2] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
        }
    }
    {
        const bool hi = lane & 2;
        const double send = hi ? v[0] : v[1];
        const double keep = hi ? v[1] : v[0];
        v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
    }
    return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
}

// The staged chunks summed over the warps and added to their destinations
// (each destination at most once per flush: a flush never spans two tiles).
__device__ void ref_flush(RefSmem& sm, int& nc, double* H, double* g) {
    __syncthreads();
    for (int j = threadIdx.x; j < nc * 16; j += kRefThreads) {
        const int d = sm.dst[j];
        if (d == -1) continue;
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kRefThreads / 32; w++) s += sm.red[w][j];
        if (d >= 0) H[d] += s;
        else g[-d - 2] += s;
    }
    __syncthreads();
    nc = 0;
}

// Stages NV values (value(q), q a compile-time index after unrolling) in
// chunks of 16, their destinations dest(q) (run time, warp 0).
template <int NV, class Val, class Dst>
__device__ __forceinline__ void ref_emit(RefSmem& sm, int& nc, double* H, double* g, Val value,
                                         Dst dest) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c0 = 0; c0 < NV; c0 += 16) {
        double v[16];
#pragma unroll
        for (int k = 0; k < 16; k++) v[k] = c0 + k < NV ? value(c0 + k) : 0.0;
        const double s = warp_reduce_scatter16(v, lane);
        const int k = lane >> 1;
        if (!(lane & 1)) {
            sm.red[warp][nc * 16 + k] = s;
            if (warp == 0) sm.dst[nc * 16 + k] = c0 + k < NV ? dest(c0 + k) : -1;
        }
        if (++nc == kRefChunks) ref_flush(sm, nc, H, g);
    }
}

// (i, j), i <= j < 7, of the q-th element of a 7 x 7 upper triangle
// (row-major; rows start at 0, 7, 13, 18, 22, 25, 27).  Branch-free, so that
// a compile-time q folds to constants.
__host__ __device__ constexpr int tri_row(int q) {
    return (q >= 7) + (q >= 13) + (q >= 18) + (q >= 22) + (q >= 25) + (q >= 27);
}
__host__ __device__ constexpr int tri_col(int q) {
    return q - (tri_row(q) * 7 - tri_row(q) * (tri_row(q) - 1) / 2) + tri_row(q);
}

// Parameter slot of column i (x y flux(band) logre ee1 ee2 n) of source sI;
// -1 where the profile has no such parameter.
__device__ __forceinline__ int ref_slot(int sI, int profile, int band, int i) {
    if (i >= 3 && profile == TB_PROFILE_POINT) return -1;
    if (i == 6 && profile != TB_PROFILE_SERSIC) return -1;
    const int base = sI * TB_FIT_NPAR;
    return i < 2 ? base + i : i == 2 ? base + 2 + band : base + 2 + i;
}

// Source R's model at (px, py) (counts x its unit-flux mixture), FP64.
__device__ __forceinline__ double ref_model(const RefSrc& R, const FitC64* cs, int px, int py) {
    if (!(px >= R.x0 && px < R.x1 && py >= R.y0 && py < R.y1)) return 0.0;
    double val = 0.0;
    for (int k = 0; k < R.K; k++) {
        const FitC64& c = cs[k];
        const double dx = px - c.mx, dy = py - c.my;
        const double ux = c.i00 * dx + c.i01 * dy, uy = c.i01 * dx + c.i11 * dy;
        const double e = -0.5 * (dx * ux + dy * uy);
        if (e >= -50.0) val += c.s * tb::exp_taylor(fmin(e, 0.0));
    }
    return R.counts * val;
}

// Source R's seven derivative columns at (px, py) (zero outside its
// rectangle) and its model there, FP64: per component the moments of
// C^-1 u (u = pixel - mean) that d/d(mean, C, amplitude) produce, combined
// once per source with dM (shape) and M (index).
__device__ __forceinline__ double ref_cols(const RefSrc& R, const FitC64* cs, int px, int py,
                                           double (&J)[7]) {
#pragma unroll
    for (int j = 0; j < 7; j++) J[j] = 0.0;
    if (!(px >= R.x0 && px < R.x1 && py >= R.y0 && py < R.y1)) return 0.0;
    double S0 = 0, Sx = 0, Sy = 0, Axx = 0, Axy = 0, Ayy = 0, At0 = 0, At1 = 0, At2 = 0;
    double Dxx = 0, Dxy = 0, Dyy = 0, Dt = 0, Sn = 0;
    for (int k = 0; k < R.K; k++) {
        const FitC64& c = cs[k];
        const double dx = px - c.mx, dy = py - c.my;
        const double ux = c.i00 * dx + c.i01 * dy, uy = c.i01 * dx + c.i11 * dy;
        const double e = -0.5 * (dx * ux + dy * uy);
        if (e < -50.0) continue;
        const double E = tb::exp_taylor(fmin(e, 0.0));
        const double val = c.s * E;
        S0 += val;
        Sx = fma(val, ux, Sx);
        Sy = fma(val, uy, Sy);
        const double vv = val * c.v;
        Axx = fma(vv * ux, ux, Axx);
        Axy = fma(vv * ux, uy, Axy);
        Ayy = fma(vv * uy, uy, Ayy);
        At0 = fma(vv, c.t[0], At0);
        At1 = fma(vv, c.t[1], At1);
        At2 = fma(vv, c.t[2], At2);
        const double vd = val * c.dv;
        Dxx = fma(vd * ux, ux, Dxx);
        Dxy = fma(vd * ux, uy, Dxy);
        Dyy = fma(vd * uy, uy, Dyy);
        Dt = fma(vd, c.t[3], Dt);
        Sn = fma(c.sn, E, Sn);
    }
    const double cn = R.counts;
    const double At[3] = {At0, At1, At2};
    J[0] = cn * Sx;
    J[1] = cn * Sy;
    J[2] = S0;
#pragma unroll
    for (int j = 0; j < 3; j++)
        J[3 + j] = cn * 0.5 * (R.dM[j][0] * Axx + 2.0 * R.dM[j][1] * Axy + R.dM[j][2] * Ayy - At[j]);
    J[6] = cn * (0.5 * (R.M[0] * Dxx + 2.0 * R.M[1] * Dxy + R.M[2] * Dyy - Dt) + Sn);
    return cn * S0;
}

// A source's own block: REFINE, its 28 A^T A products (upper triangle) and
// 7 A^T r values; VJP, the 7 contracted columns.
__device__ __forceinline__ void ref_emit_own(RefSmem& sm, int& nc, double* H, double* g,
                                             const double (&Jw)[7], double rr, int sI,
                                             const RefSrc& R, int band, int P, bool refine) {
    if (refine) {
        ref_emit<35>(sm, nc, H, g,
            [&](int q) { return q < 28 ? Jw[tri_row(q)] * Jw[tri_col(q)] : Jw[q - 28] * rr; },
            [&](int q) {
                if (q >= 28) {
                    const int s = ref_slot(sI, R.profile, band, q - 28);
                    return s < 0 ? -1 : -s - 2;
                }
                const int a = ref_slot(sI, R.profile, band, tri_row(q));
                const int c = ref_slot(sI, R.profile, band, tri_col(q));
                return a < 0 || c < 0 ? -1 : a * P + c;
            });
    } else {
        ref_emit<7>(sm, nc, H, g, [&](int q) { return Jw[q] * rr; },
            [&](int q) {
                const int s = ref_slot(sI, R.profile, band, q);
                return s < 0 ? -1 : -s - 2;
            });
    }
}

// The A^T A block of two sources sA < sB (49 products).
__device__ __forceinline__ void ref_emit_pair(RefSmem& sm, int& nc, double* H, double* g,
                                              const double (&Ja)[7], const double (&Jb)[7],
                                              int sA, int sB, int band, int P) {
    const int pa = sm.us[sA].profile, pb = sm.us[sB].profile;
    ref_emit<49>(sm, nc, H, g, [&](int q) { return Ja[q / 7] * Jb[q % 7]; },
        [&](int q) {
            const int a = ref_slot(sA, pa, band, q / 7);
            const int c = ref_slot(sB, pb, band, q % 7);
            return a < 0 || c < 0 ? -1 : a * P + c;
        });
}

// CTAs per SM the refinement kernel is compiled for (2: 128 registers)
#ifndef TB_REFINE_MINB
#define TB_REFINE_MINB 2
#endif
__global__ void __launch_bounds__(kRefThreads, TB_REFINE_MINB)
fit_refine_kernel(const tb_fit_unit* __restrict__ units, const int32_t* __restrict__ order,
                  int n_units, const tb_fit_blob* __restrict__ blobs,
                  const tb_fit_source* __restrict__ srcs, const SrcTab* __restrict__ tab,
                  const FitC64* __restrict__ gcomps, const float* __restrict__ data,
                  const float* __restrict__ inverr, double* __restrict__ hbuf,
                  double* __restrict__ gbuf, double* __restrict__ chi2_out,
                  const tb_fit_state* __restrict__ state, int n_bands,
                  const int32_t* __restrict__ tiles, int32_t* counter, tb_status* st, int mode,
                  float* __restrict__ model_out, const double* __restrict__ chi2_const) {
    // mode TB_FIT_REFINE: A^T A, A^T r and chi^2 of the running blobs, r =
    // (data - model) inverr; TB_FIT_MODEL: the model into model_out (every
    // blob); TB_FIT_VJP: the columns contracted with data = an upstream
    // gradient, unweighted
    __shared__ RefSmem sm;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const bool refine = mode == TB_FIT_REFINE;
    for (;;) {
        const int64_t oi = tb::next_unit(counter, &sm.slot);
        if (oi >= n_units) break;
        const int ui = order[oi];
        if (ui < 0 || ui >= n_units) continue;
        const tb_fit_unit& u = units[ui];
        const tb_fit_blob b = blobs[u.blob];
        if (refine && state[u.blob].status != 0) continue;   // running blobs
        const int P = b.P;
        const int nsrc = b.n_src;
        double* g = gbuf ? gbuf + b.g_off + (int64_t)u.slice * P : nullptr;
        double* H = refine ? hbuf + b.h_off + (int64_t)u.slice * P * P : nullptr;
        if (mode != TB_FIT_MODEL)
            for (int e = tid; e < P; e += kRefThreads) g[e] = 0.0;
        if (refine)
            for (int e = tid; e < P * P; e += kRefThreads) H[e] = 0.0;
        if (warp == 0) {
            const bool unit_bad = nsrc < 0 || nsrc > TB_FIT_MAX_SRC || P != nsrc * TB_FIT_NPAR ||
                                  u.band < 0 || u.band >= n_bands || u.slice < 0 ||
                                  u.slice >= b.n_slices || u.t0 < 0 || u.t1 < u.t0 ||
                                  u.t1 > b.n_active;
            bool src_bad = false;
            if (!unit_bad && lane < nsrc) {
                const SrcTab& S = tab[b.src0 + lane];
                const int K = S.K[u.band];
                src_bad = !S.ok || K < 0 || K > kCompStride;
                const tb_fit_source fs = srcs[b.src0 + lane];
                const bool live = fs.w > 0 && fs.h > 0;
                RefSrc R;
                R.x0 = live ? fs.x0 : 0;
                R.y0 = live ? fs.y0 : 0;
                R.x1 = live ? fs.x0 + fs.w : 0;
                R.y1 = live ? fs.y0 + fs.h : 0;
                R.K = K;
                R.profile = fs.profile;
                R.counts = S.flux[u.band];
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    R.M[q] = S.M64[q];
#pragma unroll
                    for (int j = 0; j < 3; j++) R.dM[j][q] = S.dM64[j][q];
                }
                sm.us[lane] = R;
            }
            const bool bad = unit_bad || __any_sync(0xffffffffu, src_bad);
            if (lane == 0) {
                sm.skip = bad;
                if (bad) tb::report(st, TB_STATUS_BAD_ITEM, ui, nsrc);
            }
        }
        __syncthreads();
        if (sm.skip) {
            if (tid == 0 && chi2_out) chi2_out[b.unit0 + u.slice] = INFINITY;
            continue;
        }
        const FitC64* band_comps = gcomps + ((int64_t)b.src0 * n_bands + u.band) * kCompStride;
        const int64_t cstride = (int64_t)n_bands * kCompStride;
        const int n_t = u.t1 - u.t0;
        const int32_t* tl = tiles + b.tile_off + u.t0;
        double chi2 = 0.0;
        int nc = 0;
        for (int t = 0; t < n_t; t++) {
            const int ox = (tl[t] & 0x3ff) * kTileW, oy = ((tl[t] >> 10) & 0x3ff) * kTileH;
            const int px = ox + lane, py = oy + warp;
            const bool in = px < u.W && py < u.H;
            // the sources whose rectangles meet the tile (the same for every thread)
            unsigned reach = 0u;
            if (lane < nsrc) {
                const RefSrc& R = sm.us[lane];
                reach = R.x1 > ox && R.x0 < ox + kTileW && R.y1 > oy && R.y0 < oy + kTileH;
            }
            reach = __ballot_sync(0xffffffffu, reach);
            const int nreach = __popc(reach);
            double d = 0.0, w = 0.0;
            const int64_t pix = u.pix_off + (int64_t)py * u.W + px;
            // MODEL reads neither data nor inverr (both may be NULL); VJP
            // reads the upstream gradient in `data` and no weights
            if (in && mode != TB_FIT_MODEL) {
                d = data[pix];
                w = mode == TB_FIT_VJP ? 1.0 : inverr[pix];
            }
            if (mode == TB_FIT_MODEL) {
                double m = 0.0;
                for (unsigned rm = reach; rm && in; rm &= rm - 1) {
                    const int sI = __ffs(rm) - 1;
                    m += ref_model(sm.us[sI], band_comps + sI * cstride, px, py);
                }
                if (in) model_out[pix] = (float)m;
                continue;
            }
            if (nreach <= 2) {
                // one or two sources: their columns and the model in one evaluation
                const int s0 = nreach > 0 ? __ffs(reach) - 1 : -1;
                const int s1 = nreach > 1 ? __ffs(reach & (reach - 1)) - 1 : -1;
                double J0[7], J1[7];
                double m = 0.0;
                if (s0 >= 0) m += ref_cols(sm.us[s0], band_comps + s0 * cstride, px, py, J0);
                if (s1 >= 0) m += ref_cols(sm.us[s1], band_comps + s1 * cstride, px, py, J1);
                const double r = refine ? (d - m) * w : d;
                if (refine) chi2 += r * r;
                if (s0 >= 0) {
#pragma unroll
                    for (int j = 0; j < 7; j++) J0[j] *= w;
                    ref_emit_own(sm, nc, H, g, J0, r, s0, sm.us[s0], u.band, P, refine);
                }
                if (s1 >= 0) {
#pragma unroll
                    for (int j = 0; j < 7; j++) J1[j] *= w;
                    ref_emit_own(sm, nc, H, g, J1, r, s1, sm.us[s1], u.band, P, refine);
                    if (refine) ref_emit_pair(sm, nc, H, g, J0, J1, s0, s1, u.band, P);
                }
            } else {
                // three or more: the model first, then each source's columns
                // (a pair's block re-evaluates the later source)
                double m = 0.0;
                if (refine)
                    for (unsigned rm = reach; rm; rm &= rm - 1) {
                        const int sI = __ffs(rm) - 1;
                        m += ref_model(sm.us[sI], band_comps + sI * cstride, px, py);
                    }
                const double r = refine ? (d - m) * w : d;
                if (refine) chi2 += r * r;
                for (unsigned ra = reach; ra; ra &= ra - 1) {
                    const int sA = __ffs(ra) - 1;
                    double Ja[7];
                    ref_cols(sm.us[sA], band_comps + sA * cstride, px, py, Ja);
#pragma unroll
                    for (int j = 0; j < 7; j++) Ja[j] *= w;
                    ref_emit_own(sm, nc, H, g, Ja, r, sA, sm.us[sA], u.band, P, refine);
                    if (!refine) continue;
                    for (unsigned rb = ra & (ra - 1); rb; rb &= rb - 1) {
                        const int sB = __ffs(rb) - 1;
                        double Jb[7];
                        ref_cols(sm.us[sB], band_comps + sB * cstride, px, py, Jb);
#pragma unroll
                        for (int j = 0; j < 7; j++) Jb[j] *= w;
                        ref_emit_pair(sm, nc, H, g, Ja, Jb, sA, sB, u.band, P);
                    }
                }
            }
            if (nc > 0) ref_flush(sm, nc, H, g);
        }
        if (mode == TB_FIT_MODEL) continue;
        // the unit's chi^2 (its active tiles; the constant part stays in chi2_const)
        for (int o = 16; o > 0; o >>= 1) chi2 += __shfl_xor_sync(0xffffffffu, chi2, o);
        if (lane == 0) sm.red[warp][0] = chi2;
        __syncthreads();
        if (tid == 0 && chi2_out) {
            // the slice's chi^2 with its constant part (the tiles no mask
            // reaches), as tb_fit_pass writes it
            double c2 = chi2_const ? chi2_const[b.unit0 + u.slice] : 0.0;
            for (int w2 = 0; w2 < kRefThreads / 32; w2++) c2 += sm.red[w2][0];
            chi2_out[b.unit0 + u.slice] = c2;
        }
        __syncthreads();
    }
}

// One CTA per blob.  The factor lives in the blob's global area (L2
// resident); shared memory and registers stay small so that five blobs
// share an SM.
__global__ void __launch_bounds__(kStepThreads, 5)
fit_step_kernel(const tb_fit_blob* __restrict__ blobs, int n_blobs, int n_bands,
                const tb_fit_source* __restrict__ srcs, double* __restrict__ params,
                double* __restrict__ trial, double* __restrict__ hbuf, double* __restrict__ gbuf,
                const double* __restrict__ chi2_part, tb_fit_state* __restrict__ state,
                double tol, int max_iter) {
    __shared__ double dsc[TB_FIT_MAX_SRC * TB_FIT_NPAR];
    __shared__ double dinv[TB_FIT_MAX_SRC * TB_FIT_NPAR];
    __shared__ double y[TB_FIT_MAX_SRC * TB_FIT_NPAR];
    __shared__ double xs[TB_FIT_MAX_SRC * TB_FIT_NPAR];
    __shared__ double rdg[TB_FIT_MAX_SRC * TB_FIT_NPAR];
    __shared__ double red[kStepThreads / 32], red2[kStepThreads / 32];
    __shared__ int s_accept, s_active;
    __shared__ double s_lambda, s_scale, s_pa, s_pb;
    const int bi = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    (void)n_bands;
    if (bi >= n_blobs) return;
    const tb_fit_blob b = blobs[bi];
    tb_fit_state& S = state[bi];
    const int status0 = S.status;
    __syncthreads();   // every thread has read the status before thread 0 updates it
    if (status0 != 0) return;
    const int P = b.P;
    const int ns = b.n_slices;
    double* Hp = hbuf + b.h_off;                        // slice partials
    double* Ha = Hp + (int64_t)ns * P * P;              // accepted H
    double* L = Ha + (int64_t)P * P;                    // factor
    double* gp = gbuf + b.g_off;
    double* ga = gp + (int64_t)ns * P;
    double* pa = params + (int64_t)b.src0 * TB_FIT_NPAR;
    double* pt = trial + (int64_t)b.src0 * TB_FIT_NPAR;

    if (tid == 0) {
        double c2 = 0.0;
        for (int k = 0; k < ns; k++) c2 += chi2_part[b.unit0 + k];
        const bool first = S.accepted == 0;
        const bool acc = isfinite(c2) && (first || c2 < S.chi2);
        int status = 0;
        if (acc) {
            // damping from the gain ratio rho = actual / predicted (Nielsen's
            // rule: lambda x max(1/3, 1 - (2 rho - 1)^3); x 0.3 without a
            // prediction)
            const double gain = first ? INFINITY : 0.5 * (S.chi2 - c2);
            double fct = 0.3;
            if (!first && S.pred > 0.0 && isfinite(S.pred)) {
                const double t = 2.0 * (gain / S.pred) - 1.0;
                fct = fmax(1.0 / 3.0, 1.0 - t * t * t);
            }
            S.dlnp = gain;
            S.chi2 = c2;
            S.accepted += 1;
            S.lambda = fmax(S.lambda * fct, 1e-9);
        } else {
            S.lambda *= 10.0;
            S.rejected += 1;
            if (!(S.lambda < 1e12) || !isfinite(c2) && first) status = 2;
        }
        S.iters += 1;
        if (status == 0 && S.iters >= max_iter) status = 3;
        s_accept = acc;
        s_lambda = S.lambda;
        s_active = status == 0;
        S.status = status;
    }
    __syncthreads();
    if (s_accept) {
        for (int e = tid; e < P; e += kStepThreads) pa[e] = pt[e];
        // accepted H (symmetric, from the slice partials' upper triangles) and g
        for (int r = warp; r < P; r += kStepThreads / 32)
            for (int c = r + lane; c < P; c += 32) {
                double s = 0.0;
                for (int k = 0; k < ns; k++) s += Hp[(int64_t)k * P * P + (int64_t)r * P + c];
                Ha[(int64_t)r * P + c] = s;
                Ha[(int64_t)c * P + r] = s;
            }
        for (int e = tid; e < P; e += kStepThreads) {
            double s = 0.0;
            for (int k = 0; k < ns; k++) s += gp[(int64_t)k * P + e];
            ga[e] = s;
        }
    }
    __syncthreads();
    if (!s_active) {
        // stopped: the trial parameters are the accepted ones
        for (int e = tid; e < P; e += kStepThreads) pt[e] = pa[e];
        return;
    }
    const double lam = s_lambda;
    // Marquardt scaling: D = sqrt(diag H); (D^-1 H D^-1 + lambda I) x = D^-1 g
    for (int i = tid; i < P; i += kStepThreads) {
        const double a = Ha[(int64_t)i * P + i];
        double d = (a > 0.0 && isfinite(a)) ? sqrt(a) : 0.0;
        // a Sersic index held at a bound that the gradient pushes against is
        // left out of the step (projected step; the bound-constrained optimum)
        if (i % TB_FIT_NPAR == TB_FIT_NPAR - 1 &&
            srcs[b.src0 + i / TB_FIT_NPAR].profile == TB_PROFILE_SERSIC &&
            ((pa[i] >= TB_FIT_SERSIC_MAX && ga[i] > 0.0) ||
             (pa[i] <= TB_FIT_SERSIC_MIN && ga[i] < 0.0)))
            d = 0.0;
        // frozen parameters are left out of the step
        if ((srcs[b.src0 + i / TB_FIT_NPAR].frozen >> (i % TB_FIT_NPAR)) & 1) d = 0.0;
        dsc[i] = d;
        dinv[i] = d == 0.0 ? 0.0 : 1.0 / d;
    }
    __syncthreads();
    // element (i, j) of the scaled matrix (H symmetric: read along i)
    auto scaled = [&](int i, int j) -> double {
        if (dinv[i] == 0.0 || dinv[j] == 0.0) return i == j ? 1.0 : 0.0;
        return Ha[(int64_t)j * P + i] * dinv[i] * dinv[j] + (i == j ? lam : 0.0);
    };
    // LDL^T of the scaled matrix, lower triangle column-major (element
    // (i, j), i >= j, at L[j P + i]), right-looking: step k subtracts
    // L[k P + i] L[k P + j] / d_k from the trailing columns and leaves column
    // k as d_k (diagonal) and d_k l_ik below it, so no column is rescaled
    // and each step takes one barrier.
    for (int j = warp; j < P; j += kStepThreads / 32)
        for (int i = j + lane; i < P; i += 32) L[(int64_t)j * P + i] = scaled(i, j);
    __syncthreads();
    bool bad = false;
    for (int k = 0; k < P; k++) {
        const double* ck = L + (int64_t)k * P;
        const double dk = ck[k];   // final since step k - 1; the same in every thread
        if (!(dk > 0.0) || !isfinite(dk)) { bad = true; break; }
        const double rk = 1.0 / dk;
        for (int j = k + 1 + warp; j < P; j += kStepThreads / 32) {
            const double cj = ck[j] * rk;
            double* colj = L + (int64_t)j * P;
            for (int i = j + lane; i < P; i += 32) colj[i] = fma(-ck[i], cj, colj[i]);
        }
        __syncthreads();
    }
    if (bad) {
        // not positive definite: treat as a rejected step with more damping
        if (tid == 0) {
            S.lambda *= 10.0;
            if (!(S.lambda < 1e12)) S.status = 2;
        }
        for (int e = tid; e < P; e += kStepThreads) pt[e] = pa[e];
        return;
    }
    for (int i = tid; i < P; i += kStepThreads) {
        rdg[i] = 1.0 / L[(int64_t)i * P + i];
        xs[i] = 0.0;
        y[i] = ga[i] * dinv[i];
    }
    __syncthreads();
    // solution and one refinement step
    for (int pass = 0; pass < 2; pass++) {
        if (pass == 1) {
            for (int i = tid; i < P; i += kStepThreads) {
                double acc = ga[i] * dinv[i];
                for (int j = 0; j < P; j++) acc -= scaled(i, j) * xs[j];
                y[i] = acc;
            }
            __syncthreads();
        }
        if (warp == 0) {
            // L z = y, w = D^-1 z, L^T x = w by columns, lane l holding rows
            // l + 32 m in registers: l_ik = L[k P + i] / d_k
            constexpr int kSlots = (TB_FIT_MAX_SRC * TB_FIT_NPAR + 31) / 32;
            double v[kSlots];
#pragma unroll
            for (int m = 0; m < kSlots; m++) {
                const int i = lane + 32 * m;
                v[m] = i < P ? y[i] : 0.0;
            }
            for (int k = 0; k < P; k++) {
                double zk = 0.0;
#pragma unroll
                for (int m = 0; m < kSlots; m++)
                    if (m == (k >> 5)) zk = v[m];
                zk = __shfl_sync(0xffffffffu, zk, k & 31) * rdg[k];
                const double* ck = L + (int64_t)k * P;
#pragma unroll
                for (int m = 0; m < kSlots; m++) {
                    const int i = lane + 32 * m;
                    if (i > k && i < P) v[m] = fma(-ck[i], zk, v[m]);
                }
            }
#pragma unroll
            for (int m = 0; m < kSlots; m++) {
                const int i = lane + 32 * m;
                if (i < P) v[m] *= rdg[i];
            }
            for (int k = P - 1; k > 0; k--) {
                double xk = 0.0;
#pragma unroll
                for (int m = 0; m < kSlots; m++)
                    if (m == (k >> 5)) xk = v[m];
                xk = __shfl_sync(0xffffffffu, xk, k & 31);
#pragma unroll
                for (int m = 0; m < kSlots; m++) {
                    const int j = lane + 32 * m;
                    if (j < k) v[m] = fma(-L[(int64_t)j * P + k] * rdg[j], xk, v[m]);
                }
            }
#pragma unroll
            for (int m = 0; m < kSlots; m++) {
                const int i = lane + 32 * m;
                if (i < P) y[i] = v[m];
            }
        }
        __syncthreads();
        for (int i = tid; i < P; i += kStepThreads) xs[i] += y[i];
        __syncthreads();
    }
    // Predicted log-likelihood gain of this damped step,
    // 1/2 (x . D^-1 g + lambda x . x); the blob has converged when it is below
    // tol while the damping is moderate (optimize_loop stops on the gain of
    // the last step, dchisq; the prediction is immune to FP32 noise in chi^2).
    {
        // a = x^T y0, b = x^T x: the gain predicted for the step is
        // (a + lambda b) / 2, for the step scaled by s it is
        // s a - s^2 (a - lambda b) / 2
        double pa_ = 0.0, pb_ = 0.0;
        for (int i = tid; i < P; i += kStepThreads) {
            const double y0 = dsc[i] == 0.0 ? 0.0 : ga[i] / dsc[i];
            pa_ += xs[i] * y0;
            pb_ += xs[i] * xs[i];
        }
        for (int o = 16; o > 0; o >>= 1) {
            pa_ += __shfl_xor_sync(0xffffffffu, pa_, o);
            pb_ += __shfl_xor_sync(0xffffffffu, pb_, o);
        }
        if (lane == 0) {
            red[warp] = pa_;
            red2[warp] = pb_;
        }
        __syncthreads();
        if (tid == 0) {
            double ta = 0.0, tb2 = 0.0;
            for (int w2 = 0; w2 < kStepThreads / 32; w2++) {
                ta += red[w2];
                tb2 += red2[w2];
            }
            s_pa = ta;
            s_pb = tb2;
            const double t = ta + lam * tb2;
            S.pred = 0.5 * t;
            s_active = !(0.5 * t < tol && lam <= 1.0);
            if (!s_active) S.status = 1;
        }
        __syncthreads();
        if (!s_active) {
            for (int e = tid; e < P; e += kStepThreads) pt[e] = pa[e];
            return;
        }
    }
    // step = x / D, limited by maximum steps and the Sersic-index bounds
    // (ConstrainedOptimizer scales the whole step, constrained_optimizer.py)
    double lim = 1.0;
    for (int i = tid; i < P; i += kStepThreads) {
        const double dlt = dsc[i] == 0.0 ? 0.0 : xs[i] / dsc[i];
        y[i] = dlt;
        const int off = i % TB_FIT_NPAR;
        const double ms = max_step(off);
        if (ms > 0.0 && fabs(dlt) > ms) lim = fmin(lim, ms / fabs(dlt));
        if (off == TB_FIT_NPAR - 1 && srcs[b.src0 + i / TB_FIT_NPAR].profile == TB_PROFILE_SERSIC) {
            const double nv = pa[i] + dlt;
            if (nv > TB_FIT_SERSIC_MAX && dlt > 0.0) lim = fmin(lim, (TB_FIT_SERSIC_MAX - pa[i]) / dlt);
            if (nv < TB_FIT_SERSIC_MIN && dlt < 0.0) lim = fmin(lim, (TB_FIT_SERSIC_MIN - pa[i]) / dlt);
        }
    }
    for (int o = 16; o > 0; o >>= 1) lim = fmin(lim, __shfl_xor_sync(0xffffffffu, lim, o));
    if (lane == 0) red[warp] = lim;
    __syncthreads();
    if (tid == 0) {
        double l = 1.0;
        for (int w2 = 0; w2 < kStepThreads / 32; w2++) l = fmin(l, red[w2]);
        s_scale = fmax(l, 0.0);
        // the gain predicted for the trial as scaled (the next call's gain
        // ratio divides by it)
        S.pred = s_scale * s_pa - 0.5 * s_scale * s_scale * (s_pa - lam * s_pb);
    }
    __syncthreads();
    for (int i = tid; i < P; i += kStepThreads) {
        double v = pa[i] + s_scale * y[i];
        if (i % TB_FIT_NPAR == TB_FIT_NPAR - 1 &&
            srcs[b.src0 + i / TB_FIT_NPAR].profile == TB_PROFILE_SERSIC)
            v = fmin(fmax(v, TB_FIT_SERSIC_MIN), TB_FIT_SERSIC_MAX);
        pt[i] = v;
    }
}

__global__ void fit_reset_kernel(tb_fit_state* state, int n, double lambda0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    tb_fit_state s;
    s.chi2 = INFINITY;
    s.dlnp = INFINITY;
    s.lambda = lambda0;
    s.pred = INFINITY;
    s.iters = 0;
    s.accepted = 0;
    s.rejected = 0;
    s.status = 0;
    state[i] = s;
}

}  // namespace

extern "C" int tb_fit_workspace(int32_t n_src, int32_t n_bands, int64_t* bytes) {
    if (n_src < 0 || n_bands < 1 || n_bands > TB_FIT_MAX_BANDS || !bytes) return TB_ERR_ARG;
    const int64_t tab = ((int64_t)n_src * (int64_t)sizeof(SrcTab) + 255) / 256 * 256;
    const int64_t nc = (int64_t)n_src * n_bands * kCompStride;
    *bytes = tab + nc * (int64_t)sizeof(FitC) + nc * (int64_t)sizeof(FitC64);
    return TB_OK;
}

namespace {
inline SrcTab* ws_tab(void* ws) { return static_cast<SrcTab*>(ws); }
inline FitC* ws_comps(void* ws, int32_t n_src) {
    const int64_t tab = ((int64_t)n_src * (int64_t)sizeof(SrcTab) + 255) / 256 * 256;
    return reinterpret_cast<FitC*>(static_cast<char*>(ws) + tab);
}
inline FitC64* ws_comps64(void* ws, int32_t n_src, int32_t n_bands) {
    return reinterpret_cast<FitC64*>(ws_comps(ws, n_src) +
                                     (int64_t)n_src * n_bands * kCompStride);
}
}  // namespace

extern "C" int tb_fit_reset(tb_fit_state* state, int32_t n_blobs, double lambda0, void* stream) {
    if (n_blobs < 0 || (n_blobs > 0 && !state)) return TB_ERR_ARG;
    if (n_blobs == 0) return TB_OK;
    fit_reset_kernel<<<(n_blobs + 255) / 256, 256, 0, (cudaStream_t)stream>>>(state, n_blobs,
                                                                             lambda0);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

extern "C" int tb_fit_prep(const tb_fit_source* srcs, int32_t n_src, const double* params,
                           int32_t n_bands, const tb_fit_unit* units, int32_t n_units,
                           const double* cd_inv, const tb_profile_tables* tables, void* workspace,
                           const tb_fit_state* state, void* stream) {
    if (n_src < 0 || n_bands < 1 || n_bands > TB_FIT_MAX_BANDS || n_units < 0) return TB_ERR_ARG;
    if (n_src == 0) return TB_OK;
    if (!srcs || !params || !units || !cd_inv || !tables || !workspace) return TB_ERR_ARG;
    const int smem = tb::tables_smem_bytes(*tables);
    if (smem > TB_PROFILE_SMEM_MAX) return TB_ERR_SIZE;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(fit_prep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
            cudaSuccess)
        return TB_ERR_LAUNCH;
    const int per_block = kPrepThreads / 32;
    fit_prep_kernel<<<(n_src + per_block - 1) / per_block, kPrepThreads, smem,
                      (cudaStream_t)stream>>>(srcs, n_src, params, n_bands, units, n_units,
                                              *tables, cd_inv[0], cd_inv[1], cd_inv[2], cd_inv[3],
                                              ws_tab(workspace), ws_comps(workspace, n_src),
                                              ws_comps64(workspace, n_src, n_bands), state);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

extern "C" int tb_fit_pass(const tb_fit_unit* units, const int32_t* order, int32_t n_units,
                           const tb_fit_blob* blobs, const tb_fit_source* srcs, int32_t n_src,
                           const void* workspace, const float* data, const float* inverr,
                           const int32_t* tiles, double* hbuf, double* gbuf, double* chi2_part,
                           double* chi2_const, const tb_fit_state* state, int32_t n_bands,
                           int32_t mode, int32_t* work_counter, tb_status* status,
                           void* stream) {
    if (n_units < 0 || n_src < 0 || n_bands < 1 || n_bands > TB_FIT_MAX_BANDS) return TB_ERR_ARG;
    if (mode != 0 && mode != 1) return TB_ERR_ARG;
    if (n_units == 0) return TB_OK;
    if (!units || !order || !blobs || !srcs || !workspace || !data || !inverr || !tiles ||
        !hbuf || !gbuf || !chi2_part || !chi2_const || !state || !work_counter)
        return TB_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const int smem = (int)sizeof(PassSmem);
    if (cudaFuncSetAttribute(fit_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
        cudaSuccess)
        return TB_ERR_LAUNCH;
    if (cudaMemsetAsync(work_counter, 0, sizeof(int32_t), s) != cudaSuccess) return TB_ERR_LAUNCH;
    if (status && cudaMemsetAsync(status, 0, sizeof(tb_status), s) != cudaSuccess)
        return TB_ERR_LAUNCH;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fit_pass_kernel, kThreads, smem) !=
            cudaSuccess || per_sm < 1)
        per_sm = 1;
    const int64_t want = (int64_t)tb::num_sms() * per_sm;
    const int grid = (int)(n_units < want ? n_units : want);
    void* ws = const_cast<void*>(workspace);
    fit_pass_kernel<<<grid, kThreads, smem, s>>>(
        units, order, n_units, blobs, srcs, ws_tab(ws), ws_comps(ws, n_src), data, inverr, hbuf,
        gbuf, chi2_part, state, n_bands, tiles, chi2_const, mode, work_counter, status);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

extern "C" int tb_fit_step(const tb_fit_blob* blobs, int32_t n_blobs, int32_t n_bands,
                           const tb_fit_source* srcs, double* params, double* trial,
                           double* hbuf, double* gbuf, const double* chi2_part,
                           tb_fit_state* state, double tol, int32_t max_iter, void* stream) {
    if (n_blobs < 0 || n_bands < 1 || n_bands > TB_FIT_MAX_BANDS) return TB_ERR_ARG;
    if (n_blobs == 0) return TB_OK;
    if (!blobs || !srcs || !params || !trial || !hbuf || !gbuf || !chi2_part || !state)
        return TB_ERR_ARG;
    fit_step_kernel<<<n_blobs, kStepThreads, 0, (cudaStream_t)stream>>>(
        blobs, n_blobs, n_bands, srcs, params, trial, hbuf, gbuf, chi2_part, state, tol, max_iter);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

extern "C" int tb_fit_refine(const tb_fit_unit* units, const int32_t* order, int32_t n_units,
                             const tb_fit_blob* blobs, const tb_fit_source* srcs, int32_t n_src,
                             const void* workspace, const float* data, const float* inverr,
                             const int32_t* tiles, double* hbuf, double* gbuf,
                             double* chi2_out, const double* chi2_const,
                             const tb_fit_state* state, int32_t n_bands, int32_t* work_counter,
                             tb_status* status, void* stream) {
    if (n_units < 0 || n_src < 0 || n_bands < 1 || n_bands > TB_FIT_MAX_BANDS) return TB_ERR_ARG;
    if (n_units == 0) return TB_OK;
    if (!units || !order || !blobs || !srcs || !workspace || !data || !inverr || !tiles ||
        !hbuf || !gbuf || !chi2_out || !state || !work_counter)
        return TB_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(work_counter, 0, sizeof(int32_t), s) != cudaSuccess) return TB_ERR_LAUNCH;
    if (status && cudaMemsetAsync(status, 0, sizeof(tb_status), s) != cudaSuccess)
        return TB_ERR_LAUNCH;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fit_refine_kernel, kRefThreads,
                                                      0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const int64_t want = (int64_t)tb::num_sms() * per_sm;
    const int grid = (int)(n_units < want ? n_units : want);
    void* ws = const_cast<void*>(workspace);
    fit_refine_kernel<<<grid, kRefThreads, 0, s>>>(
        units, order, n_units, blobs, srcs, ws_tab(ws), ws_comps64(ws, n_src, n_bands), data,
        inverr, hbuf, gbuf, chi2_out, state, n_bands, tiles, work_counter, status, TB_FIT_REFINE,
        nullptr, chi2_const);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

extern "C" int tb_fit_model_vjp(const tb_fit_unit* units, const int32_t* order, int32_t n_units,
                                const tb_fit_blob* blobs, const tb_fit_source* srcs,
                                int32_t n_src, const void* workspace, const float* grad,
                                float* model, const int32_t* tiles, double* gbuf,
                                int32_t n_bands, int32_t mode, int32_t* work_counter,
                                tb_status* status, void* stream) {
    if (n_units < 0 || n_src < 0 || n_bands < 1 || n_bands > TB_FIT_MAX_BANDS) return TB_ERR_ARG;
    if (mode != TB_FIT_MODEL && mode != TB_FIT_VJP) return TB_ERR_ARG;
    if (n_units == 0) return TB_OK;
    if (!units || !order || !blobs || !srcs || !workspace || !tiles || !work_counter ||
        (mode == TB_FIT_MODEL && !model) || (mode == TB_FIT_VJP && (!grad || !gbuf)))
        return TB_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(work_counter, 0, sizeof(int32_t), s) != cudaSuccess) return TB_ERR_LAUNCH;
    if (status && cudaMemsetAsync(status, 0, sizeof(tb_status), s) != cudaSuccess)
        return TB_ERR_LAUNCH;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fit_refine_kernel, kRefThreads,
                                                      0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const int64_t want = (int64_t)tb::num_sms() * per_sm;
    const int grid = (int)(n_units < want ? n_units : want);
    void* ws = const_cast<void*>(workspace);
    fit_refine_kernel<<<grid, kRefThreads, 0, s>>>(
        units, order, n_units, blobs, srcs, ws_tab(ws), ws_comps64(ws, n_src, n_bands), grad,
        nullptr, nullptr, gbuf, nullptr, nullptr, n_bands, tiles, work_counter, status, mode,
        model, nullptr);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

