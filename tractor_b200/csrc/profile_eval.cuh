// Galaxy profile and shape evaluation shared by the prep kernels (sm_100a).
//
// Everything here runs in FP64 (a few hundred operations per source) and
// follows the reference's host-side Python:
//   profile:  exp / deV tables (tractor/mixture_profiles.py:20-45) or the
//             Sersic mixture (tractor/sersic.py:288-342): index clamped to
//             the table range, range lookup, B-spline interpolation of
//             amplitudes and log-variances, normalisation, delta core for
//             n > 1;
//   shape:    getRaDecBasis of EllipseE / EllipseESoft (ellipses.py:126-155,
//             165-263) and GalaxyShape (galaxy.py:73-89); the pixel-space
//             factor T T^T with T = cdInverse * basis (galaxy.py:659-669).
#pragma once
#include "tb_common.cuh"

namespace tb {

// De Boor's recursion for a B-spline of degree k (1..3) with coefficients c
// at x, given its knot span l and the knots around it: tk[j] = t[l - k + 1
// + j], j = 0 .. 2k - 1.
//   d_j <- (1 - a) d_{j-1} + a d_j, a = (x - t_i) / (t_{i+k+1-r} - t_i),
//   i = j + l - k, for r = 1..k and j = k..r.
__device__ inline double deboor(const double* c, const double* tk, int k, int l, double x) {
    auto t = [&](int i) { return tk[i - (l - k + 1)]; };
    auto blend = [&](double lo, double hi, int i, int r) {
        const double den = t(i + k + 1 - r) - t(i);
        const double a = den == 0.0 ? 0.0 : (x - t(i)) / den;
        return (1.0 - a) * lo + a * hi;
    };
    if (k == 3) {
        double d0 = c[l - 3], d1 = c[l - 2], d2 = c[l - 1], d3 = c[l];
        d3 = blend(d2, d3, l, 1);
        d2 = blend(d1, d2, l - 1, 1);
        d1 = blend(d0, d1, l - 2, 1);
        d3 = blend(d2, d3, l, 2);
        d2 = blend(d1, d2, l - 1, 2);
        d3 = blend(d2, d3, l, 3);
        return d3;
    }
    if (k == 2) {
        double d0 = c[l - 2], d1 = c[l - 1], d2 = c[l];
        d2 = blend(d1, d2, l, 1);
        d1 = blend(d0, d1, l - 1, 1);
        d2 = blend(d1, d2, l, 2);
        return d2;
    }
    if (k == 1) return blend(c[l - 1], c[l], l, 1);
    return c[l];
}

// B-spline value of spline s at x (FITPACK knots / coefficients, degree
// 1..3), by de Boor's recursion with the knot span clamped to the table.
__device__ inline double bspline(const tb_profile_tables& T, int s, double x) {
    const int to = T.spline_info[4 * s], nt = T.spline_info[4 * s + 1];
    const int co = T.spline_info[4 * s + 2], k = T.spline_info[4 * s + 3];
    const double* t = T.knots + to;
    const int n = nt - k - 1;
    // knot span l: t[l] <= x < t[l+1], clamped to [k, n-1] -- the largest
    // j in (k, n-1] with t[j] <= x, else k (knots are non-decreasing), by
    // bisection: a few dependent loads instead of one per knot
    int l = k, hi = n - 1;
    while (l < hi) {
        const int mid = (l + hi + 1) >> 1;
        if (t[mid] <= x) l = mid;
        else hi = mid - 1;
    }
    double tk[6];
    for (int j = 0; j < 2 * k; j++) tk[j] = t[l - k + 1 + j];
    return deboor(T.coefs + co, tk, k, l, x);
}

// The knot span of x in a knot vector of nt <= 32 knots and degree k,
// found by the whole warp at once: lane j holds t[j]; the span is the
// largest j in (k, nt - k - 2] with t[j] <= x, else k (as bspline's
// search), and every lane receives the 2k knots around it in tk.  All 32
// lanes must call this together.
__device__ inline int warp_knot_span(const double* t, int nt, int k, double x, double* tk) {
    const int j = (int)(threadIdx.x & 31);
    const double tj = j < nt ? t[j] : 0.0;
    const int n = nt - k - 1;
    const unsigned m = __ballot_sync(0xffffffffu, j >= k + 1 && j <= n - 1 && tj <= x);
    const int l = m ? 31 - __clz((int)m) : k;
    for (int q = 0; q < 2 * k; q++) tk[q] = __shfl_sync(0xffffffffu, tj, l - k + 1 + q);
    return l;
}

// bspline() of one spline evaluated by the whole warp (all lanes get the
// value): the knot span by warp_knot_span when the spline has at most 32
// knots.  All 32 lanes must call this together.
__device__ inline double warp_bspline(const tb_profile_tables& T, int s, double x) {
    const int nt = T.spline_info[4 * s + 1];
    if (nt > 32) return bspline(T, s, x);
    const int to = T.spline_info[4 * s], co = T.spline_info[4 * s + 2];
    const int k = T.spline_info[4 * s + 3];
    double tk[6];
    const int l = warp_knot_span(T.knots + to, nt, k, x, tk);
    return deboor(T.coefs + co, tk, k, l, x);
}

// Radius of a profile in units of r_e beyond which the reference treats a
// source outside its ModelMask as absent (galaxy.py:353-374).
__device__ inline double nre_of(int kind) {
    switch (kind) {
        case TB_PROFILE_EXP: return 4.0;
        case TB_PROFILE_GAUSSIAN: return 6.0;
        default: return 8.0;   // deV, Sersic
    }
}

__host__ __device__ inline int tables_smem_bytes(const tb_profile_tables& G) {
    return 8 * (G.n_knots + G.n_coefs + 2 * G.n_ranges + 2 * G.exp_K + 2 * G.dev_K) +
           4 * (4 * G.n_ranges + 4 * G.n_splines);
}

// Copies the profile tables into shared memory (the spline evaluations make
// many dependent lookups) and returns a table view pointing there.  Every
// thread of the block must call it.
__device__ inline tb_profile_tables stage_tables(const tb_profile_tables& G, unsigned char* smem) {
    tb_profile_tables T = G;
    double* d = reinterpret_cast<double*>(smem);
    double* knots = d;
    double* coefs = knots + G.n_knots;
    double* lohi = coefs + G.n_coefs;
    double* ea = lohi + 2 * G.n_ranges;
    double* ev = ea + G.exp_K;
    double* da = ev + G.exp_K;
    double* dv = da + G.dev_K;
    int32_t* ri = reinterpret_cast<int32_t*>(dv + G.dev_K);
    int32_t* si = ri + 4 * G.n_ranges;
    for (int k = threadIdx.x; k < G.n_knots; k += blockDim.x) knots[k] = G.knots[k];
    for (int k = threadIdx.x; k < G.n_coefs; k += blockDim.x) coefs[k] = G.coefs[k];
    for (int k = threadIdx.x; k < 2 * G.n_ranges; k += blockDim.x) lohi[k] = G.range_lohi[k];
    for (int k = threadIdx.x; k < G.exp_K; k += blockDim.x) { ea[k] = G.exp_amp[k]; ev[k] = G.exp_var[k]; }
    for (int k = threadIdx.x; k < G.dev_K; k += blockDim.x) { da[k] = G.dev_amp[k]; dv[k] = G.dev_var[k]; }
    for (int k = threadIdx.x; k < 4 * G.n_ranges; k += blockDim.x) ri[k] = G.range_info[k];
    for (int k = threadIdx.x; k < 4 * G.n_splines; k += blockDim.x) si[k] = G.spline_info[k];
    T.knots = knots;
    T.coefs = coefs;
    T.range_lohi = lohi;
    T.exp_amp = ea;
    T.exp_var = ev;
    T.dev_amp = da;
    T.dev_var = dv;
    T.range_info = ri;
    T.spline_info = si;
    __syncthreads();
    return T;
}

// Sum over lanes 0..K-1 of v, accumulated in lane order (the reference's
// sequential numpy sum for these short vectors).
__device__ __forceinline__ double lane_sum(double v, int K) {
    double s = 0.0;
    for (int k = 0; k < K; k++) s += __shfl_sync(0xffffffffu, v, k);
    return s;
}

// Profile mixture across a warp: lane l < K receives component l's
// amplitude and (circular, unit r_e) variance.  Returns K, or -1 if the
// profile is unknown or has more than max_k components.  Sersic components
// come out in the spline order; the caller ranks them by variance.
__device__ inline int warp_profile(const tb_profile_tables& T, int profile, double sersic_n,
                                   int lane, int max_k, double& a, double& v) {
    a = 0.0;
    v = 0.0;
    if (profile == TB_PROFILE_EXP || profile == TB_PROFILE_DEV) {
        const bool ex = profile == TB_PROFILE_EXP;
        const int K = ex ? T.exp_K : T.dev_K;
        if (K > max_k) return -1;
        if (lane < K) {
            a = ex ? T.exp_amp[lane] : T.dev_amp[lane];
            v = ex ? T.exp_var[lane] : T.dev_var[lane];
        }
        return K;
    }
    if (profile == TB_PROFILE_GAUSSIAN) {
        if (lane == 0) { a = 1.0; v = 1.0; }
        return 1;
    }
    if (profile != TB_PROFILE_SERSIC) return -1;
    double nn = sersic_n;
    const double lowest = T.range_lohi[0], highest = T.range_lohi[2 * T.n_ranges - 1];
    int r = -1;
    if (nn <= lowest) { r = 0; nn = lowest; }
    else if (nn >= highest) { r = T.n_ranges - 1; nn = highest; }
    else {
        // the first range holding nn: lane q tests range q (one round of loads)
        for (int q0 = 0; q0 < T.n_ranges && r < 0; q0 += 32) {
            const int q = q0 + (int)(threadIdx.x & 31);
            const bool in = q < T.n_ranges && T.range_lohi[2 * q] <= nn &&
                            nn < T.range_lohi[2 * q + 1];
            const unsigned m = __ballot_sync(0xffffffffu, in);
            if (m) r = q0 + __ffs(m) - 1;
        }
    }
    if (r < 0) return -1;
    const int Kr = T.range_info[4 * r], sa = T.range_info[4 * r + 1];
    const int sv = T.range_info[4 * r + 2];
    if (Kr + 1 > max_k) return -1;
    if (T.range_info[4 * r + 3] == 1) {
        // every spline of the range has spline sa's knots (<= 32 of them):
        // one knot span for the warp, then each lane's coefficients
        const int to = T.spline_info[4 * sa], nt = T.spline_info[4 * sa + 1];
        const int kd = T.spline_info[4 * sa + 3];
        double tk[6];
        const int l = warp_knot_span(T.knots + to, nt, kd, nn, tk);
        if (lane < Kr) {
            a = deboor(T.coefs + T.spline_info[4 * (sa + lane) + 2], tk, kd, l, nn);
            v = exp(deboor(T.coefs + T.spline_info[4 * (sv + lane) + 2], tk, kd, l, nn));
        }
    } else if (lane < Kr) {
        a = bspline(T, sa + lane, nn);
        v = exp(bspline(T, sv + lane, nn));
    }
    a /= lane_sum(a, Kr);
    int K = Kr;
    if (nn > 1.0) {
        const double core = warp_bspline(T, T.core_spline, nn);
        a *= (1.0 - core) / lane_sum(a, Kr);
        if (lane == Kr) { a = core; v = 0.0; }
        K = Kr + 1;
    }
    return K;
}

// Sersic mixture of range r at index nn with the core present or not, lane l
// holding component l (the spline evaluation of warp_profile without the
// range lookup, so that both sides of a central difference use the same
// components).
__device__ inline int sersic_fixed(const tb_profile_tables& T, int r, double nn, bool core_on,
                                   int lane, double& a, double& v) {
    const int Kr = T.range_info[4 * r], sa = T.range_info[4 * r + 1];
    const int sv = T.range_info[4 * r + 2];
    a = 0.0;
    v = 0.0;
    if (lane < Kr) {
        a = bspline(T, sa + lane, nn);
        v = exp(bspline(T, sv + lane, nn));
    }
    a /= lane_sum(a, Kr);
    if (!core_on) return Kr;
    const double core = bspline(T, T.core_spline, nn);
    a *= (1.0 - core) / lane_sum(a, Kr);
    if (lane == Kr) { a = core; v = 0.0; }
    return Kr + 1;
}

// Stable rank of this lane's variance among lanes 0..K-1 (the argsort of
// sersic.py:338-341).
__device__ __forceinline__ int variance_rank(double v, int K, int lane) {
    int rank = 0;
    for (int j = 0; j < (K > 0 ? K : 0); j++) {
        const double vj = __shfl_sync(0xffffffffu, v, j);
        rank += (vj < v) || (vj == v && j < lane);
    }
    return rank;
}

// getRaDecBasis of a shape (degrees per r_e unit): G row-major, and r_e.
__device__ inline void shape_basis(int shape_type, double s0, double s1, double s2, double G[4],
                                   double& re) {
    if (shape_type == TB_SHAPE_RABPHI) {
        const double phi = (90.0 - s2) * (TB_PI / 180.0);
        re = s0;
        const double r_deg = fmax(1.0 / 30.0, s0) / 3600.0;
        const double cp = cos(phi), sp = sin(phi);
        G[0] = r_deg * cp;
        G[1] = r_deg * sp * s1;
        G[2] = -r_deg * sp;
        G[3] = r_deg * cp * s1;
        return;
    }
    double e1 = s1, e2 = s2;
    re = s0;
    if (shape_type == TB_SHAPE_ELLIPSE_ESOFT) {
        re = exp(s0);
        const double ee = hypot(s1, s2);
        const double e = fmin(0.999999, 1.0 - exp(-ee));
        const double th = atan2(s2, s1) / 2.0;
        e1 = e * cos(2.0 * th);
        e2 = e * sin(2.0 * th);
    }
    const double th = atan2(e2, e1) / 2.0;
    const double ct = cos(th), st = sin(th);
    const double e = hypot(e1, e2);
    const double ab = e >= 1.0 ? 1000.0 : fmin(1000.0, (1.0 + e) / (1.0 - e));
    const double r_deg = re / 3600.0;
    G[0] = r_deg * ct / ab;
    G[1] = r_deg * st;
    G[2] = -r_deg * st / ab;
    G[3] = r_deg * ct;
}

// M = T T^T with T = cd_inv * G (both 2x2 row-major): the pixel-space
// covariance of a unit-variance circular component.
__device__ inline void pixel_factor(const double* C, const double G[4], double& M00,
                                    double& M01, double& M11) {
    const double T0 = C[0] * G[0] + C[1] * G[2], T1 = C[0] * G[1] + C[1] * G[3];
    const double T2 = C[2] * G[0] + C[3] * G[2], T3 = C[2] * G[1] + C[3] * G[3];
    M00 = T0 * T0 + T1 * T1;
    M01 = T0 * T2 + T1 * T3;
    M11 = T2 * T2 + T3 * T3;
}

}  // namespace tb
