// Galaxy preparation for the Fourier path (sm_100a): one thread per source
// turns (position, counts, shape, profile, ModelMask) into a tb_fft_item and
// its component table.  Everything runs in FP64 (it is a few hundred
// operations per source), following the reference's host-side Python:
//   profile:  exp / deV tables (tractor/mixture_profiles.py:20-45) or the
//             Sersic mixture (tractor/sersic.py:288-342): index clamped to
//             the table range, range lookup, B-spline interpolation of
//             amplitudes and log-variances, normalisation, delta core for
//             n > 1, sort by variance;
//   shape:    T = cdInverse * getRaDecBasis (galaxy.py:659-669,
//             ellipses.py:126-155, galaxy.py:73-89); var_k = v_k T T^T;
//   geometry: half-size for a ModelMask (galaxy.py:339-351), FFT size
//             (psf.py:209-212), source-outside-mask rule (galaxy.py:353-374),
//             integer / sub-pixel split with half-to-even rounding
//             (galaxy.py:383-406).
#include "tb_common.cuh"

namespace {

constexpr int kMaxComp = 10;
constexpr int kPrepThreads = 128;   // 4 sources (warps) per block

__device__ double bspline(const tb_profile_tables& T, int s, double x) {
    const int to = T.spline_info[4 * s], nt = T.spline_info[4 * s + 1];
    const int co = T.spline_info[4 * s + 2], k = T.spline_info[4 * s + 3];
    const double* t = T.knots + to;
    const double* c = T.coefs + co;
    const int n = nt - k - 1;
    // knot span l: t[l] <= x < t[l+1], clamped to [k, n-1]
    int l = k;
    while (l + 1 < n && t[l + 1] <= x) l++;
    // de Boor's recursion, written out per degree with scalars:
    // d_j <- (1 - a) d_{j-1} + a d_j, a = (x - t_i) / (t_{i+k+1-r} - t_i),
    // i = j + l - k, for r = 1..k and j = k..r.
    auto blend = [&](double lo, double hi, int i, int r) {
        const double den = t[i + k + 1 - r] - t[i];
        const double a = den == 0.0 ? 0.0 : (x - t[i]) / den;
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

__device__ double nre_of(int kind) {
    switch (kind) {
        case TB_PROFILE_EXP: return 4.0;
        case TB_PROFILE_GAUSSIAN: return 6.0;
        default: return 8.0;   // deV, Sersic
    }
}

// Copies the profile tables into shared memory (the spline evaluations make
// many dependent lookups) and returns a table view pointing there.
__device__ tb_profile_tables stage_tables(const tb_profile_tables& G, unsigned char* smem) {
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

__host__ __device__ inline int tables_smem_bytes(const tb_profile_tables& G) {
    return 8 * (G.n_knots + G.n_coefs + 2 * G.n_ranges + 2 * G.exp_K + 2 * G.dev_K) +
           4 * (4 * G.n_ranges + 4 * G.n_splines);
}

// Sum over lanes 0..K-1 of v, accumulated in lane order (the reference's
// sequential numpy sum for these short vectors).
__device__ __forceinline__ double lane_sum(double v, int K) {
    double s = 0.0;
    for (int k = 0; k < K; k++) s += __shfl_sync(0xffffffffu, v, k);
    return s;
}

// One warp per source.  Lane l < K evaluates component l's amplitude and
// log-variance splines; sums and the stable variance ranking use shuffles;
// the shape and geometry are computed redundantly by every lane.
__global__ void __launch_bounds__(kPrepThreads)
galaxy_fft_prep_kernel(const tb_galaxy_src* __restrict__ srcs, int n, tb_fft_image img,
                       tb_profile_tables Tg, tb_fft_item* __restrict__ items,
                       double* __restrict__ camp, double* __restrict__ cvar, int stride,
                       int32_t* __restrict__ flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const tb_profile_tables T = stage_tables(Tg, smem_raw);
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * (kPrepThreads / 32) + (threadIdx.x >> 5);
    if (i >= n) return;   // whole warps leave together
    const tb_galaxy_src s = srcs[i];

    // ---- profile: lane l holds component l ----
    double a = 0.0, v = 0.0;
    int K = -1;
    if (s.profile == TB_PROFILE_EXP || s.profile == TB_PROFILE_DEV) {
        const bool ex = s.profile == TB_PROFILE_EXP;
        K = ex ? T.exp_K : T.dev_K;
        if (K > kMaxComp) K = -1;
        else if (lane < K) {
            a = ex ? T.exp_amp[lane] : T.dev_amp[lane];
            v = ex ? T.exp_var[lane] : T.dev_var[lane];
        }
    } else if (s.profile == TB_PROFILE_GAUSSIAN) {
        K = 1;
        if (lane == 0) { a = 1.0; v = 1.0; }
    } else {
        double nn = s.sersic_n;
        const double lowest = T.range_lohi[0], highest = T.range_lohi[2 * T.n_ranges - 1];
        int r = -1;
        if (nn <= lowest) { r = 0; nn = lowest; }
        else if (nn >= highest) { r = T.n_ranges - 1; nn = highest; }
        else {
            for (int q = 0; q < T.n_ranges; q++)
                if (T.range_lohi[2 * q] <= nn && nn < T.range_lohi[2 * q + 1]) { r = q; break; }
        }
        if (r >= 0) {
            const int Kr = T.range_info[4 * r], sa = T.range_info[4 * r + 1];
            const int sv = T.range_info[4 * r + 2];
            if (Kr + 1 <= kMaxComp) {
                if (lane < Kr) {
                    a = bspline(T, sa + lane, nn);
                    v = exp(bspline(T, sv + lane, nn));
                }
                a /= lane_sum(a, Kr);
                K = Kr;
                if (nn > 1.0) {
                    const double core = bspline(T, T.core_spline, nn);
                    a *= (1.0 - core) / lane_sum(a, Kr);
                    if (lane == Kr) { a = core; v = 0.0; }
                    K = Kr + 1;
                }
            }
        }
    }
    // stable rank by increasing variance (sersic.py:338-341)
    int rank = 0;
    for (int j = 0; j < (K > 0 ? K : 0); j++) {
        const double vj = __shfl_sync(0xffffffffu, v, j);
        rank += (vj < v) || (vj == v && j < lane);
    }

    // ---- shape -> basis G -> pixel covariance factor M = T T^T ----
    double re, G[4];
    if (s.shape_type == TB_SHAPE_RABPHI) {
        const double phi = (90.0 - s.s2) * (TB_PI / 180.0);
        re = s.s0;
        const double r_deg = fmax(1.0 / 30.0, s.s0) / 3600.0;
        const double cp = cos(phi), sp = sin(phi);
        G[0] = r_deg * cp;
        G[1] = r_deg * sp * s.s1;
        G[2] = -r_deg * sp;
        G[3] = r_deg * cp * s.s1;
    } else {
        double e1 = s.s1, e2 = s.s2;
        re = s.s0;
        if (s.shape_type == TB_SHAPE_ELLIPSE_ESOFT) {
            re = exp(s.s0);
            const double ee = hypot(s.s1, s.s2);
            const double e = fmin(0.999999, 1.0 - exp(-ee));
            const double th = atan2(s.s2, s.s1) / 2.0;
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
    const double* C = img.cd_inv;
    const double T0 = C[0] * G[0] + C[1] * G[2], T1 = C[0] * G[1] + C[1] * G[3];
    const double T2 = C[2] * G[0] + C[3] * G[2], T3 = C[2] * G[1] + C[3] * G[3];
    const double M00 = T0 * T0 + T1 * T1, M01 = T0 * T2 + T1 * T3, M11 = T2 * T2 + T3 * T3;

    // ---- geometry (ModelMask given) ----
    const double px = s.px, py = s.py;
    const int x0 = s.mx0, y0 = s.my0, x1 = s.mx0 + s.mw, y1 = s.my0 + s.mh;
    double hs = fmax(s.mh / 2.0, s.mw / 2.0);
    hs = fmax(hs, fmax(fmax(1 + px - x0, 1 + x1 - px), fmax(1 + py - y0, 1 + y1 - py)));
    hs = fmax(hs, fmax(img.psf_w / 2.0, img.psf_h / 2.0));
    const double hsi = ceil(hs);
    int sz = 1;
    while (sz < 2.0 * hsi && sz < (1 << 20)) sz *= 2;
    const bool out = px < x0 || px > x1 - 1 || py < y0 || py > y1 - 1;
    const int si = sz == 32 ? 0 : sz == 64 ? 1 : sz == 128 ? 2 : sz == 256 ? 3 : -1;
    int flag = 0;
    if (K < 0 || s.mw <= 0 || s.mh <= 0) {
        flag = 2;
    } else if (s.counts == 0.0) {
        flag = 1;
    } else if (out) {
        double ndx = 0.0, ndy = 0.0;
        if (px < x0) ndx = x0 - px;
        if (px > x1) ndx = px - x1;
        if (py < y0) ndy = y0 - py;
        if (py > y1) ndy = py - y1;
        const double nearest = hypot(ndx, ndy);
        flag = (nearest > nre_of(s.profile) * re / img.pixscale) ? 1 : 2;
    } else if (si < 0 || img.spec_off[si] < 0) {
        flag = 2;
    }
    const int c0 = i * stride;
    if (flag == 0 && lane < K) {
        camp[c0 + rank] = a;
        double* w = cvar + 4 * (c0 + rank);
        w[0] = v * M00;
        w[1] = v * M01;
        w[2] = v * M01;
        w[3] = v * M11;
    }
    if (lane == 0) {
        tb_fft_item it;
        it.c0 = c0;
        it.K = 0;
        it.sz = 32;
        it.mode = TB_MOG_STORE;
        it.mw = s.mw;
        it.mh = s.mh;
        it.sx = 0;
        it.sy = 0;
        it.mux = 0.0;
        it.muy = 0.0;
        it.scale = (float)s.counts;
        it.ldo = 0;
        it.out_off = s.out_off;
        it.spec_off = img.spec_off[0] >= 0 ? img.spec_off[0] : 0;
        if (flag == 0) {
            const double dx = px - img.psf_cx[si], dy = py - img.psf_cy[si];
            double mux = dx - x0, muy = dy - y0;
            const double sxd = rint(mux), syd = rint(muy);
            it.K = K;
            it.sz = sz;
            it.sx = (int)sxd;
            it.sy = (int)syd;
            it.mux = mux - sxd;
            it.muy = muy - syd;
            it.spec_off = img.spec_off[si];
        }
        items[i] = it;
        flags[i] = flag;
    }
}

}  // namespace

extern "C" int tb_galaxy_fft_prep(const tb_galaxy_src* srcs, int32_t n, const tb_fft_image* image,
                                  const tb_profile_tables* tables, tb_fft_item* items,
                                  double* comp_amp, double* comp_var, int32_t comp_stride,
                                  int32_t* flags, void* stream) {
    if (n < 0) return TB_ERR_ARG;
    if (n == 0) return TB_OK;
    if (!srcs || !image || !tables || !items || !comp_amp || !comp_var || !flags) return TB_ERR_ARG;
    if (comp_stride < kMaxComp) return TB_ERR_SIZE;
    const int smem = tables_smem_bytes(*tables);
    if (smem > TB_PROFILE_SMEM_MAX) return TB_ERR_SIZE;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(galaxy_fft_prep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem) != cudaSuccess)
        return TB_ERR_LAUNCH;
    const int per_block = kPrepThreads / 32;
    galaxy_fft_prep_kernel<<<(n + per_block - 1) / per_block, kPrepThreads, smem,
                             (cudaStream_t)stream>>>(
        srcs, n, *image, *tables, items, comp_amp, comp_var, comp_stride, flags);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}
