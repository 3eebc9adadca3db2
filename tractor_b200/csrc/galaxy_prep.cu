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
#include "galaxy_geom.cuh"

namespace {

using tb::kMaxComp;
using tb::prep_geometry;
using tb::item_geometry;
constexpr int kPrepThreads = 128;   // 4 sources (warps) per block

// One warp per source.  Lane l < K evaluates component l's amplitude and
// log-variance splines; sums and the stable variance ranking use shuffles;
// the shape and geometry are computed redundantly by every lane.
__global__ void __launch_bounds__(kPrepThreads)
galaxy_fft_prep_kernel(const tb_galaxy_src* __restrict__ srcs, int n, tb_fft_image img,
                       tb_profile_tables Tg, tb_fft_item* __restrict__ items,
                       double* __restrict__ camp, double* __restrict__ cvar, int stride,
                       int32_t* __restrict__ flags) {
    // The tables are read where they lie (L1-cached): each warp touches only
    // its range's few knots and coefficients, and copying all of them into
    // shared memory first cost each block more latency than it saved.
    const tb_profile_tables T = Tg;
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * (kPrepThreads / 32) + (threadIdx.x >> 5);
    if (i >= n) return;   // whole warps leave together
    const tb_galaxy_src s = srcs[i];
    // profile (lane l holds component l, ranked by variance), shape -> pixel
    // factor M = T T^T, geometry and the item
    double a, v, M[3];
    int rank, flag;
    tb_fft_item it;
    const int K = tb::prep_galaxy_warp(s, img, T, lane, a, v, rank, M, flag, it);
    const int c0 = i * stride;
    if (flag == 0 && lane < K) {
        camp[c0 + rank] = a;
        double* w = cvar + 4 * (c0 + rank);
        w[0] = v * M[0];
        w[1] = v * M[1];
        w[2] = v * M[1];
        w[3] = v * M[2];
    }
    if (lane == 0) {
        it.c0 = c0;
        items[i] = it;
        flags[i] = flag;
    }
}


constexpr double kHn = 1e-5;   // central-difference step in the Sersic index
constexpr double kHs = 1e-6;   // central-difference step in shape parameters

__device__ void shape_factor(const tb_fft_image& img, int shape_type, double s0, double s1,
                             double s2, double M[3], double& re) {
    double G[4];
    tb::shape_basis(shape_type, s0, s1, s2, G, re);
    tb::pixel_factor(img.cd_inv, G, M[0], M[1], M[2]);
}

// Jacobian items: per source 7 items (x, y, counts, s0, s1, s2, n) on the
// value item's geometry.  Position: the derivative Lanczos taps; counts: the
// unit-flux render; shape and index: the spectrum's derivative with
// coefficients (da_k, dC_k) in dcoef -- dC = v_k dM/ds_j for the shape, and
// (da_k, dv_k M) for the Sersic index -- by FP64 central differences of the
// exact maps (the range held fixed for n).
__global__ void __launch_bounds__(kPrepThreads)
galaxy_fft_jac_prep_kernel(const tb_galaxy_src* __restrict__ srcs, int n, tb_fft_image img,
                           tb_profile_tables Tg, tb_fft_item* __restrict__ items,
                           double* __restrict__ camp, double* __restrict__ cvar,
                           double* __restrict__ dcoef, int stride, int mode, int64_t col_stride,
                           int32_t* __restrict__ flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const tb_profile_tables T = tb::stage_tables(Tg, smem_raw);
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * (kPrepThreads / 32) + (threadIdx.x >> 5);
    if (i >= n) return;
    const tb_galaxy_src s = srcs[i];

    double a = 0.0, v = 0.0, da = 0.0, dv = 0.0;
    int K;
    if (s.profile == TB_PROFILE_SERSIC) {
        double nn = s.sersic_n;
        const double lowest = T.range_lohi[0], highest = T.range_lohi[2 * T.n_ranges - 1];
        int r = -1;
        bool clamped = false;
        if (nn <= lowest) { r = 0; nn = lowest; clamped = true; }
        else if (nn >= highest) { r = T.n_ranges - 1; nn = highest; clamped = true; }
        else {
            for (int q = 0; q < T.n_ranges; q++)
                if (T.range_lohi[2 * q] <= nn && nn < T.range_lohi[2 * q + 1]) { r = q; break; }
        }
        if (r < 0 || T.range_info[4 * r] + 1 > kMaxComp) {
            K = -1;
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
        }
    } else {
        K = tb::warp_profile(T, s.profile, s.sersic_n, lane, kMaxComp, a, v);
    }
    // sorted by variance (sersic.py:338-341), the permutation kept for the
    // derivative
    const int rank = tb::variance_rank(v, K, lane);

    double M[3], re;
    shape_factor(img, s.shape_type, s.s0, s.s1, s.s2, M, re);
    double dM[3][3];
    const double sp[3] = {s.s0, s.s1, s.s2};
#pragma unroll
    for (int j = 0; j < 3; j++) {
        double hp[3] = {sp[0], sp[1], sp[2]}, hm[3] = {sp[0], sp[1], sp[2]};
        hp[j] += kHs;
        hm[j] -= kHs;
        double Mp[3], Mm[3], rr;
        shape_factor(img, s.shape_type, hp[0], hp[1], hp[2], Mp, rr);
        shape_factor(img, s.shape_type, hm[0], hm[1], hm[2], Mm, rr);
#pragma unroll
        for (int q = 0; q < 3; q++) dM[j][q] = (Mp[q] - Mm[q]) / (2.0 * kHs);
    }

    int flag, sz, si;
    prep_geometry(s, img, K, re, flag, sz, si);
    const int c0 = i * stride;
    if (flag == 0 && lane < K) {
        const int c = c0 + rank;
        camp[c] = a;
        double* w = cvar + 4 * c;
        w[0] = v * M[0];
        w[1] = v * M[1];
        w[2] = v * M[1];
        w[3] = v * M[2];
        for (int j = 0; j < 4; j++) {
            double* d = dcoef + 4 * ((int64_t)(4 * i + j) * stride + rank);
            if (j < 3) {
                d[0] = 0.0;
                d[1] = v * dM[j][0];
                d[2] = v * dM[j][1];
                d[3] = v * dM[j][2];
            } else {
                d[0] = da;
                d[1] = dv * M[0];
                d[2] = dv * M[1];
                d[3] = dv * M[2];
            }
        }
    }
    if (lane < 7) {
        const int j = lane;
        tb_fft_item it;
        it.c0 = c0;
        it.K = 0;
        it.sz = 32;
        it.mode = mode;
        it.mw = s.mw;
        it.mh = s.mh;
        it.sx = 0;
        it.sy = 0;
        it.mux = 0.0;
        it.muy = 0.0;
        it.scale = j == 2 ? 1.0f : (float)s.counts;
        it.ldo = 0;
        it.out_off = s.out_off + j * col_stride;
        it.spec_off = img.spec_off[0] >= 0 ? img.spec_off[0] : 0;
        it.dmode = j == 0 ? TB_FFT_DX : j == 1 ? TB_FFT_DY : j == 2 ? TB_FFT_VALUE : TB_FFT_DSPEC;
        it.dc0 = j >= 3 ? (4 * i + (j - 3)) * stride : 0;
        it.dot_off = 7 * (int64_t)i + j;
        if (flag == 0) {
            it.K = K;
            item_geometry(s, img, sz, si, it);
        }
        items[7 * (int64_t)i + j] = it;
    }
    if (lane == 0) flags[i] = flag;
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
    const int per_block = kPrepThreads / 32;
    galaxy_fft_prep_kernel<<<(n + per_block - 1) / per_block, kPrepThreads, 0,
                             (cudaStream_t)stream>>>(
        srcs, n, *image, *tables, items, comp_amp, comp_var, comp_stride, flags);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

extern "C" int tb_galaxy_fft_jac_prep(const tb_galaxy_src* srcs, int32_t n, const tb_fft_image* image,
                                      const tb_profile_tables* tables, tb_fft_item* items,
                                      double* comp_amp, double* comp_var, double* comp_dcoef,
                                      int32_t comp_stride, int32_t mode, int64_t col_stride,
                                      int32_t* flags, void* stream) {
    if (n < 0) return TB_ERR_ARG;
    if (n == 0) return TB_OK;
    if (!srcs || !image || !tables || !items || !comp_amp || !comp_var || !comp_dcoef || !flags)
        return TB_ERR_ARG;
    if (mode != TB_MOG_STORE && mode != TB_MOG_ACCUM && mode != TB_FFT_DOT) return TB_ERR_ARG;
    if (comp_stride < kMaxComp) return TB_ERR_SIZE;
    const int smem = tb::tables_smem_bytes(*tables);
    if (smem > TB_PROFILE_SMEM_MAX) return TB_ERR_SIZE;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(galaxy_fft_jac_prep_kernel,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
        return TB_ERR_LAUNCH;
    const int per_block = kPrepThreads / 32;
    galaxy_fft_jac_prep_kernel<<<(n + per_block - 1) / per_block, kPrepThreads, smem,
                                 (cudaStream_t)stream>>>(srcs, n, *image, *tables, items,
                                                         comp_amp, comp_var, comp_dcoef,
                                                         comp_stride, mode, col_stride, flags);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}
