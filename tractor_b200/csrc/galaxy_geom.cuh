// Per-source geometry of the Fourier path and the warp-level preparation of
// one galaxy (sm_100a), shared by the prep kernel (galaxy_prep.cu) and the
// fused prep + render kernel (fourier_render.cu):
//   geometry: half-size for a ModelMask (tractor/galaxy.py:339-351), FFT
//             size (tractor/psf.py:209-212), source-outside-mask rule
//             (galaxy.py:353-374), integer / sub-pixel split with
//             half-to-even rounding (galaxy.py:383-406).
#pragma once
#include "profile_eval.cuh"

namespace tb {

constexpr int kMaxComp = 10;   // components per source (Sersic mixtures: <= 9 + core)

// Patch geometry for a ModelMask: half-size (galaxy.py:339-351), FFT size
// (psf.py:209-212), the source-outside-mask rule (galaxy.py:353-374).
// flag: 0 render, 1 no patch, 2 unsupported; si: index of sz in 32..256.
__device__ inline void prep_geometry(const tb_galaxy_src& s, const tb_fft_image& img, int K, double re,
                              int& flag, int& sz, int& si) {
    const double px = s.px, py = s.py;
    const int x0 = s.mx0, y0 = s.my0, x1 = s.mx0 + s.mw, y1 = s.my0 + s.mh;
    double hs = fmax(s.mh / 2.0, s.mw / 2.0);
    hs = fmax(hs, fmax(fmax(1 + px - x0, 1 + x1 - px), fmax(1 + py - y0, 1 + y1 - py)));
    hs = fmax(hs, fmax(img.psf_w / 2.0, img.psf_h / 2.0));
    const double hsi = ceil(hs);
    sz = 1;
    while (sz < 2.0 * hsi && sz < (1 << 20)) sz *= 2;
    const bool out = px < x0 || px > x1 - 1 || py < y0 || py > y1 - 1;
    si = sz == 32 ? 0 : sz == 64 ? 1 : sz == 128 ? 2 : sz == 256 ? 3 : -1;
    flag = 0;
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
        flag = (nearest > tb::nre_of(s.profile) * re / img.pixscale) ? 1 : 2;
    } else if (si < 0 || img.spec_off[si] < 0) {
        flag = 2;
    }
}

// Fills a rendered item's geometry: integer / sub-pixel split of the offset
// with half-to-even rounding (galaxy.py:383-406).
__device__ inline void item_geometry(const tb_galaxy_src& s, const tb_fft_image& img, int sz, int si,
                              tb_fft_item& it) {
    const double dx = s.px - img.psf_cx[si], dy = s.py - img.psf_cy[si];
    const double mux = dx - s.mx0, muy = dy - s.my0;
    const double sxd = rint(mux), syd = rint(muy);
    it.sz = sz;
    it.sx = (int)sxd;
    it.sy = (int)syd;
    it.mux = mux - sxd;
    it.muy = muy - syd;
    it.spec_off = img.spec_off[si];
}

// One warp prepares source s (galaxy_fft_prep_kernel's work for one
// source): lane l < K ends with component l's amplitude `a` and unit-r_e
// variance `v` at its rank by increasing variance (sersic.py:338-341), M the
// pixel-space factor T T^T, and every lane with the flag (0 render, 1 no
// patch, 2 unsupported) and, when the flag is 0, the item `it` (K, FFT size,
// offsets, ...).  Returns K (< 0: unknown profile).
__device__ inline int prep_galaxy_warp(const tb_galaxy_src& s, const tb_fft_image& img,
                                       const tb_profile_tables& T, int lane, double& a,
                                       double& v, int& rank, double M[3], int& flag,
                                       tb_fft_item& it) {
    const int K = warp_profile(T, s.profile, s.sersic_n, lane, kMaxComp, a, v);
    rank = variance_rank(v, K, lane);
    double re, G[4];
    shape_basis(s.shape_type, s.s0, s.s1, s.s2, G, re);
    pixel_factor(img.cd_inv, G, M[0], M[1], M[2]);
    int sz, si;
    prep_geometry(s, img, K, re, flag, sz, si);
    it.c0 = 0;
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
    it.dmode = TB_FFT_VALUE;
    it.dc0 = 0;
    it.dot_off = 0;
    if (flag == 0) {
        it.K = K;
        item_geometry(s, img, sz, si, it);
    }
    return K;
}

}  // namespace tb
