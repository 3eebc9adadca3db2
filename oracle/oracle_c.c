/* Oracle (test infrastructure, never the product path): a plain-C restatement
 * of the reference Tractor's native pixel kernels, used by tests/, the smoke
 * check and bench.py's CPU baseline leg to check the CUDA path.
 *
 * Each function states the reference lines it follows.  Loops keep the
 * reference's evaluation order and precision (double for the grid / ring
 * evaluators and the Fourier transform, float for the masked evaluator and the
 * Lanczos correlation) so results agree with the reference to rounding.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* Per-component constants of a 2-D Gaussian: the inverse covariance with the
 * -1/2 of the exponent and the factor 2 of the cross term folded in, and the
 * normalisation amp / (2 pi sqrt(det)).  tractor/approx3.c:101-125. */
typedef struct {
    double q0, q1, q2; /* exponent = q0 dx^2 + q1 dx dy + q2 dy^2 */
    double scale;
    double floor_;     /* smallest exponent that is evaluated */
} orc_gauss;

static void orc_prepare(int K, const double* amp, const double* var,
                        double minval, orc_gauss* g) {
    const double twopi2 = 4.0 * M_PI * M_PI; /* (2 pi)^D, D = 2 */
    double ampsum = 0.0;
    for (int k = 0; k < K; k++) ampsum += amp[k];
    for (int k = 0; k < K; k++) {
        const double* V = var + 4 * k;
        double vxx = V[0], vxy = 0.5 * (V[1] + V[2]), vyy = V[3];
        double det = vxx * vyy - vxy * vxy;
        double f = -0.5 / det;
        g[k].q0 = vyy * f;
        g[k].q1 = -2.0 * vxy * f;
        g[k].q2 = vxx * f;
        g[k].scale = amp[k] / sqrt(twopi2 * det);
        double fl = -100.0;
        if (minval > 0.0) {
            fl = log(minval * sqrt(twopi2 * det) / ampsum);
            if (fl < -100.0) fl = -100.0;
        }
        g[k].floor_ = fl;
    }
}

/* Value (and optional d/dmean) of the mixture at offset (x, y) from the
 * mixture origin.  tractor/mix.i:44-82 (eval_all_dxy). */
static double orc_eval(int K, const orc_gauss* g, const double* mean,
                       double x, double y, double* dmx, double* dmy) {
    double r = 0.0;
    if (dmx) *dmx = 0.0;
    if (dmy) *dmy = 0.0;
    for (int k = 0; k < K; k++) {
        double dx = x - mean[2 * k], dy = y - mean[2 * k + 1];
        double e = g[k].q0 * dx * dx + g[k].q1 * dx * dy + g[k].q2 * dy * dy;
        if (!(e >= g[k].floor_) || !isfinite(e)) continue;
        double G = g[k].scale * exp(e);
        r += G;
        if (dmx) *dmx += -G * (2.0 * g[k].q0 * dx + g[k].q1 * dy);
        if (dmy) *dmy += -G * (2.0 * g[k].q2 * dy + g[k].q1 * dx);
    }
    return r;
}

/* Plain mixture value (no floor other than -100), tractor/mix.i:19-42. */
static double orc_eval_plain(int K, const orc_gauss* g, const double* mean,
                             double x, double y) {
    double r = 0.0;
    for (int k = 0; k < K; k++) {
        double dx = x - mean[2 * k], dy = y - mean[2 * k + 1];
        double e = g[k].q0 * dx * dx + g[k].q1 * dx * dy + g[k].q2 * dy * dy;
        if (e < -100.0) continue;
        r += g[k].scale * exp(e);
    }
    return r;
}

/* Exact rectangle evaluation, accumulated into out[(y-y0)*(x1-x0) + x-x0].
 * Components with Mahalanobis^2 >= 100 at a pixel are skipped there.
 * tractor/mix.i:452-524 (c_gauss_2d_grid).  Returns 0, or -1 on bad sizes. */
int orc_mog_grid(int x0, int x1, int y0, int y1, double fx, double fy, int K,
                 const double* amp, const double* mean, const double* var,
                 double* out) {
    if (x1 < x0 || y1 < y0 || K < 0) return -1;
    const double tpd = 4.0 * M_PI * M_PI;
    double* iv = (double*)malloc(sizeof(double) * 4 * (K > 0 ? K : 1));
    for (int k = 0; k < K; k++) {
        const double* V = var + 4 * k;
        double det = V[0] * V[3] - V[1] * V[2];
        iv[4 * k + 0] = V[3] / det;
        iv[4 * k + 1] = -(V[1] + V[2]) / det;
        iv[4 * k + 2] = V[0] / det;
        iv[4 * k + 3] = amp[k] / sqrt(tpd * det);
    }
    int i = 0;
    for (int iy = y0; iy < y1; iy++) {
        for (int ix = x0; ix < x1; ix++, i++) {
            for (int k = 0; k < K; k++) {
                double dx = ix - fx - mean[2 * k];
                double dy = iy - fy - mean[2 * k + 1];
                double d2 = iv[4 * k] * dx * dx + iv[4 * k + 1] * dx * dy +
                            iv[4 * k + 2] * dy * dy;
                if (d2 >= 100.0) continue;
                out[i] += iv[4 * k + 3] * exp(-0.5 * d2);
            }
        }
    }
    free(iv);
    return 0;
}

/* Ring-growing evaluation with a value floor (c_gauss_2d_approx3,
 * tractor/approx3.c:1-465).  Starting at pixel (xc, yc) -- or, if it is
 * outside the box, at the brightest pixel on the nearest box edge(s)
 * (approx3.c:127-168) -- square rings of radius R = 1, 2, ... are visited.
 * A ring pixel is evaluated if a neighbour in the previous ring marked it;
 * an evaluated pixel marks its outward neighbours if R <= minradius or its
 * value is >= minval.  Top/bottom rows own the ring corners.  Growth stops
 * when a ring evaluates nothing.  out / dx / dy (may be NULL) receive values
 * (assigned, not accumulated) at evaluated pixels; bbox[4] receives the
 * tight extent [sx0, sx1) x [sy0, sy1) of evaluated pixels in box-relative
 * coordinates.  The derivative outputs are d/dmean. */
int orc_mog_approx3(int x0, int x1, int y0, int y1, double fx, double fy,
                    double minval, int K, const double* amp,
                    const double* mean, const double* var, double* out,
                    double* dxo, double* dyo, int xc, int yc, int minradius,
                    int* bbox) {
    const int W = x1 - x0, H = y1 - y0;
    if (W <= 0 || H <= 0 || K <= 0) return -1;
    orc_gauss* g = (orc_gauss*)malloc(sizeof(orc_gauss) * K);
    orc_prepare(K, amp, var, minval, g);

    if (xc < x0 || yc < y0 || xc >= x1 || yc >= y1) {
        int bx = (x0 + x1) / 2, by = (y0 + y1) / 2;
        double best = 0.0;
        if (xc < x0 || xc >= x1) {
            int ex = (xc < x0) ? x0 : x1 - 1;
            for (int iy = y0; iy < y1; iy++) {
                double v = orc_eval_plain(K, g, mean, ex - fx, iy - fy);
                if (v > best) { best = v; bx = ex; by = iy; }
            }
        }
        if (yc < y0 || yc >= y1) {
            int ey = (yc < y0) ? y0 : y1 - 1;
            for (int ix = x0; ix < x1; ix++) {
                double v = orc_eval_plain(K, g, mean, ix - fx, ey - fy);
                if (v > best) { best = v; bx = ix; by = ey; }
            }
        }
        xc = bx;
        yc = by;
    }

    /* Row (top/bottom, indexed by x) and column (left/right, indexed by y)
     * marks for the current ring and the next one. */
    uint8_t* buf = (uint8_t*)calloc(4 * (size_t)W + 4 * (size_t)H, 1);
    uint8_t *curT = buf, *curB = buf + W, *nxtT = buf + 2 * W, *nxtB = buf + 3 * W;
    uint8_t *curL = buf + 4 * W, *curR = curL + H, *nxtL = curL + 2 * H,
            *nxtR = curL + 3 * H;
#define MARK(a, i, lo, hi) do { int _i = (i); if (_i >= (lo) && _i < (hi)) (a)[_i - (lo)] = 1; } while (0)

    if (yc > y0) { MARK(nxtB, xc - 1, x0, x1); MARK(nxtB, xc, x0, x1); MARK(nxtB, xc + 1, x0, x1); }
    if (yc < y1 - 1) { MARK(nxtT, xc - 1, x0, x1); MARK(nxtT, xc, x0, x1); MARK(nxtT, xc + 1, x0, x1); }
    if (xc > x0) MARK(nxtL, yc, y0, y1);
    if (xc < x1 - 1) MARK(nxtR, yc, y0, y1);

    {
        size_t o = (size_t)(yc - y0) * W + (xc - x0);
        out[o] = orc_eval(K, g, mean, xc - fx, yc - fy, dxo ? dxo + o : NULL,
                          dyo ? dyo + o : NULL);
    }
    int sx0 = xc - x0, sx1 = sx0, sy0 = yc - y0, sy1 = sy0;

    for (int R = 1;; R++) {
        uint8_t* t;
        t = curT; curT = nxtT; nxtT = t;
        t = curB; curB = nxtB; nxtB = t;
        t = curL; curL = nxtL; nxtL = t;
        t = curR; curR = nxtR; nxtR = t;
        memset(nxtT, 0, W); memset(nxtB, 0, W);
        memset(nxtL, 0, H); memset(nxtR, 0, H);
        int any = 0;

        /* Top and bottom rows of the ring (they own the corners). */
        for (int side = 0; side < 2; side++) {
            int yy = side == 0 ? yc + R : yc - R;
            if (side == 0 ? (yy >= y1) : (yy < y0)) continue;
            uint8_t* cur = side == 0 ? curT : curB;
            uint8_t* nxt = side == 0 ? nxtT : nxtB;
            int inward = side == 0 ? -1 : +1; /* the row toward the centre */
            int rowhit = 0;
            for (int i = 0; i < W; i++) {
                if (!cur[i]) continue;
                any = rowhit = 1;
                int xx = x0 + i;
                size_t o = (size_t)(yy - y0) * W + i;
                double r = orc_eval(K, g, mean, xx - fx, yy - fy,
                                    dxo ? dxo + o : NULL, dyo ? dyo + o : NULL);
                out[o] = r;
                if (R > minradius && r < minval) continue;
                if (xx == xc - R && xx > x0) { MARK(nxtL, yy, y0, y1); MARK(nxtL, yy + inward, y0, y1); }
                if (xx == xc + R && xx < x1 - 1) { MARK(nxtR, yy, y0, y1); MARK(nxtR, yy + inward, y0, y1); }
                if (side == 0 ? (yy < y1 - 1) : (yy > y0)) {
                    MARK(nxt, xx - 1, x0, x1); MARK(nxt, xx, x0, x1); MARK(nxt, xx + 1, x0, x1);
                }
            }
            if (rowhit) {
                if (side == 0) sy1 = yy - y0; else sy0 = yy - y0;
            }
        }
        /* Left and right columns. */
        for (int side = 0; side < 2; side++) {
            int xx = side == 0 ? xc - R : xc + R;
            if (side == 0 ? (xx < x0) : (xx >= x1)) continue;
            uint8_t* cur = side == 0 ? curL : curR;
            uint8_t* nxt = side == 0 ? nxtL : nxtR;
            int colhit = 0;
            for (int j = 0; j < H; j++) {
                if (!cur[j]) continue;
                any = colhit = 1;
                int yy = y0 + j;
                size_t o = (size_t)j * W + (xx - x0);
                double r = orc_eval(K, g, mean, xx - fx, yy - fy,
                                    dxo ? dxo + o : NULL, dyo ? dyo + o : NULL);
                out[o] = r;
                if (R > minradius && r < minval) continue;
                if (side == 0 ? (xx > x0) : (xx < x1 - 1)) {
                    MARK(nxt, yy - 1, y0, y1); MARK(nxt, yy, y0, y1); MARK(nxt, yy + 1, y0, y1);
                }
            }
            if (colhit) {
                if (side == 0) sx0 = xx - x0; else sx1 = xx - x0;
            }
        }
        if (!any) break;
    }
#undef MARK
    bbox[0] = sx0;
    bbox[1] = sx1 + 1;
    bbox[2] = sy0;
    bbox[3] = sy1 + 1;
    free(buf);
    free(g);
    return 0;
}

/* Float evaluation on a boolean mask with d/dmean outputs
 * (c_gauss_2d_masked, tractor/gauss_masked.c:1-159 with eval_all_dxy_f,
 * tractor/mix.i:85-142).  Components whose constants are not finite are
 * dropped; exponents below -30 are skipped.  Returns 1 when every component
 * was dropped (nothing written), else 0. */
int orc_mog_masked(int x0, int y0, int W, int H, double fxd, double fyd,
                   int K, const float* amp, const float* mean,
                   const float* var, float* out, float* dxo, float* dyo,
                   const uint8_t* mask) {
    const float fx = (float)fxd, fy = (float)fyd;
    const float tpd = (float)(4.0 * M_PI * M_PI);
    float* c = (float*)malloc(sizeof(float) * 4 * (K > 0 ? K : 1));
    int live = 0;
    for (int k = 0; k < K; k++) {
        float vxx = var[4 * k], vxy = (var[4 * k + 1] + var[4 * k + 2]) * 0.5f,
              vyy = var[4 * k + 3];
        float det = vxx * vyy - vxy * vxy;
        float f = (float)(-0.5 / det);
        float q0 = vyy * f, q1 = (float)(-vxy * f * 2.0), q2 = vxx * f;
        float s = (float)(amp[k] / sqrt(tpd * det));
        if (!(isfinite(vxx) && isfinite(vxy) && isfinite(vyy) && isfinite(q0) &&
              isfinite(q1) && isfinite(q2) && isfinite(s))) {
            s = 0.f;
            q0 = q1 = q2 = -1.f;
        }
        c[4 * k] = q0; c[4 * k + 1] = q1; c[4 * k + 2] = q2; c[4 * k + 3] = s;
        if (s != 0.f) live = 1;
    }
    if (!live) { free(c); return 1; }
    for (int j = 0; j < H; j++) {
        for (int i = 0; i < W; i++) {
            size_t o = (size_t)j * W + i;
            if (!mask[o]) continue;
            float x = (float)(x0 + i) - fx, y = (float)(y0 + j) - fy;
            float r = 0.f, gx = 0.f, gy = 0.f;
            for (int k = 0; k < K; k++) {
                const float* q = c + 4 * k;
                if (q[3] == 0.f) continue;
                float dx = x - mean[2 * k], dy = y - mean[2 * k + 1];
                float e = q[0] * dx * dx + q[1] * dx * dy + q[2] * dy * dy;
                if (!(e >= -30.f) || !isfinite(e)) continue;
                float G = q[3] * expf(e);
                r += G;
                /* the reference accumulates these in double, one store to
                 * float per term */
                gx = (float)((double)gx - (double)G * (2.0 * q[0] * dx + (double)(q[1] * dy)));
                gy = (float)((double)gy - (double)G * (2.0 * q[2] * dy + (double)(q[1] * dx)));
            }
            out[o] = r;
            if (dxo) dxo[o] = gx;
            if (dyo) dyo[o] = gy;
        }
    }
    free(c);
    return 0;
}

/* Normalised Lanczos-3 taps for a shift dx in [-0.5, 0.5]
 * (tractor/mp_fourier.i:355-402): the 7 taps sample the kernel at
 * i - 3 + dx; the one tap that falls outside |t| < 3 is zero and the other six
 * are normalised to sum to 1. */
void orc_lanczos3_taps(double dx, double* taps) {
    for (int i = 0; i < 7; i++) taps[i] = 0.0;
    if (dx == 0.0) { taps[3] = 1.0; return; }
    int lo = dx > 0.0 ? 0 : 1, hi = dx > 0.0 ? 6 : 7;
    double s = 0.0;
    for (int i = lo; i < hi; i++) {
        double t = M_PI * (i - 3.0 + dx);
        taps[i] = 3.0 * sin(t) * sin(t / 3.0) / (t * t);
        s += taps[i];
    }
    for (int i = lo; i < hi; i++) taps[i] /= s;
}

/* One 7-tap correlation pass along rows of a (rows x n) float array, with
 * zero samples beyond both ends, written transposed into dst (n x rows).
 * Taps are rounded to float first and sums run tap by tap in float, as in
 * tractor/mp_fourier.i:267-352. */
static void orc_corr7_rows_T(const float* src, int rows, int n,
                             const float* f, float* dst) {
    for (int j = 0; j < rows; j++) {
        const float* s = src + (size_t)j * n;
        for (int i = 0; i < n; i++) {
            /* output i sums f[k] * s[i - 3 + k] over the in-range k, in
             * increasing k */
            float acc = 0.0f;
            int k0 = 3 - i > 0 ? 3 - i : 0;
            int k1 = n + 3 - i < 7 ? n + 3 - i : 7;
            for (int k = k0; k < k1; k++) acc += f[k] * s[i - 3 + k];
            dst[(size_t)i * rows + j] = acc;
        }
    }
}

/* Separable Lanczos-3 shift of an H x W float image by (dx, dy)
 * (lanczos_shift_3f, tractor/mp_fourier.i:405-429).  work holds H*W floats. */
void orc_lanczos_shift3f(const float* in, float* out, int H, int W, double dx,
                         double dy, float* work) {
    double tx[7], ty[7];
    float fx[7], fy[7];
    orc_lanczos3_taps(dx, tx);
    orc_lanczos3_taps(dy, ty);
    for (int i = 0; i < 7; i++) { fx[i] = (float)tx[i]; fy[i] = (float)ty[i]; }
    orc_corr7_rows_T(in, H, W, fx, work);   /* work is W x H */
    orc_corr7_rows_T(work, W, H, fy, out);  /* out is H x W */
}

/* Zero-mean mixture spectrum on an rfft grid
 * (gaussian_fourier_transform_zero_mean, tractor/mp_fourier.i:431-478):
 * out[j, i] = sum_k amp_k exp(-2 pi^2 (a v_i^2 + 2 b v_i w_j + d w_j^2)),
 * with a delta component (a = b = d = 0) contributing amp_k. */
void orc_fourier_mog(int K, const double* amp, const double* var, int NV,
                     const double* v, int NW, const double* w, double* out) {
    const double c = -2.0 * M_PI * M_PI;
    for (int j = 0; j < NW; j++) {
        for (int i = 0; i < NV; i++) {
            double s = 0.0;
            for (int k = 0; k < K; k++) {
                double a = var[4 * k], b = var[4 * k + 1], d = var[4 * k + 3];
                if (a == 0.0 && b == 0.0 && d == 0.0) { s += amp[k]; continue; }
                double vv = v[i] * v[i], ww = w[j] * w[j];
                s += amp[k] * exp(c * (a * vv + 2.0 * b * v[i] * w[j] + d * ww));
            }
            out[(size_t)j * NV + i] = s;
        }
    }
}
