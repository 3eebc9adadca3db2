/* Test infrastructure (oracle only): exported entry points for the reference's
 * Fourier / Lanczos kernels, whose C text oracle/build_ref.sh copies verbatim
 * out of tractor/mp_fourier.i into ref_mpf_blocks.c (static functions there).
 *
 *   correlate7f                          tractor/mp_fourier.i:154-249
 *   correlate7f_inout                    tractor/mp_fourier.i:267-352
 *   lanczos_filter_3                     tractor/mp_fourier.i:355-402
 *   lanczos_shift_3f                     tractor/mp_fourier.i:405-429
 *   gaussian_fourier_transform_zero_mean tractor/mp_fourier.i:431-478
 *
 * The signatures are the SWIG-expanded (pointer, dims...) forms, so ctypes
 * can call them with numpy buffers directly.
 */
#include <string.h>
#include "ref_mpf_blocks.c"

void ref_correlate7f(float* img, int h, int w, double* fx, int nfx, double* fy,
                     int nfy, float* work, int wh, int ww) {
    correlate7f(img, h, w, fx, nfx, fy, nfy, work, wh, ww);
}

void ref_correlate7f_inout(float* in, int ih, int iw, float* out, int oh,
                           int ow, double* fx, int nfx, double* fy, int nfy,
                           float* work, int wh, int ww) {
    correlate7f_inout(in, ih, iw, out, oh, ow, fx, nfx, fy, nfy, work, wh, ww);
}

void ref_lanczos_filter_3(double* filt, double dx) { lanczos_filter_3(filt, dx); }

void ref_lanczos_shift_3f(float* in, int ih, int iw, float* out, int oh,
                          int ow, double dx, double dy, float* work, int wh,
                          int ww) {
    lanczos_shift_3f(in, ih, iw, out, oh, ow, dx, dy, work, wh, ww);
}

void ref_gaussian_fourier_transform_zero_mean(double* amps, int K,
                                              double* vars, int d1, int d2,
                                              int d3, double* v, int nv,
                                              double* w, int nw, double* out,
                                              int o1, int o2) {
    gaussian_fourier_transform_zero_mean(amps, K, vars, d1, d2, d3, v, nv, w,
                                         nw, out, o1, o2);
}
