/*
 * tractor_b200 -- C ABI of the B200 (sm_100a) forward-model kernels.
 *
 * Every pointer argument is a DEVICE pointer unless stated otherwise, every
 * call is asynchronous on the given CUDA stream (a cudaStream_t passed as
 * void*, NULL = legacy default stream), and every call returns an int status
 * (TB_OK = 0) after validating its arguments on the host; it never aborts the
 * process.  Kernels additionally write per-call status words to device memory
 * (tb_status, may be NULL; zeroed by the call on its stream before the
 * launch) that the caller reads after synchronising.  The library allocates
 * no memory: callers own every buffer, including workspaces, and may call
 * from one stream per host thread.  Its only global state is the scratch
 * array of tb_solve_update_noalloc with that array's cached per-device
 * addresses, and the device counter of tensor-core wait timeouts read by
 * tb_tensor_core_timeouts.
 *
 * Each entry point names the reference interface (file:line in the Tractor
 * source tree) whose computation it replaces.
 */
#ifndef TRACTOR_B200_H
#define TRACTOR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TB_OK 0
#define TB_ERR_ARG -1        /* invalid argument (null pointer, bad size) */
#define TB_ERR_LAUNCH -2     /* CUDA launch or attribute error */
#define TB_ERR_SIZE -3       /* a size exceeds what this kernel supports */

/* Device-written status: code 0 = ok; otherwise the first failing work item
 * and a kernel-specific detail (non-finite value, unsupported size, ...). */
typedef struct {
    int32_t code;
    int32_t item;
    int32_t detail;
    int32_t count;
} tb_status;

#define TB_STATUS_NONFINITE 1
#define TB_STATUS_BAD_ITEM 2
#define TB_STATUS_NOT_SPD 3

/* ------------------------------------------------------------------------
 * Mixture-of-Gaussians pixel evaluation
 *
 * One item = one 2-D Gaussian mixture evaluated on one rectangle
 * [x0, x0+w) x [y0, y0+h).  Component k of an item (k in [0, K)) is
 * comp_amp[c0+k], comp_mean[2(c0+k)..], comp_var[4(c0+k)..] (2x2 row-major,
 * FP64, as MixtureOfGaussians stores them), evaluated at pixel (x, y) as
 *     scale * amp / (2 pi sqrt(det V)) * exp(-0.5 d^T V^-1 d),
 *     d = (x - fx - mean_x, y - fy - mean_y).
 * A component is skipped at a pixel when its exponent is below `floor`
 * (natural-log units): -50 reproduces c_gauss_2d_grid's Mahalanobis^2 >= 100
 * cut, -30 c_gauss_2d_masked's, and approx3's per-component minval floor is
 * log(minval * 2 pi sqrt(det) / sum(amp)) clamped at -100.
 * Output: out[out_off + (y-y0)*ldo + (x-x0)] (float32; ldo = 0 means w).
 * mask_off >= 0 selects a uint8 mask, masks[mask_off + (y-y0)*w + (x-x0)] --
 * unmasked pixels are written 0 -- and mask_off < 0 means the full
 * rectangle.
 * ------------------------------------------------------------------------ */
typedef struct {
    int32_t x0, y0, w, h;
    int32_t c0, K;
    int32_t mode;      /* TB_MOG_STORE, TB_MOG_ACCUM or TB_MOG_ATOMIC */
    int32_t ldo;       /* output row stride in elements (0 = w) */
    double fx, fy;     /* evaluation offset added to every mean */
    double floor;      /* TB_FLOOR_FIXED: exponent floor (natural-log units);
                          TB_FLOOR_MINVAL: minval (see below) */
    float scale;       /* output multiplier (counts for a model patch) */
    int32_t floor_mode;
    int64_t out_off;   /* element offset of this item's output */
    int64_t mask_off;  /* element offset of this item's mask, or -1 */
    int64_t tile0;     /* exclusive prefix of tiles (32x32) over items */
    int64_t deriv_off; /* >= 0: also write d/dmean_x and d/dmean_y (times
                          scale), two w x h planes at out + deriv_off */
    int32_t diff_c0;   /* >= 0: a difference item (see below); -1 otherwise */
    int32_t pad;
} tb_mog_item;

/* Difference items (diff_c0 >= 0): the item evaluates
 *     scale * sum_k [G'_k(x, y) - G_k(x, y)]
 * where G_k is component c0+k and G'_k component diff_c0+k, both with the
 * MEAN of component c0+k: the difference of two renders of the same
 * rectangle (a finite-difference derivative column, e.g. the Sersic-index
 * step of SersicGalaxy.getParamDerivatives, tractor/sersic.py:416-444)
 * computed as G_k (s'_k expm1(e'_k - e_k) + (s'_k - s_k)), so that its
 * error is relative to the difference, not to the two renders.  The floor
 * is tested on the base exponent.  Requires floor_mode TB_FLOOR_FIXED and
 * deriv_off < 0. */

/* TB_FLOOR_MINVAL: each component k gets the floor
 * max(-100, log(minval * 2 pi sqrt(det V_k) / sum(amp))), the per-component
 * cut of c_gauss_2d_approx3 (tractor/approx3.c:101-125); `floor` holds
 * minval. */
#define TB_FLOOR_FIXED 0
#define TB_FLOOR_MINVAL 1

/* Output modes: STORE writes, ACCUM adds (items must not overlap in the
 * output), ATOMIC adds with atomics (overlapping items allowed, e.g. many
 * sources into one image; the summation order is then unspecified). */
#define TB_MOG_STORE 0
#define TB_MOG_ACCUM 1
#define TB_MOG_ATOMIC 2
#define TB_MOG_TILE 32
#define TB_MOG_MAX_K 256

/* Batched MoG evaluation into per-item patches.  Replaces
 * c_gauss_2d_grid (tractor/mix.i:452-524) and c_gauss_2d_masked
 * (tractor/gauss_masked.c:1-159, values only), called per source by
 * MixtureOfGaussians.evaluate_grid / evaluate_grid_masked
 * (tractor/mixture_profiles.py:248-331).
 * n_tiles = sum over items of ceil(w/32)*ceil(h/32) (= the last item's tile0
 * plus its own tiles).  work_counter: one int32 of device scratch, zeroed by
 * this call on `stream` before the launch. */
int tb_mog_render(const tb_mog_item* items, int32_t n_items, int64_t n_tiles,
                  const double* comp_amp, const double* comp_mean,
                  const double* comp_var, const uint8_t* masks, float* out,
                  int32_t* work_counter, tb_status* status, void* stream);

/* tb_mog_render over HOST buffers, the way c_gauss_2d_grid /
 * c_gauss_2d_masked (tractor/mix.i:452-524, tractor/gauss_masked.c:1-159)
 * take and fill numpy arrays: items[n_items], comp_amp[n_comp],
 * comp_mean[2 n_comp], comp_var[4 n_comp], masks[mask_bytes] (may be NULL
 * when mask_bytes = 0) are read from host memory, the n_out output elements
 * are written to host `out` and the launch's status word to host `status`.
 * Staging goes through two caller-owned buffers of
 * tb_mog_render_host_bytes() bytes each: `pinned` (page-locked host memory,
 * e.g. cudaHostAlloc) and `workspace` (device memory); the call packs the
 * inputs into `pinned`, copies them to `workspace` in one copy, renders,
 * copies the output and status back in one copy and synchronises `stream`
 * before returning, so both buffers may be reused at once.  Every item must
 * lie inside the given sizes (components, mask, output; tile0 the exclusive
 * prefix of its tiles, n_tiles their total), else TB_ERR_ARG before any
 * copy; ws_bytes smaller than needed gives TB_ERR_SIZE.  Outputs that no
 * item writes, and the targets of TB_MOG_ACCUM / TB_MOG_ATOMIC items, start
 * at zero. */
int tb_mog_render_host_bytes(int32_t n_items, int64_t n_comp, int64_t mask_bytes,
                             int64_t n_out, int64_t* bytes);
int tb_mog_render_host(const tb_mog_item* items, int32_t n_items, int64_t n_tiles,
                       const double* comp_amp, const double* comp_mean,
                       const double* comp_var, int64_t n_comp, const uint8_t* masks,
                       int64_t mask_bytes, float* out, int64_t n_out, tb_status* status,
                       void* pinned, void* workspace, int64_t ws_bytes, void* stream);

/* c_gauss_2d_approx3's evaluated region (tractor/approx3.c:126-442) over
 * values tb_mog_render has already written for a whole box with the
 * TB_FLOOR_MINVAL floors: starting at (xc, yc) -- or, when that is outside
 * the box, at the largest value of the edge column / row the caller
 * evaluated (edge_col_off / edge_row_off, -1 for none; column first, ties to
 * the first, the default start (dcx, dcy) when no value is above 0) -- square
 * rings R = 1, 2, ... are visited; a ring pixel counts as evaluated when a
 * pixel of the previous ring marked it (the reference's next-T/B/L/R arrays:
 * a passing pixel -- R <= minradius or value >= minval -- marks its
 * neighbours on the next ring, top and bottom rows own the corners), and the
 * walk stops at the first ring with nothing evaluated.  Every other pixel of
 * the box is set to 0 (and of the d/dx, d/dy planes when deriv_off >= 0),
 * and extent[4 i ..] = (sx0, sx1, sy0, sy1), box-relative with exclusive
 * upper ends, updated per ring by its rows (y) and columns (x) as
 * approx3.c does.  w, h <= TB_RING_MAX.  One CTA per item. */
#define TB_RING_MAX 4096
typedef struct {
    int64_t val_off;       /* the box's w x h values in vals */
    int64_t deriv_off;     /* >= 0: two more w x h planes, zeroed alike */
    int64_t edge_col_off;  /* >= 0: h values of column edge_x (start search) */
    int64_t edge_row_off;  /* >= 0: w values of row edge_y */
    int32_t w, h;
    int32_t xc, yc;        /* start pixel, box-relative */
    int32_t edge_x, edge_y;
    int32_t dcx, dcy;      /* default start, box-relative */
    int32_t minradius;
    int32_t start_inside;  /* 1: (xc, yc) is inside the box */
    double minval;
} tb_ring_item;

int tb_approx3_region(const tb_ring_item* items, int32_t n_items, float* vals,
                      int32_t* extent, tb_status* status, void* stream);

/* ------------------------------------------------------------------------
 * Lanczos-3 sub-pixel shift
 * ------------------------------------------------------------------------ */

/* Batched separable Lanczos-3 shift of n float32 images of h x w (contiguous,
 * image i at in + i*h*w) by (shift[2i], shift[2i+1]) in [-0.5, 0.5], with
 * zero samples outside each image.  Replaces lanczos_shift_3f
 * (tractor/mp_fourier.i:405-429; taps mp_fourier.i:355-402, correlation
 * mp_fourier.i:267-352) as called by lanczos_shift_image
 * (tractor/psf.py:26-58).  in and out must not overlap. */
int tb_lanczos3_shift(const float* in, float* out, const double* shift,
                      int32_t n, int32_t h, int32_t w, void* stream);

/* ------------------------------------------------------------------------
 * Pixelized-PSF (Fourier) galaxy rendering
 *
 * One item = one galaxy rendered through the FFT path of
 * ProfileGalaxy._realGetUnitFluxModelPatch with a ModelMask
 * (tractor/galaxy.py:336-519, non-hybrid): the zero-mean mixture spectrum
 * (gaussian_fourier_transform_zero_mean, mp_fourier.i:431-478) times the
 * PSF spectrum, inverse real FFT of size sz x sz (numpy irfftn,
 * galaxy.py:457-465), Lanczos-3 shift by (mux, muy), integer shift by
 * (sx, sy) into the mh x mw mask.  sz is a power of two in [32, 256].
 * psf_spec: sz x (sz/2+1) complex64 (interleaved re, im) per PSF, stored
 * column-major (element (row j, column v) at v*sz + j), an item's spectrum
 * at psf_spec + spec_off floats, as written by tb_psf_spectrum.  Components: amp[c0+k] and the
 * sheared 2x2 covariance var[4(c0+k)..] (FP64); a zero covariance is a delta
 * component.  Output: float32 mh x mw at out + out_off (row stride ldo, or
 * mw if ldo = 0), times `scale`.  Items taller than 128 pixels at sz = 256
 * are rendered in row chunks.
 * ------------------------------------------------------------------------ */
typedef struct {
    int32_t c0, K;
    int32_t sz;
    int32_t mode;      /* TB_MOG_STORE, TB_MOG_ACCUM or TB_MOG_ATOMIC */
    int32_t mw, mh;
    int32_t sx, sy;
    double mux, muy;
    float scale;
    int32_t ldo;       /* output row stride in elements (0 = mw) */
    int64_t out_off;
    int64_t spec_off;  /* float offset of this item's PSF spectrum in psf_spec */
    int32_t dmode;     /* TB_FFT_VALUE, or a derivative (see below) */
    int32_t dc0;       /* TB_FFT_DSPEC: coefficients at comp_dcoef[4 (dc0 + k) ..] */
    int64_t dot_off;   /* mode TB_FFT_DOT: result slot in dots */
} tb_fft_item;

#define TB_FFT_MAX_SZ 256
/* Derivative items (tb_fourier_render_deriv): DSPEC renders
 * d/dtheta sum_k a_k exp(-2 pi^2 f^T C_k f) from per-component (da_k,
 * dC_k00, dC_k01, dC_k11); DX / DY render the derivative with respect to the
 * sub-pixel shift mux / muy (the Lanczos-3 taps' derivative). */
#define TB_FFT_VALUE 0
#define TB_FFT_DSPEC 1
#define TB_FFT_DX 2
#define TB_FFT_DY 3
/* DIFF renders the difference of two mixtures with the same geometry:
 * per component the spectrum a'_k exp(-2 pi^2 f^T C'_k f) - a_k exp(-2 pi^2
 * f^T C_k f) = exp(-2 pi^2 f^T C_k f) (a'_k expm1(-2 pi^2 f^T (C'_k - C_k) f)
 * + (a'_k - a_k)), from per-component (a'_k - a_k, C'_k - C_k) in
 * comp_dcoef -- a finite-difference column (the Sersic-index step of
 * tractor/sersic.py:416-444) with its error relative to the difference. */
#define TB_FFT_DIFF 4
/* Output mode of a Fourier item: instead of writing its pixels, accumulate
 * sum over its pixels of out[pixel] * value into dots[dot_off] (out then
 * holds the upstream gradient, read only): the vector-Jacobian product. */
#define TB_FFT_DOT 3

int tb_fourier_render(const tb_fft_item* items, int32_t n_items,
                      const double* comp_amp, const double* comp_var,
                      const float* psf_spec, float* out, int32_t* work_counter,
                      tb_status* status, void* stream);

/* tb_fourier_render with derivative items and the TB_FFT_DOT output mode:
 * the analytic parameter derivatives of the Fourier path that
 * Galaxy.getParamDerivatives / SersicGalaxy.getParamDerivatives
 * (tractor/galaxy.py:137-223, tractor/sersic.py:402-445) approximate by
 * finite differences, and their contraction with an upstream gradient.
 * comp_dcoef may be NULL when no item is DSPEC, dots when none is DOT. */
int tb_fourier_render_deriv(const tb_fft_item* items, int32_t n_items,
                            const double* comp_amp, const double* comp_var,
                            const double* comp_dcoef, const float* psf_spec, float* out,
                            double* dots, int32_t* work_counter, tb_status* status,
                            void* stream);

/* The same renders (values, derivative items, TB_FFT_DOT) through the
 * split spectral path: a column kernel (units of 16 rfft columns of one
 * item: the mixture spectrum times the PSF spectrum and the y taps'
 * response, inverse FFT along y, the real parts only of the DC and Nyquist
 * columns) writes the kept rows of every column to `workspace`
 * (L2-resident: at most 256 items per column / row launch pair), and a row
 * kernel (units of 16 kept rows: times the x taps' response, inverse FFT
 * along x, two real rows per complex transform) writes the output.  Items
 * whose Lanczos-3 window reaches the FFT box edge, and TB_FFT_DOT items, go
 * to tb_fourier_render_deriv's kernel in a third launch.  Results equal
 * tb_fourier_render's up to FP32 rounding.  workspace: device, 256-byte
 * aligned, at least tb_fourier_workspace(n_items) bytes. */
int tb_fourier_workspace(int32_t n_items, int64_t* bytes);
int tb_fourier_render_split(const tb_fft_item* items, int32_t n_items,
                            const double* comp_amp, const double* comp_var,
                            const double* comp_dcoef, const float* psf_spec, float* out,
                            double* dots, void* workspace, int64_t workspace_bytes,
                            tb_status* status, void* stream);

/* ------------------------------------------------------------------------
 * Galaxy preparation for the Fourier path
 *
 * Turns source parameters into tb_fft_item work items and component tables
 * on the device: the profile mixture (exp, deV, Gaussian, or the Sersic
 * mixture of tractor/sersic.py:288-342 evaluated from its spline knots and
 * coefficients), the shape's pixel-space covariance T V T^T with
 * T = cdInverse * getRaDecBasis() (HoggGalaxy._getShearedProfile,
 * tractor/galaxy.py:659-669; EllipseE / EllipseESoft / GalaxyShape bases),
 * the patch half-size and FFT size for a ModelMask (galaxy.py:339-351,
 * psf.py:209-212), and the integer / sub-pixel split of the offset
 * (galaxy.py:383-406, np.round's half-to-even rounding).
 * ------------------------------------------------------------------------ */
typedef struct {
    double px, py;       /* pixel position */
    double counts;       /* brightness in counts: the output scale */
    double s0, s1, s2;   /* shape parameters, see shape_type */
    double sersic_n;     /* Sersic index (profile TB_PROFILE_SERSIC) */
    int64_t out_off;     /* element offset of this source's mh x mw output */
    int32_t profile;     /* TB_PROFILE_* */
    int32_t shape_type;  /* TB_SHAPE_* */
    int32_t mx0, my0, mw, mh;  /* ModelMask */
} tb_galaxy_src;

#define TB_PROFILE_EXP 0
#define TB_PROFILE_DEV 1
#define TB_PROFILE_SERSIC 2
#define TB_PROFILE_GAUSSIAN 3
#define TB_SHAPE_ELLIPSE_E 0      /* (re, e1, e2), tractor/ellipses.py:13-155 */
#define TB_SHAPE_ELLIPSE_ESOFT 1  /* (log re, ee1, ee2), ellipses.py:165-263 */
#define TB_SHAPE_RABPHI 2         /* GalaxyShape (re, ab, phi), galaxy.py:37-89 */

/* Constants of one image: WCS inverse CD matrix and pixel scale, PSF size,
 * and for each FFT size 32, 64, 128, 256 the PSF centre in the padded PSF
 * image and the float offset of its spectrum (-1 if not provided).  Passed by
 * host pointer, read at call time. */
typedef struct {
    double cd_inv[4];
    double pixscale;
    int32_t psf_w, psf_h;
    double psf_cx[4], psf_cy[4];
    int64_t spec_off[4];
} tb_fft_image;

/* Profile tables in device memory (pointers), passed by host pointer. */
typedef struct {
    int32_t n_ranges;
    int32_t core_spline;          /* spline index of the core fraction */
    const double* range_lohi;     /* 2 per Sersic-index range */
    const int32_t* range_info;    /* 4 per range: K, first amp spline, first log-var spline,
                                     1 if all its splines share the first one's knots
                                     (at most 32) and degree, else 0 */
    const int32_t* spline_info;   /* 4 per spline: knot offset, knot count, coef offset, degree */
    const double* knots;
    const double* coefs;
    const double* exp_amp;
    const double* exp_var;
    const double* dev_amp;
    const double* dev_var;
    int32_t exp_K, dev_K;
    int32_t n_splines, n_knots, n_coefs, pad;
} tb_profile_tables;

#define TB_PROFILE_SMEM_MAX 49152  /* bytes of tables the prep kernels that stage them hold */

/* flags[i]: 0 = item written; 1 = no patch (zero counts, or the source lies
 * outside its mask farther than its radius: getModelPatch returns None);
 * 2 = unsupported here (source outside its mask but within its radius -- the
 * reference raises for a non-hybrid PSF -- or an FFT size above 256).
 * Items not written get K = 0.  Components: comp_stride (>= 10) slots per
 * source at comp_amp + i*comp_stride, comp_var + 4*i*comp_stride. */
int tb_galaxy_fft_prep(const tb_galaxy_src* srcs, int32_t n, const tb_fft_image* image,
                       const tb_profile_tables* tables, tb_fft_item* items,
                       double* comp_amp, double* comp_var, int32_t comp_stride,
                       int32_t* flags, void* stream);

/* Mixture spectrum times PSF spectrum on the full sz x (sz/2 + 1) rfft grid,
 * for Fourier-path galaxies whose FFT size exceeds 256 (tb_fourier_render's
 * limit): out[w][v] (row-major, interleaved complex64: the input of an
 * inverse 2-D real FFT) = psf_spec[v][w] (column-major, as
 * tb_psf_spectrum writes it) x sum_k amp_k exp(-2 pi^2 f^T var_k f),
 * f = (v, fftfreq(w)) / sz; with comp_dcoef (K rows of a'_k - a_k, dC00,
 * dC01, dC11; may be NULL) the difference of the two mixtures as
 * TB_FFT_DIFF items render it.  K <= 128.  Replaces
 * MixtureOfGaussians.getFourierTransform(v, w, zero_mean=True) times P in
 * ProfileGalaxy._realGetUnitFluxModelPatch (tractor/galaxy.py:457-470,
 * tractor/mp_fourier.i:405-430); the caller runs the inverse transform, the
 * Lanczos-3 shift (tb_lanczos3_shift) and the crop. */
int tb_fourier_spectrum_grid(const double* comp_amp, const double* comp_var,
                             const double* comp_dcoef, int32_t K, const float* psf_spec,
                             int32_t sz, float* out, void* stream);

/* tb_galaxy_fft_prep and tb_fourier_render in one persistent launch: each
 * source is prepared (as tb_galaxy_fft_prep) by one warp straight into
 * shared memory and rendered (as tb_fourier_render) by its block, so no
 * component tables go through global memory; the patches are bit-for-bit
 * those of the two-launch path.  The per-source work of
 * ProfileGalaxy._realGetUnitFluxModelPatch's FFT branch times its counts
 * (tractor/galaxy.py:336-519) for a non-hybrid PixelizedPSF, as the two
 * entry points it joins.  psf_spec: the spectra image->spec_off points into
 * (tb_psf_spectrum).  flags as tb_galaxy_fft_prep; items (may be NULL):
 * receives each source's item (c0 = 0: its components stay on chip).
 * work_counter: one int32 of device scratch. */
int tb_galaxy_fft_render(const tb_galaxy_src* srcs, int32_t n, const tb_fft_image* image,
                         const tb_profile_tables* tables, const float* psf_spec, float* out,
                         tb_fft_item* items, int32_t* flags, int32_t* work_counter,
                         tb_status* status, void* stream);

/* Jacobian items of n galaxies: items[7 i + j] for the parameters j = x, y,
 * counts, s0, s1, s2 (shape, per shape_type), Sersic n of source i, on the
 * geometry tb_galaxy_fft_prep gives its value item, with out_off =
 * srcs[i].out_off + j * col_stride and dot_off = 7 i + j.  comp_dcoef:
 * 4 * n * comp_stride * 4 doubles (per source and shape / index parameter,
 * per component: da, dC00, dC01, dC11), by FP64 central differences of the
 * profile (Sersic range held fixed) and of the shape's T T^T.  mode:
 * TB_MOG_STORE / TB_MOG_ACCUM (Jacobian patches) or TB_FFT_DOT (with
 * col_stride 0: the upstream gradient patch at srcs[i].out_off). */
int tb_galaxy_fft_jac_prep(const tb_galaxy_src* srcs, int32_t n, const tb_fft_image* image,
                           const tb_profile_tables* tables, tb_fft_item* items,
                           double* comp_amp, double* comp_var, double* comp_dcoef,
                           int32_t comp_stride, int32_t mode, int64_t col_stride,
                           int32_t* flags, void* stream);

/* Forward real FFT of n zero-padded sz x sz float32 PSF images (prepared by
 * the caller, image i at pad + i*sz*sz) into complex64 spectra
 * sz x (sz/2+1) (interleaved, column-major as tb_fourier_render reads them),
 * optionally divided by |P[0,0]|.  Replaces
 * np.fft.rfft2 + astype(complex64) in PixelizedPSF.getFourierTransform
 * (tractor/psf.py:249-280) and NormalizedPsf (psf.py:947-953). */
int tb_psf_spectrum(const float* pad, float* spec, int32_t n, int32_t sz,
                    int32_t normalize, void* stream);

/* ------------------------------------------------------------------------
 * Scene rendering: many sources into whole images (mixture-of-Gaussians PSFs)
 *
 * The batched form of Tractor.getModelImage (tractor/engine.py:424-445) for
 * images whose PSF is a Gaussian mixture: every source's getModelPatch with
 * a rectangular ModelMask (galaxy.py:266-326 run_mog with evaluate_grid,
 * PointSource via GaussianMixturePSF.getPointSourcePatch, psf.py:458-528),
 * times its counts, added into a float32 image (Patch.addTo clips to the
 * image, patch.py:341-354).  One record per (source, image): a source seen
 * in several images (bands) has one record per image, each with its counts.
 * ------------------------------------------------------------------------ */
typedef struct {
    double px, py;          /* pixel position in this image */
    double counts;          /* brightness in this image's counts */
    double fdev;            /* TB_PROFILE_COMPOSITE: deV fraction, clamped to [0, 1] */
    double sa0, sa1, sa2;   /* shape (see shape_type): the galaxy's, or the exp
                               part of a composite */
    double sb0, sb1, sb2;   /* deV shape of a composite */
    double sersic_n;        /* TB_PROFILE_SERSIC */
    int32_t profile;        /* TB_PROFILE_* (incl. POINT and COMPOSITE) */
    int32_t shape_type;     /* TB_SHAPE_* (both shapes of a composite) */
    int32_t image;          /* index into the image table */
    int32_t mx0, my0, mw, mh;  /* ModelMask rectangle (image pixels) */
    int32_t pad;
} tb_scene_src;

#define TB_PROFILE_POINT 4       /* PointSource (tractor/pointsource.py) */
#define TB_PROFILE_COMPOSITE 5   /* FixedCompositeGalaxy (galaxy.py:779-1029) */

/* One image: size, output placement, PSF mixture and WCS.  tile0 = the
 * exclusive prefix over images of ceil(W/32) * ceil(H/tile_h) for the tile
 * height passed to tb_scene_render; n_tiles = the total. */
typedef struct {
    int32_t W, H;
    int32_t ldo;            /* row stride in elements (0 = W) */
    int32_t psf_c0, psf_K;  /* PSF components psf_amp[psf_c0 + k] (k < psf_K <= 32) */
    int32_t pad;
    int64_t out_off;        /* element offset of pixel (0, 0) in `out` */
    int64_t tile0;
    double cd_inv[4];       /* WCS cdInverse (row-major), NullWCS: I * 3600 / pixscale */
    double pixscale;
} tb_scene_image;

/* A prepared (source, image) record.  flag: 0 = rendered; 1 = no patch
 * (zero counts, or the mask misses the image); 2 = unsupported (bad image
 * index, unknown profile, too many components). */
typedef struct {
    int32_t x0, y0, w, h;   /* rectangle: the mask clipped to the image */
    int32_t c0, K;          /* components comp_*[c0 .. c0+K) */
    int32_t image;
    int32_t flag;
    double fx, fy;          /* evaluation offset (point sources: the position) */
    float scale;            /* counts */
    float floor;            /* exponent floor, natural-log units (-50: the grid cut) */
} tb_scene_item;

/* Prepares n records: profile mixture (exp / deV / Sersic / Gaussian /
 * composite / point), shape to pixel covariance, convolution with the
 * image's PSF mixture (mixture_profiles.py:158-172: PSF component outer,
 * galaxy component inner), rectangle.  Components of record i go to
 * comp_*[i * comp_stride ...] (FP64; mean 2, var 4 values per component),
 * K = (galaxy components) x psf_K <= comp_stride <= 256. */
int tb_scene_prep(const tb_scene_src* srcs, int32_t n, const tb_scene_image* images,
                  int32_t n_images, const double* psf_amp, const double* psf_mean,
                  const double* psf_var, const tb_profile_tables* tables,
                  tb_scene_item* items, double* comp_amp, double* comp_mean,
                  double* comp_var, int32_t comp_stride, void* stream);

/* Workspace bytes tb_scene_render needs for n_tiles tiles and at most
 * max_pairs (item, tile) overlaps (host call, writes *bytes). */
int tb_scene_workspace(int64_t n_tiles, int64_t max_pairs, int64_t* bytes);

/* Renders every image: bins the items by image tile (32 x tile_h pixels,
 * tile_h 16, 32 or 64), then one persistent launch evaluates each tile's
 * sources in item order (each source's components summed first, as a
 * patch, then added inside its rectangle) and writes the tile once.
 * mode TB_MOG_STORE writes every pixel of every image (0 where no source
 * reaches), TB_MOG_ACCUM adds to `out`.  Summation order is the item order
 * for tiles reached by at most 1024 items.  max_pairs bounds the (item,
 * tile) overlaps; more are reported as TB_STATUS_BAD_ITEM (detail -3). */
int tb_scene_render(const tb_scene_item* items, int32_t n_items,
                    const tb_scene_image* images, int32_t n_images, int64_t n_tiles,
                    int32_t tile_h, const double* comp_amp, const double* comp_mean,
                    const double* comp_var, float* out, int32_t mode, void* workspace,
                    int64_t workspace_bytes, int64_t max_pairs, tb_status* status,
                    void* stream);

/* ------------------------------------------------------------------------
 * Least-squares step
 * ------------------------------------------------------------------------ */

/* Normal equations of one or more independent least-squares problems.
 * Problem b has P[b] parameters and R[b] rows; its design matrix is stored
 * column-major at A + a_off[b] with leading dimension lda[b] (rows), its
 * right-hand side at rhs + r_off[b].  Writes (FP64) AtA[b] (P x P, at
 * ata_off[b], exactly symmetric) and Atr[b] (P, at atr_off[b]).  For
 * max_p <= 255 the products run on the tensor cores (tcgen05 kind::tf32):
 * each value is split into TF32 hi + lo parts and hi*hi + hi*lo + lo*hi is
 * accumulated in FP32 over at most 128 rows, then summed in FP64 (about 22
 * significant bits per product).  For 255 < max_p <= 320 FP32 CUDA-core
 * products are accumulated by compensated (two-sum) FP32 partial sums
 * combined in FP64.  max_p must bound every P[b]; a problem above it is
 * skipped.  A tensor-core wait that times out (1 s) writes NaN into that
 * problem's outputs and counts in tb_tensor_core_timeouts.
 * Replaces the sparse A / b assembly and LSQR solve of
 * LsqrOptimizer.getUpdateDirection (tractor/lsqr_optimizer.py:328-644). */
int tb_normal_equations(const float* A, const float* rhs, const int64_t* a_off,
                        const int64_t* r_off, const int32_t* lda,
                        const int32_t* P, const int32_t* R,
                        const int64_t* ata_off, const int64_t* atr_off,
                        double* AtA, double* Atr, int32_t n_problems,
                        int32_t max_p, void* stream);

/* Number of tensor-core waits that timed out since the library was loaded
 * on the current device (0 in a healthy run).  Synchronous. */
int tb_tensor_core_timeouts(uint32_t* count);

/* Solves each problem's column-scaled normal equations in FP64 on the device
 * (column scaling as lsqr_optimizer.py:470-489 with scale = sqrt(diag),
 * Cholesky with a `damp`^2 ridge, one step of iterative refinement) and
 * writes X[x_off[b] + i] = update / colscale (zero for empty columns).
 * info[b] = 0 ok, >0 the failing pivot (not positive definite; X is then
 * zero, as LsqrOptimizer returns a zero update on failure,
 * lsqr_optimizer.py:586-604), -1 if P[b] > 320 or P[b] > max_p (the
 * problem is skipped and its X left as it was).  work: caller-owned FP64
 * scratch of n_problems * max_p * max_p elements (the Cholesky factors). */
int tb_solve_update(const double* AtA, const double* Atr,
                    const int64_t* ata_off, const int64_t* atr_off,
                    const int32_t* P, const int64_t* x_off, double* X,
                    int32_t* info, double damp, int32_t n_problems,
                    int32_t max_p, double* work, void* stream);

/* Allocation-free variant of tb_solve_update (no counterpart in the
 * reference).  For callers that cannot allocate device memory when they
 * call -- code that runs under another allocator that owns the device
 * memory, or latency-bound loops where an allocation, which can
 * synchronise the device, is not acceptable -- and so cannot provide the
 * `work` buffer.  The Cholesky factors go to a file-scope scratch array of
 * TB_SOLVE_NOALLOC_MAX_DOUBLES doubles (8 MiB) that the library holds on
 * every GPU that loads it, until the process exits.  Requires
 * n_problems * max_p * max_p <= TB_SOLVE_NOALLOC_MAX_DOUBLES, else returns
 * TB_ERR_SIZE.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) with that device current; make that first
 * call before any stream capture.  All calls share the one array: calls
 * whose kernels overlap on the GPU (different streams, or different host
 * threads) race and must be serialised by the caller.  The array keeps the
 * previous call's contents; the solver writes every factor entry it reads,
 * so nothing needs clearing.  Allocates nothing (no cudaMalloc / cudaFree).
 * info[b] as tb_solve_update (-1 for P[b] > max_p: the factors of one
 * problem never reach another's slice of the array).  The cached address
 * (an atomic per device) belongs to the device's primary context: after
 * cudaDeviceReset the library must be unloaded and loaded again. */
#define TB_SOLVE_NOALLOC_MAX_DOUBLES 1048576
int tb_solve_update_noalloc(const double* AtA, const double* Atr,
                            const int64_t* ata_off, const int64_t* atr_off,
                            const int32_t* P, const int64_t* x_off, double* X,
                            int32_t* info, double damp, int32_t n_problems,
                            int32_t max_p, void* stream);

/* ------------------------------------------------------------------------
 * Batched blob fitting (Levenberg-Marquardt over many independent blobs)
 *
 * The batched form of Tractor.optimize_loop with LsqrOptimizer
 * (tractor/lsqr_optimizer.py:280-326; engine.py:279-339 getDerivs,
 * engine.py:455-473 getChiImage) and ConstrainedOptimizer's step limits
 * (tractor/constrained_optimizer.py:12-159) for galaxies and point sources
 * seen in up to 3 bands through mixture-of-Gaussians PSFs.  A blob is a set
 * of sources and one image per band (all of one size, aligned); every
 * (blob, band) image is a "unit".
 *
 * Parameters: TB_FIT_NPAR slots per source, in the reference's order for a
 * SersicGalaxy with NanoMaggies brightness and an EllipseESoft shape:
 * x, y (pixels), flux[3] (counts; LinearPhotoCal(1)), log r_e, ee1, ee2,
 * Sersic n.  Unused slots (missing bands, the index of exp / deV galaxies,
 * the shape of point sources) have zero derivative and never move.
 * Source k of blob b is sources[b.src0 + k]; its parameters start at
 * params[TB_FIT_NPAR * (b.src0 + k)].
 * ------------------------------------------------------------------------ */
#define TB_FIT_NPAR 9
#define TB_FIT_MAX_BANDS 3
#define TB_FIT_MAX_SRC 32
#define TB_FIT_MAX_PSF 4
#define TB_FIT_SERSIC_MIN 0.29   /* SersicIndex bounds, tractor/sersic.py:349-351 */
#define TB_FIT_SERSIC_MAX 6.3

typedef struct {
    int32_t profile;          /* TB_PROFILE_SERSIC, _EXP, _DEV or _POINT */
    int32_t x0, y0, w, h;     /* ModelMask in blob pixels (fixed during a fit) */
    int32_t blob;             /* the blob it belongs to */
    int32_t frozen;           /* bit k set: parameter slot k held at its start value
                                 (frozen parameters, utils.py:195-320) */
    int32_t pad;
} tb_fit_source;

/* Buffers of blob b: hbuf + h_off holds (n_slices + 2) P x P FP64 blocks
 * (per-slice partial A^T A, accepted A^T A, Cholesky factor); gbuf + g_off
 * holds (n_slices + 1) P-vectors (per-slice A^T r, accepted).  A slice is
 * one pass unit's share: a band's image, or a range of its active tiles. */
typedef struct {
    int32_t n_src;            /* sources (<= TB_FIT_MAX_SRC) */
    int32_t src0;             /* first source */
    int32_t P;                /* n_src * TB_FIT_NPAR */
    int32_t unit0;            /* chi2_part[unit0 + slice] holds a slice's chi^2 */
    int64_t h_off, g_off;
    int64_t tile_off;         /* the blob's 32 x 8 tiles in `tiles`: first the n_active */
    int32_t n_active;         /* tiles some source mask reaches, then the others */
    int32_t n_tiles;          /* (each entry tx | ty << 16) */
    int32_t n_slices;         /* partial blocks summed by tb_fit_step (>= 1) */
    int32_t pad;
} tb_fit_blob;

/* One (blob, band) image: W x H float32 pixels of data and inverr at
 * pix_off (row stride W), and the band's PSF mixture (psf_K <= 4).
 * tb_fit_prep takes the table of (blob, band) images in blob-major,
 * band-minor order (unit blob * n_bands + band).  tb_fit_pass takes units
 * that may split an image's active tiles into ranges [t0, t1) (t0 = t1 = 0
 * and t1 = n_active describe the whole list); each unit owns the blob's
 * partial blocks and chi^2 of its `slice`, and the unit with t0 = 0 also
 * covers the image's inactive tiles in mode 1. */
typedef struct {
    int32_t blob, band;
    int32_t W, H;
    int64_t pix_off;
    int32_t psf_K;
    int32_t slice;            /* partial block of the blob this unit owns */
    int32_t t0, t1;           /* range of the blob's active tiles */
    double psf_amp[4];
    double psf_mean[8];
    double psf_var[16];
} tb_fit_unit;

/* Per-blob optimiser state.  status: 0 running, 1 converged (the predicted
 * log-likelihood gain of the next step is below tol), 2 stopped (damping
 * exhausted, or non-finite chi^2 at the start), 3 iteration limit. */
typedef struct {
    double chi2;              /* chi^2 of the accepted parameters */
    double dlnp;              /* log-likelihood gain of the last accepted step */
    double lambda;            /* Marquardt damping (relative to the scaled diagonal) */
    double pred;              /* predicted log-likelihood gain of the next step */
    int32_t iters, accepted, rejected, status;
} tb_fit_state;

/* Bytes of the workspace tb_fit_prep writes and tb_fit_pass reads: per
 * source a summary and its PSF-convolved components in every band (host
 * call). */
int tb_fit_workspace(int32_t n_src, int32_t n_bands, int64_t* bytes);

/* Initialises n_blobs states (status 0, chi^2 = inf, lambda = lambda0). */
int tb_fit_reset(tb_fit_state* state, int32_t n_blobs, double lambda0, void* stream);

/* Per-source tables at `params` (the trial parameters): profile mixture and
 * its derivative in n (tractor/sersic.py:288-342), shape factor T T^T and
 * its derivatives in (log r_e, ee1, ee2) (ellipses.py:165-263,
 * galaxy.py:659-669) by FP64 central differences, and from them every
 * band's PSF-convolved components (mixture_profiles.py:158-172) with their
 * derivative coefficients.  cd_inv: the WCS cdInverse, 4 doubles in HOST
 * memory (one WCS for every blob).  state (optional, n_blobs entries):
 * sources of blobs whose status is not 0 (converged or stopped) are left
 * as they are -- the pass and the step skip those blobs. */
int tb_fit_prep(const tb_fit_source* srcs, int32_t n_src, const double* params,
                int32_t n_bands, const tb_fit_unit* units, int32_t n_units,
                const double* cd_inv, const tb_profile_tables* tables, void* workspace,
                const tb_fit_state* state, void* stream);

/* mode 0: for every unit of a running blob, over its range of the tiles its
 * sources' masks reach: the model (each source's PSF-convolved mixture on
 * its mask, summed), r = (data - model) * inverr, the analytic derivative
 * columns A = dmodel/dparams * inverr, and the unit's A^T A (upper
 * triangle), A^T r and r^T r + chi2_const into its slice
 * (chi2_part[blob.unit0 + slice]).  mode 1 (once per data set):
 * chi2_const[blob.unit0 + slice] = r^T r over the image's other tiles
 * (where the model is zero) for units with t0 = 0, else 0.  Replaces getDerivs / getChiImage / the A and b
 * assembly of lsqr_optimizer.py:328-520.  A persistent grid takes units
 * in the order `order` lists them (e.g. largest first) from work_counter
 * (one int32 of device scratch). */
int tb_fit_pass(const tb_fit_unit* units, const int32_t* order, int32_t n_units,
                const tb_fit_blob* blobs, const tb_fit_source* srcs, int32_t n_src,
                const void* workspace, const float* data, const float* inverr,
                const int32_t* tiles, double* hbuf, double* gbuf, double* chi2_part,
                double* chi2_const, const tb_fit_state* state, int32_t n_bands,
                int32_t mode, int32_t* work_counter, tb_status* status, void* stream);

/* One Levenberg-Marquardt step per running blob: accept the trial
 * parameters if chi^2 fell (the first pass is always accepted; the damping
 * then follows the ratio rho of the actual to the predicted gain, lambda x
 * max(1/3, 1 - (2 rho - 1)^3)), else raise the damping x 10; solve (D^-1 H D^-1 + lambda I) x = D^-1 g, D = sqrt(diag H),
 * by FP64 Cholesky with one refinement step; scale the step to respect the
 * maximum steps (PixPos 1, log r_e 1, ee 0.1, n 0.1) and the Sersic-index
 * bounds; write params + step into `trial`.  Stops a blob when the step's
 * predicted log-likelihood gain is below `tol` with lambda <= 1
 * (optimize_loop's dchisq, tested on the prediction). */
int tb_fit_step(const tb_fit_blob* blobs, int32_t n_blobs, int32_t n_bands,
                const tb_fit_source* srcs, double* params, double* trial, double* hbuf,
                double* gbuf, const double* chi2_part, tb_fit_state* state, double tol,
                int32_t max_iter, void* stream);

/* FP64 evaluation for the final iterations of a fit (no reference
 * counterpart beyond the optimum LsqrOptimizer.optimize_loop converges to,
 * lsqr_optimizer.py:317-326): for every running blob (status 0), A^T A,
 * A^T r and chi^2 over the units' active tiles with the model, the
 * derivative columns, the residuals and the sums in FP64 (FP64 exp from the
 * FP64 component tables tb_fit_prep writes into the workspace), written into
 * the hbuf, gbuf and chi2 slices that tb_fit_pass fills (call it in place
 * of the pass, before tb_fit_step); chi2_const (may be NULL) is added to
 * each slice's chi^2 as the pass does. */
int tb_fit_refine(const tb_fit_unit* units, const int32_t* order, int32_t n_units,
                  const tb_fit_blob* blobs, const tb_fit_source* srcs, int32_t n_src,
                  const void* workspace, const float* data, const float* inverr,
                  const int32_t* tiles, double* hbuf, double* gbuf, double* chi2_out,
                  const double* chi2_const, const tb_fit_state* state, int32_t n_bands,
                  int32_t* work_counter, tb_status* status, void* stream);

/* The blobs' model and its vector-Jacobian product, in FP64 (the
 * refinement pass's evaluation): mode TB_FIT_MODEL writes every unit's
 * model (sum of the sources' PSF-convolved mixtures over their masks) into
 * `model` at the active tiles' pixels (the caller zeroes the rest); mode
 * TB_FIT_VJP contracts each source's derivative columns (x, y, flux of the
 * band, log r_e, ee1, ee2, n: the derivatives Galaxy.getParamDerivatives and
 * PointSource.getParamDerivatives approximate, tractor/galaxy.py:137-223,
 * tractor/pointsource.py:130-241) with the upstream gradient `grad` (laid
 * out as the data), into the gbuf slices (summed over a blob's slices, the
 * gradient with respect to its parameters).  Run tb_fit_prep with state =
 * NULL at the parameters first. */
#define TB_FIT_REFINE 0
#define TB_FIT_MODEL 1
#define TB_FIT_VJP 2
int tb_fit_model_vjp(const tb_fit_unit* units, const int32_t* order, int32_t n_units,
                     const tb_fit_blob* blobs, const tb_fit_source* srcs, int32_t n_src,
                     const void* workspace, const float* grad, float* model,
                     const int32_t* tiles, double* gbuf, int32_t n_bands, int32_t mode,
                     int32_t* work_counter, tb_status* status, void* stream);


/* Chi-square of n images: sum over pixels of ((data - model) * inverr)^2,
 * FP32 terms with compensated FP32 block sums combined in FP64; out[i] for
 * image i of npix[i] pixels starting at offset off[i].  Replaces
 * Tractor.getLogLikelihood's sum (tractor/engine.py:475-479). */
int tb_chi2(const float* data, const float* model, const float* inverr,
            const int64_t* off, const int64_t* npix, int32_t n, double* out,
            void* stream);

/* EM fit of K-component 2-D Gaussian mixtures to n images, the batched
 * em_fit_2d_reg (tractor/emfit.i:274-557) that GaussianMixturePSF.fromStamp
 * (tractor/psf.py:536-597) runs on a PSF stamp.  Image s is ny x nx FP64
 * values, row-major, at img + s*ny*nx; pixel (ix, iy) sits at
 * (x0 + ix, y0 + iy) with (x0, y0) = xy0[2s], xy0[2s + 1], or
 * (-(nx/2), -(ny/2)) when xy0 is NULL.  amp (n x K), mean (n x K x 2) and
 * var (n x K x 2 x 2, row-major) hold the initial mixtures and receive the
 * fitted ones after `steps` iterations; alpha is the reference's
 * inverse-Wishart prior strength (alpha I added to the scatter matrix,
 * alpha to its weight).  status[s] (optional) is 0, or 1 when a component's
 * covariance determinant became non-positive: that image's fit stops there
 * with the previous iteration's mixture, as the reference returns -1.
 * FP64 throughout; every pointer is device memory.  1 <= K <= TB_EM_MAX_K,
 * ny * nx <= 2^24. */
#define TB_EM_MAX_K 8
int tb_em_fit_2d(const double* img, int32_t n, int32_t ny, int32_t nx, const int32_t* xy0,
                 double* amp, double* mean, double* var, int32_t K, double alpha,
                 int32_t steps, int32_t* status, void* stream);

/* The EM fit with a flat sky term, em_fit_2d_reg2 (tractor/emfit2.c), that
 * GaussianMixturePSF.fromStamp(v2=True) runs (tractor/psf.py:579-588), in
 * the layout of tb_em_fit_2d.  Pixels at or below zero count toward the sky
 * only; a component's responsibility is cut where its squared Mahalanobis
 * distance reaches -2 log(approx sqrt((2 pi)^2 det C)) (approx > 0);
 * second moments are taken about the previous iteration's mean, as the
 * reference accumulates them.  skyamp[s] (optional) receives the fit's
 * final sky level per pixel (the reference's skyamp output). */
int tb_em_fit_2d_sky(const double* img, int32_t n, int32_t ny, int32_t nx, const int32_t* xy0,
                     double* amp, double* mean, double* var, int32_t K, double alpha,
                     int32_t steps, double approx, double* skyamp, int32_t* status,
                     void* stream);

/* Blob segmentation for callers that cut images into blobs before
 * Tractor.setModelMasks / the batched fitter (the callers of
 * tractor/engine.py:341-361).  tb_label_components labels the connected
 * components of mask (H x W bytes, nonzero = foreground, row-major) with
 * 4-connectivity (conn8 = 0, scipy.ndimage.label's default structure) or
 * 8-connectivity (conn8 = 1): labels (H x W int32) receives 0 for
 * background and 1..n for the components, numbered in the raster order of
 * each component's first pixel (scipy.ndimage.label's numbering); *n_labels
 * (device int32) receives n.  workspace: tb_label_workspace_bytes(H, W)
 * bytes of device memory, 16-byte aligned.  *error (device int32) is set to
 * 1 if a merge ran out of its retry bound (never expected).  H * W <= 2^30.
 * Every pointer is device memory. */
int64_t tb_label_workspace_bytes(int32_t H, int32_t W);
int tb_label_components(const uint8_t* mask, int32_t H, int32_t W, int32_t conn8,
                        int32_t* labels, int32_t* n_labels, void* workspace, int32_t* error,
                        void* stream);

/* Bounding boxes of labels 1..n_labels (scipy.ndimage.find_objects):
 * boxes[4(l-1) ..] = y0, x0, y1, x1 (y1, x1 exclusive); a label with no
 * pixel keeps (H, W, 0, 0). */
int tb_component_boxes(const int32_t* labels, int32_t H, int32_t W, int32_t n_labels,
                       int32_t* boxes, void* stream);

/* Library version string (host memory, static). */
const char* tb_version(void);

/* ABI guard for bindings: writes sizeof(tb_mog_item), sizeof(tb_fft_item),
 * sizeof(tb_status), sizeof(tb_galaxy_src), sizeof(tb_fft_image),
 * sizeof(tb_scene_src), sizeof(tb_scene_image), sizeof(tb_scene_item),
 * sizeof(tb_fit_source), sizeof(tb_fit_blob), sizeof(tb_fit_unit),
 * sizeof(tb_fit_state), sizeof(tb_ring_item) into sizes[0..12] (host memory)
 * and returns 13.  No reference counterpart (bindings check their struct
 * layouts with it). */
int tb_abi_sizes(int32_t* sizes);

#ifdef __cplusplus
}
#endif

#endif /* TRACTOR_B200_H */
