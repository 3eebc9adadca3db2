/*
 * tractor_b200 -- C ABI of the B200 (sm_100a) forward-model kernels.
 *
 * Every pointer argument is a DEVICE pointer unless stated otherwise, every
 * call is asynchronous on the given CUDA stream (a cudaStream_t passed as
 * void*, NULL = legacy default stream), and every call returns an int status
 * (TB_OK = 0) after validating its arguments on the host; it never aborts the
 * process.  Kernels additionally write per-call status words to device memory
 * (tb_status) that the caller reads after synchronising.  The library holds no
 * mutable global state and allocates no memory: callers own every buffer,
 * including workspaces, and may call from one stream per host thread.
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
    double floor;      /* exponent floor, natural-log units */
    float scale;       /* output multiplier (counts for a model patch) */
    int32_t pad1;
    int64_t out_off;   /* element offset of this item's output */
    int64_t mask_off;  /* element offset of this item's mask, or -1 */
    int64_t tile0;     /* exclusive prefix of tiles (32x32) over items */
} tb_mog_item;

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
 * column-major (element (row j, column v) at v*sz + j), PSF p at
 * psf_spec + p * sz*(sz/2+1)*2 floats, as written by tb_psf_spectrum.  Components: amp[c0+k] and the
 * sheared 2x2 covariance var[4(c0+k)..] (FP64); a zero covariance is a delta
 * component.  Output: float32 mh x mw at out + out_off (row stride ldo, or
 * mw if ldo = 0), times `scale`.  Items taller than 128 pixels at sz = 256
 * are rendered in row chunks.
 * ------------------------------------------------------------------------ */
typedef struct {
    int32_t c0, K;
    int32_t sz;
    int32_t psf;       /* PSF spectrum index */
    int32_t mw, mh;
    int32_t sx, sy;
    double mux, muy;
    float scale;
    int32_t mode;      /* TB_MOG_STORE, TB_MOG_ACCUM or TB_MOG_ATOMIC */
    int64_t out_off;
    int32_t ldo;       /* output row stride in elements (0 = mw) */
    int32_t pad0;
} tb_fft_item;

#define TB_FFT_MAX_SZ 256

int tb_fourier_render(const tb_fft_item* items, int32_t n_items,
                      const double* comp_amp, const double* comp_var,
                      const float* psf_spec, float* out, int32_t* work_counter,
                      tb_status* status, void* stream);

/* Forward real FFT of n zero-padded sz x sz float32 PSF images (prepared by
 * the caller, image i at pad + i*sz*sz) into complex64 spectra
 * sz x (sz/2+1) (interleaved, column-major as tb_fourier_render reads them),
 * optionally divided by |P[0,0]|.  Replaces
 * np.fft.rfft2 + astype(complex64) in PixelizedPSF.getFourierTransform
 * (tractor/psf.py:249-280) and NormalizedPsf (psf.py:947-953). */
int tb_psf_spectrum(const float* pad, float* spec, int32_t n, int32_t sz,
                    int32_t normalize, void* stream);

/* ------------------------------------------------------------------------
 * Least-squares step
 * ------------------------------------------------------------------------ */

/* Normal equations of one or more independent least-squares problems.
 * Problem b has P[b] parameters and R[b] rows; its design matrix is stored
 * column-major at A + a_off[b] with leading dimension lda[b] (rows), its
 * right-hand side at rhs + r_off[b].  Writes (FP64) AtA[b] (P x P, at
 * ata_off[b]) and Atr[b] (P, at atr_off[b]) with FP32 products accumulated
 * by compensated (two-sum) FP32 partial sums combined in FP64.
 * Replaces the sparse A / b assembly and LSQR solve of
 * LsqrOptimizer.getUpdateDirection (tractor/lsqr_optimizer.py:328-644). */
int tb_normal_equations(const float* A, const float* rhs, const int64_t* a_off,
                        const int64_t* r_off, const int32_t* lda,
                        const int32_t* P, const int32_t* R,
                        const int64_t* ata_off, const int64_t* atr_off,
                        double* AtA, double* Atr, int32_t n_problems,
                        int32_t max_p, void* stream);

/* Solves each problem's column-scaled normal equations in FP64 on the device
 * (column scaling as lsqr_optimizer.py:470-489 with scale = sqrt(diag),
 * Cholesky with a `damp`^2 ridge, one step of iterative refinement) and
 * writes X[x_off[b] + i] = update / colscale (zero for empty columns).
 * info[b] = 0 ok, >0 the failing pivot (not positive definite; X is then
 * zero, as LsqrOptimizer returns a zero update on failure,
 * lsqr_optimizer.py:586-604), -1 if P[b] > 320.  work: caller-owned FP64
 * scratch of n_problems * max_p * max_p elements (the Cholesky factors). */
int tb_solve_update(const double* AtA, const double* Atr,
                    const int64_t* ata_off, const int64_t* atr_off,
                    const int32_t* P, const int64_t* x_off, double* X,
                    int32_t* info, double damp, int32_t n_problems,
                    int32_t max_p, double* work, void* stream);

/* Chi-square of n images: sum over pixels of ((data - model) * inverr)^2,
 * FP32 terms with compensated FP32 block sums combined in FP64; out[i] for
 * image i of npix[i] pixels starting at offset off[i].  Replaces
 * Tractor.getLogLikelihood's sum (tractor/engine.py:475-479). */
int tb_chi2(const float* data, const float* model, const float* inverr,
            const int64_t* off, const int64_t* npix, int32_t n, double* out,
            void* stream);

/* Library version string (host memory, static). */
const char* tb_version(void);

/* ABI guard for bindings: writes sizeof(tb_mog_item), sizeof(tb_fft_item),
 * sizeof(tb_status) into sizes[0..2] (host memory) and returns 3.  No
 * reference counterpart (bindings check their struct layouts with it). */
int tb_abi_sizes(int32_t* sizes);

#ifdef __cplusplus
}
#endif

#endif /* TRACTOR_B200_H */
