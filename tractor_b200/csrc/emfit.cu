// Batched EM fit of 2-D Gaussian mixtures to images (sm_100a): the batched
// form of em_fit_2d_reg (tractor/emfit.i:274-557), which
// GaussianMixturePSF.fromStamp (tractor/psf.py:536-597) runs on a PSF stamp.
//
// One CTA per image, all iterations inside the kernel, FP64 throughout (as
// the reference).  Each iteration:
//   * per component: C^-1 and amp / (2 pi sqrt det C) (a non-positive
//     determinant stops the fit, as the reference returns -1 there);
//   * E step: the responsibility of component k at pixel (x, y) is
//     z_k / sum_j z_j (as z_k times the sum's reciprocal) with
//     z_k = scale_k exp(-dsq_k / 2), 0 for dsq >= 100 (z itself where the
//     sum is 0, as the reference leaves it);
//   * M step from the weighted moments w = img z_k / sum z (sum w, sum w x,
//     sum w y, sum w x^2, sum w x y, sum w y^2), summed per thread over a
//     fixed pixel stride and then over the block in a fixed order (every
//     launch gives the same result): mean = (sum w x, sum w y) / sum w,
//     covariance = (alpha I + sum w (x - mean)(x - mean)^T) / (sum w + alpha)
//     with sum w (x - m)^2 = sum w x^2 - m sum w x, amplitude = sum w.
// The reference sums the second moments about the new mean in a second pass
// over the pixels; the expansion above is the same sum in one pass (the
// difference is FP64 rounding).
#include "tb_common.cuh"

namespace {

constexpr int kEmThreads = 64;
constexpr int kWarps = kEmThreads / 32;

template <int K>
__global__ void __launch_bounds__(kEmThreads, 8)
em_fit_kernel(const double* __restrict__ img, int n, int ny, int nx,
              const int32_t* __restrict__ xy0, double* __restrict__ amp,
              double* __restrict__ mean, double* __restrict__ var, double alpha, int steps,
              int32_t* __restrict__ status) {
    constexpr int kM = 6 * K;   // moments per image
    __shared__ double w_s[K], mu_s[K][2], v_s[K][4];
    __shared__ double iv_s[K][4], sc_s[K];
    __shared__ double red[kWarps][kM];
    __shared__ int bad;
    const int s = blockIdx.x;
    if (s >= n) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double* im = img + (int64_t)s * ny * nx;
    double* A = amp + (int64_t)s * K;
    double* Mu = mean + (int64_t)s * K * 2;
    double* V = var + (int64_t)s * K * 4;
    const int x0 = xy0 ? xy0[2 * s] : -(nx / 2);
    const int y0 = xy0 ? xy0[2 * s + 1] : -(ny / 2);
    const int npix = nx * ny;
    const int ix0 = tid % nx, iy0 = tid / nx;                       // this thread's first pixel
    const int step_x = kEmThreads % nx, step_y = kEmThreads / nx;   // and its stride
    const double tpd = 4.0 * TB_PI * TB_PI;   // (2 pi)^D, D = 2
    if (tid < K) {
        w_s[tid] = A[tid];
        mu_s[tid][0] = Mu[2 * tid];
        mu_s[tid][1] = Mu[2 * tid + 1];
#pragma unroll
        for (int d = 0; d < 4; d++) v_s[tid][d] = V[4 * tid + d];
    }
    if (tid == 0) bad = 0;
    __syncthreads();
    for (int step = 0; step < steps; step++) {
        if (tid < K) {
            const double* Vk = v_s[tid];
            const double det = Vk[0] * Vk[3] - Vk[1] * Vk[2];
            if (det <= 0.0) bad = 1;
            iv_s[tid][0] = Vk[3] / det;
            iv_s[tid][1] = -Vk[1] / det;
            iv_s[tid][2] = -Vk[2] / det;
            iv_s[tid][3] = Vk[0] / det;
            sc_s[tid] = w_s[tid] / sqrt(tpd * det);
        }
        __syncthreads();
        if (bad) break;   // the same value in every thread
        double acc[kM];
#pragma unroll
        for (int v = 0; v < kM; v++) acc[v] = 0.0;
        // pixel i = tid + kEmThreads j at (ix, iy), advanced without a division
        int ix = ix0, iy = iy0;
        for (int i = tid; i < npix; i += kEmThreads) {
            const double x = (double)(x0 + ix), y = (double)(y0 + iy);
            ix += step_x;
            iy += step_y;
            if (ix >= nx) {
                ix -= nx;
                iy++;
            }
            double z[K];
            double zsum = 0.0;
#pragma unroll
            for (int k = 0; k < K; k++) {
                const double dx = x - mu_s[k][0], dy = y - mu_s[k][1];
                const double dsq = iv_s[k][0] * dx * dx + iv_s[k][1] * dx * dy +
                                   iv_s[k][2] * dx * dy + iv_s[k][3] * dy * dy;
                z[k] = dsq >= 100.0 ? 0.0 : sc_s[k] * exp(-0.5 * dsq);
                zsum += z[k];
            }
            // a pixel whose z sum to 0 keeps them unnormalised (all 0 unless
            // some amplitude is negative), as the reference does; one
            // reciprocal per pixel instead of a division per component
            const double rz = zsum != 0.0 ? 1.0 / zsum : 1.0;
            const double d = im[i];
#pragma unroll
            for (int k = 0; k < K; k++) {
                const double wi = d * (z[k] * rz);
                acc[6 * k + 0] += wi;
                acc[6 * k + 1] += wi * x;
                acc[6 * k + 2] += wi * y;
                acc[6 * k + 3] += wi * x * x;
                acc[6 * k + 4] += wi * x * y;
                acc[6 * k + 5] += wi * y * y;
            }
        }
#pragma unroll
        for (int v = 0; v < kM; v++) {
            double a = acc[v];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
            if (lane == 0) red[warp][v] = a;
        }
        __syncthreads();
        if (tid < K) {
            double m[6];
#pragma unroll
            for (int q = 0; q < 6; q++) {
                double t = 0.0;
                for (int w2 = 0; w2 < kWarps; w2++) t += red[w2][6 * tid + q];
                m[q] = t;
            }
            const double ws = m[0];
            const double mx = m[1] / ws, my = m[2] / ws;
            mu_s[tid][0] = mx;
            mu_s[tid][1] = my;
            const double den = ws + alpha;
            v_s[tid][0] = (alpha + (m[3] - mx * m[1])) / den;
            v_s[tid][1] = (m[4] - mx * m[2]) / den;
            v_s[tid][2] = v_s[tid][1];
            v_s[tid][3] = (alpha + (m[5] - my * m[2])) / den;
            w_s[tid] = ws;
        }
        __syncthreads();
    }
    if (tid < K) {
        A[tid] = w_s[tid];
        Mu[2 * tid] = mu_s[tid][0];
        Mu[2 * tid + 1] = mu_s[tid][1];
#pragma unroll
        for (int d = 0; d < 4; d++) V[4 * tid + d] = v_s[tid][d];
    }
    if (tid == 0 && status) status[s] = bad;
}

// The EM fit with a flat sky term (em_fit_2d_reg2, tractor/emfit2.c), the
// fit GaussianMixturePSF.fromStamp(v2=True) runs (tractor/psf.py:579-588).
// Per iteration, per component: the symmetrised covariance's determinant (a
// non-positive one stops the fit), its inverse, amp / sqrt((2 pi)^2 det) and
// the cut maxD = -2 log(approx sqrt((2 pi)^2 det)); per pixel: a pixel <= 0
// adds |img| to the sky and nothing else; z_k = 0 where dsq >= maxD_k; a
// pixel whose z sum to 0 adds img to the sky; otherwise psky joins the sum,
// img psky / sum goes to the sky and w_k = img z_k / sum; the weighted
// moments (sum w, sum w x, sum w y and the second moments about the OLD
// mean, as emfit2.c accumulates them in one pass) and the sky sum are
// summed per thread over a fixed pixel stride, then over the block in a
// fixed order; then mean = sum w x / sum w, covariance = (alpha I + second
// moments) / (sum w + alpha), amplitude = sum w, psky = sky / npix.  psky
// starts at 0.01 x the image mean; its last value is the fit's sky level.
template <int K>
__global__ void __launch_bounds__(kEmThreads, 8)
em_fit_sky_kernel(const double* __restrict__ img, int n, int ny, int nx,
                  const int32_t* __restrict__ xy0, double* __restrict__ amp,
                  double* __restrict__ mean, double* __restrict__ var, double alpha, int steps,
                  double approx, double* __restrict__ skyamp, int32_t* __restrict__ status) {
    constexpr int kM = 6 * K + 1;   // moments per image, then the sky sum
    __shared__ double w_s[K], mu_s[K][2], v_s[K][4];
    __shared__ double iv_s[K][3], sc_s[K], maxd_s[K];
    __shared__ double red[kWarps][kM];
    __shared__ double psky_s;
    __shared__ int bad;
    const int s = blockIdx.x;
    if (s >= n) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double* im = img + (int64_t)s * ny * nx;
    double* A = amp + (int64_t)s * K;
    double* Mu = mean + (int64_t)s * K * 2;
    double* V = var + (int64_t)s * K * 4;
    const int x0 = xy0 ? xy0[2 * s] : -(nx / 2);
    const int y0 = xy0 ? xy0[2 * s + 1] : -(ny / 2);
    const int npix = nx * ny;
    const int ix0 = tid % nx, iy0 = tid / nx;
    const int step_x = kEmThreads % nx, step_y = kEmThreads / nx;
    const double tpd = 4.0 * TB_PI * TB_PI;
    if (tid < K) {
        w_s[tid] = A[tid];
        mu_s[tid][0] = Mu[2 * tid];
        mu_s[tid][1] = Mu[2 * tid + 1];
#pragma unroll
        for (int d = 0; d < 4; d++) v_s[tid][d] = V[4 * tid + d];
    }
    if (tid == 0) {
        bad = 0;
        psky_s = 0.0;
    }
    // the image sum (fixed-order block reduction) for the first sky level
    {
        double t = 0.0;
        for (int i = tid; i < npix; i += kEmThreads) t += im[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) red[warp][0] = t;
        __syncthreads();
        if (tid == 0 && steps > 0) {
            double sum = 0.0;
            for (int w2 = 0; w2 < kWarps; w2++) sum += red[w2][0];
            psky_s = 0.01 * sum / (double)npix;
        }
        __syncthreads();
    }
    for (int step = 0; step < steps; step++) {
        if (tid < K) {
            const double* Vk = v_s[tid];
            const double v12 = (Vk[1] + Vk[2]) / 2.0;
            const double det = Vk[0] * Vk[3] - v12 * v12;
            if (det <= 0.0) bad = 1;
            iv_s[tid][0] = Vk[3] / det;
            iv_s[tid][1] = -2.0 * v12 / det;
            iv_s[tid][2] = Vk[0] / det;
            sc_s[tid] = w_s[tid] / sqrt(tpd * det);
            maxd_s[tid] = log(approx * sqrt(tpd * det)) / -0.5;
        }
        __syncthreads();
        if (bad) break;   // the same value in every thread
        const double psky = psky_s;
        double acc[kM];
#pragma unroll
        for (int v = 0; v < kM; v++) acc[v] = 0.0;
        int ix = ix0, iy = iy0;
        for (int i = tid; i < npix; i += kEmThreads) {
            const double x = (double)(x0 + ix), y = (double)(y0 + iy);
            ix += step_x;
            iy += step_y;
            if (ix >= nx) {
                ix -= nx;
                iy++;
            }
            const double d = im[i];
            if (d <= 0.0) {
                acc[6 * K] += fabs(d);
                continue;
            }
            double z[K];
            double zsum = 0.0;
#pragma unroll
            for (int k = 0; k < K; k++) {
                const double dx = x - mu_s[k][0], dy = y - mu_s[k][1];
                const double dsq = iv_s[k][0] * dx * dx + iv_s[k][1] * dx * dy +
                                   iv_s[k][2] * dy * dy;
                z[k] = dsq >= maxd_s[k] ? 0.0 : sc_s[k] * exp(-0.5 * dsq);
                zsum += z[k];
            }
            if (zsum == 0.0) {
                acc[6 * K] += d;
                continue;
            }
            zsum += psky;
            acc[6 * K] += d * (psky / zsum);
#pragma unroll
            for (int k = 0; k < K; k++) {
                const double wi = d * z[k] / zsum;
                const double dx = x - mu_s[k][0], dy = y - mu_s[k][1];
                acc[6 * k + 0] += wi;
                acc[6 * k + 1] += wi * x;
                acc[6 * k + 2] += wi * y;
                acc[6 * k + 3] += wi * dx * dx;
                acc[6 * k + 4] += wi * dx * dy;
                acc[6 * k + 5] += wi * dy * dy;
            }
        }
#pragma unroll
        for (int v = 0; v < kM; v++) {
            double a = acc[v];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
            if (lane == 0) red[warp][v] = a;
        }
        __syncthreads();
        if (tid < K) {
            double m[6];
#pragma unroll
            for (int q = 0; q < 6; q++) {
                double t = 0.0;
                for (int w2 = 0; w2 < kWarps; w2++) t += red[w2][6 * tid + q];
                m[q] = t;
            }
            const double ws = m[0];
            mu_s[tid][0] = m[1] / ws;
            mu_s[tid][1] = m[2] / ws;
            const double den = ws + alpha;
            v_s[tid][0] = (alpha + m[3]) / den;
            v_s[tid][1] = m[4] / den;
            v_s[tid][2] = v_s[tid][1];
            v_s[tid][3] = (alpha + m[5]) / den;
            w_s[tid] = ws;
        }
        if (tid == 0) {
            double t = 0.0;
            for (int w2 = 0; w2 < kWarps; w2++) t += red[w2][6 * K];
            psky_s = t / (double)npix;
        }
        __syncthreads();
    }
    if (tid < K) {
        A[tid] = w_s[tid];
        Mu[2 * tid] = mu_s[tid][0];
        Mu[2 * tid + 1] = mu_s[tid][1];
#pragma unroll
        for (int d = 0; d < 4; d++) V[4 * tid + d] = v_s[tid][d];
    }
    if (tid == 0) {
        if (skyamp) skyamp[s] = psky_s;
        if (status) status[s] = bad;
    }
}

template <int K>
int launch_sky(const double* img, int n, int ny, int nx, const int32_t* xy0, double* amp,
               double* mean, double* var, double alpha, int steps, double approx, double* sky,
               int32_t* status, cudaStream_t s) {
    em_fit_sky_kernel<K><<<n, kEmThreads, 0, s>>>(img, n, ny, nx, xy0, amp, mean, var, alpha,
                                                  steps, approx, sky, status);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

template <int K>
int launch(const double* img, int n, int ny, int nx, const int32_t* xy0, double* amp,
           double* mean, double* var, double alpha, int steps, int32_t* status,
           cudaStream_t s) {
    em_fit_kernel<K><<<n, kEmThreads, 0, s>>>(img, n, ny, nx, xy0, amp, mean, var, alpha, steps,
                                              status);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

}  // namespace

extern "C" int tb_em_fit_2d(const double* img, int32_t n, int32_t ny, int32_t nx,
                            const int32_t* xy0, double* amp, double* mean, double* var,
                            int32_t K, double alpha, int32_t steps, int32_t* status,
                            void* stream) {
    if (n < 0 || ny < 1 || nx < 1 || (int64_t)ny * nx > (1 << 24) || K < 1 ||
        K > TB_EM_MAX_K || steps < 0)
        return TB_ERR_ARG;
    if (n == 0) return TB_OK;
    if (!img || !amp || !mean || !var) return TB_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    switch (K) {
        case 1: return launch<1>(img, n, ny, nx, xy0, amp, mean, var, alpha, steps, status, s);
        case 2: return launch<2>(img, n, ny, nx, xy0, amp, mean, var, alpha, steps, status, s);
        case 3: return launch<3>(img, n, ny, nx, xy0, amp, mean, var, alpha, steps, status, s);
        case 4: return launch<4>(img, n, ny, nx, xy0, amp, mean, var, alpha, steps, status, s);
        case 5: return launch<5>(img, n, ny, nx, xy0, amp, mean, var, alpha, steps, status, s);
        case 6: return launch<6>(img, n, ny, nx, xy0, amp, mean, var, alpha, steps, status, s);
        case 7: return launch<7>(img, n, ny, nx, xy0, amp, mean, var, alpha, steps, status, s);
        default: return launch<8>(img, n, ny, nx, xy0, amp, mean, var, alpha, steps, status, s);
    }
}

extern "C" int tb_em_fit_2d_sky(const double* img, int32_t n, int32_t ny, int32_t nx,
                                const int32_t* xy0, double* amp, double* mean, double* var,
                                int32_t K, double alpha, int32_t steps, double approx,
                                double* skyamp, int32_t* status, void* stream) {
    if (n < 0 || ny < 1 || nx < 1 || (int64_t)ny * nx > (1 << 24) || K < 1 ||
        K > TB_EM_MAX_K || steps < 0 || !(approx > 0.0))
        return TB_ERR_ARG;
    if (n == 0) return TB_OK;
    if (!img || !amp || !mean || !var) return TB_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    switch (K) {
        case 1: return launch_sky<1>(img, n, ny, nx, xy0, amp, mean, var, alpha, steps, approx, skyamp, status, s);
        case 2: return launch_sky<2>(img, n, ny, nx, xy0, amp, mean, var, alpha, steps, approx, skyamp, status, s);
        case 3: return launch_sky<3>(img, n, ny, nx, xy0, amp, mean, var, alpha, steps, approx, skyamp, status, s);
        case 4: return launch_sky<4>(img, n, ny, nx, xy0, amp, mean, var, alpha, steps, approx, skyamp, status, s);
        case 5: return launch_sky<5>(img, n, ny, nx, xy0, amp, mean, var, alpha, steps, approx, skyamp, status, s);
        case 6: return launch_sky<6>(img, n, ny, nx, xy0, amp, mean, var, alpha, steps, approx, skyamp, status, s);
        case 7: return launch_sky<7>(img, n, ny, nx, xy0, amp, mean, var, alpha, steps, approx, skyamp, status, s);
        default: return launch_sky<8>(img, n, ny, nx, xy0, amp, mean, var, alpha, steps, approx, skyamp, status, s);
    }
}
