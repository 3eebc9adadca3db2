// Mixture spectrum x PSF spectrum on a full rfft grid, for Fourier-path
// galaxies whose FFT size exceeds the 256 that the fused renderer (K3) holds
// in shared memory (sm_100a).
//
// One thread per element (v, w) of the N x (N/2 + 1) grid:
//   S(v, w) = P(v, w) * sum_k amp_k exp(-2 pi^2 f^T C_k f),  f = (v/N, w'/N)
// with w' = w for w < N/2 and w - N otherwise (numpy's fftfreq / rfftfreq),
// evaluated in FP32 with one SFU ex2 per element and component as K3 does
// (the FP64 components folded into FP32 exponent coefficients in log2 units),
// and for difference items (TB_FFT_DIFF) the difference of two mixtures of
// one size, sum_k exp(e_k) (a'_k expm1(de_k) + (a'_k - a_k)).  The PSF
// spectrum is read column-major (v-major, K3's layout) and the result is
// written row-major, S[w][v], the layout an inverse 2-D real FFT takes
// (torch.fft.irfft2 on a (N, N/2 + 1) complex tensor).
//
// This is MixtureOfGaussians.getFourierTransform(v, w, zero_mean=True)
// (tractor/mixture_profiles.py, mp_fourier.i:405-430) times the PSF's
// getFourierTransform, the product galaxy.py:457-470 hands to irfftn.
#include "tb_common.cuh"

namespace {

constexpr int kGridThreads = 256;
constexpr int kMaxKGrid = 128;

__global__ void __launch_bounds__(kGridThreads)
spectrum_grid_kernel(const double* __restrict__ amp, const double* __restrict__ var,
                     const double* __restrict__ dcoef, int K, const float2* __restrict__ psf,
                     int N, float2* __restrict__ out) {
    __shared__ float4 comp[kMaxKGrid];
    __shared__ float4 dcomp[kMaxKGrid];
    const double c2 = -2.0 * TB_PI * TB_PI * TB_LOG2E;
    const double n2 = -2.0 * TB_PI * TB_PI;
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        comp[k] = make_float4((float)amp[k], (float)(c2 * var[4 * k]),
                              (float)(c2 * 2.0 * var[4 * k + 1]), (float)(c2 * var[4 * k + 3]));
        if (dcoef) {
            const double* dc = dcoef + 4 * k;
            dcomp[k] = make_float4((float)dc[0], (float)(n2 * dc[1]), (float)(n2 * 2.0 * dc[2]),
                                   (float)(n2 * dc[3]));
        }
    }
    __syncthreads();
    const int NH = N / 2 + 1;
    const int64_t total = (int64_t)N * NH;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        // consecutive threads take consecutive v of one row w (coalesced writes)
        const int w = (int)(e / NH), v = (int)(e % NH);
        const float vf = (float)v / (float)N;
        const float wf = (float)(w < N / 2 ? w : w - N) / (float)N;
        float acc = 0.f;
        if (dcoef) {
            for (int k = 0; k < K; k++) {
                const float4 c = comp[k];
                const float4 d = dcomp[k];
                const float ex = fmaf(wf, fmaf(c.w, wf, c.z * vf), c.y * vf * vf);
                const float de = fmaf(wf, fmaf(d.w, wf, d.z * vf), d.y * vf * vf);
                const float pre = fmaf(c.x + d.x, expm1f(de), d.x);
                acc = fmaf(pre, tb::ex2(ex), acc);
            }
        } else {
            for (int k = 0; k < K; k++) {
                const float4 c = comp[k];
                const float ex = fmaf(wf, fmaf(c.w, wf, c.z * vf), c.y * vf * vf);
                acc = fmaf(c.x, tb::ex2(ex), acc);
            }
        }
        const float2 p = __ldg(psf + (int64_t)v * N + w);
        out[e] = make_float2(acc * p.x, acc * p.y);
    }
}

}  // namespace

extern "C" int tb_fourier_spectrum_grid(const double* comp_amp, const double* comp_var,
                                        const double* comp_dcoef, int32_t K,
                                        const float* psf_spec, int32_t sz, float* out,
                                        void* stream) {
    if (K < 0 || sz < 2 || (sz & (sz - 1)) != 0) return TB_ERR_ARG;
    if (K > kMaxKGrid) return TB_ERR_SIZE;
    if (!psf_spec || !out || (K > 0 && (!comp_amp || !comp_var))) return TB_ERR_ARG;
    const int64_t total = (int64_t)sz * (sz / 2 + 1);
    int64_t blocks = (total + kGridThreads - 1) / kGridThreads;
    const int64_t cap = (int64_t)tb::num_sms() * 8;
    if (blocks > cap) blocks = cap;
    spectrum_grid_kernel<<<(int)blocks, kGridThreads, 0, (cudaStream_t)stream>>>(
        comp_amp, comp_var, comp_dcoef, K, reinterpret_cast<const float2*>(psf_spec), sz,
        reinterpret_cast<float2*>(out));
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}
