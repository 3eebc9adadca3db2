// K2: batched separable Lanczos-3 sub-pixel shift (sm_100a).
//
// Each CTA produces one 32x32 output tile of one image: it loads the
// (32+6)^2 input window (zeros outside the image) into shared memory, runs the
// 7-tap pass along x into a (32+6) x 32 buffer and then the pass along y.
// Taps are built in FP64 exactly as lanczos_filter_3
// (tractor/mp_fourier.i:355-402) and rounded to float; every sum runs tap by
// tap with separate float multiply and add (no FMA contraction), which is the
// arithmetic of correlate7f_inout (mp_fourier.i:267-352).  The zero samples
// outside the image add exact zeros, so results are bit-identical to the
// reference's C kernel.
#include "tb_common.cuh"

namespace {

constexpr int kT = 32;     // output tile
constexpr int kH = 3;      // halo
constexpr int kW = kT + 2 * kH;

__device__ void lanczos3_taps(double dx, float* f) {
    double t[7] = {0, 0, 0, 0, 0, 0, 0};
    if (dx == 0.0) {
        t[3] = 1.0;
    } else {
        const int lo = dx > 0.0 ? 0 : 1, hi = dx > 0.0 ? 6 : 7;
        double s = 0.0;
        for (int i = lo; i < hi; i++) {
            const double p = TB_PI * (i - 3.0 + dx);
            t[i] = 3.0 * sin(p) * sin(p / 3.0) / (p * p);
            s += t[i];
        }
        for (int i = lo; i < hi; i++) t[i] /= s;
    }
    for (int i = 0; i < 7; i++) f[i] = (float)t[i];
}

__global__ void __launch_bounds__(256)
lanczos3_kernel(const float* __restrict__ in, float* __restrict__ out,
                const double* __restrict__ shift, int h, int w) {
    __shared__ float src[kW][kW + 1];
    __shared__ float xs[kW][kT + 1];
    __shared__ float taps[14];
    const int img = blockIdx.z;
    const int X0 = blockIdx.x * kT, Y0 = blockIdx.y * kT;
    const float* I = in + (int64_t)img * h * w;
    float* O = out + (int64_t)img * h * w;
    if (threadIdx.x == 0) {
        lanczos3_taps(shift[2 * img], taps);
        lanczos3_taps(shift[2 * img + 1], taps + 7);
    }
    for (int i = threadIdx.x; i < kW * kW; i += blockDim.x) {
        const int r = i / kW, c = i % kW;
        const int y = Y0 - kH + r, x = X0 - kH + c;
        src[r][c] = (y >= 0 && y < h && x >= 0 && x < w) ? I[(int64_t)y * w + x] : 0.f;
    }
    __syncthreads();
    float fx[7], fy[7];
#pragma unroll
    for (int k = 0; k < 7; k++) { fx[k] = taps[k]; fy[k] = taps[7 + k]; }
    for (int i = threadIdx.x; i < kW * kT; i += blockDim.x) {
        const int r = i / kT, c = i % kT;
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < 7; k++) acc = __fadd_rn(acc, __fmul_rn(fx[k], src[r][c + k]));
        xs[r][c] = acc;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kT * kT; i += blockDim.x) {
        const int r = i / kT, c = i % kT;
        const int y = Y0 + r, x = X0 + c;
        if (y >= h || x >= w) continue;
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < 7; k++) acc = __fadd_rn(acc, __fmul_rn(fy[k], xs[r + k][c]));
        O[(int64_t)y * w + x] = acc;
    }
}

}  // namespace

extern "C" int tb_lanczos3_shift(const float* in, float* out, const double* shift, int32_t n,
                                 int32_t h, int32_t w, void* stream) {
    if (n < 0 || h < 0 || w < 0) return TB_ERR_ARG;
    if (n == 0 || h == 0 || w == 0) return TB_OK;
    if (!in || !out || !shift || in == out) return TB_ERR_ARG;
    if (n > 65535) return TB_ERR_SIZE;
    dim3 grid((w + kT - 1) / kT, (h + kT - 1) / kT, n);
    lanczos3_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(in, out, shift, h, w);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}
