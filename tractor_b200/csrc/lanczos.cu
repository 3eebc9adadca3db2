// K2: batched separable Lanczos-3 sub-pixel shift (sm_100a).
//
// Each warp produces a strip of 32 output columns by kRowsPerWarp rows of one
// image.  Lane l owns column X0 + l: for every input row of the strip (its
// rows plus 3 above and 3 below) it loads its pixel, lanes 0-5 also the three
// halo columns on each side, and the 7-tap pass along x takes its neighbours'
// pixels by warp shuffles; the last seven results of that pass stay in
// registers, a sliding window from which the pass along y produces one output
// row per input row.  No shared memory and no block barrier.
// Taps are built in FP64 exactly as lanczos_filter_3
// (tractor/mp_fourier.i:355-402) and rounded to float; every sum runs tap by
// tap with separate float multiply and add (no FMA contraction), which is the
// arithmetic of correlate7f_inout (mp_fourier.i:267-352).  The zero samples
// outside the image add exact zeros, so results are bit-identical to the
// reference's C kernel.
#include "tb_common.cuh"

namespace {

constexpr int kT = 32;               // output columns per warp
constexpr int kRowsPerWarp = 16;     // output rows per warp
constexpr int kWarpsPerCta = 8;
constexpr int kRowsPerCta = kRowsPerWarp * kWarpsPerCta;

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

__global__ void __launch_bounds__(kWarpsPerCta * 32)
lanczos3_kernel(const float* __restrict__ in, float* __restrict__ out,
                const double* __restrict__ shift, int h, int w) {
    __shared__ float taps[14];
    const int img = blockIdx.z;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int X0 = blockIdx.x * kT;
    const int Y0 = (blockIdx.y * kWarpsPerCta + warp) * kRowsPerWarp;
    const float* I = in + (int64_t)img * h * w;
    float* O = out + (int64_t)img * h * w;
    if (threadIdx.x == 0) {
        lanczos3_taps(shift[2 * img], taps);
        lanczos3_taps(shift[2 * img + 1], taps + 7);
    }
    __syncthreads();
    float fx[7], fy[7];
#pragma unroll
    for (int k = 0; k < 7; k++) {
        fx[k] = taps[k];
        fy[k] = taps[7 + k];
    }
    const int x = X0 + lane;
    // halo columns: lanes 0-2 hold X0 - 3 .. X0 - 1, lanes 3-5 X0 + 32 .. X0 + 34
    const int xe = lane < 3 ? X0 - 3 + lane : X0 + kT + (lane - 3);
    const bool has_e = lane < 6 && xe >= 0 && xe < w;
    float win[7];
#pragma unroll
    for (int k = 0; k < 7; k++) win[k] = 0.f;
    for (int i = 0; i < kRowsPerWarp + 6; i++) {
        const int y = Y0 - 3 + i;
        const bool rowin = y >= 0 && y < h;
        const float* row = I + (int64_t)y * w;
        const float mid = (rowin && x < w) ? row[x] : 0.f;
        const float ext = (rowin && has_e) ? row[xe] : 0.f;
        // pass along x: input column x - 3 + k, tap by tap
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < 7; k++) {
            const int sl = lane + k - 3;
            const float a = __shfl_sync(0xffffffffu, mid, sl & 31);
            const float b = __shfl_sync(0xffffffffu, ext, (sl < 0 ? sl + 3 : sl - 29) & 31);
            acc = __fadd_rn(acc, __fmul_rn(fx[k], (sl < 0 || sl >= kT) ? b : a));
        }
#pragma unroll
        for (int k = 0; k < 6; k++) win[k] = win[k + 1];
        win[6] = acc;
        // pass along y: output row y - 3 from input rows y - 6 .. y
        const int yo = y - 3;
        if (i >= 6 && yo < h && x < w) {
            float o = 0.f;
#pragma unroll
            for (int k = 0; k < 7; k++) o = __fadd_rn(o, __fmul_rn(fy[k], win[k]));
            O[(int64_t)yo * w + x] = o;
        }
    }
}

}  // namespace

extern "C" int tb_lanczos3_shift(const float* in, float* out, const double* shift, int32_t n,
                                 int32_t h, int32_t w, void* stream) {
    if (n < 0 || h < 0 || w < 0) return TB_ERR_ARG;
    if (n == 0 || h == 0 || w == 0) return TB_OK;
    if (!in || !out || !shift || in == out) return TB_ERR_ARG;
    if (n > 65535) return TB_ERR_SIZE;
    dim3 grid((w + kT - 1) / kT, (h + kRowsPerCta - 1) / kRowsPerCta, n);
    lanczos3_kernel<<<grid, kWarpsPerCta * 32, 0, (cudaStream_t)stream>>>(in, out, shift, h, w);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}
