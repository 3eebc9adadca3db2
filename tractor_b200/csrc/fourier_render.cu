// K3: fused pixelized-PSF galaxy renderer (sm_100a).
//
// One CTA renders one item (galaxy) at a time, persistent over items taken
// from a global counter, entirely in shared memory:
//   1. column pass: for each rfft column v (sz/2+1 of them) a thread group
//      evaluates the zero-mean mixture spectrum sum_k amp_k exp2(e_k(v, w))
//      for all sz rows w (one SFU ex2 per element and component), multiplies
//      by the PSF spectrum column (stored column-major, so loads coalesce),
//      and runs an inverse complex FFT along w; only the rows the output
//      window needs are kept, in a [row][v] buffer S1.
//   2. row pass: pairs of kept rows are packed as H1 + i H2 with their
//      Hermitian extension and one inverse complex FFT along v yields both
//      real rows (the imaginary parts of the DC and Nyquist bins are dropped,
//      as numpy's irfft does); only the needed columns are kept, in place.
//   3. Lanczos-3 along x (in place, per row) and along y, then the integer
//      shift and crop into the mh x mw output, scaled by scale / sz^2
//      (irfftn's normalisation).
// This is ProfileGalaxy._realGetUnitFluxModelPatch's FFT branch with a
// ModelMask (tractor/galaxy.py:336-519) for a non-hybrid PixelizedPSF.
// Masks taller than 128 rows at sz = 256 are processed in row chunks (the
// column pass is repeated per chunk).
#include "fft_warp.cuh"

namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxK = 128;
constexpr int kXbufPerWarp = 528;                  // floats, any N in [32, 256]
constexpr int kRmax256 = 134;                      // kept rows at sz = 256

__host__ __device__ constexpr int s1_bytes(int N, int rmax) { return rmax * (N / 2 + 1) * 8; }

constexpr int kS1Bytes = s1_bytes(256, kRmax256) > s1_bytes(128, 128) ? s1_bytes(256, kRmax256)
                                                                       : s1_bytes(128, 128);
constexpr int kSmemBytes = 256 * 8               /* twiddles */
                           + kMaxK * 16           /* components */
                           + 16 * 4               /* taps */
                           + kWarps * kXbufPerWarp * 4 + kS1Bytes;

struct Shared {
    float2* tw;
    float4* comp;   // (amp, ca, cb, cd): exponent = ca v^2 + cb v w + cd w^2 (log2 units)
    float* taps;    // fx[0..6], fy[0..6]
    float* xbuf;
    float2* s1;
};

__device__ void taps3(double dx, float* f) {
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

template <int N>
__device__ void render_item(const tb_fft_item& it, int K, const float* __restrict__ spec,
                            float* __restrict__ out, const Shared& sh, int rmax) {
    constexpr int NH = N / 2 + 1;
    constexpr int T = N / 8;            // threads per FFT
    constexpr int GPW = 32 / T;         // FFT groups per warp
    constexpr int XB = tb::fft_xbuf_floats<N>();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = lane % T;
    const int ngroups = kWarps * GPW;
    float* xr = sh.xbuf + warp * kXbufPerWarp + (lane / T) * XB;
    float* xi = xr + XB / 2;

    const int mw = it.mw, mh = it.mh, sx = it.sx, sy = it.sy;
    const float osc = it.scale / (float)(N * N);
    const bool accum = it.mode == TB_MOG_ACCUM || it.mode == TB_MOG_ATOMIC;
    float* O = out + it.out_off;
    const int64_t ldo = it.ldo > 0 ? it.ldo : mw;

    const int gr0 = max(0, -sy), gr1 = min(N, mh - sy);
    const int gc0 = max(0, -sx), gc1 = min(N, mw - sx);
    const bool empty = gr0 >= gr1 || gc0 >= gc1;
    // Output rows whose source row is outside [gr0, gr1) are zero.
    if (!accum) {
        for (int i = threadIdx.x; i < mh * mw; i += kThreads) {
            const int r = i / mw - sy;
            if (empty || r < gr0 || r >= gr1) O[(int64_t)(i / mw) * ldo + i % mw] = 0.f;
        }
    }
    if (empty) return;
    const int c0 = max(0, gc0 - 3), c1 = min(N, gc1 + 3);
    const int chunk = rmax - 6;
    const float* fx = sh.taps;
    const float* fy = sh.taps + 7;

    for (int a = gr0; a < gr1; a += chunk) {
        const int b = min(gr1, a + chunk);
        const int rlo = max(0, a - 3), rhi = min(N, b + 3);
        const int nrows = rhi - rlo;

        // ---- 1. column pass ----
        // Every lane of a warp runs the same number of iterations (groups past
        // the end compute on a clamped column and store nothing), so the
        // warp-wide syncs inside the FFT see all 32 lanes.
        for (int v0 = warp * GPW; v0 < NH; v0 += ngroups) {
            const bool act = v0 + lane / T < NH;
            const int v = act ? v0 + lane / T : NH - 1;
            const float vf = (float)v / (float)N;
            float acc[8];
            float wf[8];
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const int j = t + m * T;
                wf[m] = (float)(j < N / 2 ? j : j - N) / (float)N;
                acc[m] = 0.f;
            }
            for (int k = 0; k < K; k++) {
                const float4 c = sh.comp[k];
                const float al = c.y * vf * vf, be = c.z * vf;
#pragma unroll
                for (int m = 0; m < 8; m++) {
                    const float e = fmaf(wf[m], fmaf(c.w, wf[m], be), al);
                    acc[m] = fmaf(c.x, tb::ex2(e), acc[m]);
                }
            }
            float2 x[8];
            const float2* P = reinterpret_cast<const float2*>(spec) + (int64_t)v * N;
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const float2 p = __ldg(P + t + m * T);
                x[m] = make_float2(acc[m] * p.x, acc[m] * p.y);
            }
            float2* S1 = sh.s1;
            tb::fft_run<N, +1>(x, t, xr, xi, sh.tw, [&](int row, float2 z) {
                if (act && row >= rlo && row < rhi) S1[(row - rlo) * NH + v] = z;
            });
            __syncwarp();
        }
        __syncthreads();

        // ---- 2. row pass (two real rows per complex FFT) ----
        const int npairs = (nrows + 1) / 2;
        for (int p0 = warp * GPW; p0 < npairs; p0 += ngroups) {
            const bool act = p0 + lane / T < npairs;
            const int p = act ? p0 + lane / T : npairs - 1;
            const int ia = 2 * p, ib = 2 * p + 1;
            const bool hasb = ib < nrows;
            const float2* H1 = sh.s1 + ia * NH;
            const float2* H2 = sh.s1 + (hasb ? ib : ia) * NH;
            float2 x[8];
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const int n = t + m * T;
                const int q = n <= N / 2 ? n : N - n;
                float2 h1 = H1[q];
                float2 h2 = hasb ? H2[q] : make_float2(0.f, 0.f);
                if (q == 0 || q == N / 2) { h1.y = 0.f; h2.y = 0.f; }
                x[m] = n <= N / 2 ? make_float2(h1.x - h2.y, h1.y + h2.x)
                                  : make_float2(h1.x + h2.y, h2.x - h1.y);
            }
            float* rowA = reinterpret_cast<float*>(sh.s1 + ia * NH);
            float* rowB = reinterpret_cast<float*>(sh.s1 + ib * NH);
            tb::fft_run<N, +1>(x, t, xr, xi, sh.tw, [&](int col, float2 z) {
                if (act && col >= c0 && col < c1) {
                    rowA[col - c0] = z.x;
                    if (hasb) rowB[col - c0] = z.y;
                }
            });
            __syncwarp();
        }
        __syncthreads();

        // ---- 3a. Lanczos along x, in place per row (columns [gc0, gc1)) ----
        const int ncol = gc1 - gc0;
        for (int r = warp; r < nrows; r += kWarps) {
            float* row = reinterpret_cast<float*>(sh.s1 + r * NH);
            float res[8];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int cc = lane + 32 * i;
                float acc = 0.f;
                if (cc < ncol) {
                    const int c = gc0 + cc;
#pragma unroll
                    for (int k = 0; k < 7; k++) {
                        const int xsrc = c - 3 + k;
                        const float g = (xsrc >= c0 && xsrc < c1) ? row[xsrc - c0] : 0.f;
                        acc = fmaf(fx[k], g, acc);
                    }
                }
                res[i] = acc;
            }
            __syncwarp();
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int cc = lane + 32 * i;
                if (cc < ncol) row[cc] = res[i];
            }
        }
        __syncthreads();

        // ---- 3b. Lanczos along y, shift, crop, write ----
        const int orows = b - a;
        for (int idx = threadIdx.x; idx < orows * mw; idx += kThreads) {
            const int r = a + idx / mw;
            const int j = idx % mw;
            const int c = j - sx;
            float val = 0.f;
            if (c >= gc0 && c < gc1) {
#pragma unroll
                for (int k = 0; k < 7; k++) {
                    const int rr = r - 3 + k;
                    if (rr >= rlo && rr < rhi) {
                        const float* row = reinterpret_cast<const float*>(sh.s1 + (rr - rlo) * NH);
                        val = fmaf(fy[k], row[c - gc0], val);
                    }
                }
            }
            float* o = O + (int64_t)(r + sy) * ldo + j;
            const float res = val * osc;
            if (it.mode == TB_MOG_ATOMIC) atomicAdd(o, res);
            else if (accum) *o += res;
            else *o = res;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kThreads, 1)
fourier_render_kernel(const tb_fft_item* __restrict__ items, int n_items,
                      const double* __restrict__ amp, const double* __restrict__ var,
                      const float* __restrict__ psf_spec, float* __restrict__ out,
                      int32_t* counter, tb_status* st) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Shared sh;
    sh.tw = reinterpret_cast<float2*>(smem_raw);
    sh.comp = reinterpret_cast<float4*>(smem_raw + 256 * 8);
    sh.taps = reinterpret_cast<float*>(smem_raw + 256 * 8 + kMaxK * 16);
    sh.xbuf = sh.taps + 16;
    sh.s1 = reinterpret_cast<float2*>(sh.xbuf + kWarps * kXbufPerWarp);
    __shared__ int64_t slot;
    __shared__ int cur_n;
    if (threadIdx.x == 0) cur_n = 0;

    for (;;) {
        const int64_t u = tb::next_unit(counter, &slot);
        if (u >= n_items) break;
        const tb_fft_item& it = items[u];
        const int N = it.sz, K = it.K;
        const bool okN = N == 32 || N == 64 || N == 128 || N == 256;
        if (!okN || K < 0 || K > kMaxK || it.mw <= 0 || it.mh <= 0 ||
            !(fabs(it.mux) <= 0.5) || !(fabs(it.muy) <= 0.5)) {
            if (threadIdx.x == 0) tb::report(st, TB_STATUS_BAD_ITEM, (int)u, N);
            continue;
        }
        // components (FP64 -> FP32 exponent coefficients in log2 units)
        const double c2 = -2.0 * TB_PI * TB_PI * TB_LOG2E;
        for (int k = threadIdx.x; k < K; k += kThreads) {
            const int c = it.c0 + k;
            const double a = var[4 * c], bb = var[4 * c + 1], d = var[4 * c + 3];
            sh.comp[k] = make_float4((float)amp[c], (float)(c2 * a), (float)(c2 * 2.0 * bb),
                                     (float)(c2 * d));
        }
        if (threadIdx.x == 32) taps3(it.mux, sh.taps);
        if (threadIdx.x == 64) taps3(it.muy, sh.taps + 7);
        __syncthreads();
        if (cur_n != N) {
            __syncthreads();
            switch (N) {
                case 256: tb::build_twiddles<256>(sh.tw); break;
                case 128: tb::build_twiddles<128>(sh.tw); break;
                case 64: tb::build_twiddles<64>(sh.tw); break;
                default: tb::build_twiddles<32>(sh.tw); break;
            }
            __syncthreads();
            if (threadIdx.x == 0) cur_n = N;
        }
        __syncthreads();
        const float* spec = psf_spec + it.spec_off;
        switch (N) {
            case 256: render_item<256>(it, K, spec, out, sh, kRmax256); break;
            case 128: render_item<128>(it, K, spec, out, sh, 128 + 6); break;
            case 64: render_item<64>(it, K, spec, out, sh, 64 + 6); break;
            default: render_item<32>(it, K, spec, out, sh, 32 + 6); break;
        }
    }
}

}  // namespace

extern "C" int tb_fourier_render(const tb_fft_item* items, int32_t n_items,
                                 const double* comp_amp, const double* comp_var,
                                 const float* psf_spec, float* out, int32_t* work_counter,
                                 tb_status* status, void* stream) {
    if (n_items < 0) return TB_ERR_ARG;
    if (n_items == 0) return TB_OK;
    if (!items || !comp_amp || !comp_var || !psf_spec || !out || !work_counter) return TB_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaFuncSetAttribute(fourier_render_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kSmemBytes) != cudaSuccess)
        return TB_ERR_LAUNCH;
    if (cudaMemsetAsync(work_counter, 0, sizeof(int32_t), s) != cudaSuccess) return TB_ERR_LAUNCH;
    if (status && cudaMemsetAsync(status, 0, sizeof(tb_status), s) != cudaSuccess)
        return TB_ERR_LAUNCH;
    const int grid = n_items < tb::num_sms() ? n_items : tb::num_sms();
    fourier_render_kernel<<<grid, kThreads, kSmemBytes, s>>>(items, n_items, comp_amp, comp_var,
                                                             psf_spec, out, work_counter, status);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

// ---------------------------------------------------------------------------
// PSF spectra: forward rfft2 of zero-padded PSF images, stored column-major
// (element (row j, column v) at v * sz + j) so the column pass above reads
// contiguous memory.
// ---------------------------------------------------------------------------
namespace {

constexpr int kSpecThreads = 256;

template <int N>
__device__ void spec_rows(const float* __restrict__ pad, float* __restrict__ spec, int img,
                          float* xbuf, const float2* tw) {
    constexpr int T = N / 8, GPW = 32 / T, XB = tb::fft_xbuf_floats<N>();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = lane % T;
    float* xr = xbuf + warp * kXbufPerWarp + (lane / T) * XB;
    float* xi = xr + XB / 2;
    const int nwarps = kSpecThreads / 32;
    const float* I = pad + (int64_t)img * N * N;
    float2* S = reinterpret_cast<float2*>(spec) + (int64_t)img * N * (N / 2 + 1);
    for (int y0 = blockIdx.x * nwarps * GPW + warp * GPW; y0 < N; y0 += gridDim.x * nwarps * GPW) {
        const int y = y0 + lane / T;   // N rows, groups never run past the end
        float2 x[8];
#pragma unroll
        for (int m = 0; m < 8; m++) x[m] = make_float2(I[(int64_t)y * N + t + m * T], 0.f);
        tb::fft_run<N, -1>(x, t, xr, xi, tw, [&](int k, float2 z) {
            if (k <= N / 2) S[(int64_t)k * N + y] = z;
        });
        __syncwarp();
    }
}

template <int N>
__device__ void spec_cols(float* __restrict__ spec, int img, float* xbuf, const float2* tw) {
    constexpr int T = N / 8, GPW = 32 / T, XB = tb::fft_xbuf_floats<N>(), NH = N / 2 + 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int t = lane % T;
    float* xr = xbuf + warp * kXbufPerWarp + (lane / T) * XB;
    float* xi = xr + XB / 2;
    const int nwarps = kSpecThreads / 32;
    float2* S = reinterpret_cast<float2*>(spec) + (int64_t)img * N * NH;
    for (int v0 = blockIdx.x * nwarps * GPW + warp * GPW; v0 < NH; v0 += gridDim.x * nwarps * GPW) {
        const bool act = v0 + lane / T < NH;
        const int v = act ? v0 + lane / T : NH - 1;
        float2 x[8];
#pragma unroll
        for (int m = 0; m < 8; m++) x[m] = S[(int64_t)v * N + t + m * T];
        __syncwarp();
        tb::fft_run<N, -1>(x, t, xr, xi, tw, [&](int j, float2 z) {
            if (act) S[(int64_t)v * N + j] = z;
        });
        __syncwarp();
    }
}

template <int N>
__global__ void __launch_bounds__(kSpecThreads) spec_kernel(const float* pad, float* spec, int pass) {
    __shared__ float2 tw[N];
    __shared__ float xbuf[(kSpecThreads / 32) * kXbufPerWarp];
    tb::build_twiddles<N>(tw);
    __syncthreads();
    if (pass == 0) spec_rows<N>(pad, spec, blockIdx.y, xbuf, tw);
    else spec_cols<N>(spec, blockIdx.y, xbuf, tw);
}

__global__ void spec_normalize_kernel(float* spec, int N) {
    const int img = blockIdx.y;
    float2* S = reinterpret_cast<float2*>(spec) + (int64_t)img * N * (N / 2 + 1);
    const float2 p00 = S[0];
    const float n = sqrtf(p00.x * p00.x + p00.y * p00.y);
    __syncthreads();
    if (n == 0.f) return;
    const int total = N * (N / 2 + 1);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        if (i == 0) continue;
        float2 z = S[i];
        S[i] = make_float2(z.x / n, z.y / n);
    }
}

__global__ void spec_normalize_dc_kernel(float* spec, int N) {
    float2* S = reinterpret_cast<float2*>(spec) + (int64_t)blockIdx.x * N * (N / 2 + 1);
    const float2 p00 = S[0];
    const float n = sqrtf(p00.x * p00.x + p00.y * p00.y);
    if (threadIdx.x == 0 && n != 0.f) S[0] = make_float2(p00.x / n, p00.y / n);
}

template <int N>
int launch_spec(const float* pad, float* spec, int n, cudaStream_t s) {
    constexpr int GPW = 32 / (N / 8);
    const int lines_per_cta = (kSpecThreads / 32) * GPW;
    dim3 g0((N + lines_per_cta - 1) / lines_per_cta, n);
    spec_kernel<N><<<g0, kSpecThreads, 0, s>>>(pad, spec, 0);
    dim3 g1((N / 2 + 1 + lines_per_cta - 1) / lines_per_cta, n);
    spec_kernel<N><<<g1, kSpecThreads, 0, s>>>(pad, spec, 1);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

}  // namespace

extern "C" int tb_psf_spectrum(const float* pad, float* spec, int32_t n, int32_t sz,
                               int32_t normalize, void* stream) {
    if (n < 0) return TB_ERR_ARG;
    if (n == 0) return TB_OK;
    if (!pad || !spec) return TB_ERR_ARG;
    if (n > 65535) return TB_ERR_SIZE;
    cudaStream_t s = (cudaStream_t)stream;
    int r;
    switch (sz) {
        case 32: r = launch_spec<32>(pad, spec, n, s); break;
        case 64: r = launch_spec<64>(pad, spec, n, s); break;
        case 128: r = launch_spec<128>(pad, spec, n, s); break;
        case 256: r = launch_spec<256>(pad, spec, n, s); break;
        default: return TB_ERR_SIZE;
    }
    if (r != TB_OK || !normalize) return r;
    // Divide every element by |P[0,0]| (the DC element last, after all blocks
    // have read it).
    dim3 g(64, n);
    spec_normalize_kernel<<<g, 256, 0, s>>>(spec, sz);
    spec_normalize_dc_kernel<<<n, 32, 0, s>>>(spec, sz);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}
