// K5: least-squares step kernels (sm_100a).
//
//  * normal equations A^T A, A^T r of many independent problems: FP32
//    products, compensated (Kahan) FP32 running sums per output, final values
//    in FP64;
//  * FP64 column-scaled Cholesky solve with a damping ridge and one step of
//    iterative refinement, one CTA per problem;
//  * per-image chi^2 with compensated FP32 sums reduced in FP64 in a fixed
//    order (deterministic).
// These replace the sparse-matrix assembly and LSQR solve of
// LsqrOptimizer.getUpdateDirection (tractor/lsqr_optimizer.py:328-644) and
// the chi-square sum of Tractor.getLogLikelihood (tractor/engine.py:475-479).
#include "tb_common.cuh"

namespace {

constexpr int kNeThreads = 256;
constexpr int kRowChunk = 32;
constexpr int kOutPerThread = 8;
constexpr int kMaxSmemP = 320;

// Output index o in [0, P(P+1)/2 + P): the upper triangle (i <= j) row by row,
// then the P entries of A^T r (j = P means the right-hand side).
__device__ __forceinline__ void out_pair(int o, int P, int& i, int& j) {
    const int ntri = P * (P + 1) / 2;
    if (o >= ntri) { i = o - ntri; j = P; return; }
    // row i holds P - i entries
    int r = 0, base = 0;
    while (base + (P - r) <= o) { base += P - r; r++; }
    i = r;
    j = r + (o - base);
}

__global__ void __launch_bounds__(kNeThreads)
normal_eq_kernel(const float* __restrict__ A, const float* __restrict__ rhs,
                 const int64_t* a_off, const int64_t* r_off, const int32_t* lda,
                 const int32_t* Pv, const int32_t* Rv, const int64_t* ata_off,
                 const int64_t* atr_off, double* AtA, double* Atr) {
    __shared__ float tile[kRowChunk][kMaxSmemP + 1 + 1];
    const int b = blockIdx.x;
    const int P = Pv[b], R = Rv[b], ld = lda[b];
    if (P <= 0 || P > kMaxSmemP) return;
    const float* Ab = A + a_off[b];
    const float* rb = rhs + r_off[b];
    const int nout = P * (P + 1) / 2 + P;
    for (int o0 = 0; o0 < nout; o0 += kNeThreads * kOutPerThread) {
        int oi[kOutPerThread], oj[kOutPerThread];
        float s[kOutPerThread], c[kOutPerThread];
#pragma unroll
        for (int q = 0; q < kOutPerThread; q++) {
            const int o = o0 + q * kNeThreads + threadIdx.x;
            if (o < nout) out_pair(o, P, oi[q], oj[q]); else { oi[q] = 0; oj[q] = 0; }
            s[q] = 0.f;
            c[q] = 0.f;
        }
        for (int r0 = 0; r0 < R; r0 += kRowChunk) {
            const int nr = min(kRowChunk, R - r0);
            __syncthreads();
            for (int e = threadIdx.x; e < kRowChunk * (P + 1); e += kNeThreads) {
                const int col = e / kRowChunk, r = e % kRowChunk;
                float v = 0.f;
                if (r < nr) v = (col < P) ? Ab[(int64_t)col * ld + r0 + r] : rb[r0 + r];
                tile[r][col] = v;
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < kOutPerThread; q++) {
                if (o0 + q * kNeThreads + threadIdx.x >= nout) continue;
                const int i = oi[q], j = oj[q];
                float sq = s[q], cq = c[q];
                for (int r = 0; r < nr; r++) {
                    const float p = tile[r][i] * tile[r][j];
                    const float y = p - cq;
                    const float t = sq + y;
                    cq = (t - sq) - y;
                    sq = t;
                }
                s[q] = sq;
                c[q] = cq;
            }
        }
#pragma unroll
        for (int q = 0; q < kOutPerThread; q++) {
            const int o = o0 + q * kNeThreads + threadIdx.x;
            if (o >= nout) continue;
            const double v = (double)s[q] - (double)c[q];
            const int i = oi[q], j = oj[q];
            if (j == P) {
                Atr[atr_off[b] + i] = v;
            } else {
                AtA[ata_off[b] + (int64_t)i * P + j] = v;
                AtA[ata_off[b] + (int64_t)j * P + i] = v;
            }
        }
    }
}

constexpr int kSolveThreads = 256;

// Solves (D^-1 AtA D^-1 + damp^2 I) x = D^-1 Atr with D = sqrt(diag(AtA)),
// X = x / D.  L (P x P, lower) lives in `work`.
__global__ void __launch_bounds__(kSolveThreads)
solve_kernel(const double* __restrict__ AtA, const double* __restrict__ Atr,
             const int64_t* ata_off, const int64_t* atr_off, const int32_t* Pv,
             const int64_t* x_off, double* X, int32_t* info, double damp, double* work,
             int64_t work_stride) {
    __shared__ double d[kMaxSmemP];
    __shared__ double y[kMaxSmemP];
    __shared__ double xs[kMaxSmemP];
    __shared__ double red[kSolveThreads];
    __shared__ int bad;
    const int b = blockIdx.x;
    const int P = Pv[b];
    const int tid = threadIdx.x;
    if (P <= 0) return;
    if (P > kMaxSmemP) {
        if (tid == 0) info[b] = -1;
        return;
    }
    const double* M = AtA + ata_off[b];
    const double* g = Atr + atr_off[b];
    double* L = work + (int64_t)b * work_stride;
    if (tid == 0) bad = 0;
    for (int i = tid; i < P; i += kSolveThreads) {
        const double a = M[(int64_t)i * P + i];
        d[i] = (a > 0.0 && isfinite(a)) ? sqrt(a) : 0.0;
    }
    __syncthreads();
    const double d2 = damp * damp;
    // Scaled matrix (lower triangle); a dropped column becomes a unit row.
    for (int e = tid; e < P * P; e += kSolveThreads) {
        const int i = e / P, j = e % P;
        if (j > i) continue;
        double v;
        if (d[i] == 0.0 || d[j] == 0.0) v = (i == j) ? 1.0 : 0.0;
        else v = M[(int64_t)i * P + j] / (d[i] * d[j]) + (i == j ? d2 : 0.0);
        L[(int64_t)i * P + j] = v;
    }
    __syncthreads();
    // Right-looking Cholesky.
    for (int k = 0; k < P; k++) {
        if (tid == 0) {
            const double a = L[(int64_t)k * P + k];
            if (!(a > 0.0) || !isfinite(a)) bad = k + 1;
            else L[(int64_t)k * P + k] = sqrt(a);
        }
        __syncthreads();
        if (bad) break;
        const double lkk = L[(int64_t)k * P + k];
        for (int i = k + 1 + tid; i < P; i += kSolveThreads) L[(int64_t)i * P + k] /= lkk;
        __syncthreads();
        const int m = P - k - 1;
        for (int e = tid; e < m * m; e += kSolveThreads) {
            const int i = k + 1 + e / m, j = k + 1 + e % m;
            if (j > i) continue;
            L[(int64_t)i * P + j] -= L[(int64_t)i * P + k] * L[(int64_t)j * P + k];
        }
        __syncthreads();
    }
    if (bad) {
        for (int i = tid; i < P; i += kSolveThreads) X[x_off[b] + i] = 0.0;
        if (tid == 0) info[b] = bad;
        return;
    }
    // rhs and two solves (solution + one refinement step)
    for (int i = tid; i < P; i += kSolveThreads) {
        xs[i] = 0.0;
        y[i] = (d[i] == 0.0) ? 0.0 : g[i] / d[i];
    }
    __syncthreads();
    for (int pass = 0; pass < 2; pass++) {
        if (pass == 1) {
            // residual r = rhs - M_scaled x, into y
            for (int i = tid; i < P; i += kSolveThreads) {
                double acc = (d[i] == 0.0) ? 0.0 : g[i] / d[i];
                for (int j = 0; j < P; j++) {
                    double mij;
                    if (d[i] == 0.0 || d[j] == 0.0) mij = (i == j) ? 1.0 : 0.0;
                    else mij = M[(int64_t)i * P + j] / (d[i] * d[j]) + (i == j ? d2 : 0.0);
                    acc -= mij * xs[j];
                }
                y[i] = acc;
            }
            __syncthreads();
        }
        // forward: L z = y (in place in y)
        for (int i = 0; i < P; i++) {
            double part = 0.0;
            for (int j = tid; j < i; j += kSolveThreads) part += L[(int64_t)i * P + j] * y[j];
            red[tid] = part;
            __syncthreads();
            for (int s = kSolveThreads / 2; s > 0; s >>= 1) {
                if (tid < s) red[tid] += red[tid + s];
                __syncthreads();
            }
            if (tid == 0) y[i] = (y[i] - red[0]) / L[(int64_t)i * P + i];
            __syncthreads();
        }
        // backward: L^T w = z (in place in y)
        for (int i = P - 1; i >= 0; i--) {
            double part = 0.0;
            for (int j = i + 1 + tid; j < P; j += kSolveThreads) part += L[(int64_t)j * P + i] * y[j];
            red[tid] = part;
            __syncthreads();
            for (int s = kSolveThreads / 2; s > 0; s >>= 1) {
                if (tid < s) red[tid] += red[tid + s];
                __syncthreads();
            }
            if (tid == 0) y[i] = (y[i] - red[0]) / L[(int64_t)i * P + i];
            __syncthreads();
        }
        for (int i = tid; i < P; i += kSolveThreads) xs[i] += y[i];
        __syncthreads();
    }
    for (int i = tid; i < P; i += kSolveThreads)
        X[x_off[b] + i] = (d[i] == 0.0) ? 0.0 : xs[i] / d[i];
    if (tid == 0) info[b] = 0;
}

constexpr int kChiThreads = 1024;

__global__ void __launch_bounds__(kChiThreads)
chi2_kernel(const float* __restrict__ data, const float* __restrict__ model,
            const float* __restrict__ inverr, const int64_t* off, const int64_t* npix,
            double* out) {
    __shared__ double red[kChiThreads];
    const int b = blockIdx.x;
    const int64_t o = off[b], n = npix[b];
    float s = 0.f, c = 0.f;
    for (int64_t i = threadIdx.x; i < n; i += kChiThreads) {
        const float chi = (data[o + i] - model[o + i]) * inverr[o + i];
        const float y = chi * chi - c;
        const float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    red[threadIdx.x] = (double)s - (double)c;
    __syncthreads();
    for (int k = kChiThreads / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[b] = red[0];
}

}  // namespace

extern "C" int tb_normal_equations(const float* A, const float* rhs, const int64_t* a_off,
                                   const int64_t* r_off, const int32_t* lda, const int32_t* P,
                                   const int32_t* R, const int64_t* ata_off,
                                   const int64_t* atr_off, double* AtA, double* Atr,
                                   int32_t n_problems, int32_t max_p, void* stream) {
    if (n_problems < 0 || max_p < 0) return TB_ERR_ARG;
    if (n_problems == 0) return TB_OK;
    if (max_p > kMaxSmemP) return TB_ERR_SIZE;
    if (!A || !rhs || !a_off || !r_off || !lda || !P || !R || !ata_off || !atr_off || !AtA || !Atr)
        return TB_ERR_ARG;
    normal_eq_kernel<<<n_problems, kNeThreads, 0, (cudaStream_t)stream>>>(
        A, rhs, a_off, r_off, lda, P, R, ata_off, atr_off, AtA, Atr);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

extern "C" int tb_solve_update(const double* AtA, const double* Atr, const int64_t* ata_off,
                               const int64_t* atr_off, const int32_t* P, const int64_t* x_off,
                               double* X, int32_t* info, double damp, int32_t n_problems,
                               int32_t max_p, double* work, void* stream) {
    if (n_problems < 0 || max_p < 0) return TB_ERR_ARG;
    if (n_problems == 0) return TB_OK;
    if (max_p > kMaxSmemP) return TB_ERR_SIZE;
    if (!AtA || !Atr || !ata_off || !atr_off || !P || !x_off || !X || !info || !work)
        return TB_ERR_ARG;
    solve_kernel<<<n_problems, kSolveThreads, 0, (cudaStream_t)stream>>>(
        AtA, Atr, ata_off, atr_off, P, x_off, X, info, damp, work, (int64_t)max_p * max_p);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

// ---------------------------------------------------------------------------
// Allocation-free solve: the factor workspace is a file-scope device array,
// held by every GPU that loads the library.  Host code cannot use the
// array's name as a device address; its address is looked up once per device
// (with that device current) and cached here.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double g_solve_scratch[TB_SOLVE_NOALLOC_MAX_DOUBLES];

namespace {
constexpr int kMaxDevices = 64;
double* g_solve_scratch_addr[kMaxDevices] = {nullptr};
}  // namespace

extern "C" int tb_solve_update_noalloc(const double* AtA, const double* Atr,
                                       const int64_t* ata_off, const int64_t* atr_off,
                                       const int32_t* P, const int64_t* x_off, double* X,
                                       int32_t* info, double damp, int32_t n_problems,
                                       int32_t max_p, void* stream) {
    if (n_problems < 0 || max_p < 0) return TB_ERR_ARG;
    if (n_problems == 0) return TB_OK;
    if (max_p > kMaxSmemP) return TB_ERR_SIZE;
    if ((int64_t)n_problems * max_p * max_p > (int64_t)TB_SOLVE_NOALLOC_MAX_DOUBLES)
        return TB_ERR_SIZE;
    if (!AtA || !Atr || !ata_off || !atr_off || !P || !x_off || !X || !info) return TB_ERR_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TB_ERR_LAUNCH;
    if (g_solve_scratch_addr[dev] == nullptr) {
        double* addr = nullptr;
        if (cudaGetSymbolAddress((void**)&addr, g_solve_scratch) != cudaSuccess || !addr)
            return TB_ERR_LAUNCH;
        g_solve_scratch_addr[dev] = addr;
    }
    solve_kernel<<<n_problems, kSolveThreads, 0, (cudaStream_t)stream>>>(
        AtA, Atr, ata_off, atr_off, P, x_off, X, info, damp, g_solve_scratch_addr[dev],
        (int64_t)max_p * max_p);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

extern "C" int tb_chi2(const float* data, const float* model, const float* inverr,
                       const int64_t* off, const int64_t* npix, int32_t n, double* out,
                       void* stream) {
    if (n < 0) return TB_ERR_ARG;
    if (n == 0) return TB_OK;
    if (!data || !model || !inverr || !off || !npix || !out) return TB_ERR_ARG;
    chi2_kernel<<<n, kChiThreads, 0, (cudaStream_t)stream>>>(data, model, inverr, off, npix, out);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

extern "C" const char* tb_version(void) { return "tractor_b200 0.1 (sm_100a)"; }

extern "C" int tb_abi_sizes(int32_t* sizes) {
    if (!sizes) return TB_ERR_ARG;
    sizes[0] = (int32_t)sizeof(tb_mog_item);
    sizes[1] = (int32_t)sizeof(tb_fft_item);
    sizes[2] = (int32_t)sizeof(tb_status);
    sizes[3] = (int32_t)sizeof(tb_galaxy_src);
    sizes[4] = (int32_t)sizeof(tb_fft_image);
    sizes[5] = (int32_t)sizeof(tb_scene_src);
    sizes[6] = (int32_t)sizeof(tb_scene_image);
    sizes[7] = (int32_t)sizeof(tb_scene_item);
    sizes[8] = (int32_t)sizeof(tb_fit_source);
    sizes[9] = (int32_t)sizeof(tb_fit_blob);
    sizes[10] = (int32_t)sizeof(tb_fit_unit);
    sizes[11] = (int32_t)sizeof(tb_fit_state);
    return 12;
}
