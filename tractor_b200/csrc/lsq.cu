// K5: least-squares step kernels (sm_100a).
//
//  * normal equations A^T A, A^T r of many independent problems: on the
//    tensor cores (tcgen05 kind::tf32, three-term TF32 split, FP32 partial
//    sums over at most 128 rows, FP64 totals) for P <= 255; above that
//    FP32 CUDA-core products with compensated (Kahan) FP32 running sums;
//  * FP64 column-scaled Cholesky solve with a damping ridge and one step of
//    iterative refinement, one CTA per problem;
//  * per-image chi^2 with compensated FP32 sums reduced in FP64 in a fixed
//    order (deterministic).
// These replace the sparse-matrix assembly and LSQR solve of
// LsqrOptimizer.getUpdateDirection (tractor/lsqr_optimizer.py:328-644) and
// the chi-square sum of Tractor.getLogLikelihood (tractor/engine.py:475-479).
#include <atomic>

#include "tb_common.cuh"
#include "tc_sm100.cuh"

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

// ---------------------------------------------------------------------------
// Normal equations on the tensor cores (tcgen05, kind::tf32).
//
// Problem b's operand is the Q x R matrix [A^T; r^T] (Q = P + 1 rows: the P
// design-matrix columns, then the right-hand side), K-major: the R pixel rows
// are the contraction dimension.  A pass covers the 128 operand rows
// [r0, r0 + 128) against the columns [r0, Q): one pass for Q <= 128, two
// (r0 = 0, 128) for Q <= 256, which together give the upper triangle.  Within
// a pass (Qp = Q - r0 operand rows, Q8 = Qp rounded up to 8) a stage covers
// KC pixel rows (KC = 32 .. 128, the largest power of two with Q8 KC <=
// 32 QM, so a stage moves up to 16 KB (QM = 128) or 32 KB (QM = 256)):
//  * every thread copies its quads (4 consecutive pixel rows of one operand
//    row) of a stage with cp.async into its own slots of a ring of raw
//    stages (kRaw stages in flight, no registers held): one 16-byte copy when
//    the problem's columns are 16-byte aligned, else four 4-byte copies;
//  * when its copies of stage s have landed, the thread splits each value into
//    TF32 hi and lo parts and stores each quad as one 16-byte core-matrix row
//    of the canonical no-swizzle K-major layout (two operand stages; the K
//    chunks Q8 * 16 + 16 bytes apart keep the stores bank-conflict-free);
//  * one thread issues S += Hi_t Hi^T, E += Hi_t Lo^T + Lo_t Hi^T (three TF32
//    MMAs of M = 128 per K = 8 step) into two TMEM accumulators and commits
//    to the stage's mbarrier.
// The tensor core's FP32 accumulation truncates, so its error grows with the
// number of accumulations: every 128 rows (16 accumulations into S) the
// accumulators are drained, and S and E are kept apart so that the small
// cross terms add no roundings to S.  QM = 128 drains S + E into a
// compensated (Kahan) FP32 total T, C held in TMEM next to S and E (512
// columns) and writes the FP64 results once at the end; QM = 256 (S and E
// already take 512 columns) adds the drains in FP64 at AtA[j P + i]
// (coalesced over i) and Atr[i] and mirrors the lower triangle at the end.
// Either way AtA is exactly symmetric.  Operand rows Qp .. 127 and columns
// Qp .. N of the MMAs hold stale values; they only reach rows and columns of
// D that are never read.
namespace tcne {
constexpr int kThreads = 256;
constexpr int kChunkRows = 128;     // rows per FP32 accumulation chunk
constexpr uint64_t kWaitNs = 1000000000ull;   // 1 s: far above any real MMA batch
__host__ __device__ constexpr int elems(int qm) { return 32 * qm; }        // per raw stage
__host__ __device__ constexpr int qpt(int qm) { return elems(qm) / 4 / kThreads; }   // quads
// raw stages in flight (QM = 128: the copies of 3 stages ahead of the one
// being converted)
#ifndef TB_NE_RAW128
#define TB_NE_RAW128 4
#endif
__host__ __device__ constexpr int raw_stages(int qm) { return qm == 128 ? TB_NE_RAW128 : 2; }
__host__ __device__ constexpr int kc_of(int qm, int q8) {
    int kc = 128;
    while (kc > 32 && kc * q8 > elems(qm)) kc >>= 1;
    return kc;
}
// bytes one operand buffer spans, the MMA's reads of all 128 A rows and N B
// rows past the last K chunk included
__host__ __device__ constexpr int cbuf_need(int qm, int q8) {
    const int kc = kc_of(qm, q8), lbo = q8 * 16 + 16, n = (q8 + 15) / 16 * 16;
    return (kc / 4 - 1) * lbo + (n * 16 > 2048 ? n * 16 : 2048);
}
__host__ __device__ constexpr int cbuf_bytes(int qm) {
    int m = 0;
    for (int q8 = 8; q8 <= qm; q8 += 8) m = cbuf_need(qm, q8) > m ? cbuf_need(qm, q8) : m;
    return (m + 127) / 128 * 128;
}
__host__ __device__ constexpr int raw_bytes(int qm) { return raw_stages(qm) * elems(qm) * 4; }
__host__ __device__ constexpr int smem_bytes(int qm) {
    return raw_bytes(qm) + 4 * cbuf_bytes(qm) + 64;
}
// QM = 128: S, E, T, C at columns 0, 128, 256, 384; QM = 256: S, E at 0, 256
constexpr uint32_t kTmemCols = 512;
}  // namespace tcne

__device__ unsigned int g_ne_timeouts = 0;

__device__ __forceinline__ void cp_async4(uint32_t dst, const float* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src),
                 "r"(valid ? 4 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const float* src, int bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int QM>
__global__ void __launch_bounds__(tcne::kThreads, 1)
normal_eq_tc_kernel(const float* __restrict__ A, const float* __restrict__ rhs,
                    const int64_t* a_off, const int64_t* r_off, const int32_t* lda,
                    const int32_t* Pv, const int32_t* Rv, const int64_t* ata_off,
                    const int64_t* atr_off, double* AtA, double* Atr) {
    using namespace tb::tc;
    constexpr int QPT = tcne::qpt(QM);
    constexpr int NRAW = tcne::raw_stages(QM);
    constexpr int CBUF = tcne::cbuf_bytes(QM);
    constexpr int RAW = tcne::raw_bytes(QM);
    constexpr uint32_t NCOLS = tcne::kTmemCols;
    extern __shared__ __align__(128) unsigned char smem[];
    float4* raw = reinterpret_cast<float4*>(smem);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + RAW + 4 * CBUF);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + RAW + 4 * CBUF + 16);

    const int b = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int P = Pv[b], R = Rv[b], ld = lda[b];
    const int Q = P + 1;
    if (P <= 0 || Q > QM) return;
    double* M = AtA + ata_off[b];
    double* g = Atr + atr_off[b];
    if (R <= 0) {
        for (int e = tid; e < P * P; e += tcne::kThreads) M[e] = 0.0;
        for (int e = tid; e < P; e += tcne::kThreads) g[e] = 0.0;
        return;
    }
    const float* Ab = A + a_off[b];
    const float* rb = rhs + r_off[b];
    // 16-byte copies when every column starts on a 16-byte boundary
    const bool vec = ((reinterpret_cast<uintptr_t>(Ab) | reinterpret_cast<uintptr_t>(rb)) & 15) == 0 &&
                     (ld & 3) == 0;

    if (warp == 0) tmem_alloc(tslot, NCOLS);
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tS = *tslot, tE = tS + QM;
    const uint32_t tT = tS + 256, tC = tS + 384;   // QM = 128 only
    const uint32_t lane_sel = (uint32_t)((warp & 3) * 32) << 16;
    const uint32_t raw_base = smem_u32(raw);

    bool fail = false;
    int gs = 0;              // stage counter over both passes (operand buffer, phase)
    int last_commit = -1;
    int nchunk = 0;          // drains so far (QM = 128: T and C hold data after the first)
    for (int r0 = 0; r0 < Q && !fail; r0 += 128) {
        const int Qp = Q - r0;                        // operand rows of this pass
        const int Q8 = (Qp + 7) & ~7;
        const int N = (Qp + 15) & ~15;                // columns r0 .. r0 + N
        const int KC = tcne::kc_of(QM, Q8);
        const int KQ = KC / 4;                        // quads per operand row and stage
        const int LBO = Q8 * 16 + 16;
        const int nst = (R + KC - 1) / KC;
        const int chunk_st = tcne::kChunkRows / KC;   // stages per accumulation chunk
        const uint32_t idesc = idesc_tf32(128, N);
        // this thread's quads: pixel rows k .. k + 3 of operand rows c0 + m * cs
        const int k = 4 * (tid % KQ), c0 = tid / KQ, cs = tcne::kThreads / KQ;
        const float* src[QPT];
        int soff[QPT];
#pragma unroll
        for (int m = 0; m < QPT; m++) {
            const int c = c0 + m * cs, col = r0 + c;
            src[m] = c < Qp ? (col < P ? Ab + (int64_t)col * ld : rb) + k : nullptr;
            soff[m] = (k >> 2) * LBO + (c >> 3) * 128 + (c & 7) * 16;
        }
        auto issue = [&](int s) {
            const int slot = s % NRAW;
            const int row = s * KC + k;
            const int nv = s < nst ? min(max(R - row, 0), 4) : 0;   // valid rows of the quad
#pragma unroll
            for (int m = 0; m < QPT; m++) {
                if (src[m] == nullptr || s >= nst) continue;
                const uint32_t dst = raw_base + 16 * ((slot * QPT + m) * tcne::kThreads + tid);
                const float* p = src[m] + (int64_t)s * KC;
                if (vec) {
                    cp_async16(dst, nv > 0 ? p : Ab, 4 * nv);
                } else {
#pragma unroll
                    for (int q = 0; q < 4; q++) cp_async4(dst + 4 * q, q < nv ? p + q : Ab, q < nv);
                }
            }
            cp_async_commit();
        };
        for (int s = 0; s < NRAW - 1; s++) issue(s);
        for (int s = 0; s < nst; s++, gs++) {
            issue(s + NRAW - 1);
            cp_async_wait<NRAW - 1>();    // this thread's copies of stage s have landed
            const int bi = gs & 1;
            unsigned char* hi = smem + RAW + (2 * bi) * CBUF;
            unsigned char* lo = smem + RAW + (2 * bi + 1) * CBUF;
            // operand buffer bi is free once the MMAs of stage gs - 2 have completed
            bool ok = true;
            if (s >= 2) ok = mbar_wait(&bar[bi], ((gs >> 1) - 1) & 1, tcne::kWaitNs);
            const int slot = s % NRAW;
#pragma unroll
            for (int m = 0; m < QPT; m++) {
                if (src[m] == nullptr) continue;
                const float4 v = raw[(slot * QPT + m) * tcne::kThreads + tid];
                float4 h, l;
                split_tf32(v.x, h.x, l.x);
                split_tf32(v.y, h.y, l.y);
                split_tf32(v.z, h.z, l.z);
                split_tf32(v.w, h.w, l.w);
                *reinterpret_cast<float4*>(hi + soff[m]) = h;
                *reinterpret_cast<float4*>(lo + soff[m]) = l;
            }
            fence_async_smem();
            if (__syncthreads_or(!ok)) { fail = true; break; }
            if (tid == 0) {
                fence_after_sync();
                const bool fresh = (s % chunk_st) == 0;
                const uint32_t ha = smem_u32(hi), la = smem_u32(lo);
                for (int kk = 0; kk < KC / 8; kk++) {
                    const uint32_t o = kk * 2 * LBO;
                    const uint64_t dh = smem_desc(ha + o, LBO, 128);
                    const uint64_t dl = smem_desc(la + o, LBO, 128);
                    const uint32_t acc = (fresh && kk == 0) ? 0u : 1u;
                    mma_tf32(tS, dh, dh, idesc, acc);
                    mma_tf32(tE, dh, dl, idesc, acc);
                    mma_tf32(tE, dl, dh, idesc, 1u);
                }
                commit(&bar[bi]);
            }
            last_commit = gs;
            const bool drain = (s % chunk_st) == chunk_st - 1 || s == nst - 1;
            if (!drain) continue;
            ok = mbar_wait(&bar[bi], (gs >> 1) & 1, tcne::kWaitNs);
            if (__syncthreads_or(!ok)) { fail = true; break; }
            fence_after_sync();
            const int row0 = r0 + (warp & 3) * 32;     // first D row of this warp
            const int i = row0 + lane;
            for (int cb = warp >> 2; cb < (N + 31) / 32; cb += 2) {
                // blocks wholly below the diagonal or past row P - 1 hold nothing needed
                if (r0 + cb * 32 + 31 < row0 || row0 >= P) continue;
                float vs[32], ve[32];
                tmem_ld32(tS + cb * 32 + lane_sel, vs);
                tmem_ld32(tE + cb * 32 + lane_sel, ve);
                if constexpr (QM == 128) {
                    // T, C += S + E (Kahan)
                    if (nchunk == 0) {
#pragma unroll
                        for (int jj = 0; jj < 32; jj++) { vs[jj] += ve[jj]; ve[jj] = 0.f; }
                    } else {
                        float vt[32], vc[32];
                        tmem_ld32(tT + cb * 32 + lane_sel, vt);
                        tmem_ld32(tC + cb * 32 + lane_sel, vc);
#pragma unroll
                        for (int jj = 0; jj < 32; jj++) {
                            const float y = (vs[jj] + ve[jj]) - vc[jj];
                            const float t = vt[jj] + y;
                            ve[jj] = (t - vt[jj]) - y;
                            vs[jj] = t;
                        }
                    }
                    tmem_st32(tT + cb * 32 + lane_sel, vs);
                    tmem_st32(tC + cb * 32 + lane_sel, ve);
                } else {
                    if (i >= P) continue;
                    const bool first = s < chunk_st;
                    // all loads of the block first, then the stores
                    double old[32];
#pragma unroll
                    for (int jj = 0; jj < 32; jj++) {
                        const int j = r0 + cb * 32 + jj;
                        old[jj] = 0.0;
                        if (first || j < i || j > P) continue;
                        old[jj] = j == P ? g[i] : M[(int64_t)j * P + i];
                    }
#pragma unroll
                    for (int jj = 0; jj < 32; jj++) {
                        const int j = r0 + cb * 32 + jj;
                        if (j < i || j > P) continue;
                        const double x = old[jj] + ((double)vs[jj] + (double)ve[jj]);
                        if (j == P) g[i] = x;
                        else M[(int64_t)j * P + i] = x;
                    }
                }
            }
            nchunk++;
            fence_before_sync();
            __syncthreads();   // the next chunk's first MMAs overwrite the accumulators
        }
        cp_async_wait<0>();
    }
    if (fail) {
        if (tid == 0) atomicAdd(&g_ne_timeouts, 1u);
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        for (int e = tid; e < P * P; e += tcne::kThreads) M[e] = nan;
        for (int e = tid; e < P; e += tcne::kThreads) g[e] = nan;
        // let the MMAs in flight finish (bounded) before the TMEM is freed
        if (last_commit >= 0)
            mbar_wait(&bar[last_commit & 1], (last_commit >> 1) & 1, tcne::kWaitNs);
    } else if constexpr (QM == 128) {
        // FP64 results from the compensated totals: D[i][j], i <= j
        fence_after_sync();
        const int row0 = (warp & 3) * 32, i = row0 + lane;
        for (int cb = warp >> 2; cb < (((Q + 15) & ~15) + 31) / 32; cb += 2) {
            if (cb * 32 + 31 < row0 || row0 >= P) continue;
            float vt[32], vc[32];
            tmem_ld32(tT + cb * 32 + lane_sel, vt);
            tmem_ld32(tC + cb * 32 + lane_sel, vc);
            if (i >= P) continue;
#pragma unroll
            for (int jj = 0; jj < 32; jj++) {
                const int j = cb * 32 + jj;
                if (j < i || j > P) continue;
                const double x = (double)vt[jj] - (double)vc[jj];
                if (j == P) {
                    g[i] = x;
                } else {
                    M[(int64_t)j * P + i] = x;
                    M[(int64_t)i * P + j] = x;
                }
            }
        }
    } else {
        // lower triangle from the accumulated upper one (M[j P + i], i <= j)
        __syncthreads();
        for (int e = tid; e < P * P; e += tcne::kThreads) {
            const int i = e / P, j = e % P;
            if (i < j) M[e] = M[(int64_t)j * P + i];
        }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        tmem_dealloc(tS, NCOLS);
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
    // P[b] is device data: a problem larger than the shared arrays or than
    // its slice of the workspace (work_stride = max_p^2 doubles) is refused
    // instead of writing into its neighbours' factors
    if (P > kMaxSmemP || (int64_t)P * P > work_stride) {
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

// ---------------------------------------------------------------------------
// Normal equations on the tensor cores for Q = P + 1 <= 64 (warp-specialised,
// one MMA per K step).
//
// The A operand of the MMA is the stacked 128-row tile [Hi; Lo] of the
// problem's Q operand rows (hi parts in rows 0-63, lo parts in rows 64-127)
// and the B operand its hi rows, so ONE kind::tf32 MMA of M = 128 per K = 8
// step gives S = Hi Hi^T (D rows 0-63) and E = Lo Hi^T (D rows 64-127);
// D = S + E + E^T, the cross terms symmetrised when the accumulators are
// drained.  Warps 0-7 (converters) stage KC = 32 pixel rows per stage (4-
// or 16-byte cp.async into their own slots of a raw ring, split into TF32 hi
// and lo, one 16-byte core-matrix row each in the canonical no-swizzle
// K-major layout) and arrive on `full`; warp 8 issues the stage's 4 MMAs and
// commits to `empty`.  Chunks of 128 rows alternate between two
// accumulator sets (TMEM columns 0 and 128); the converters drain chunk c
// after staging the first stage of chunk c + 1, whose MMAs wait until that
// drain is done: TMEM loads that ran while MMAs into the other set were in
// flight returned wrong values on B200 (two column layouts tried), so a drain
// never overlaps an MMA.  A set holds two tiles (columns +0 and +64) that
// take alternate K steps, so each FP32 accumulator takes 8 accumulations per
// chunk: the tensor core's accumulation truncates, and its error grows with
// that count.  A drain: the warps
// holding E rows copy their 32 x 32 blocks to shared memory, a converter
// barrier, then the warps holding S rows add S + E + E^T of their blocks on
// or above the diagonal into compensated (Kahan) FP32 totals in shared
// memory, and arrive on `accfree` (the set may be overwritten).  The FP64
// results are written once at the end, AtA exactly symmetric.
// ---------------------------------------------------------------------------
namespace tc64 {
constexpr int kConv = 256;                 // converter threads
constexpr int kThreads = kConv + 32;       // + the MMA warp
constexpr int kKc = 32;                    // pixel rows per stage
constexpr int kChunkSt = 4;                // stages per 128-row accumulation chunk
#ifndef TB_NE64_RAW
#define TB_NE64_RAW 3
#endif
constexpr int kRaw = TB_NE64_RAW;          // raw stages in flight
constexpr int kKq = kKc / 4;               // quads per operand row and stage
constexpr int kRowStep = kConv / kKq;      // operand rows between a thread's quads
constexpr int kQpt = 64 / kRowStep;        // quads per thread and stage (64 x 32 / 4 / 256)
constexpr int kLbo = 128 / 8 * 128 + 16;   // bytes between K chunks (128 stacked rows)
constexpr int kCbuf = 16512;               // kKc / 4 chunks of kLbo bytes, MMA over-read included
constexpr int kRawBytes = kRaw * kQpt * kConv * 16;
constexpr int kEsLd = 65;                  // E staging row stride (floats)
constexpr int kEsBytes = 64 * kEsLd * 4;
constexpr int kTotBytes = 3 * 2 * 32 * 32 * 4;   // T, C of blocks (0,0), (0,1), (1,1)
constexpr int kBarOff = kRawBytes + 2 * kCbuf + kEsBytes + kTotBytes;
constexpr int kSmem = kBarOff + 128;
constexpr uint32_t kTmemCols = 256;
constexpr uint64_t kWaitNs = 1000000000ull;
static_assert((kKc / 4 - 1) * kLbo + 2048 <= kCbuf, "MMA reads stay inside the operand buffer");
// two CTAs per SM (shared memory), whose 2 x 256 TMEM columns always fit
static_assert(kSmem + 1024 > 232448 / 3 && 2 * (kSmem + 1024) <= 232448, "two CTAs per SM");
}  // namespace tc64

__device__ __forceinline__ void conv_barrier() {
    asm volatile("bar.sync 1, 256;" ::: "memory");
}

__global__ void __launch_bounds__(tc64::kThreads, 2)
normal_eq_tc64_kernel(const float* __restrict__ A, const float* __restrict__ rhs,
                      const int64_t* a_off, const int64_t* r_off, const int32_t* lda,
                      const int32_t* Pv, const int32_t* Rv, const int64_t* ata_off,
                      const int64_t* atr_off, double* AtA, double* Atr) {
    using namespace tb::tc;
    using namespace tc64;
    extern __shared__ __align__(128) unsigned char smem[];
    float4* raw = reinterpret_cast<float4*>(smem);
    unsigned char* cbuf = smem + kRawBytes;
    float* Es = reinterpret_cast<float*>(smem + kRawBytes + 2 * kCbuf);
    float* tot = reinterpret_cast<float*>(smem + kRawBytes + 2 * kCbuf + kEsBytes);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kBarOff);
    uint64_t* full = bar;          // [2] converters -> MMA warp: operand buffer written
    uint64_t* empty = bar + 2;     // [2] MMA warp -> converters: the stage's MMAs completed
    uint64_t* accfree = bar + 4;   // [2] converters -> MMA warp: accumulator set drained
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 6);
    int* flag = reinterpret_cast<int*>(bar + 7);   // a wait timed out

    const int b = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int P = Pv[b], R = Rv[b], ld = lda[b];
    const int Q = P + 1;
    if (P <= 0 || Q > 64) return;
    double* M = AtA + ata_off[b];
    double* g = Atr + atr_off[b];
    if (R <= 0) {
        for (int e = tid; e < P * P; e += kThreads) M[e] = 0.0;
        for (int e = tid; e < P; e += kThreads) g[e] = 0.0;
        return;
    }
    const float* Ab = A + a_off[b];
    const float* rb = rhs + r_off[b];
    const bool vec = ((reinterpret_cast<uintptr_t>(Ab) | reinterpret_cast<uintptr_t>(rb)) & 15) == 0 &&
                     (ld & 3) == 0;
    const int N = (Q + 15) & ~15;
    const int nst = (R + kKc - 1) / kKc;

    if (warp == 0) tmem_alloc(tslot, kTmemCols);
    if (tid == 0) {
        for (int i = 0; i < 2; i++) {
            mbar_init(&full[i], kConv);
            mbar_init(&empty[i], 1);
            mbar_init(&accfree[i], kConv);
        }
        *flag = 0;
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tbase = *tslot;

    if (warp == 8) {
        // ---------------- MMA warp ----------------
        const uint32_t idesc = idesc_tf32(128, N);
        int last = -1;
        bool ok = true;
        for (int s = 0; s < nst && ok; s++) {
            const int bi = s & 1, c = s / kChunkSt;
            if (lane == 0) {
                ok = mbar_wait(&full[bi], (s >> 1) & 1, kWaitNs);
                // the previous chunk has been drained: no TMEM load of a drain
                // runs while MMAs are in flight
                if (ok && s % kChunkSt == 0 && c >= 1)
                    ok = mbar_wait(&accfree[(c - 1) & 1], ((c - 1) >> 1) & 1, kWaitNs);
                if (ok) {
                    fence_after_sync();
                    const uint32_t base = smem_u32(cbuf + bi * kCbuf);
                    const uint32_t d = tbase + (uint32_t)(128 * (c & 1));
                    // K steps alternate between the set's two tiles (columns
                    // +0, +64): 8 accumulations per tile and chunk
                    for (int kk = 0; kk < kKc / 8; kk++) {
                        const uint64_t desc = smem_desc(base + kk * 2 * kLbo, kLbo, 128);
                        mma_tf32(d + 64 * (kk & 1), desc, desc, idesc,
                                 (s % kChunkSt == 0 && kk < 2) ? 0u : 1u);
                    }
                } else {
                    atomicExch(flag, 1);
                }
                commit(&empty[bi]);   // in every case: no converter waits on a stage never committed
                last = s;
            }
            ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
            if (*reinterpret_cast<volatile int*>(flag)) ok = false;
        }
        // every MMA this warp issued has completed before the TMEM is freed
        if (lane == 0 && last >= 0 && !mbar_wait(&empty[last & 1], (last >> 1) & 1, kWaitNs))
            atomicExch(flag, 1);
        __syncwarp();
    } else {
        // ---------------- converter warps ----------------
        const int q = warp & 3;                       // TMEM lane quarter
        const uint32_t lane_sel = (uint32_t)(q * 32) << 16;
        const uint32_t raw_base = smem_u32(raw);
        // this thread's quads: pixel rows k .. k + 3 of operand rows
        // c0 + kRowStep m
        const int k = 4 * (tid % kKq), c0 = tid / kKq;
        const float* src[kQpt];
        int soff[kQpt];
#pragma unroll
        for (int m = 0; m < kQpt; m++) {
            const int c = c0 + kRowStep * m;
            src[m] = c < Q ? (c < P ? Ab + (int64_t)c * ld : rb) + k : nullptr;
            soff[m] = (k >> 2) * kLbo + (c >> 3) * 128 + (c & 7) * 16;
        }
        auto issue = [&](int s) {
            const int slot = s % kRaw;
            const int row = s * kKc + k;
            const int nv = s < nst ? min(max(R - row, 0), 4) : 0;
#pragma unroll
            for (int m = 0; m < kQpt; m++) {
                if (src[m] == nullptr || s >= nst) continue;
                const uint32_t dst = raw_base + 16 * ((slot * kQpt + m) * kConv + tid);
                const float* p = src[m] + (int64_t)s * kKc;
                if (vec) {
                    cp_async16(dst, nv > 0 ? p : Ab, 4 * nv);
                } else {
#pragma unroll
                    for (int j = 0; j < 4; j++) cp_async4(dst + 4 * j, j < nv ? p + j : Ab, j < nv);
                }
            }
            cp_async_commit();
        };
        int drains = 0;
        // Drain of chunk `drains` (accumulator set drains & 1), last stage
        // s_last.  Every converter thread runs every drain and its barrier in
        // the same order, also after a wait has timed out (`skip`: the waits
        // are left out, the values then are garbage and the outputs NaN).
        auto drain = [&](int s_last, bool skip) -> bool {
            const bool ok = __all_sync(
                0xffffffffu, !skip && mbar_wait(&empty[s_last & 1], (s_last >> 1) & 1, kWaitNs));
            const uint32_t d = tbase + (uint32_t)(128 * (drains & 1));
            const int cb = warp >> 2;                  // 32-column block
            if (ok) {
                fence_after_sync();
                // E rows (q - 2) * 32 .. + 31 of this column block -> shared memory
                const int e0 = (q - 2) * 32;
                if (q >= 2 && e0 < Q && cb * 32 < N) {
                    float v[32], v2[32];
                    tmem_ld32(d + cb * 32 + lane_sel, v);
                    tmem_ld32(d + 64 + cb * 32 + lane_sel, v2);
#pragma unroll
                    for (int jj = 0; jj < 32; jj++)
                        Es[(e0 + lane) * kEsLd + cb * 32 + jj] = v[jj] + v2[jj];
                }
            }
            conv_barrier();
            if (ok && q < 2 && cb >= q && q * 32 < P && cb * 32 <= P) {
                // S block (I = q, J = cb) on or above the diagonal: T, C += S + E + E^T
                float v[32], v2[32];
                tmem_ld32(d + cb * 32 + lane_sel, v);
                tmem_ld32(d + 64 + cb * 32 + lane_sel, v2);
#pragma unroll
                for (int jj = 0; jj < 32; jj++) v[jj] += v2[jj];
                const int i = q * 32 + lane;
                float* Tt = tot + (q + cb) * 2 * 1024;    // blocks (0,0) 0, (0,1) 1, (1,1) 2
                float* Cc = Tt + 1024;
#pragma unroll 8
                for (int jj = 0; jj < 32; jj++) {
                    const int j = cb * 32 + jj;
                    const float x = v[jj] + (Es[i * kEsLd + j] + Es[j * kEsLd + i]);
                    if (drains == 0) {
                        Tt[jj * 32 + lane] = x;
                        Cc[jj * 32 + lane] = 0.f;
                    } else {
                        const float t0 = Tt[jj * 32 + lane], c0v = Cc[jj * 32 + lane];
                        const float y = x - c0v;
                        const float t = t0 + y;
                        Cc[jj * 32 + lane] = (t - t0) - y;
                        Tt[jj * 32 + lane] = t;
                    }
                }
            }
            // the E block copies are read by other warps: no warp refills Es
            // before every S warp has read it (the next drain needs the next
            // chunk, whose stages need every converter's arrival)
            fence_before_sync();
            tb::tc::mbar_arrive(&accfree[drains & 1]);
            drains++;
            return ok;
        };
        bool fail = false;
        for (int s = 0; s < kRaw - 1; s++) issue(s);
        for (int s = 0; s < nst; s++) {
            issue(s + kRaw - 1);
            cp_async_wait<kRaw - 1>();    // this thread's copies of stage s have landed
            const int bi = s & 1;
            unsigned char* buf = cbuf + bi * kCbuf;
            // operand buffer bi is free once the MMAs of stage s - 2 have completed
            if (s >= 2 && !fail && !mbar_wait(&empty[bi], ((s >> 1) - 1) & 1, kWaitNs)) fail = true;
            const int slot = s % kRaw;
#pragma unroll
            for (int m = 0; m < kQpt; m++) {
                if (src[m] == nullptr) continue;
                const float4 v = raw[(slot * kQpt + m) * kConv + tid];
                float4 h, l;
                split_tf32(v.x, h.x, l.x);
                split_tf32(v.y, h.y, l.y);
                split_tf32(v.z, h.z, l.z);
                split_tf32(v.w, h.w, l.w);
                *reinterpret_cast<float4*>(buf + soff[m]) = h;          // row c
                *reinterpret_cast<float4*>(buf + soff[m] + 1024) = l;   // row 64 + c
            }
            fence_async_smem();
            tb::tc::mbar_arrive(&full[bi]);
            // the previous chunk's accumulators, while this chunk is multiplied
            if (s % kChunkSt == 0 && s > 0 && !drain(s - 1, fail)) fail = true;
        }
        cp_async_wait<0>();
        if (!drain(nst - 1, fail)) fail = true;
        if (fail) atomicExch(flag, 1);
        conv_barrier();
        // FP64 results from the compensated totals: D[i][j], i <= j <= P
        const int cb = warp >> 2;
        if (!fail && !*reinterpret_cast<volatile int*>(flag) && q < 2 && cb >= q && q * 32 < P &&
            cb * 32 <= P) {
            const int i = q * 32 + lane;
            const float* Tt = tot + (q + cb) * 2 * 1024;
            const float* Cc = Tt + 1024;
            if (i < P) {
                for (int jj = 0; jj < 32; jj++) {
                    const int j = cb * 32 + jj;
                    if (j < i || j > P) continue;
                    const double x = (double)Tt[jj * 32 + lane] - (double)Cc[jj * 32 + lane];
                    if (j == P) {
                        g[i] = x;
                    } else {
                        M[(int64_t)j * P + i] = x;
                        M[(int64_t)i * P + j] = x;
                    }
                }
            }
        }
    }
    __syncthreads();
    if (*reinterpret_cast<volatile int*>(flag)) {
        if (tid == 0) atomicAdd(&g_ne_timeouts, 1u);
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        for (int e = tid; e < P * P; e += kThreads) M[e] = nan;
        for (int e = tid; e < P; e += kThreads) g[e] = nan;
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        tmem_dealloc(tbase, kTmemCols);
    }
}

int launch_normal_eq_tc64(const float* A, const float* rhs, const int64_t* a_off,
                          const int64_t* r_off, const int32_t* lda, const int32_t* P,
                          const int32_t* R, const int64_t* ata_off, const int64_t* atr_off,
                          double* AtA, double* Atr, int32_t n_problems, cudaStream_t s) {
    if (cudaFuncSetAttribute(normal_eq_tc64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             tc64::kSmem) != cudaSuccess)
        return TB_ERR_LAUNCH;
    normal_eq_tc64_kernel<<<n_problems, tc64::kThreads, tc64::kSmem, s>>>(
        A, rhs, a_off, r_off, lda, P, R, ata_off, atr_off, AtA, Atr);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

// One CTA per problem and, by its shared memory, per SM: the 512 TMEM
// columns it takes are always free.
template <int QM>
int launch_normal_eq_tc(const float* A, const float* rhs, const int64_t* a_off,
                        const int64_t* r_off, const int32_t* lda, const int32_t* P,
                        const int32_t* R, const int64_t* ata_off, const int64_t* atr_off,
                        double* AtA, double* Atr, int32_t n_problems, cudaStream_t s) {
    constexpr int smem = tcne::smem_bytes(QM);
    static_assert(smem > 114 * 1024, "one CTA per SM");
    static_assert(smem <= 227 * 1024, "shared memory per CTA");
    if (cudaFuncSetAttribute(normal_eq_tc_kernel<QM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem) != cudaSuccess)
        return TB_ERR_LAUNCH;
    normal_eq_tc_kernel<QM><<<n_problems, tcne::kThreads, smem, s>>>(
        A, rhs, a_off, r_off, lda, P, R, ata_off, atr_off, AtA, Atr);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
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
    const cudaStream_t s = (cudaStream_t)stream;
    if (max_p + 1 <= 64)
        return launch_normal_eq_tc64(A, rhs, a_off, r_off, lda, P, R, ata_off, atr_off, AtA, Atr,
                                     n_problems, s);
    if (max_p + 1 <= 128)
        return launch_normal_eq_tc<128>(A, rhs, a_off, r_off, lda, P, R, ata_off, atr_off, AtA,
                                        Atr, n_problems, s);
    if (max_p + 1 <= 256)
        return launch_normal_eq_tc<256>(A, rhs, a_off, r_off, lda, P, R, ata_off, atr_off, AtA,
                                        Atr, n_problems, s);
    normal_eq_kernel<<<n_problems, kNeThreads, 0, s>>>(A, rhs, a_off, r_off, lda, P, R, ata_off,
                                                        atr_off, AtA, Atr);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

extern "C" int tb_tensor_core_timeouts(uint32_t* count) {
    if (!count) return TB_ERR_ARG;
    unsigned int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_ne_timeouts, sizeof(v)) != cudaSuccess) return TB_ERR_LAUNCH;
    *count = v;
    return TB_OK;
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
// Per-device address of g_solve_scratch.  Host threads may call at once:
// relaxed atomics (every thread that looks the address up stores the same
// value).  The address belongs to the device's primary context; a caller
// that destroys it (cudaDeviceReset) must reload the library.
std::atomic<double*> g_solve_scratch_addr[kMaxDevices];
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
    double* scratch = g_solve_scratch_addr[dev].load(std::memory_order_relaxed);
    if (scratch == nullptr) {
        if (cudaGetSymbolAddress((void**)&scratch, g_solve_scratch) != cudaSuccess || !scratch)
            return TB_ERR_LAUNCH;
        g_solve_scratch_addr[dev].store(scratch, std::memory_order_relaxed);
    }
    solve_kernel<<<n_problems, kSolveThreads, 0, (cudaStream_t)stream>>>(
        AtA, Atr, ata_off, atr_off, P, x_off, X, info, damp, scratch, (int64_t)max_p * max_p);
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
    sizes[12] = (int32_t)sizeof(tb_ring_item);
    return 13;
}
