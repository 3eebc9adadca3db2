// K1: batched mixture-of-Gaussians pixel evaluator (sm_100a).
//
// Work unit = one 32x32 tile of one item's rectangle.  A persistent grid takes
// units from a global counter.  For each unit the CTA stages the item's
// components in shared memory -- folding the FP64 covariance into FP32
// exponent coefficients in log2 units, with the means taken relative to the
// tile origin so FP32 offsets stay small -- and culls the components whose
// evaluated region (exponent >= floor) misses the tile.  Each thread then owns
// one column and four rows of the tile and evaluates every surviving
// component with one SFU ex2 per pixel.  Component order (and so summation
// order) is the item's order, as in c_gauss_2d_grid (tractor/mix.i:452-524).
#include "tb_common.cuh"

namespace {

struct GaussC {
    float mx, my;       // mean relative to the tile origin
    float qxx, qxy, qyy;  // exponent (log2 units) = qxx dx^2 + qxy dx dy + qyy dy^2
    float s;            // amp / (2 pi sqrt(det))
    float fl;           // exponent floor, log2 units
    float pad;
};

// Difference items: the perturbed mixture relative to the base one, for
// G'_k - G_k = exp2(e_k) (s'_k expm1(de_k) + (s'_k - s_k)) with
// de_k = e'_k - e_k (natural-log units, same mean).
struct GaussD {
    float dxx, dxy, dyy;  // de = dxx dx^2 + dxy dx dy + dyy dy^2
    float sp;             // s'_k = amp'_k / (2 pi sqrt(det V'_k))
    float ds;             // s'_k - s_k (from FP64)
    float pad0, pad1, pad2;
};

constexpr int kThreads = 256;
constexpr int kRowsPerThread = TB_MOG_TILE / (kThreads / 32);  // 4

// Evaluates the staged components on one tile: thread column `lane`, rows
// warp + 8 j.  With kDerivs, also the derivatives with respect to the mean
// (-G (2 I0 dx + I1 dy), tractor/mix.i:44-82), written to two planes.
template <bool kDerivs, bool kDiff>
__device__ __forceinline__ void eval_tile(const tb_mog_item& it, const GaussC* comps,
                                          const GaussD* dcomps, int total,
                                          int tw, int th, int ox, int oy,
                                          const uint8_t* __restrict__ masks,
                                          float* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float acc[kRowsPerThread], gx[kRowsPerThread], gy[kRowsPerThread];
#pragma unroll
    for (int j = 0; j < kRowsPerThread; j++) acc[j] = gx[j] = gy[j] = 0.f;
    const float xf = (float)lane;
    for (int c = 0; c < total; c++) {
        const GaussC q = comps[c];
        const float dx = xf - q.mx;
        const float A = q.qxx * dx * dx;
        const float B = q.qxy * dx;
#pragma unroll
        for (int j = 0; j < kRowsPerThread; j++) {
            const float dy = (float)(warp + 8 * j) - q.my;
            const float e = fmaf(dy, fmaf(q.qyy, dy, B), A);
            float sv = (e >= q.fl) ? q.s : 0.f;
            const float ev = tb::ex2(e);
            if (kDiff) {
                const GaussD d = dcomps[c];
                const float de = fmaf(dy, fmaf(d.dyy, dy, d.dxy * dx), d.dxx * dx * dx);
                sv = (e >= q.fl) ? fmaf(d.sp, expm1f(de), d.ds) : 0.f;
            }
            acc[j] = fmaf(sv, ev, acc[j]);
            if (kDerivs) {
                const float v = sv * ev;
                // d/dmean in natural-log units: ln2 * (2 qxx dx + qxy dy) etc.
                gx[j] = fmaf(-v, 0.69314718f * fmaf(2.f * q.qxx, dx, q.qxy * dy), gx[j]);
                gy[j] = fmaf(-v, 0.69314718f * fmaf(2.f * q.qyy, dy, q.qxy * dx), gy[j]);
            }
        }
    }
    const float sc = it.scale;
    const int w = it.w, h = it.h;
    const int64_t ldo = it.ldo > 0 ? it.ldo : w;
#pragma unroll
    for (int j = 0; j < kRowsPerThread; j++) {
        const int y = warp + 8 * j;
        if (lane < tw && y < th) {
            const int64_t o = (int64_t)(oy + y) * w + (ox + lane);
            const bool on = !(it.mask_off >= 0 && !masks[it.mask_off + o]);
            const float val = on ? acc[j] * sc : 0.f;
            float* p = out + it.out_off + (int64_t)(oy + y) * ldo + (ox + lane);
            if (it.mode == TB_MOG_ACCUM) *p += val;
            else if (it.mode == TB_MOG_ATOMIC) atomicAdd(p, val);
            else *p = val;
            if (kDerivs) {
                out[it.deriv_off + o] = on ? gx[j] * sc : 0.f;
                out[it.deriv_off + (int64_t)w * h + o] = on ? gy[j] * sc : 0.f;
            }
        }
    }
}

__global__ void __launch_bounds__(kThreads)
mog_render_kernel(const tb_mog_item* __restrict__ items, int n_items, int64_t n_tiles,
                  const double* __restrict__ amp, const double* __restrict__ mean,
                  const double* __restrict__ var, const uint8_t* __restrict__ masks,
                  float* __restrict__ out, int32_t* counter, tb_status* st) {
    __shared__ GaussC comps[TB_MOG_MAX_K];
    __shared__ GaussD dcomps[TB_MOG_MAX_K];
    __shared__ int64_t slot;
    __shared__ int item_idx;
    __shared__ int warp_count[kThreads / 32];

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;

    for (;;) {
        const int64_t u = tb::next_unit(counter, &slot);
        if (u >= n_tiles) break;
        if (threadIdx.x == 0) {
            int lo = 0, hi = n_items - 1;
            while (lo < hi) {
                int mid = (lo + hi + 1) >> 1;
                if (items[mid].tile0 <= u) lo = mid; else hi = mid - 1;
            }
            item_idx = lo;
        }
        __syncthreads();
        const int ii = item_idx;
        const tb_mog_item& it = items[ii];
        const int w = it.w, h = it.h, K = it.K;
        const int tiles_x = (w + TB_MOG_TILE - 1) / TB_MOG_TILE;
        const int64_t t = u - it.tile0;
        const int ox = (int)(t % tiles_x) * TB_MOG_TILE;
        const int oy = (int)(t / tiles_x) * TB_MOG_TILE;
        const int tw = min(TB_MOG_TILE, w - ox);
        const int th = min(TB_MOG_TILE, h - oy);
        const double tx0 = (double)it.x0 + ox, ty0 = (double)it.y0 + oy;
        const bool diff = it.diff_c0 >= 0;
        if (K < 0 || K > TB_MOG_MAX_K || w <= 0 || h <= 0 ||
            (diff && (it.deriv_off >= 0 || it.floor_mode != TB_FLOOR_FIXED))) {
            if (threadIdx.x == 0) tb::report(st, TB_STATUS_BAD_ITEM, ii, K);
            continue;
        }

        // ---- stage + cull components (one thread per component) ----
        bool keep = false;
        GaussC g;
        GaussD gd;
        if (threadIdx.x < K) {
            const int c = it.c0 + threadIdx.x;
            const double a = amp[c];
            const double v0 = var[4 * c], v3 = var[4 * c + 3];
            const double vxy = 0.5 * (var[4 * c + 1] + var[4 * c + 2]);
            const double det = v0 * v3 - vxy * vxy;
            const double s = a / (2.0 * TB_PI * sqrt(det));
            const double f = -0.5 / det * TB_LOG2E;
            double fl = it.floor;
            if (it.floor_mode == TB_FLOOR_MINVAL) {
                double asum = 0.0;
                for (int k = 0; k < K; k++) asum += amp[it.c0 + k];
                fl = -100.0;
                if (it.floor > 0.0) fl = fmax(-100.0, log(it.floor * 2.0 * TB_PI * sqrt(det) / asum));
            }
            g.qxx = (float)(v3 * f);
            g.qxy = (float)(-2.0 * vxy * f);
            g.qyy = (float)(v0 * f);
            g.s = (float)s;
            g.fl = (float)(fl * TB_LOG2E);
            const double mx = (mean[2 * c] + it.fx) - tx0;
            const double my = (mean[2 * c + 1] + it.fy) - ty0;
            g.mx = (float)mx;
            g.my = (float)my;
            g.pad = 0.f;
            bool finite = det > 0.0 && isfinite(s) && isfinite(f) && isfinite(mx) &&
                          isfinite(my) && isfinite(fl);
            double rx2 = 0.0, ry2 = 0.0;
            bool live = a != 0.0;
            if (diff) {
                // perturbed component: same mean, its own amplitude and
                // covariance; exponent differences in natural-log units
                const int c2 = it.diff_c0 + threadIdx.x;
                const double a2 = amp[c2];
                const double w0 = var[4 * c2], w3 = var[4 * c2 + 3];
                const double wxy = 0.5 * (var[4 * c2 + 1] + var[4 * c2 + 2]);
                const double det2 = w0 * w3 - wxy * wxy;
                const double s2 = a2 / (2.0 * TB_PI * sqrt(det2));
                gd.dxx = (float)(-0.5 * (w3 / det2 - v3 / det));
                gd.dxy = (float)(wxy / det2 - vxy / det);
                gd.dyy = (float)(-0.5 * (w0 / det2 - v0 / det));
                gd.sp = (float)s2;
                gd.ds = (float)(s2 - s);
                gd.pad0 = gd.pad1 = gd.pad2 = 0.f;
                finite = finite && det2 > 0.0 && isfinite(s2);
                rx2 = w0;
                ry2 = w3;
                live = live || a2 != 0.0;
            }
            if (!finite) {
                tb::report(st, TB_STATUS_NONFINITE, ii, threadIdx.x);
            } else if (live) {
                // Region where the exponent is >= floor: Mahalanobis^2 <= -2 floor
                // (for a difference item, the larger of the two covariances').
                const double r2 = -2.0 * fl;
                const double rx = sqrt(r2 * fmax(v0, rx2)), ry = sqrt(r2 * fmax(v3, ry2));
                keep = (mx + rx >= 0.0) && (mx - rx <= tw - 1) && (my + ry >= 0.0) &&
                       (my - ry <= th - 1);
            }
        }
        // Order-preserving compaction of the surviving components.
        const unsigned ballot = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) warp_count[warp] = __popc(ballot);
        __syncthreads();
        int base = 0, total = 0;
#pragma unroll
        for (int i = 0; i < kThreads / 32; i++) {
            base += (i < warp) ? warp_count[i] : 0;
            total += warp_count[i];
        }
        if (keep) {
            const int slot_k = base + __popc(ballot & ((1u << lane) - 1u));
            comps[slot_k] = g;
            if (diff) dcomps[slot_k] = gd;
        }
        __syncthreads();

        if (diff)
            eval_tile<false, true>(it, comps, dcomps, total, tw, th, ox, oy, masks, out);
        else if (it.deriv_off >= 0)
            eval_tile<true, false>(it, comps, dcomps, total, tw, th, ox, oy, masks, out);
        else
            eval_tile<false, false>(it, comps, dcomps, total, tw, th, ox, oy, masks, out);
    }
}

}  // namespace

extern "C" int tb_mog_render(const tb_mog_item* items, int32_t n_items, int64_t n_tiles,
                             const double* comp_amp, const double* comp_mean,
                             const double* comp_var, const uint8_t* masks, float* out,
                             int32_t* work_counter, tb_status* status, void* stream) {
    if (n_items < 0 || n_tiles < 0) return TB_ERR_ARG;
    if (n_items == 0 || n_tiles == 0) return TB_OK;
    if (!items || !comp_amp || !comp_mean || !comp_var || !out || !work_counter)
        return TB_ERR_ARG;
    if (n_tiles > (int64_t)0x7fffffff) return TB_ERR_SIZE;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(work_counter, 0, sizeof(int32_t), s) != cudaSuccess) return TB_ERR_LAUNCH;
    if (status && cudaMemsetAsync(status, 0, sizeof(tb_status), s) != cudaSuccess)
        return TB_ERR_LAUNCH;
    const int64_t want = (int64_t)tb::num_sms() * 8;
    const int grid = (int)(n_tiles < want ? n_tiles : want);
    mog_render_kernel<<<grid, kThreads, 0, s>>>(items, n_items, n_tiles, comp_amp, comp_mean,
                                               comp_var, masks, out, work_counter, status);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}
