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
#include <cstring>

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

// ---------------------------------------------------------------------------
// tb_mog_render over host buffers: the items, components and masks are
// packed into the caller's page-locked staging buffer, copied to the caller's
// device workspace in one copy, rendered, and the packed output and status
// word brought back in one copy; the stream is synchronised before return.
// One call per render instead of a staging copy, an output allocation, a
// launch and a read-back issued one by one from the host language.
// ---------------------------------------------------------------------------
namespace {

inline int64_t up256(int64_t x) { return (x + 255) & ~(int64_t)255; }

struct MogHostLayout {
    int64_t items, amp, mean, var, mask, in_end, counter, out, status, total;
};

MogHostLayout mog_host_layout(int64_t n_items, int64_t n_comp, int64_t mask_bytes,
                              int64_t n_out) {
    MogHostLayout L;
    int64_t o = 0;
    L.items = o;   o = up256(o + n_items * (int64_t)sizeof(tb_mog_item));
    L.amp = o;     o = up256(o + n_comp * 8);
    L.mean = o;    o = up256(o + n_comp * 16);
    L.var = o;     o = up256(o + n_comp * 32);
    L.mask = o;    o = up256(o + mask_bytes);
    L.in_end = o;
    L.counter = o; o = up256(o + 4);
    L.out = o;     o = o + n_out * 4;
    L.status = (o + 15) & ~(int64_t)15;
    L.total = L.status + (int64_t)sizeof(tb_status);
    return L;
}

// Every item's components, mask and output inside the sizes given, so that
// the device never reads or writes outside the workspace.
bool mog_items_fit(const tb_mog_item* items, int32_t n_items, int64_t n_tiles, int64_t n_comp,
                   int64_t mask_bytes, int64_t n_out, bool* any_accum) {
    int64_t tiles = 0;
    *any_accum = false;
    for (int32_t i = 0; i < n_items; i++) {
        const tb_mog_item& it = items[i];
        if (it.w < 0 || it.h < 0 || it.K < 0 || it.c0 < 0 || it.ldo < 0) return false;
        if ((int64_t)it.c0 + it.K > n_comp) return false;
        if (it.diff_c0 >= 0 && (int64_t)it.diff_c0 + it.K > n_comp) return false;
        if (it.tile0 != tiles) return false;
        tiles += (int64_t)((it.w + TB_MOG_TILE - 1) / TB_MOG_TILE) *
                 ((it.h + TB_MOG_TILE - 1) / TB_MOG_TILE);
        if (it.w == 0 || it.h == 0) continue;
        const int64_t ldo = it.ldo ? it.ldo : it.w;
        if (ldo < it.w || it.out_off < 0) return false;
        if (it.out_off + (int64_t)(it.h - 1) * ldo + it.w > n_out) return false;
        if (it.deriv_off >= 0 && it.deriv_off + 2 * (int64_t)it.w * it.h > n_out) return false;
        if (it.mask_off >= 0 && it.mask_off + (int64_t)it.w * it.h > mask_bytes) return false;
        if (it.mode != TB_MOG_STORE) *any_accum = true;
    }
    return tiles == n_tiles;
}

}  // namespace

extern "C" int tb_mog_render_host_bytes(int32_t n_items, int64_t n_comp, int64_t mask_bytes,
                                        int64_t n_out, int64_t* bytes) {
    if (n_items < 0 || n_comp < 0 || mask_bytes < 0 || n_out < 0 || !bytes) return TB_ERR_ARG;
    *bytes = mog_host_layout(n_items, n_comp, mask_bytes, n_out).total;
    return TB_OK;
}

extern "C" int tb_mog_render_host(const tb_mog_item* items, int32_t n_items, int64_t n_tiles,
                                  const double* comp_amp, const double* comp_mean,
                                  const double* comp_var, int64_t n_comp, const uint8_t* masks,
                                  int64_t mask_bytes, float* out, int64_t n_out,
                                  tb_status* status, void* pinned, void* workspace,
                                  int64_t ws_bytes, void* stream) {
    if (n_items < 0 || n_tiles < 0 || n_comp < 0 || mask_bytes < 0 || n_out < 0 || !status)
        return TB_ERR_ARG;
    if ((n_items > 0 && !items) || (n_comp > 0 && (!comp_amp || !comp_mean || !comp_var)) ||
        (mask_bytes > 0 && !masks) || (n_out > 0 && !out) || !pinned || !workspace)
        return TB_ERR_ARG;
    const MogHostLayout L = mog_host_layout(n_items, n_comp, mask_bytes, n_out);
    if (ws_bytes < L.total) return TB_ERR_SIZE;
    bool any_accum = false;
    if (!mog_items_fit(items, n_items, n_tiles, n_comp, mask_bytes, n_out, &any_accum))
        return TB_ERR_ARG;
    char* P = static_cast<char*>(pinned);
    char* D = static_cast<char*>(workspace);
    std::memcpy(P + L.items, items, (size_t)n_items * sizeof(tb_mog_item));
    std::memcpy(P + L.amp, comp_amp, (size_t)n_comp * 8);
    std::memcpy(P + L.mean, comp_mean, (size_t)n_comp * 16);
    std::memcpy(P + L.var, comp_var, (size_t)n_comp * 32);
    if (mask_bytes > 0) std::memcpy(P + L.mask, masks, (size_t)mask_bytes);
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemcpyAsync(D, P, (size_t)L.in_end, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return TB_ERR_LAUNCH;
    // ACCUM / ATOMIC targets start at zero, as does an output no tile writes
    const bool launches = n_items > 0 && n_tiles > 0;
    if ((any_accum || !launches) && n_out > 0 &&
        cudaMemsetAsync(D + L.out, 0, (size_t)n_out * 4, s) != cudaSuccess)
        return TB_ERR_LAUNCH;
    // (tb_mog_render zeroes the status word itself when it launches)
    if (!launches && cudaMemsetAsync(D + L.status, 0, sizeof(tb_status), s) != cudaSuccess)
        return TB_ERR_LAUNCH;
    const int rc = tb_mog_render(reinterpret_cast<const tb_mog_item*>(D + L.items), n_items,
                                 n_tiles, reinterpret_cast<const double*>(D + L.amp),
                                 reinterpret_cast<const double*>(D + L.mean),
                                 reinterpret_cast<const double*>(D + L.var),
                                 mask_bytes > 0 ? reinterpret_cast<const uint8_t*>(D + L.mask)
                                                : nullptr,
                                 reinterpret_cast<float*>(D + L.out),
                                 reinterpret_cast<int32_t*>(D + L.counter),
                                 reinterpret_cast<tb_status*>(D + L.status), stream);
    if (rc != TB_OK) return rc;
    if (cudaMemcpyAsync(P + L.out, D + L.out, (size_t)(L.total - L.out), cudaMemcpyDeviceToHost,
                        s) != cudaSuccess)
        return TB_ERR_LAUNCH;
    if (cudaStreamSynchronize(s) != cudaSuccess) return TB_ERR_LAUNCH;
    if (n_out > 0) std::memcpy(out, P + L.out, (size_t)n_out * 4);
    std::memcpy(status, P + L.status, sizeof(tb_status));
    return TB_OK;
}

// ---------------------------------------------------------------------------
// approx3's evaluated region (tractor/approx3.c:126-442) over values that
// tb_mog_render wrote for the whole box: the ring walk of the reference, one
// CTA per item, with the do / next mark arrays in shared memory.  A pixel of
// ring R lies on exactly one side (top and bottom rows own the corners; the
// left and right columns hold the rows strictly between), marks only ever
// land inside the next ring's sides, and a ring pixel is evaluated iff it is
// marked; so each unmarked pixel of a visited ring is zeroed in the same
// pass, and after the walk everything from the first empty ring outward.
// ---------------------------------------------------------------------------
namespace {

constexpr int kRingThreads = 256;

struct RingShared {
    uint8_t m[8][TB_RING_MAX];   // doT, doB, doL, doR, nextT, nextB, nextL, nextR
    int any, anyT, anyB, anyL, anyR;
    int cx, cy;
};

__device__ __forceinline__ void ring_set(uint8_t* a, int i, int n) {
    if (i >= 0 && i < n) a[i] = 1;
}

// Zeroes pixel o of the value plane and, when present, of the two
// derivative planes (dv: their start, both planes w x h).
__device__ __forceinline__ void ring_zero(float* v, float* dv, int64_t plane, int64_t o) {
    v[o] = 0.f;
    if (dv) {
        dv[o] = 0.f;
        dv[plane + o] = 0.f;
    }
}

__global__ void __launch_bounds__(kRingThreads)
approx3_ring_kernel(const tb_ring_item* __restrict__ items, int n_items, float* __restrict__ vals,
                    int32_t* __restrict__ extent, tb_status* st) {
    __shared__ RingShared sh;
    const int ii = blockIdx.x;
    if (ii >= n_items) return;
    const tb_ring_item it = items[ii];
    const int W = it.w, H = it.h;
    if (W <= 0 || H <= 0 || W > TB_RING_MAX || H > TB_RING_MAX) {
        if (threadIdx.x == 0) tb::report(st, TB_STATUS_BAD_ITEM, ii, W > H ? W : H);
        return;
    }
    float* v = vals + it.val_off;
    float* d = it.deriv_off >= 0 ? vals + it.deriv_off : nullptr;
    const int64_t plane = (int64_t)W * H;
    const double minval = it.minval;
    const int tid = threadIdx.x;
    uint8_t* dT = sh.m[0];
    uint8_t* dB = sh.m[1];
    uint8_t* dL = sh.m[2];
    uint8_t* dR = sh.m[3];
    uint8_t* nT = sh.m[4];
    uint8_t* nB = sh.m[5];
    uint8_t* nL = sh.m[6];
    uint8_t* nR = sh.m[7];
    const int wh = W > H ? W : H;
    for (int i = tid; i < wh; i += kRingThreads)
#pragma unroll
        for (int a = 4; a < 8; a++) sh.m[a][i] = 0;
    if (tid == 0) {
        int cx = it.xc, cy = it.yc;
        if (!it.start_inside) {
            // the largest value of the edge column, then of the edge row
            double best = 0.0;
            cx = it.dcx;
            cy = it.dcy;
            if (it.edge_col_off >= 0)
                for (int y = 0; y < H; y++) {
                    const double val = vals[it.edge_col_off + y];
                    if (val > best) { best = val; cx = it.edge_x; cy = y; }
                }
            if (it.edge_row_off >= 0)
                for (int x = 0; x < W; x++) {
                    const double val = vals[it.edge_row_off + x];
                    if (val > best) { best = val; cx = x; cy = it.edge_y; }
                }
        }
        sh.cx = cx;
        sh.cy = cy;
    }
    __syncthreads();
    const int cx = sh.cx, cy = sh.cy;
    if (tid == 0) {
        // the eight neighbours of the start pixel
        if (cy > 0) { ring_set(nB, cx - 1, W); ring_set(nB, cx, W); ring_set(nB, cx + 1, W); }
        if (cy < H - 1) { ring_set(nT, cx - 1, W); ring_set(nT, cx, W); ring_set(nT, cx + 1, W); }
        if (cx > 0) ring_set(nL, cy, H);
        if (cx < W - 1) ring_set(nR, cy, H);
    }
    int sx0 = cx, sx1 = cx, sy0 = cy, sy1 = cy;
    int R = 1;
    for (;; R++) {
        __syncthreads();
        // swap: the next arrays become the do arrays
        uint8_t* t;
        t = dT; dT = nT; nT = t;
        t = dB; dB = nB; nB = t;
        t = dL; dL = nL; nL = t;
        t = dR; dR = nR; nR = t;
        for (int i = tid; i < W; i += kRingThreads) { nT[i] = 0; nB[i] = 0; }
        for (int i = tid; i < H; i += kRingThreads) { nL[i] = 0; nR[i] = 0; }
        if (tid == 0) sh.anyT = sh.anyB = sh.anyL = sh.anyR = 0;
        __syncthreads();
        const bool pass_all = R <= it.minradius;
        // top (y = cy + R) and bottom (y = cy - R) rows, x in [cx - R, cx + R]
        for (int x = tid; x < W; x += kRingThreads) {
            if (x < cx - R || x > cx + R) continue;
            for (int side = 0; side < 2; side++) {
                const int y = side == 0 ? cy + R : cy - R;
                if (y < 0 || y >= H) continue;
                const int64_t o = (int64_t)y * W + x;
                const uint8_t* dm = side == 0 ? dT : dB;
                if (!dm[x]) { ring_zero(v, d, plane, o); continue; }
                if (side == 0) sh.anyT = 1; else sh.anyB = 1;
                if (!pass_all && (double)v[o] < minval) continue;
                const int inward = side == 0 ? -1 : 1;
                if (x == cx - R && x > 0) { ring_set(nL, y, H); ring_set(nL, y + inward, H); }
                if (x == cx + R && x < W - 1) { ring_set(nR, y, H); ring_set(nR, y + inward, H); }
                if (side == 0 ? y < H - 1 : y > 0) {
                    uint8_t* nm = side == 0 ? nT : nB;
                    ring_set(nm, x - 1, W); ring_set(nm, x, W); ring_set(nm, x + 1, W);
                }
            }
        }
        // left (x = cx - R) and right (x = cx + R) columns, y strictly inside the ring
        for (int y = tid; y < H; y += kRingThreads) {
            if (y <= cy - R || y >= cy + R) continue;
            for (int side = 0; side < 2; side++) {
                const int x = side == 0 ? cx - R : cx + R;
                if (x < 0 || x >= W) continue;
                const int64_t o = (int64_t)y * W + x;
                const uint8_t* dm = side == 0 ? dL : dR;
                if (!dm[y]) { ring_zero(v, d, plane, o); continue; }
                if (side == 0) sh.anyL = 1; else sh.anyR = 1;
                if (!pass_all && (double)v[o] < minval) continue;
                if (side == 0 ? x > 0 : x < W - 1) {
                    uint8_t* nm = side == 0 ? nL : nR;
                    ring_set(nm, y - 1, H); ring_set(nm, y, H); ring_set(nm, y + 1, H);
                }
            }
        }
        __syncthreads();
        if (sh.anyT) sy1 = cy + R;
        if (sh.anyB) sy0 = cy - R;
        if (sh.anyL) sx0 = cx - R;
        if (sh.anyR) sx1 = cx + R;
        if (!(sh.anyT | sh.anyB | sh.anyL | sh.anyR)) break;
    }
    // nothing was evaluated from ring R outward
    for (int64_t o = tid; o < plane; o += kRingThreads) {
        const int y = (int)(o / W), x = (int)(o % W);
        const int dist = max(abs(x - cx), abs(y - cy));
        if (dist >= R) ring_zero(v, d, plane, o);
    }
    if (tid == 0) {
        extent[4 * ii + 0] = sx0;
        extent[4 * ii + 1] = sx1 + 1;
        extent[4 * ii + 2] = sy0;
        extent[4 * ii + 3] = sy1 + 1;
    }
}

}  // namespace

extern "C" int tb_approx3_region(const tb_ring_item* items, int32_t n_items, float* vals,
                                 int32_t* extent, tb_status* status, void* stream) {
    if (n_items < 0) return TB_ERR_ARG;
    if (n_items == 0) return TB_OK;
    if (!items || !vals || !extent) return TB_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (status && cudaMemsetAsync(status, 0, sizeof(tb_status), s) != cudaSuccess)
        return TB_ERR_LAUNCH;
    approx3_ring_kernel<<<n_items, kRingThreads, 0, s>>>(items, n_items, vals, extent, status);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}
