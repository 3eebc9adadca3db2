// Scene rendering (sm_100a): many sources into whole images, the batched
// Tractor.getModelImage (tractor/engine.py:424-445) for mixture-of-Gaussians
// PSFs.
//
// 1. tb_scene_prep: one warp per (source, image) record builds the source's
//    PSF-convolved mixture (galaxy.py:307-326 run_mog; point sources
//    psf.py:458-528) and its pixel rectangle (the ModelMask clipped to the
//    image, as Patch.addTo clips, patch.py:341-354).
// 2. Binning: every item is listed in each image tile (32 x tile_h) that its
//    rectangle touches -- a count pass, an exclusive scan, a fill pass.
// 3. tb_scene_render: a persistent kernel takes image tiles from a global
//    counter.  For a tile it sorts the listed items by index (catalog order),
//    stages their components -- culled against the part of the tile inside
//    each item's rectangle -- in shared memory, evaluates them with one SFU
//    ex2 per pixel and component, sums each source's components into a
//    per-source partial (the reference's patch), adds the partial inside the
//    rectangle to the tile accumulator, and writes every tile pixel once.
//    No float atomics; the result does not depend on scheduling.
#include "profile_eval.cuh"

namespace {

constexpr int kPrepThreads = 128;   // 4 records (warps) per block
constexpr int kMaxGal = 32;         // galaxy components of one source (one per lane)
constexpr int kThreads = 256;       // render CTA
constexpr int kSlots = kThreads;    // components staged per pass
constexpr int kCap = 1024;          // items of one tile handled per chunk

// ---------------------------------------------------------------------------
// 1. prep
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kPrepThreads)
scene_prep_kernel(const tb_scene_src* __restrict__ srcs, int n,
                  const tb_scene_image* __restrict__ images, int n_images,
                  const double* __restrict__ pamp, const double* __restrict__ pmean,
                  const double* __restrict__ pvar, tb_profile_tables Tg,
                  tb_scene_item* __restrict__ items, double* __restrict__ camp,
                  double* __restrict__ cmean, double* __restrict__ cvar, int stride) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const tb_profile_tables T = tb::stage_tables(Tg, smem_raw);
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * (kPrepThreads / 32) + (threadIdx.x >> 5);
    if (i >= n) return;   // whole warps leave together
    const tb_scene_src s = srcs[i];
    int flag = 0;
    const bool img_ok = s.image >= 0 && s.image < n_images;
    tb_scene_image im;
    if (img_ok) im = images[s.image];
    else {
        flag = 2;
        im = tb_scene_image{};
        im.cd_inv[0] = im.cd_inv[3] = 1.0;
    }

    // rectangle = ModelMask clipped to the image
    const int x0 = max(s.mx0, 0), y0 = max(s.my0, 0);
    const int x1 = min(s.mx0 + s.mw, im.W), y1 = min(s.my0 + s.mh, im.H);
    if (flag == 0 && (x1 <= x0 || y1 <= y0 || s.counts == 0.0)) flag = 1;
    const int Kp = im.psf_K;
    if (flag == 0 && (Kp <= 0 || Kp > 32)) flag = 2;

    // galaxy components: lane l holds component `slot` of the whole source
    // (composite: deV block, then exp block; galaxy.py:847-876)
    double a = 0.0, V00 = 0.0, V01 = 0.0, V11 = 0.0;
    int Kg = 0, slot = lane;
    const bool point = s.profile == TB_PROFILE_POINT;
    if (point) {
        Kg = 1;
        a = lane == 0 ? 1.0 : 0.0;
    } else if (s.profile == TB_PROFILE_COMPOSITE) {
        const double f = fmin(1.0, fmax(0.0, s.fdev));
        int Kd = 0, Ke = 0;
        double G[4], re, M00, M01, M11;
        if (f > 0.0) {
            double ad, vd;
            Kd = tb::warp_profile(T, TB_PROFILE_DEV, 0.0, lane, kMaxGal, ad, vd);
            tb::shape_basis(s.shape_type, s.sb0, s.sb1, s.sb2, G, re);
            tb::pixel_factor(im.cd_inv, G, M00, M01, M11);
            if (lane < Kd) {
                a = ad * f;
                V00 = vd * M00;
                V01 = vd * M01;
                V11 = vd * M11;
            }
        }
        if (f < 1.0 && Kd >= 0) {
            // exp component index of this lane (>= 32: none)
            const int el = lane >= Kd ? lane - Kd : 32 + lane;
            double ae, ve;
            Ke = tb::warp_profile(T, TB_PROFILE_EXP, 0.0, el, kMaxGal, ae, ve);
            tb::shape_basis(s.shape_type, s.sa0, s.sa1, s.sa2, G, re);
            tb::pixel_factor(im.cd_inv, G, M00, M01, M11);
            if (el < Ke) {
                a = ae * (1.0 - f);
                V00 = ve * M00;
                V01 = ve * M01;
                V11 = ve * M11;
            }
        }
        if (Kd < 0 || Ke < 0 || Kd + Ke > kMaxGal) flag = 2;
        else Kg = Kd + Ke;
    } else {
        double ab, vb;
        const int Kb = tb::warp_profile(T, s.profile, s.sersic_n, lane, kMaxGal, ab, vb);
        // Sersic components sorted by variance (sersic.py:338-341)
        const int rank = s.profile == TB_PROFILE_SERSIC ? tb::variance_rank(vb, Kb, lane) : lane;
        double G[4], re, M00, M01, M11;
        tb::shape_basis(s.shape_type, s.sa0, s.sa1, s.sa2, G, re);
        tb::pixel_factor(im.cd_inv, G, M00, M01, M11);
        if (Kb < 0) {
            flag = 2;
        } else {
            Kg = Kb;
            if (lane < Kb) {
                a = ab;
                V00 = vb * M00;
                V01 = vb * M01;
                V11 = vb * M11;
                slot = rank;
            }
        }
    }
    const int K = Kg * Kp;
    if (flag == 0 && K > stride) flag = 2;
    const int c0 = i * stride;
    if (flag == 0 && lane < Kg) {
        // MixtureOfGaussians.convolve (mixture_profiles.py:158-172): PSF
        // component p (outer) x galaxy component k (inner)
        const double mx = point ? 0.0 : s.px, my = point ? 0.0 : s.py;
        for (int p = 0; p < Kp; p++) {
            const int pc = im.psf_c0 + p;
            const int c = c0 + p * Kg + slot;
            camp[c] = a * pamp[pc];
            cmean[2 * c] = mx + pmean[2 * pc];
            cmean[2 * c + 1] = my + pmean[2 * pc + 1];
            cvar[4 * c] = V00 + pvar[4 * pc];
            cvar[4 * c + 1] = V01 + pvar[4 * pc + 1];
            cvar[4 * c + 2] = V01 + pvar[4 * pc + 2];
            cvar[4 * c + 3] = V11 + pvar[4 * pc + 3];
        }
    }
    if (lane == 0) {
        tb_scene_item it;
        it.x0 = x0;
        it.y0 = y0;
        it.w = flag == 0 ? x1 - x0 : 0;
        it.h = flag == 0 ? y1 - y0 : 0;
        it.c0 = c0;
        it.K = flag == 0 ? K : 0;
        it.image = s.image;
        it.flag = flag;
        it.fx = point ? s.px : 0.0;
        it.fy = point ? s.py : 0.0;
        it.scale = (float)s.counts;
        it.floor = -50.0f;   // c_gauss_2d_grid: Mahalanobis^2 >= 100 is skipped
        items[i] = it;
    }
}

// ---------------------------------------------------------------------------
// 2. binning
// ---------------------------------------------------------------------------

__device__ __forceinline__ bool item_tiles(const tb_scene_item& it, const tb_scene_image& im,
                                           int tile_h, int& tx0, int& tx1, int& ty0, int& ty1) {
    if (it.flag != 0 || it.w <= 0 || it.h <= 0 || it.K <= 0) return false;
    tx0 = it.x0 / TB_MOG_TILE;
    tx1 = (it.x0 + it.w - 1) / TB_MOG_TILE;
    ty0 = it.y0 / tile_h;
    ty1 = (it.y0 + it.h - 1) / tile_h;
    return true;
}

template <bool kFill>
__global__ void scene_bin_kernel(const tb_scene_item* __restrict__ items, int n_items,
                                 const tb_scene_image* __restrict__ images, int n_images,
                                 int64_t n_tiles, int tile_h, int32_t* __restrict__ counts,
                                 const int32_t* __restrict__ offsets, int32_t* __restrict__ list,
                                 int64_t max_pairs, tb_status* st) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_items) return;
    const tb_scene_item it = items[i];
    if (it.image < 0 || it.image >= n_images) {
        if (!kFill && it.flag == 0) tb::report(st, TB_STATUS_BAD_ITEM, i, -1);
        return;
    }
    const tb_scene_image im = images[it.image];
    int tx0, tx1, ty0, ty1;
    if (!item_tiles(it, im, tile_h, tx0, tx1, ty0, ty1)) return;
    const int tiles_x = (im.W + TB_MOG_TILE - 1) / TB_MOG_TILE;
    for (int ty = ty0; ty <= ty1; ty++) {
        for (int tx = tx0; tx <= tx1; tx++) {
            const int64_t t = im.tile0 + (int64_t)ty * tiles_x + tx;
            if (t < 0 || t >= n_tiles) {
                if (!kFill) tb::report(st, TB_STATUS_BAD_ITEM, i, -2);
                continue;
            }
            const int pos = atomicAdd(&counts[t], 1);
            if (kFill) {
                const int64_t at = (int64_t)offsets[t] + pos;
                if (at < max_pairs) list[at] = i;
                else tb::report(st, TB_STATUS_BAD_ITEM, i, -3);
            }
        }
    }
}

// Exclusive scan of counts[0..n) into offsets[0..n] in three passes:
// per-block scans (1024 values per block), a scan of the block totals, and
// the block offsets added back.
constexpr int kScanThreads = 1024;

__device__ __forceinline__ int block_exclusive_scan(int v, int* warp_tot, int& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        warp_tot[lane] = w;   // inclusive over warps
    }
    __syncthreads();
    total = warp_tot[(blockDim.x >> 5) - 1];
    const int before = warp > 0 ? warp_tot[warp - 1] : 0;
    __syncthreads();
    return before + x - v;
}

__global__ void __launch_bounds__(kScanThreads)
scan_blocks_kernel(const int32_t* __restrict__ counts, int64_t n, int32_t* __restrict__ offsets,
                   int32_t* __restrict__ bsum) {
    __shared__ int warp_tot[32];
    const int64_t i = (int64_t)blockIdx.x * kScanThreads + threadIdx.x;
    const int v = i < n ? counts[i] : 0;
    int total;
    const int ex = block_exclusive_scan(v, warp_tot, total);
    if (i < n) offsets[i] = ex;
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads)
scan_sums_kernel(int32_t* __restrict__ bsum, int nb, int32_t* __restrict__ offsets, int64_t n) {
    __shared__ int warp_tot[32];
    int carry = 0;
    for (int b0 = 0; b0 < nb; b0 += kScanThreads) {
        const int b = b0 + threadIdx.x;
        const int v = b < nb ? bsum[b] : 0;
        int total;
        const int ex = block_exclusive_scan(v, warp_tot, total);
        if (b < nb) bsum[b] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) offsets[n] = carry;
}

__global__ void __launch_bounds__(kScanThreads)
scan_add_kernel(int32_t* __restrict__ offsets, int64_t n, const int32_t* __restrict__ bsum) {
    const int64_t i = (int64_t)blockIdx.x * kScanThreads + threadIdx.x;
    if (i < n) offsets[i] += bsum[blockIdx.x];
}

// ---------------------------------------------------------------------------
// 3. tile renderer
// ---------------------------------------------------------------------------

struct SceneC {
    float mx, my;           // mean relative to the tile origin
    float qxx, qxy, qyy;    // exponent (log2 units) = qxx dx^2 + qxy dx dy + qyy dy^2
    float s;                // counts * amp / (2 pi sqrt(det))
    float fl;               // exponent floor, log2 units
    int32_t src;            // position of the source in the tile's sorted list
    uint32_t rect;          // source rectangle in tile coordinates: x0 | x1<<8 | y0<<16 | y1<<24
    int32_t pad;
};

template <int ROWS>
__global__ void __launch_bounds__(kThreads)
scene_render_kernel(const tb_scene_item* __restrict__ items, int n_items,
                    const tb_scene_image* __restrict__ images, int n_images, int64_t n_tiles,
                    int64_t max_pairs,
                    const double* __restrict__ amp, const double* __restrict__ mean,
                    const double* __restrict__ var, const int32_t* __restrict__ offsets,
                    const int32_t* __restrict__ list, float* __restrict__ out, int mode,
                    int32_t* counter, tb_status* st) {
    constexpr int TH = 8 * ROWS;   // tile height (8 warps x ROWS rows)
    __shared__ SceneC comps[kSlots];
    __shared__ int ids[kCap];
    __shared__ int raw[kCap];
    __shared__ int prefK[kCap + 1];
    __shared__ int64_t slot;
    __shared__ int img_idx;
    __shared__ int warp_count[kThreads / 32];
    __shared__ int warp_tot[32];

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const float xf = (float)lane;

    // More overlaps than the list holds: the fill dropped some, so no tile
    // list can be trusted (tb_scene_render reports it from the fill pass).
    if ((int64_t)offsets[n_tiles] > max_pairs) return;

    for (;;) {
        const int64_t u = tb::next_unit(counter, &slot);
        if (u >= n_tiles) break;
        if (tid == 0) {
            int lo = 0, hi = n_images - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (images[mid].tile0 <= u) lo = mid; else hi = mid - 1;
            }
            img_idx = lo;
        }
        __syncthreads();
        const tb_scene_image im = images[img_idx];
        const int tiles_x = (im.W + TB_MOG_TILE - 1) / TB_MOG_TILE;
        const int64_t t = u - im.tile0;
        const int ox = (int)(t % tiles_x) * TB_MOG_TILE;
        const int oy = (int)(t / tiles_x) * TH;
        const int tw = min(TB_MOG_TILE, im.W - ox);
        const int th = min(TH, im.H - oy);
        if (tw <= 0 || th <= 0) {   // a tile index beyond its image
            if (tid == 0) tb::report(st, TB_STATUS_BAD_ITEM, img_idx, (int)t);
            continue;
        }

        float acc[ROWS];
#pragma unroll
        for (int j = 0; j < ROWS; j++) acc[j] = 0.f;

        const int beg = offsets[u];
        const int n = offsets[u + 1] - beg;
        for (int cb = 0; cb < n; cb += kCap) {
            const int m = min(kCap, n - cb);
            for (int q = tid; q < m; q += kThreads) {
                const int v = list[beg + cb + q];
                // an index outside the item table is reported and becomes a
                // distinct negative placeholder with no components
                if (v < 0 || v >= n_items) tb::report(st, TB_STATUS_BAD_ITEM, v, -4);
                raw[q] = (v < 0 || v >= n_items) ? -1 - q : v;
            }
            __syncthreads();
            // rank sort (ids in one tile are distinct): catalog order
            for (int q = tid; q < m; q += kThreads) {
                const int v = raw[q];
                int r = 0;
                for (int z = 0; z < m; z++) r += raw[z] < v;
                ids[r] = v;
            }
            __syncthreads();
            // exclusive prefix of component counts over the sorted items,
            // 4 consecutive items per thread
            {
                int k4[4], sum = 0;
#pragma unroll
                for (int z = 0; z < 4; z++) {
                    const int q = 4 * tid + z;
                    k4[z] = (q < m && ids[q] >= 0) ? items[ids[q]].K : 0;
                    sum += k4[z];
                }
                int total;
                int ex = block_exclusive_scan(sum, warp_tot, total);
#pragma unroll
                for (int z = 0; z < 4; z++) {
                    const int q = 4 * tid + z;
                    if (q < m) prefK[q] = ex;
                    ex += k4[z];
                }
                if (tid == 0) prefK[m] = total;
            }
            __syncthreads();
            const int total = prefK[m];

            float part[ROWS];
#pragma unroll
            for (int j = 0; j < ROWS; j++) part[j] = 0.f;
            int cur = -1;
            bool colin = false;
            unsigned rowmask = 0u;

            for (int base = 0; base < total; base += kSlots) {
                const int g = base + tid;
                bool keep = false;
                SceneC c;
                if (g < total) {
                    // the item holding global component g: largest q with prefK[q] <= g
                    int lo = 0, hi = m - 1;
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (prefK[mid] <= g) lo = mid; else hi = mid - 1;
                    }
                    const int ii = ids[lo];
                    const tb_scene_item& it = items[ii];
                    const int k = g - prefK[lo];
                    const int ci = it.c0 + k;
                    const int rx0 = max(it.x0 - ox, 0), rx1 = min(it.x0 + it.w - ox, tw);
                    const int ry0 = max(it.y0 - oy, 0), ry1 = min(it.y0 + it.h - oy, th);
                    const double a = amp[ci];
                    const double v0 = var[4 * ci], v3 = var[4 * ci + 3];
                    const double vxy = 0.5 * (var[4 * ci + 1] + var[4 * ci + 2]);
                    const double det = v0 * v3 - vxy * vxy;
                    const double sc = (double)it.scale * a / (2.0 * TB_PI * sqrt(det));
                    const double f = -0.5 / det * TB_LOG2E;
                    const double fl = (double)it.floor;
                    const double mx = (mean[2 * ci] + it.fx) - (double)ox;
                    const double my = (mean[2 * ci + 1] + it.fy) - (double)oy;
                    c.qxx = (float)(v3 * f);
                    c.qxy = (float)(-2.0 * vxy * f);
                    c.qyy = (float)(v0 * f);
                    c.s = (float)sc;
                    c.fl = (float)(fl * TB_LOG2E);
                    c.mx = (float)mx;
                    c.my = (float)my;
                    c.src = lo;
                    c.rect = (uint32_t)rx0 | ((uint32_t)rx1 << 8) | ((uint32_t)ry0 << 16) |
                             ((uint32_t)ry1 << 24);
                    c.pad = 0;
                    const bool finite = det > 0.0 && isfinite(sc) && isfinite(f) &&
                                        isfinite(mx) && isfinite(my);
                    if (!finite) {
                        tb::report(st, TB_STATUS_NONFINITE, ii, k);
                    } else if (a != 0.0 && rx0 < rx1 && ry0 < ry1) {
                        // evaluated region (exponent >= floor) against the
                        // part of the tile inside the rectangle
                        const double r2 = -2.0 * fl;
                        const double ex = sqrt(r2 * v0), ey = sqrt(r2 * v3);
                        keep = (mx + ex >= rx0) && (mx - ex <= rx1 - 1) && (my + ey >= ry0) &&
                               (my - ey <= ry1 - 1);
                    }
                }
                // order-preserving compaction of the kept components
                const unsigned ballot = __ballot_sync(0xffffffffu, keep);
                if (lane == 0) warp_count[warp] = __popc(ballot);
                __syncthreads();
                int wbase = 0, kept = 0;
#pragma unroll
                for (int w = 0; w < kThreads / 32; w++) {
                    wbase += (w < warp) ? warp_count[w] : 0;
                    kept += warp_count[w];
                }
                if (keep) comps[wbase + __popc(ballot & ((1u << lane) - 1u))] = c;
                __syncthreads();

                for (int q = 0; q < kept; q++) {
                    const SceneC g2 = comps[q];
                    if (g2.src != cur) {
                        // previous source done: add its patch inside its rectangle
#pragma unroll
                        for (int j = 0; j < ROWS; j++) {
                            acc[j] += colin ? part[j] : 0.f;
                            part[j] = 0.f;
                        }
                        cur = g2.src;
                        const int rx0 = g2.rect & 0xff, rx1 = (g2.rect >> 8) & 0xff;
                        const int ry0 = (g2.rect >> 16) & 0xff, ry1 = g2.rect >> 24;
                        colin = lane >= rx0 && lane < rx1;
                        rowmask = 0u;
#pragma unroll
                        for (int j = 0; j < ROWS; j++) {
                            const int y = warp + 8 * j;
                            rowmask |= (y >= ry0 && y < ry1) ? (1u << j) : 0u;
                        }
                    }
                    const float dx = xf - g2.mx;
                    const float A = g2.qxx * dx * dx;
                    const float B = g2.qxy * dx;
#pragma unroll
                    for (int j = 0; j < ROWS; j++) {
                        if (rowmask & (1u << j)) {
                            const float dy = (float)(warp + 8 * j) - g2.my;
                            const float e = fmaf(dy, fmaf(g2.qyy, dy, B), A);
                            const float sv = (e >= g2.fl) ? g2.s : 0.f;
                            part[j] = fmaf(sv, tb::ex2(e), part[j]);
                        }
                    }
                }
                __syncthreads();   // comps is overwritten by the next pass
            }
#pragma unroll
            for (int j = 0; j < ROWS; j++) acc[j] += colin ? part[j] : 0.f;
        }

        const int64_t ldo = im.ldo > 0 ? im.ldo : im.W;
#pragma unroll
        for (int j = 0; j < ROWS; j++) {
            const int y = warp + 8 * j;
            if (lane < tw && y < th) {
                float* p = out + im.out_off + (int64_t)(oy + y) * ldo + (ox + lane);
                if (mode == TB_MOG_ACCUM) *p += acc[j];
                else *p = acc[j];
            }
        }
    }
}

template <int ROWS>
int launch_render(const tb_scene_item* items, int n_items, const tb_scene_image* images,
                  int n_images, int64_t n_tiles, int64_t max_pairs, const double* a, const double* m, const double* v,
                  const int32_t* offsets, const int32_t* list, float* out, int mode,
                  int32_t* counter, tb_status* st, cudaStream_t s) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, scene_render_kernel<ROWS>, kThreads,
                                                      0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const int64_t want = (int64_t)tb::num_sms() * per_sm;
    const int grid = (int)(n_tiles < want ? n_tiles : want);
    scene_render_kernel<ROWS><<<grid, kThreads, 0, s>>>(items, n_items, images, n_images, n_tiles,
                                                        max_pairs, a, m, v, offsets, list, out,
                                                        mode, counter, st);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

// Workspace layout (bytes, each section 256-aligned): counts[n_tiles] int32,
// offsets[n_tiles + 1] int32, block sums int32, list[max_pairs] int32, the
// work counter.
struct Workspace {
    int32_t* counts;
    int32_t* offsets;
    int32_t* bsum;
    int32_t* list;
    int32_t* counter;
    int64_t bytes;
};

inline int64_t align256(int64_t x) { return (x + 255) / 256 * 256; }

Workspace carve(void* base, int64_t n_tiles, int64_t max_pairs) {
    Workspace w;
    const int64_t nb = (n_tiles + kScanThreads - 1) / kScanThreads;
    int64_t o = 0;
    char* b = static_cast<char*>(base);
    w.counts = reinterpret_cast<int32_t*>(b + o);
    o += align256(4 * n_tiles);
    w.offsets = reinterpret_cast<int32_t*>(b + o);
    o += align256(4 * (n_tiles + 1));
    w.bsum = reinterpret_cast<int32_t*>(b + o);
    o += align256(4 * (nb > 0 ? nb : 1));
    w.list = reinterpret_cast<int32_t*>(b + o);
    o += align256(4 * (max_pairs > 0 ? max_pairs : 1));
    w.counter = reinterpret_cast<int32_t*>(b + o);
    o += 256;
    w.bytes = o;
    return w;
}

}  // namespace

extern "C" int tb_scene_prep(const tb_scene_src* srcs, int32_t n, const tb_scene_image* images,
                             int32_t n_images, const double* psf_amp, const double* psf_mean,
                             const double* psf_var, const tb_profile_tables* tables,
                             tb_scene_item* items, double* comp_amp, double* comp_mean,
                             double* comp_var, int32_t comp_stride, void* stream) {
    if (n < 0 || n_images < 0) return TB_ERR_ARG;
    if (n == 0) return TB_OK;
    if (!srcs || !images || !psf_amp || !psf_mean || !psf_var || !tables || !items ||
        !comp_amp || !comp_mean || !comp_var)
        return TB_ERR_ARG;
    if (comp_stride < 1 || comp_stride > TB_MOG_MAX_K) return TB_ERR_SIZE;
    const int smem = tb::tables_smem_bytes(*tables);
    if (smem > TB_PROFILE_SMEM_MAX) return TB_ERR_SIZE;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(scene_prep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem) != cudaSuccess)
        return TB_ERR_LAUNCH;
    const int per_block = kPrepThreads / 32;
    scene_prep_kernel<<<(n + per_block - 1) / per_block, kPrepThreads, smem,
                        (cudaStream_t)stream>>>(srcs, n, images, n_images, psf_amp, psf_mean,
                                                psf_var, *tables, items, comp_amp, comp_mean,
                                                comp_var, comp_stride);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

extern "C" int tb_scene_workspace(int64_t n_tiles, int64_t max_pairs, int64_t* bytes) {
    if (n_tiles < 0 || max_pairs < 0 || !bytes) return TB_ERR_ARG;
    if (n_tiles > 0x7ffffffeLL || max_pairs > 0x7fffffffLL) return TB_ERR_SIZE;
    *bytes = carve(nullptr, n_tiles, max_pairs).bytes;
    return TB_OK;
}

extern "C" int tb_scene_render(const tb_scene_item* items, int32_t n_items,
                               const tb_scene_image* images, int32_t n_images, int64_t n_tiles,
                               int32_t tile_h, const double* comp_amp, const double* comp_mean,
                               const double* comp_var, float* out, int32_t mode, void* workspace,
                               int64_t workspace_bytes, int64_t max_pairs, tb_status* status,
                               void* stream) {
    if (n_items < 0 || n_images < 0 || n_tiles < 0 || max_pairs < 0) return TB_ERR_ARG;
    if (mode != TB_MOG_STORE && mode != TB_MOG_ACCUM) return TB_ERR_ARG;
    if (tile_h != 16 && tile_h != 32 && tile_h != 64) return TB_ERR_SIZE;
    if (n_tiles > 0x7ffffffeLL || max_pairs > 0x7fffffffLL) return TB_ERR_SIZE;
    if (n_tiles == 0 || n_images == 0) return TB_OK;
    if (!images || !out || !workspace || (n_items > 0 && (!items || !comp_amp || !comp_mean ||
                                                           !comp_var)))
        return TB_ERR_ARG;
    const Workspace w = carve(workspace, n_tiles, max_pairs);
    if (workspace_bytes < w.bytes) return TB_ERR_SIZE;
    cudaStream_t s = (cudaStream_t)stream;
    if (status && cudaMemsetAsync(status, 0, sizeof(tb_status), s) != cudaSuccess)
        return TB_ERR_LAUNCH;
    if (cudaMemsetAsync(w.counts, 0, 4 * n_tiles, s) != cudaSuccess) return TB_ERR_LAUNCH;
    if (cudaMemsetAsync(w.counter, 0, 4, s) != cudaSuccess) return TB_ERR_LAUNCH;
    const int nb_items = (n_items + 255) / 256;
    if (n_items > 0) {
        scene_bin_kernel<false><<<nb_items, 256, 0, s>>>(items, n_items, images, n_images, n_tiles,
                                                         tile_h, w.counts, nullptr, nullptr,
                                                         max_pairs, status);
    }
    const int nb = (int)((n_tiles + kScanThreads - 1) / kScanThreads);
    scan_blocks_kernel<<<nb, kScanThreads, 0, s>>>(w.counts, n_tiles, w.offsets, w.bsum);
    scan_sums_kernel<<<1, kScanThreads, 0, s>>>(w.bsum, nb, w.offsets, n_tiles);
    scan_add_kernel<<<nb, kScanThreads, 0, s>>>(w.offsets, n_tiles, w.bsum);
    if (n_items > 0) {
        if (cudaMemsetAsync(w.counts, 0, 4 * n_tiles, s) != cudaSuccess) return TB_ERR_LAUNCH;
        scene_bin_kernel<true><<<nb_items, 256, 0, s>>>(items, n_items, images, n_images, n_tiles,
                                                        tile_h, w.counts, w.offsets, w.list,
                                                        max_pairs, status);
    }
    if (cudaGetLastError() != cudaSuccess) return TB_ERR_LAUNCH;
    switch (tile_h) {
        case 16:
            return launch_render<2>(items, n_items, images, n_images, n_tiles, max_pairs, comp_amp, comp_mean, comp_var,
                                    w.offsets, w.list, out, mode, w.counter, status, s);
        case 32:
            return launch_render<4>(items, n_items, images, n_images, n_tiles, max_pairs, comp_amp, comp_mean, comp_var,
                                    w.offsets, w.list, out, mode, w.counter, status, s);
        default:
            return launch_render<8>(items, n_items, images, n_images, n_tiles, max_pairs, comp_amp, comp_mean, comp_var,
                                    w.offsets, w.list, out, mode, w.counter, status, s);
    }
}
