// Blob segmentation on the device (sm_100a): connected components of a
// detection mask with scipy.ndimage.label's numbering, and their bounding
// boxes (scipy.ndimage.find_objects), for callers that cut an image into
// blobs and hand them to Tractor.setModelMasks / the batched fitter
// (callers of tractor/engine.py:341-361).
//
// Labelling is union-find over the pixel grid:
//   1. per 32 x 32 tile, in shared memory: every foreground pixel merges with
//      its foreground neighbours above and to the left (and the two upper
//      diagonals with 8-connectivity) inside the tile; a merge links the
//      larger root under the smaller with atomicMin, retrying when another
//      thread moved the root first, so every set's root is its smallest
//      index -- in row-major tile order, the same order as the raster order
//      -- and each pixel's global parent becomes its tile-local root;
//   2. pixels on a tile's top / left edge (and right edge, for the
//      8-connected upper-right diagonal) merge with their neighbours across
//      the edge in global memory by the same rule, so every set's root is
//      its smallest raster index;
//   3. every pixel's parent is replaced by its root;
//   4. roots are counted per block, the block counts scanned by one CTA, and
//      each root numbered 1 + (roots before it in raster order) -- the order
//      of each component's first pixel, which is scipy's numbering;
//   5. every foreground pixel takes its root's number.
// The result does not depend on the order the threads run in.  Reads of the
// parent array inside a merge bypass L1 (other SMs update it through L2).
#include "tb_common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kScanThreads = 1024;

__device__ __forceinline__ int find_root(const int32_t* parent, int x) {
    int p = __ldcg(parent + x);
    while (p != x) {
        x = p;
        p = __ldcg(parent + x);
    }
    return x;
}

// Joins the sets of a and b; returns false if the retry bound ran out (an
// impossible case kept as an error instead of an unbounded loop).
__device__ __forceinline__ bool unite(int32_t* parent, int a, int b, int bound) {
    for (int it = 0; it < bound; it++) {
        a = find_root(parent, a);
        b = find_root(parent, b);
        if (a == b) return true;
        if (a > b) {
            const int t = a;
            a = b;
            b = t;
        }
        const int old = atomicMin(parent + b, a);
        if (old == b) return true;   // b was still a root: linked under a
        b = old;                     // b had been linked meanwhile: retry from there
    }
    return false;
}

constexpr int kTile = 32;   // tile side of the shared-memory pass

__device__ __forceinline__ int find_local(volatile int* lp, int x) {
    int p = lp[x];
    while (p != x) {
        x = p;
        p = lp[x];
    }
    return x;
}

__device__ __forceinline__ bool unite_local(int* lp, int a, int b, int bound) {
    for (int it = 0; it < bound; it++) {
        a = find_local(lp, a);
        b = find_local(lp, b);
        if (a == b) return true;
        if (a > b) {
            const int t = a;
            a = b;
            b = t;
        }
        const int old = atomicMin(lp + b, a);
        if (old == b) return true;
        b = old;
    }
    return false;
}

// One CTA per 32 x 32 tile (kThreads threads, 4 rows each): the tile's
// components in shared memory, then every pixel's global parent = the global
// index of its tile-local root (-1 for background).
__global__ void __launch_bounds__(kThreads)
ccl_local(const uint8_t* __restrict__ mask, int H, int W, int conn8, int tiles_x,
          int32_t* __restrict__ parent, int* err) {
    __shared__ int lp[kTile * kTile];
    const int tx = blockIdx.x % tiles_x, ty = blockIdx.x / tiles_x;
    const int lx = threadIdx.x % kTile, ly0 = threadIdx.x / kTile;
    constexpr int kRows = kTile * kTile / kThreads;
    const int gx = tx * kTile + lx;
#pragma unroll
    for (int k = 0; k < kRows; k++) {
        const int ly = ly0 + k * (kThreads / kTile), gy = ty * kTile + ly;
        const int l = ly * kTile + lx;
        lp[l] = (gx < W && gy < H && mask[(int64_t)gy * W + gx]) ? l : -1;
    }
    __syncthreads();
    bool ok = true;
#pragma unroll
    for (int k = 0; k < kRows; k++) {
        const int ly = ly0 + k * (kThreads / kTile);
        const int l = ly * kTile + lx;
        if (lp[l] < 0) continue;
        if (lx > 0 && lp[l - 1] >= 0) ok &= unite_local(lp, l, l - 1, 1 << 20);
        if (ly > 0) {
            const int u = l - kTile;
            if (lp[u] >= 0) ok &= unite_local(lp, l, u, 1 << 20);
            if (conn8) {
                if (lx > 0 && lp[u - 1] >= 0) ok &= unite_local(lp, l, u - 1, 1 << 20);
                if (lx + 1 < kTile && lp[u + 1] >= 0) ok &= unite_local(lp, l, u + 1, 1 << 20);
            }
        }
    }
    if (!ok) atomicExch(err, 1);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kRows; k++) {
        const int ly = ly0 + k * (kThreads / kTile), gy = ty * kTile + ly;
        if (gx >= W || gy >= H) continue;
        const int l = ly * kTile + lx;
        int32_t g = -1;
        if (lp[l] >= 0) {
            const int r = find_local(lp, l);
            g = (ty * kTile + r / kTile) * W + tx * kTile + r % kTile;
        }
        parent[(int64_t)gy * W + gx] = g;
    }
}

// Merges across tile edges in global memory (pairs inside a tile were
// merged by ccl_local).
__global__ void ccl_edges(const uint8_t* __restrict__ mask, int H, int W, int conn8,
                          int32_t* parent, int* err) {
    const int64_t n = (int64_t)H * W;
    const int bound = 1 << 26;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / W), x = (int)(i - (int64_t)y * W);
        const int lx = x % kTile, ly = y % kTile;
        const bool left = lx == 0, top = ly == 0, right = lx == kTile - 1;
        if (!(left || top || (conn8 && right))) continue;
        if (!mask[i]) continue;
        bool ok = true;
        if (left && x > 0 && mask[i - 1]) ok &= unite(parent, (int)i, (int)(i - 1), bound);
        if (y > 0) {
            const int64_t u = i - W;
            if (top && mask[u]) ok &= unite(parent, (int)i, (int)u, bound);
            if (conn8) {
                if ((left || top) && x > 0 && mask[u - 1])
                    ok &= unite(parent, (int)i, (int)(u - 1), bound);
                if ((right || top) && x + 1 < W && mask[u + 1])
                    ok &= unite(parent, (int)i, (int)(u + 1), bound);
            }
        }
        if (!ok) atomicExch(err, 1);
    }
}

__global__ void ccl_flatten(int64_t n, int32_t* parent) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (parent[i] >= 0) parent[i] = find_root(parent, (int)i);
    }
}

// Roots per block of kThreads consecutive pixels.
__global__ void ccl_count(int64_t n, const int32_t* __restrict__ parent,
                          int32_t* __restrict__ block_roots) {
    const int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
    const bool root = i < n && parent[i] == (int32_t)i;
    const int c = __syncthreads_count(root);
    if (threadIdx.x == 0) block_roots[blockIdx.x] = c;
}

// Exclusive scan of the block counts by one CTA; the total is the number of
// components.
__global__ void ccl_scan(int nb, int32_t* __restrict__ block_roots, int32_t* __restrict__ n_labels) {
    __shared__ int32_t part[kScanThreads];
    const int tid = threadIdx.x;
    const int per = (nb + kScanThreads - 1) / kScanThreads;
    const int b0 = min(tid * per, nb), b1 = min(b0 + per, nb);
    int32_t s = 0;
    for (int b = b0; b < b1; b++) s += block_roots[b];
    part[tid] = s;
    __syncthreads();
    for (int o = 1; o < kScanThreads; o <<= 1) {
        const int32_t v = tid >= o ? part[tid - o] : 0;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    int32_t run = part[tid] - s;   // exclusive prefix of this thread's range
    for (int b = b0; b < b1; b++) {
        const int32_t c = block_roots[b];
        block_roots[b] = run;
        run += c;
    }
    if (tid == kScanThreads - 1) *n_labels = part[tid];
}

// Numbers every root: 1 + roots before it (block offset + rank in block).
__global__ void ccl_number_roots(int64_t n, const int32_t* __restrict__ parent,
                                 const int32_t* __restrict__ block_off, int32_t* __restrict__ labels) {
    __shared__ int32_t warp_cnt[kThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t i = blockIdx.x * (int64_t)kThreads + tid;
    const bool root = i < n && parent[i] == (int32_t)i;
    const unsigned bal = __ballot_sync(0xffffffffu, root);
    if (lane == 0) warp_cnt[warp] = __popc(bal);
    __syncthreads();
    int before = 0;
    for (int w = 0; w < warp; w++) before += warp_cnt[w];
    if (root) labels[i] = 1 + block_off[blockIdx.x] + before + __popc(bal & ((1u << lane) - 1u));
}

__global__ void ccl_relabel(int64_t n, const int32_t* __restrict__ parent, int32_t* labels) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t p = parent[i];
        labels[i] = p < 0 ? 0 : labels[p];   // a root keeps its own number
    }
}

__global__ void boxes_init(int n_labels, int32_t* boxes, int W, int H) {
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < n_labels; l += gridDim.x * blockDim.x) {
        boxes[4 * l + 0] = H;   // y0
        boxes[4 * l + 1] = W;   // x0
        boxes[4 * l + 2] = 0;   // y1 (exclusive)
        boxes[4 * l + 3] = 0;   // x1 (exclusive)
    }
}

__global__ void boxes_fill(const int32_t* __restrict__ labels, int H, int W, int n_labels,
                           int32_t* boxes) {
    const int64_t n = (int64_t)H * W;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int l = labels[i];
        if (l <= 0 || l > n_labels) continue;
        const int y = (int)(i / W), x = (int)(i - (int64_t)y * W);
        int32_t* b = boxes + 4 * (l - 1);
        atomicMin(b + 0, y);
        atomicMin(b + 1, x);
        atomicMax(b + 2, y + 1);
        atomicMax(b + 3, x + 1);
    }
}

int grid_for(int64_t n) {
    const int64_t want = (n + kThreads - 1) / kThreads;
    const int64_t cap = (int64_t)tb::num_sms() * 16;
    return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

}  // namespace

extern "C" int64_t tb_label_workspace_bytes(int32_t H, int32_t W) {
    if (H < 1 || W < 1 || (int64_t)H * W > ((int64_t)1 << 30)) return -1;
    const int64_t n = (int64_t)H * W;
    const int64_t nb = (n + kThreads - 1) / kThreads;
    return n * 4 + nb * 4 + 16;
}

extern "C" int tb_label_components(const uint8_t* mask, int32_t H, int32_t W, int32_t conn8,
                                   int32_t* labels, int32_t* n_labels, void* workspace,
                                   int32_t* error, void* stream) {
    if (H < 1 || W < 1 || (int64_t)H * W > ((int64_t)1 << 30) || (conn8 != 0 && conn8 != 1))
        return TB_ERR_ARG;
    if (!mask || !labels || !n_labels || !workspace || !error) return TB_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t n = (int64_t)H * W;
    const int64_t nb64 = (n + kThreads - 1) / kThreads;
    if (nb64 > INT32_MAX) return TB_ERR_ARG;
    const int nb = (int)nb64;
    int32_t* parent = static_cast<int32_t*>(workspace);
    int32_t* block_roots = parent + n;
    if (cudaMemsetAsync(error, 0, sizeof(int32_t), s) != cudaSuccess) return TB_ERR_LAUNCH;
    const int g = grid_for(n);
    const int tiles_x = (W + kTile - 1) / kTile, tiles_y = (H + kTile - 1) / kTile;
    const int64_t ntiles = (int64_t)tiles_x * tiles_y;
    if (ntiles > INT32_MAX) return TB_ERR_ARG;
    ccl_local<<<(int)ntiles, kThreads, 0, s>>>(mask, H, W, conn8, tiles_x, parent, error);
    ccl_edges<<<g, kThreads, 0, s>>>(mask, H, W, conn8, parent, error);
    ccl_flatten<<<g, kThreads, 0, s>>>(n, parent);
    ccl_count<<<nb, kThreads, 0, s>>>(n, parent, block_roots);
    ccl_scan<<<1, kScanThreads, 0, s>>>(nb, block_roots, n_labels);
    ccl_number_roots<<<nb, kThreads, 0, s>>>(n, parent, block_roots, labels);
    ccl_relabel<<<g, kThreads, 0, s>>>(n, parent, labels);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}

extern "C" int tb_component_boxes(const int32_t* labels, int32_t H, int32_t W, int32_t n_labels,
                                  int32_t* boxes, void* stream) {
    if (H < 1 || W < 1 || n_labels < 0 || (int64_t)H * W > ((int64_t)1 << 30)) return TB_ERR_ARG;
    if (n_labels == 0) return TB_OK;
    if (!labels || !boxes) return TB_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    boxes_init<<<(n_labels + kThreads - 1) / kThreads, kThreads, 0, s>>>(n_labels, boxes, W, H);
    boxes_fill<<<grid_for((int64_t)H * W), kThreads, 0, s>>>(labels, H, W, n_labels, boxes);
    return cudaGetLastError() == cudaSuccess ? TB_OK : TB_ERR_LAUNCH;
}
