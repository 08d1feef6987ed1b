// k_sort.cu -- bounding box, Morton codes, LSD radix sort and the sorted gather.
//
// Stage 1-2 of the step (reference: BarnesHutCuda.cu:648-711).  The box is
// reduced in one launch (last-block-done) and squared on the device, so the
// step never returns to the host; Morton codes are bit-exact with CU:54-69;
// the sort is a project-written stable LSD radix sort over all 64 key bits,
// so its order equals cub::DeviceRadixSort::SortPairs at CU:692 (any stable
// sort of (code, current index) gives the same permutation).
#include <cuda_runtime.h>
#include <stdint.h>

#include "nb_internal.cuh"

namespace nb {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kBoxThreads = 512;

__device__ __forceinline__ double warp_min(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(kFull, v, o));
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

// Chooses this step's radix passes (the top bytes of the key the sort orders
// by) and resets the counters of the tie pass; the histogram of the last tree
// is consumed.  Without `adaptive` (or with a forced count) no histogram is
// used.
__device__ __forceinline__ void start_sort(DeviceScalars* s, int64_t n, int adaptive) {
    int passes = adaptive ? choose_sort_passes(s->lcp_hist, n) : 8;
    if (s->sort_passes_forced > 0) passes = min(s->sort_passes_forced, 8);
    s->sort_passes = passes;
    for (int d = 0; d <= 32; ++d) s->lcp_hist[d] = 0;
    s->tie_count[0] = 0;
    s->tie_count[1] = 0;
}

// Exact FP64 min/max of all positions, reduced per block, then folded and
// squared by the last block to finish (CU:78-114 + the host squaring at
// CU:665-677, done here on the device in the same FP64 operations).  Min and
// max are exact in any order, so the reduction tree is free: each thread
// keeps four loads in flight, and the last block folds the partials with all
// its threads.
__device__ __forceinline__ void box_fold(double& xmin, double& xmax, double& ymin, double& ymax,
                                         double (*red)[kBoxThreads / 32]) {
    xmin = warp_min(xmin);
    xmax = warp_max(xmax);
    ymin = warp_min(ymin);
    ymax = warp_max(ymax);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        red[0][warp] = xmin;
        red[1][warp] = xmax;
        red[2][warp] = ymin;
        red[3][warp] = ymax;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kBoxThreads / 32; ++w) {
            xmin = fmin(xmin, red[0][w]);
            xmax = fmax(xmax, red[1][w]);
            ymin = fmin(ymin, red[2][w]);
            ymax = fmax(ymax, red[3][w]);
        }
    }
}

__global__ void __launch_bounds__(kBoxThreads)
bbox_kernel(const double2* __restrict__ pos, int64_t n, double* __restrict__ partials,
            DeviceScalars* __restrict__ s, int adaptive) {
    double xmin = INFINITY, xmax = -INFINITY, ymin = INFINITY, ymax = -INFINITY;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (; i + 3 * stride < n; i += 4 * stride) {
        double2 p[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) p[u] = __ldg(pos + i + u * stride);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            xmin = fmin(xmin, p[u].x);
            xmax = fmax(xmax, p[u].x);
            ymin = fmin(ymin, p[u].y);
            ymax = fmax(ymax, p[u].y);
        }
    }
    for (; i < n; i += stride) {
        const double2 p = __ldg(pos + i);
        xmin = fmin(xmin, p.x);
        xmax = fmax(xmax, p.x);
        ymin = fmin(ymin, p.y);
        ymax = fmax(ymax, p.y);
    }
    __shared__ double red[4][kBoxThreads / 32];
    __shared__ bool last_block;
    box_fold(xmin, xmax, ymin, ymax, red);
    if (threadIdx.x == 0) {
        double* out = partials + 4 * blockIdx.x;
        out[0] = xmin;
        out[1] = xmax;
        out[2] = ymin;
        out[3] = ymax;
        __threadfence();
        last_block = atomicAdd(&s->bbox_ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last_block) return;
    __threadfence();
    // CU:649-654 seeds with +-DBL_MAX; folding from there is identical.
    double bx0 = 1.7976931348623157e308, bx1 = -1.7976931348623157e308;
    double by0 = 1.7976931348623157e308, by1 = -1.7976931348623157e308;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        const double* in = partials + 4 * b;
        bx0 = fmin(bx0, __ldcg(in + 0));
        bx1 = fmax(bx1, __ldcg(in + 1));
        by0 = fmin(by0, __ldcg(in + 2));
        by1 = fmax(by1, __ldcg(in + 3));
    }
    __syncthreads();  // red[] is reused
    box_fold(bx0, bx1, by0, by1, red);
    if (threadIdx.x == 0) {
        const double x_range = bx1 - bx0;
        const double y_range = by1 - by0;
        if (x_range > y_range) {
            const double mid = (by0 + by1) * 0.5;
            by0 = mid - x_range * 0.5;
            by1 = mid + x_range * 0.5;
        } else {
            const double mid = (bx0 + bx1) * 0.5;
            bx0 = mid - y_range * 0.5;
            bx1 = mid + y_range * 0.5;
        }
        s->box[0] = bx0;
        s->box[1] = bx1;
        s->box[2] = by0;
        s->box[3] = by1;
        s->center[0] = 0.5 * (bx0 + bx1);
        s->center[1] = 0.5 * (by0 + by1);
        // the Morton kernel's scale factors (CU:122-123), divided once here
        s->inv_wh[0] = 1.0 / (bx1 - bx0);
        s->inv_wh[1] = 1.0 / (by1 - by0);
        // CU:717 root width_sq, then CU:216 child_wsq = parent * 0.25 per level.
        const double w = bx1 - bx0;
        double wsq = w * w;
        for (int l = 0; l <= kMaxLevel; ++l) {
            s->wsq[l] = wsq;
            wsq *= 0.25;
        }
        s->bbox_ticket = 0;
        start_sort(s, n, adaptive);
    }
}

__device__ __forceinline__ uint64_t expand_bits_2d(uint32_t v) {
    uint64_t x = v;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x;
}

// CU:117-132: code from (p - min) * (1 / width), quantised to 32 bits per axis
// with round-down; x bits land on odd positions.  val = current slot.  The
// codes go to the buffer the first radix pass reads: pass k reads buffer
// k & 1, and the first of the step's sort_passes passes is 8 - sort_passes,
// so the last one always writes buffer 0.
__global__ void morton_kernel(const double2* __restrict__ pos, int64_t n,
                              const DeviceScalars* __restrict__ s, uint64_t* __restrict__ key0,
                              uint64_t* __restrict__ key1, uint32_t* __restrict__ val0,
                              uint32_t* __restrict__ val1) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool odd = s->sort_passes & 1;
    uint64_t* __restrict__ key = odd ? key1 : key0;
    uint32_t* __restrict__ val = odd ? val1 : val0;
    const double x0 = s->box[0], y0 = s->box[2];
    const double inv_w = s->inv_wh[0], inv_h = s->inv_wh[1];
    const double2 p = __ldg(pos + i);
    const double nx = (p.x - x0) * inv_w;
    const double ny = (p.y - y0) * inv_h;
    const uint32_t ix = __double2uint_rd(fmin(fmax(nx * 4294967296.0, 0.0), 4294967295.0));
    const uint32_t iy = __double2uint_rd(fmin(fmax(ny * 4294967296.0, 0.0), 4294967295.0));
    key[i] = (expand_bits_2d(ix) << 1) | expand_bits_2d(iy);
    val[i] = (uint32_t)i;
}

// ---------------------------------------------------------------------------
// Batched universes: per-universe boxes and 54-bit Morton codes under the
// universe id.  Doubles are reduced through an order-preserving integer image
// so plain 64-bit atomicMin/atomicMax give the exact FP64 min/max.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long ordered_bits(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double from_ordered(unsigned long long o) {
    const unsigned long long b = (o >> 63) ? (o & 0x7fffffffffffffffull) : ~o;
    return __longlong_as_double((long long)b);
}

__global__ void __launch_bounds__(256)
bbox_batch_kernel(const double2* __restrict__ pos, int64_t n, Batch b) {
    const int lane = threadIdx.x & 31;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i - lane < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const bool valid = i < n;
        const int u = valid ? b.uid[i] : -1;
        const double2 p = valid ? pos[i] : make_double2(0.0, 0.0);
        unsigned long long e[4] = {ordered_bits(p.x), ~ordered_bits(p.x), ordered_bits(p.y),
                                   ~ordered_bits(p.y)};  // min-encoded: max via the complement
        const int u0 = __shfl_sync(kFull, u, 0);
        const bool uniform = __all_sync(kFull, valid && u == u0);
        if (uniform) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const unsigned long long t = __shfl_xor_sync(kFull, e[k], o);
                    e[k] = t < e[k] ? t : e[k];
                }
            if (lane == 0)
#pragma unroll
                for (int k = 0; k < 4; ++k) atomicMin(b.boxbits + 4 * u0 + k, e[k]);
        } else if (valid) {
#pragma unroll
            for (int k = 0; k < 4; ++k) atomicMin(b.boxbits + 4 * u + k, e[k]);
        }
    }
}

// Squares every universe's box as the single-universe path does, and resets
// the reduction slots for the next step.
__global__ void bbox_batch_finish(Batch b, DeviceScalars* __restrict__ s, int64_t n) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u == 0) start_sort(s, n, 1);
    if (u >= b.nuni) return;
    unsigned long long* e = b.boxbits + 4 * u;
    double x0 = from_ordered(e[0]), x1 = from_ordered(~e[1]);
    double y0 = from_ordered(e[2]), y1 = from_ordered(~e[3]);
    const double x_range = x1 - x0, y_range = y1 - y0;
    if (x_range > y_range) {
        const double mid = (y0 + y1) * 0.5;
        y0 = mid - x_range * 0.5;
        y1 = mid + x_range * 0.5;
    } else {
        const double mid = (x0 + x1) * 0.5;
        x0 = mid - y_range * 0.5;
        x1 = mid + y_range * 0.5;
    }
    const double w = x1 - x0;
    b.lo[u] = make_double2(x0, y0);
    b.center[u] = make_double2(0.5 * (x0 + x1), 0.5 * (y0 + y1));
    b.w2[u] = w > 0.0 ? w * w : 1.0;  // a one-point universe: any width
    e[0] = ~0ull;
    e[1] = ~0ull;
    e[2] = ~0ull;
    e[3] = ~0ull;
}

__global__ void morton_batch_kernel(const double2* __restrict__ pos, int64_t n, Batch b,
                                    const DeviceScalars* __restrict__ s,
                                    uint64_t* __restrict__ key0, uint64_t* __restrict__ key1,
                                    uint32_t* __restrict__ val0, uint32_t* __restrict__ val1) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool odd = s->sort_passes & 1;
    uint64_t* __restrict__ key = odd ? key1 : key0;
    uint32_t* __restrict__ val = odd ? val1 : val0;
    const int u = b.uid[i];
    const double2 lo = b.lo[u];
    const double inv_w = 1.0 / sqrt(b.w2[u]);
    const double2 p = __ldg(pos + i);
    const double scale = (double)(1u << kBatchMortonBits);
    const double top = scale - 1.0;
    const uint32_t ix = __double2uint_rd(fmin(fmax((p.x - lo.x) * inv_w * scale, 0.0), top));
    const uint32_t iy = __double2uint_rd(fmin(fmax((p.y - lo.y) * inv_w * scale, 0.0), top));
    key[i] = ((uint64_t)u << (2 * kBatchMortonBits)) | (expand_bits_2d(ix) << 1) | expand_bits_2d(iy);
    val[i] = (uint32_t)i;
}

// ---------------------------------------------------------------------------
// LSD radix sort, 8-bit digits, 8 passes.  Each pass: per-tile digit counts
// (upsweep), a per-digit scan over tiles, and a stable scatter (downsweep)
// that ranks keys inside the tile with warp-private histograms and
// __match_any_sync, stages the tile in shared memory sorted by digit, and
// writes each digit's run with consecutive threads (coalesced).
// ---------------------------------------------------------------------------
constexpr int kWarps = kSortThreads / 32;

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Exclusive scan of one value per thread over a 256-thread block.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_tot,
                                                         uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kWarps ? warp_tot[lane] : 0;
        uint32_t winc = w;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(kFull, winc, o);
            if (lane >= o) winc += t;
        }
        if (lane < kWarps) warp_tot[lane] = winc - w;
        if (lane == kWarps - 1 && total) *total = winc;
    }
    __syncthreads();
    const uint32_t r = warp_tot[warp] + inc - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kSortThreads)
sort_upsweep(const uint64_t* __restrict__ key, int64_t n, int shift, uint32_t* __restrict__ counts,
             int tiles) {
    __shared__ uint32_t hist[256];
    hist[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < kSortTileItems; ++k) {
        const int64_t i = base + k * kSortThreads + threadIdx.x;
        const bool valid = i < n;
        const uint32_t d = valid ? (uint32_t)((__ldg(key + i) >> shift) & 0xFF) : 0x100u + lane;
        const unsigned peers = __match_any_sync(kFull, d);
        if (valid && lane == __ffs(peers) - 1) atomicAdd(&hist[d], (uint32_t)__popc(peers));
    }
    __syncthreads();
    counts[(int64_t)threadIdx.x * tiles + blockIdx.x] = hist[threadIdx.x];
}

// Block d turns row d of counts into exclusive offsets and writes its total.
__global__ void __launch_bounds__(kSortThreads)
sort_scan_rows(uint32_t* __restrict__ counts, int tiles, uint32_t* __restrict__ totals) {
    __shared__ uint32_t warp_tot[kWarps];
    __shared__ uint32_t chunk_total;
    uint32_t* row = counts + (int64_t)blockIdx.x * tiles;
    uint32_t carry = 0;
    for (int b = 0; b < tiles; b += kSortThreads) {
        const int t = b + threadIdx.x;
        const uint32_t v = t < tiles ? row[t] : 0;
        const uint32_t ex = block_exclusive_scan(v, warp_tot, &chunk_total);
        if (t < tiles) row[t] = carry + ex;
        carry += chunk_total;
        __syncthreads();
    }
    if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

__global__ void __launch_bounds__(kSortThreads)
sort_downsweep(const uint64_t* __restrict__ key_in, const uint32_t* __restrict__ val_in,
               uint64_t* __restrict__ key_out, uint32_t* __restrict__ val_out, int64_t n, int shift,
               const uint32_t* __restrict__ counts, const uint32_t* __restrict__ totals, int tiles) {
    __shared__ uint32_t whist[kWarps][256];
    __shared__ uint32_t tile_start[256];
    __shared__ uint32_t goff[256];
    __shared__ uint32_t warp_tot[kWarps];
    __shared__ uint64_t skey[kSortTile];
    __shared__ uint32_t sval[kSortTile];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) whist[w][tid] = 0;
    {
        const uint32_t tot = totals[tid];
        const uint32_t pre = block_exclusive_scan(tot, warp_tot, nullptr);
        goff[tid] = pre + counts[(int64_t)tid * tiles + blockIdx.x];
    }
    __syncthreads();

    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    const int64_t seg = base + warp * (32 * kSortTileItems);
    uint64_t k_reg[kSortTileItems];
    uint32_t v_reg[kSortTileItems];
    uint32_t r_reg[kSortTileItems];
    const unsigned below = lanemask_lt();
#pragma unroll
    for (int k = 0; k < kSortTileItems; ++k) {
        const int64_t i = seg + k * 32 + lane;
        const bool valid = i < n;
        k_reg[k] = valid ? key_in[i] : 0ull;
        v_reg[k] = valid ? val_in[i] : 0u;
        const uint32_t d = valid ? (uint32_t)((k_reg[k] >> shift) & 0xFF) : 0x100u + lane;
        const unsigned peers = __match_any_sync(kFull, d);
        const int leader = __ffs(peers) - 1;
        uint32_t b = 0;
        if (valid && lane == leader) {
            b = whist[warp][d];
            whist[warp][d] = b + __popc(peers);
        }
        b = __shfl_sync(kFull, b, leader);
        r_reg[k] = b + __popc(peers & below);
        __syncwarp();
    }
    __syncthreads();
    {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t c = whist[w][tid];
            whist[w][tid] = run;
            run += c;
        }
        tile_start[tid] = block_exclusive_scan(run, warp_tot, nullptr);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSortTileItems; ++k) {
        const int64_t i = seg + k * 32 + lane;
        if (i < n) {
            const uint32_t d = (uint32_t)((k_reg[k] >> shift) & 0xFF);
            const uint32_t lp = tile_start[d] + whist[warp][d] + r_reg[k];
            skey[lp] = k_reg[k];
            sval[lp] = v_reg[k];
        }
    }
    __syncthreads();
    const int tile_n = (int)min((int64_t)kSortTile, n - base);
    for (int p = tid; p < tile_n; p += kSortThreads) {
        const uint64_t kk = skey[p];
        const uint32_t d = (uint32_t)((kk >> shift) & 0xFF);
        const uint32_t gp = goff[d] + (uint32_t)p - tile_start[d];
        key_out[gp] = kk;
        val_out[gp] = sval[p];
    }
}

// ---------------------------------------------------------------------------
// Onesweep LSD radix sort (the step's sort).  One pass over the keys builds
// the histograms of all eight digits; each digit pass is then a single kernel
// whose tiles learn their global offsets by decoupled look-back: a tile
// publishes its per-digit count, then sums its predecessors' counts until it
// meets one that already holds an inclusive prefix.  Tiles take their index
// from an atomic counter in the order they start, so a tile only ever waits
// on tiles that are already running.  Every wait is bounded; a wait that runs
// out sets kErrTimeout and the step reports NB_ERR_TIMEOUT.
// ---------------------------------------------------------------------------
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kCountMask = (1u << 30) - 1;
constexpr int kSpinLimit = 1 << 22;

// Histograms of the digits the radix passes sort (the top sort_passes bytes;
// the passes below return at once and need none).  A warp reads rows of 32
// consecutive keys (one coalesced load) and, per digit, finds the runs of
// equal digits in the row with one ballot: each run's first lane adds the
// run's length to the digit's bin.  The keys arrive nearly sorted (the bodies
// keep last step's order), so the high digits form long runs and most rows
// cost one shared-memory atomic per digit.
constexpr int kHistRows = 4;

__global__ void __launch_bounds__(kSortThreads)
onesweep_histogram(const uint64_t* __restrict__ key0, const uint64_t* __restrict__ key1, int64_t n,
                   const DeviceScalars* __restrict__ s, uint32_t* __restrict__ hist) {
    // the Morton pass wrote the codes where the first radix pass reads them
    const uint64_t* __restrict__ key = (s->sort_passes & 1) ? key1 : key0;
    const int dmin = 8 - s->sort_passes;  // digits below are not sorted by a pass
    __shared__ uint32_t h[8][256];
    for (int k = threadIdx.x; k < 8 * 256; k += kSortThreads) (&h[0][0])[k] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (kSortThreads / 32);
    const int64_t w = (int64_t)blockIdx.x * (kSortThreads / 32) + (threadIdx.x >> 5);
    const unsigned after_me = ~((2u << lane) - 1u);  // lanes above this one (none for lane 31)
    // kHistRows rows per warp and iteration: their loads are in flight together
    for (int64_t row0 = w * 32 * kHistRows; row0 < n; row0 += warps * 32 * kHistRows) {
        uint64_t k[kHistRows];
#pragma unroll
        for (int r = 0; r < kHistRows; ++r) {
            const int64_t i = row0 + 32 * r + lane;
            k[r] = i < n ? __ldg(key + i) : 0ull;
        }
#pragma unroll
        for (int r = 0; r < kHistRows; ++r) {
            const int64_t left = n - (row0 + 32 * r);  // valid lanes of the row are a prefix
            if (left <= 0) break;
            const int end = left < 32 ? (int)left : 32;
            const bool valid = lane < end;
            const uint64_t kp = __shfl_up_sync(kFull, k[r], 1);
            const uint64_t diff = k[r] ^ kp;
#pragma unroll
            for (int d = 0; d < 8; ++d) {
                if (d < dmin) continue;
                const bool head = valid && (lane == 0 || ((diff >> (8 * d)) & 0xFF) != 0);
                const unsigned later = __ballot_sync(kFull, head) & after_me;
                if (head)
                    atomicAdd(&h[d][(uint32_t)(k[r] >> (8 * d)) & 0xFF],
                              (uint32_t)((later ? __ffs(later) - 1 : end) - lane));
            }
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < 8 * 256; k += kSortThreads) {
        const uint32_t v = (&h[0][0])[k];
        if (v) atomicAdd(hist + k, v);
    }
}

// Lanes holding the same 8-bit digit, from eight ballots (the ballot path
// keeps this off the pipe that serialises __match_any_sync).
__device__ __forceinline__ unsigned digit_peers(uint32_t d, bool valid) {
    unsigned peers = __ballot_sync(kFull, valid);
    if (!valid) peers = 0;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const bool bit = (d >> b) & 1u;
        const unsigned m = __ballot_sync(kFull, bit);
        peers &= bit ? m : ~m;
    }
    return valid ? peers : (1u << (threadIdx.x & 31));
}

// Exclusive scan of each digit position's 256 bins (block d = position d).
__global__ void __launch_bounds__(kSortThreads)
onesweep_bins(uint32_t* __restrict__ hist) {
    __shared__ uint32_t warp_tot[kWarps];
    uint32_t* row = hist + 256 * blockIdx.x;
    const uint32_t v = row[threadIdx.x];
    const uint32_t ex = block_exclusive_scan(v, warp_tot, nullptr);
    row[threadIdx.x] = ex;
}

__device__ __forceinline__ uint32_t ld_status(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_status(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ---- one-CTA bulk copies (cp.async.bulk, no multicast) into shared memory --
__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    // the barrier must be visible to the async proxy before a copy signals it
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// bytes: a multiple of 16; both addresses 16-byte aligned
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, unsigned phase) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return done != 0;
}
// Bounded wait for phase 0 of a barrier; false if it ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar) {
    for (int k = 0; k < kSpinLimit; ++k)
        if (mbar_test(bar, 0)) return true;
    return false;
}

// Four blocks per SM (at most 64 registers): tiles of 3072 keys keep enough
// loads in flight per block, and the occupancy hides the look-back.  The
// tile's keys and values arrive in shared memory by two bulk copies (the
// copy engine moves the 36 KB while the block's threads are free), then each
// thread ranks its 12 keys, and the tile leaves sorted by digit through the
// same shared buffers with coalesced stores.  The scatter itself cannot be a
// bulk copy: a digit's run starts at an arbitrary 8-byte offset of the output.
// Passes below the step's first pass (shift < 64 - 8 sort_passes) return at
// once; passes == nullptr runs every pass.
__global__ void __launch_bounds__(kSortThreads, 4)
onesweep_pass(const uint64_t* __restrict__ key_in, const uint32_t* __restrict__ val_in,
              uint64_t* __restrict__ key_out, uint32_t* __restrict__ val_out, int64_t n, int shift,
              const uint32_t* __restrict__ bins, uint32_t* __restrict__ status,
              unsigned* __restrict__ tile_counter, unsigned* __restrict__ err,
              const int32_t* __restrict__ passes) {
    if (passes && shift < 64 - 8 * *passes) return;
    __shared__ uint32_t whist[kWarps][256];
    __shared__ uint32_t tile_start[256];
    __shared__ uint32_t goff[256];
    __shared__ uint32_t warp_tot[kWarps];
    __shared__ __align__(16) uint64_t skey[kSortTile];
    __shared__ __align__(16) uint32_t sval[kSortTile];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int tile_sh;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        const int tile = (int)atomicAdd(tile_counter, 1u);
        tile_sh = tile;
        const int64_t base = (int64_t)tile * kSortTile;
        const int tile_n = (int)min((int64_t)kSortTile, n - base);
        const int bulk = tile_n & ~3;  // whole 16-byte chunks of both arrays
        mbar_init(&bar);
        mbar_expect_tx(&bar, (unsigned)bulk * 12u);
        if (bulk > 0) {
            bulk_load(skey, key_in + base, (unsigned)bulk * 8u, &bar);
            bulk_load(sval, val_in + base, (unsigned)bulk * 4u, &bar);
        }
    }
#pragma unroll
    for (int w = 0; w < kWarps; ++w) whist[w][tid] = 0;
    __syncthreads();
    const int tile = tile_sh;
    const int64_t base = (int64_t)tile * kSortTile;
    const int tile_n = (int)min((int64_t)kSortTile, n - base);
    {
        const int bulk = tile_n & ~3;
        if (tid < tile_n - bulk) {  // the last tile's ragged end, at most 3 keys
            skey[bulk + tid] = key_in[base + bulk + tid];
            sval[bulk + tid] = val_in[base + bulk + tid];
        }
        bool ok = mbar_wait_bounded(&bar);
        if (!ok) {
            atomicOr(err, kErrTimeout);
            ok = mbar_wait_bounded(&bar);  // let the copies land before the block moves on
        }
    }
    __syncthreads();
    const int seg = warp * (32 * kSortTileItems);
    uint64_t k_reg[kSortTileItems];
    uint32_t v_reg[kSortTileItems];
    uint32_t r_reg[kSortTileItems];
    const unsigned below = lanemask_lt();
#pragma unroll
    for (int k = 0; k < kSortTileItems; ++k) {
        const int li = seg + k * 32 + lane;
        const bool valid = li < tile_n;
        k_reg[k] = valid ? skey[li] : 0ull;
        v_reg[k] = valid ? sval[li] : 0u;
        const uint32_t d = (uint32_t)((k_reg[k] >> shift) & 0xFF);
        const unsigned peers = digit_peers(d, valid);
        const int leader = __ffs(peers) - 1;
        uint32_t b = 0;
        if (valid && lane == leader) {
            b = whist[warp][d];
            whist[warp][d] = b + __popc(peers);
        }
        b = __shfl_sync(kFull, b, leader);
        r_reg[k] = b + __popc(peers & below);
        __syncwarp();
    }
    __syncthreads();
    uint32_t count;
    {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t c = whist[w][tid];
            whist[w][tid] = run;
            run += c;
        }
        count = run;
        tile_start[tid] = block_exclusive_scan(run, warp_tot, nullptr);
    }
    // look-back for digit tid
    uint32_t* st = status + (int64_t)tile * 256 + tid;
    uint32_t excl = 0;
    if (tile == 0) {
        st_status(st, kFlagPrefix | count);
    } else {
        st_status(st, kFlagAgg | count);
        for (int j = tile - 1; j >= 0; --j) {
            const uint32_t* pj = status + (int64_t)j * 256 + tid;
            uint32_t v = ld_status(pj);
            int spins = 0;
            while ((v & ~kCountMask) == 0) {
                if (++spins > kSpinLimit) {
                    atomicOr(err, kErrTimeout);
                    break;
                }
                v = ld_status(pj);
            }
            excl += v & kCountMask;
            if ((v & ~kCountMask) == kFlagPrefix) break;
        }
        st_status(st, kFlagPrefix | (excl + count));
    }
    goff[tid] = bins[tid] + excl;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSortTileItems; ++k) {
        const int li = seg + k * 32 + lane;
        if (li < tile_n) {
            const uint32_t d = (uint32_t)((k_reg[k] >> shift) & 0xFF);
            const uint32_t lp = tile_start[d] + whist[warp][d] + r_reg[k];
            skey[lp] = k_reg[k];
            sval[lp] = v_reg[k];
        }
    }
    __syncthreads();
    for (int p = tid; p < tile_n; p += kSortThreads) {
        const uint64_t kk = skey[p];
        const uint32_t d = (uint32_t)((kk >> shift) & 0xFF);
        const uint32_t gp = goff[d] + (uint32_t)p - tile_start[d];
        key_out[gp] = kk;
        val_out[gp] = sval[p];
    }
}

// ---------------------------------------------------------------------------
// Tie pass.  After radix passes over the top P bytes only, keys that agree in
// those bytes sit together in their input order; putting each such group in
// order of its low bytes (ties kept in input order) gives exactly the full
// stable sort.  tie_mark lists the groups, tie_sort_small orders groups of
// up to 32 keys one warp each in registers, tie_sort_big orders larger ones
// one warp each by an LSD radix sort of the low bytes through the free
// ping-pong buffers.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
tie_mark(const uint64_t* __restrict__ key, int64_t n, DeviceScalars* __restrict__ s,
         uint2* __restrict__ small, uint2* __restrict__ big) {
    const int passes = s->sort_passes;
    if (passes >= 8) return;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int sh = 64 - 8 * passes;
    const int lane = threadIdx.x & 31;
    // each key is read once; the neighbours come from the next and previous
    // lanes (the row's end lanes read theirs)
    const uint64_t ki = i < n ? key[i] : 0ull;
    uint64_t kn = __shfl_down_sync(kFull, ki, 1), kp = __shfl_up_sync(kFull, ki, 1);
    if (lane == 31 && i + 1 < n) kn = key[i + 1];
    if (lane == 0 && i > 0 && i < n) kp = key[i - 1];
    bool start = false;
    int64_t e = i;
    if (i + 1 < n) {
        const uint64_t top = ki >> sh;
        start = (kn >> sh) == top && (i == 0 || (kp >> sh) != top);
        if (start) {  // last key of the group: galloping search
            int64_t step = 1, good = i + 1;
            while (good + step < n && (key[good + step] >> sh) == top) {
                good += step;
                step <<= 1;
            }
            int64_t lo = good, hi = min(n - 1, good + step - 1);
            while (lo < hi) {
                const int64_t mid = (lo + hi + 1) >> 1;
                if ((key[mid] >> sh) == top) lo = mid; else hi = mid - 1;
            }
            e = lo;
        }
    }
    const unsigned size = (unsigned)(e - i + 1);
    const bool is_small = start && size <= 32, is_big = start && size > 32;
    const unsigned ms = __ballot_sync(kFull, is_small), mb = __ballot_sync(kFull, is_big);
    unsigned b0 = 0, b1 = 0;
    if (lane == 0) {
        if (ms) b0 = atomicAdd(&s->tie_count[0], __popc(ms));
        if (mb) b1 = atomicAdd(&s->tie_count[1], __popc(mb));
    }
    b0 = __shfl_sync(kFull, b0, 0);
    b1 = __shfl_sync(kFull, b1, 0);
    const unsigned lt = lanemask_lt();
    if (is_small) small[b0 + __popc(ms & lt)] = make_uint2((unsigned)i, size);
    if (is_big) big[b1 + __popc(mb & lt)] = make_uint2((unsigned)i, size);
}

// Groups of 2..32 keys: lane l holds key l of the group and counts the keys
// that go before it (smaller, or equal and earlier).  The keys share their top
// bytes, so comparing whole keys compares the low bytes.
__global__ void __launch_bounds__(256)
tie_sort_small(uint64_t* __restrict__ key, uint32_t* __restrict__ val,
               const uint2* __restrict__ small, const DeviceScalars* __restrict__ s) {
    if (s->sort_passes >= 8) return;
    const unsigned count = s->tie_count[0];
    const int lane = threadIdx.x & 31;
    const unsigned warps = gridDim.x * (blockDim.x >> 5);
    for (unsigned g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); g < count; g += warps) {
        const uint2 grp = small[g];
        const bool on = lane < (int)grp.y;
        const uint64_t k = on ? key[grp.x + lane] : ~0ull;
        const uint32_t v = on ? val[grp.x + lane] : 0u;
        int rank = 0;
        for (int j = 0; j < (int)grp.y; ++j) {
            const uint64_t kj = __shfl_sync(kFull, k, j);
            rank += (kj < k || (kj == k && j < lane)) ? 1 : 0;
        }
        __syncwarp();
        if (on) {
            key[grp.x + rank] = k;
            val[grp.x + rank] = v;
        }
    }
}

// Groups of more than 32 keys (rare: many bodies within 2^-4P of the box
// width of each other): one warp per group, a stable LSD radix sort of the
// 8 - P low bytes, 32 keys at a time, between the group's range of the
// sorted buffers and the same range of the free ping-pong buffers.
__global__ void __launch_bounds__(128)
tie_sort_big(uint64_t* __restrict__ key0, uint32_t* __restrict__ val0, uint64_t* __restrict__ key1,
             uint32_t* __restrict__ val1, const uint2* __restrict__ big,
             const DeviceScalars* __restrict__ s) {
    const int passes = s->sort_passes;
    if (passes >= 8) return;
    __shared__ uint32_t off[4][256];
    const unsigned count = s->tie_count[1];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned below = lanemask_lt();
    for (unsigned g = blockIdx.x * 4 + w; g < count; g += gridDim.x * 4) {
        const uint2 grp = big[g];
        const unsigned first = grp.x, size = grp.y;
        for (int d = 0; d < 8 - passes; ++d) {
            const int sh = 8 * d;
            const bool from0 = (d & 1) == 0;
            const uint64_t* ks = from0 ? key0 : key1;
            const uint32_t* vs = from0 ? val0 : val1;
            uint64_t* kd = from0 ? key1 : key0;
            uint32_t* vd = from0 ? val1 : val0;
            for (int b = lane; b < 256; b += 32) off[w][b] = 0;
            __syncwarp();
            for (unsigned b = 0; b < size; b += 32) {
                if (b + lane < size) atomicAdd(&off[w][(ks[first + b + lane] >> sh) & 0xFF], 1u);
            }
            __syncwarp();
            // exclusive scan of the 256 bins, 8 per lane
            uint32_t c[8], tot = 0;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                c[q] = off[w][lane * 8 + q];
                tot += c[q];
            }
            uint32_t inc = tot;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(kFull, inc, o);
                if (lane >= o) inc += t;
            }
            uint32_t run = inc - tot;
            __syncwarp();
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                off[w][lane * 8 + q] = run;
                run += c[q];
            }
            __syncwarp();
            for (unsigned b = 0; b < size; b += 32) {
                const bool on = b + lane < size;
                const uint64_t k = on ? ks[first + b + lane] : 0ull;
                const uint32_t v = on ? vs[first + b + lane] : 0u;
                const uint32_t dg = (uint32_t)((k >> sh) & 0xFF);
                const unsigned peers = digit_peers(dg, on);
                const int leader = __ffs(peers) - 1;
                uint32_t pos = 0;
                if (on && lane == leader) {
                    pos = off[w][dg];
                    off[w][dg] = pos + __popc(peers);
                }
                pos = __shfl_sync(kFull, pos, leader) + __popc(peers & below);
                if (on) {
                    kd[first + pos] = k;
                    vd[first + pos] = v;
                }
                __syncwarp();
            }
        }
        if ((8 - passes) & 1) {  // the result is in the second buffers: copy it back
            for (unsigned b = lane; b < size; b += 32) {
                key0[first + b] = key1[first + b];
                val0[first + b] = val1[first + b];
            }
        }
        __syncwarp();
    }
}

// CU:135-147: gather the bodies into Morton order.  In SPLIT mode it also
// writes the FP32 source record of each body relative to the box centre.
__global__ void gather_kernel(const uint32_t* __restrict__ order, int64_t n, BodyBuffers src,
                              BodyBuffers dst, float4* __restrict__ body4,
                              const DeviceScalars* __restrict__ s, Batch bt) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t j = __ldg(order + i);
    const double2 p = __ldg(src.pos + j);
    const double m = __ldg(src.mass + j);
    dst.pos[i] = p;
    dst.vel[i] = __ldg(src.vel + j);
    dst.mass[i] = m;
    dst.orig[i] = __ldg(src.orig + j);
    if (body4) {
        const double2 c = frame_center(s, bt, (int)i);
        body4[i] = make_float4((float)(p.x - c.x), (float)(p.y - c.y), (float)m,
                               __int_as_float((int)i));
    }
}

inline unsigned blocks_for(int64_t n, int threads) {
    return (unsigned)((n + threads - 1) / threads);
}

}  // namespace

void launch_bbox(nb_ctx* c, const double2* pos) {
    if (c->batch.nuni > 0) {
        c->launches += 2;
        bbox_batch_kernel<<<2 * c->sm_count * 8, 256, 0, c->stream>>>(pos, c->n, c->batch);
        bbox_batch_finish<<<blocks_for(c->batch.nuni, 128), 128, 0, c->stream>>>(c->batch, c->scal,
                                                                                c->n);
        return;
    }
    c->launches += 1;
    bbox_kernel<<<c->bbox_blocks, kBoxThreads, 0, c->stream>>>(pos, c->n, c->bbox_partials, c->scal,
                                                               1);
}

void launch_morton(nb_ctx* c, const double2* pos) {
    c->launches += 1;
    if (c->batch.nuni > 0) {
        morton_batch_kernel<<<blocks_for(c->n, 256), 256, 0, c->stream>>>(
            pos, c->n, c->batch, c->scal, c->sort.key[0], c->sort.key[1], c->sort.val[0],
            c->sort.val[1]);
        return;
    }
    morton_kernel<<<blocks_for(c->n, 256), 256, 0, c->stream>>>(
        pos, c->n, c->scal, c->sort.key[0], c->sort.key[1], c->sort.val[0], c->sort.val[1]);
}

// One radix pass over two tiles of keys in which only the second tile runs:
// its look-back waits on a predecessor that never publishes, so the bounded
// wait must give up and raise kErrTimeout.  Returns the error bits.
unsigned sort_timeout_probe(cudaStream_t st) {
    constexpr int n = 2 * kSortTile;
    uint64_t *key_in = nullptr, *key_out = nullptr;
    uint32_t *val_in = nullptr, *val_out = nullptr, *hist = nullptr, *status = nullptr;
    unsigned *counter = nullptr, *err = nullptr;
    unsigned flags = ~0u;
    if (cudaMalloc(&key_in, n * sizeof(uint64_t)) == cudaSuccess &&
        cudaMalloc(&key_out, n * sizeof(uint64_t)) == cudaSuccess &&
        cudaMalloc(&val_in, n * sizeof(uint32_t)) == cudaSuccess &&
        cudaMalloc(&val_out, n * sizeof(uint32_t)) == cudaSuccess &&
        cudaMalloc(&hist, 256 * sizeof(uint32_t)) == cudaSuccess &&
        cudaMalloc(&status, 2 * 256 * sizeof(uint32_t)) == cudaSuccess &&
        cudaMalloc(&counter, sizeof(unsigned)) == cudaSuccess &&
        cudaMalloc(&err, sizeof(unsigned)) == cudaSuccess) {
        // all keys zero: digit 0 holds every key, bins are all 0
        cudaMemsetAsync(key_in, 0, n * sizeof(uint64_t), st);
        cudaMemsetAsync(val_in, 0, n * sizeof(uint32_t), st);
        cudaMemsetAsync(hist, 0, 256 * sizeof(uint32_t), st);
        cudaMemsetAsync(status, 0, 2 * 256 * sizeof(uint32_t), st);
        cudaMemsetAsync(err, 0, sizeof(unsigned), st);
        const unsigned one = 1u;  // the single block takes tile 1
        cudaMemcpyAsync(counter, &one, sizeof(unsigned), cudaMemcpyHostToDevice, st);
        onesweep_pass<<<1, kSortThreads, 0, st>>>(key_in, val_in, key_out, val_out, n, 0, hist, status,
                                                  counter, err, nullptr);
        cudaMemcpyAsync(&flags, err, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) flags = ~0u;
    }
    cudaFree(key_in);
    cudaFree(key_out);
    cudaFree(val_in);
    cudaFree(val_out);
    cudaFree(hist);
    cudaFree(status);
    cudaFree(counter);
    cudaFree(err);
    return flags;
}

void launch_sort(nb_ctx* c) {
    const int tiles = c->sort.tiles;
    c->launches += 2 + 8 + 3;
    // histograms, per-pass status words and tile counters start at zero
    cudaMemsetAsync(c->sort.hist, 0, sizeof(uint32_t) * 8 * 256, c->stream);
    cudaMemsetAsync(c->sort.status, 0, sizeof(uint32_t) * 8 * 256 * (size_t)tiles, c->stream);
    cudaMemsetAsync(c->sort.tile_counter, 0, sizeof(unsigned) * 8, c->stream);
    onesweep_histogram<<<4 * c->sm_count, kSortThreads, 0, c->stream>>>(
        c->sort.key[0], c->sort.key[1], c->n, c->scal, c->sort.hist);
    onesweep_bins<<<8, kSortThreads, 0, c->stream>>>(c->sort.hist);
    for (int pass = 0; pass < 8; ++pass) {
        const int src = pass & 1, dst = src ^ 1;
        onesweep_pass<<<tiles, kSortThreads, 0, c->stream>>>(
            c->sort.key[src], c->sort.val[src], c->sort.key[dst], c->sort.val[dst], c->n, 8 * pass,
            c->sort.hist + 256 * pass, c->sort.status + (size_t)pass * 256 * tiles,
            c->sort.tile_counter + pass, &c->scal->error, &c->scal->sort_passes);
    }
    // keys tied in the sorted top bytes, in order of their low bytes
    tie_mark<<<blocks_for(c->n, 256), 256, 0, c->stream>>>(c->sort.key[0], c->n, c->scal,
                                                           c->sort.ties_small, c->sort.ties_big);
    tie_sort_small<<<c->sm_count * 8, 256, 0, c->stream>>>(c->sort.key[0], c->sort.val[0],
                                                          c->sort.ties_small, c->scal);
    tie_sort_big<<<c->sm_count, 128, 0, c->stream>>>(c->sort.key[0], c->sort.val[0],
                                                     c->sort.key[1], c->sort.val[1],
                                                     c->sort.ties_big, c->scal);
}

void launch_morton_sort_raw(const double2* pos, int64_t n, uint64_t* const key[2],
                            uint32_t* const val[2], uint64_t* key_out, uint32_t* val_out,
                            uint32_t* counts, uint32_t* totals, double* partials, int bbox_blocks,
                            DeviceScalars* scal, cudaStream_t st) {
    const int tiles = (int)((n + kSortTile - 1) / kSortTile);
    bbox_kernel<<<bbox_blocks, kBoxThreads, 0, st>>>(pos, n, partials, scal, 0);  // all 8 passes
    morton_kernel<<<blocks_for(n, 256), 256, 0, st>>>(pos, n, scal, key[0], key[1], val[0], val[1]);
    for (int pass = 0; pass < 8; ++pass) {
        const int src = pass & 1, dst = src ^ 1;
        const int shift = 8 * pass;
        uint64_t* kd = pass == 7 ? key_out : key[dst];
        uint32_t* vd = pass == 7 ? val_out : val[dst];
        sort_upsweep<<<tiles, kSortThreads, 0, st>>>(key[src], n, shift, counts, tiles);
        sort_scan_rows<<<256, kSortThreads, 0, st>>>(counts, tiles, totals);
        sort_downsweep<<<tiles, kSortThreads, 0, st>>>(key[src], val[src], kd, vd, n, shift, counts,
                                                       totals, tiles);
    }
}

void launch_gather(nb_ctx* c, const BodyBuffers& src, const BodyBuffers& dst, float4* body4) {
    c->launches += 1;
    gather_kernel<<<blocks_for(c->n, 256), 256, 0, c->stream>>>(c->sort.val[0], c->n, src, dst,
                                                                body4, c->scal, c->batch);
}

}  // namespace nb
