// k_tree.cu -- compressed quadtree from sorted Morton codes, and its moments.
//
// Replaces the reference's level-by-level build (BarnesHutCuda.cu:153-240 and
// the host loop at CU:713-777, up to 31 launches each followed by a
// device-to-host copy) and its per-level COM passes (CU:251-344, CU:787-807).
//
// Construction (Karras-style, no host round trips):
//   For the boundary i between sorted bodies i and i+1 let d_i be the number
//   of leading 2-bit digits their codes share.  Every boundary with d_i < 30
//   separates two children of the cell "bodies sharing d_i digits with body
//   i", whose level is d_i.  That cell is created once, by its first child
//   boundary (the one whose left neighbour run starts the cell), found with
//   an O(1) test after one galloping search.  Cells are numbered by an
//   exclusive scan over those boundaries, which lays every subtree out as a
//   contiguous id range.  A third pass links children (<= 4 per cell) and
//   parents.
//
// The reference tree is uncompressed: a cell with one non-empty child is
// followed by a chain of single-child cells down to the next split, all with
// the same mass and centre of mass.  The reference accepts a chain at its
// first level that passes width^2 < theta^2 d^2, and because widths shrink
// with depth that happens iff the deepest level of the chain passes.  This
// tree therefore keeps only the deepest level of every chain and stores that
// level, so opening decisions and force terms equal the reference's
// (cell widths come from the level, never from the body range).
#include <climits>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "nb_internal.cuh"

namespace nb {
namespace {

constexpr int kThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kThreads * kScanItems;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int lcp_digits(uint64_t a, uint64_t b) {
    const uint64_t x = a ^ b;
    return x ? (__clzll((long long)x) >> 1) : 32;
}

__device__ __forceinline__ bool share(uint64_t a, uint64_t b, int digits) {
    return digits <= 0 ? true : (digits >= 32 ? a == b : ((a ^ b) >> (64 - 2 * digits)) == 0);
}

// Last index e in [i, hi] whose code shares `digits` leading digits with key[i].
__device__ int gallop_right(const uint64_t* __restrict__ key, int i, int hi, int digits) {
    const uint64_t ki = key[i];
    int j = i, step = 1;
    while (true) {
        const int cand = i + step;
        if (cand > hi || !share(key[cand], ki, digits)) break;
        j = cand;
        step <<= 1;
    }
    int a = j, b = min(hi, i + step - 1);
    while (a < b) {
        const int mid = (a + b + 1) >> 1;
        if (share(key[mid], ki, digits)) a = mid; else b = mid - 1;
    }
    return a;
}

// ---- cell structure from the boundary levels ---------------------------
// Boundary i lies between bodies i and i + 1; its level c_i is the number of
// leading digits codes i and i + 1 share (capped at kMaxLevel: codes sharing
// 30 or more digits sit in one leaf).  The cell whose children boundary i
// separates spans the bodies between the nearest boundaries on either side
// with a smaller level, and the boundaries of equal level between those are
// its other child separators.  So the whole build reduces to nearest smaller
// values over c (ANSV), which three passes find without a search:
//   tree_lcp         c_i per boundary, and per tile and level v the first
//                    and last boundary with a level below v;
//   tree_ansv_tiles  those tables scanned over the tiles (prefix maximum of
//                    the last, suffix minimum of the first);
//   tree_ansv        per boundary the nearest smaller (and smaller-or-equal)
//                    level on each side: inside its warp row from the row's
//                    ballot for that level, inside its tile from the rows'
//                    summaries, beyond the tile from the scanned tables.
// A tile is kAnsvTile boundaries; warp w holds rows 8w..8w+7 of 32.  Lane v
// of a row needs the row's mask "level < v": each lane writes its level as a
// thermometer word (bit v set for every v above its level) and a 32 x 32 bit
// transpose across the warp (five butterfly shuffles) hands lane v bit v of
// every lane, which is that mask.
constexpr int kAnsvItems = kAnsvTile / kThreads;  // rows per warp
constexpr int kAnsvRows = kAnsvTile / 32;           // 64 rows
constexpr int kNoLevel = kMaxLevel + 1;             // past the last body: never below a level
static_assert(kAnsvItems == 8 && kAnsvLevels == 32, "one lane per level, 8 rows per warp");

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Lane v receives bit v of every lane's word x (bit l from lane l): the 32 x
// 32 bit matrix of the warp's words transposed by swapping off-diagonal
// blocks of 16, 8, 4, 2 and 1 between lane pairs.
__device__ __forceinline__ unsigned warp_transpose_bits(unsigned x) {
    const int lane = threadIdx.x & 31;
    constexpr unsigned keep[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int j = 16 >> k;
        const unsigned p = __shfl_xor_sync(kFull, x, j);
        x = (lane & j) ? (x & ~keep[k]) | ((p >> j) & keep[k])
                       : (x & keep[k]) | ((p << j) & ~keep[k]);
    }
    return x;
}

// Bit v set for every v above level c (v = 0..31).
__device__ __forceinline__ unsigned thermometer(int c) {
    return c >= 31 ? 0u : (0xFFFFFFFFu << (c + 1));
}

// Tables are level-major: tab[v * tiles + t].
__global__ void __launch_bounds__(kThreads)
tree_lcp(const uint64_t* __restrict__ key, int n, int tiles, uint8_t* __restrict__ lcp8,
         int32_t* __restrict__ tile_first, int32_t* __restrict__ tile_last,
         unsigned* __restrict__ lcp_hist) {
    __shared__ unsigned hist[33];
    __shared__ int sfirst[kAnsvLevels], slast[kAnsvLevels];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < 33) hist[threadIdx.x] = 0;
    if (threadIdx.x < kAnsvLevels) {
        sfirst[threadIdx.x] = INT_MAX;
        slast[threadIdx.x] = -1;
    }
    __syncthreads();
    const int base = blockIdx.x * kAnsvTile + warp * (32 * kAnsvItems);
    // lane v (1..30): first and last boundary of the warp's rows with level < v;
    // lane v (1..31) and lane 0 (for 32): how many have a level < v
    int myfirst = INT_MAX, mylast = -1;
    unsigned mycnt = 0, nbound = 0;
#pragma unroll 1
    for (int r = 0; r < kAnsvItems; ++r) {
        const int row0 = base + 32 * r;
        const int i = row0 + lane;
        int c = 64;  // not a boundary
        if (i < n - 1) c = lcp_digits(key[i], key[i + 1]);
        if (i < n) lcp8[i] = (uint8_t)(i < n - 1 ? min(c, kMaxLevel) : kNoLevel);
        // lane v (1..31): the row's mask of levels below v; lane 0: below 32
        unsigned mine = warp_transpose_bits(thermometer(c));
        const unsigned below32 = __ballot_sync(kFull, c < 32);
        if (lane == 0) mine = below32;
        nbound += __popc(__ballot_sync(kFull, i < n - 1));
        mycnt += __popc(mine);
        if (mine && lane >= 1 && lane <= kMaxLevel) {
            if (myfirst == INT_MAX) myfirst = row0 + __ffs(mine) - 1;
            mylast = row0 + 31 - __clz(mine);
        }
    }
    if (myfirst != INT_MAX) atomicMin(&sfirst[lane], myfirst);
    if (mylast >= 0) atomicMax(&slast[lane], mylast);
    {   // histogram of levels 0..32 from the counts below each level
        const unsigned c32 = __shfl_sync(kFull, mycnt, 0);
        const unsigned x = lane == 0 ? 0u : mycnt;         // count below level `lane`
        const unsigned up = __shfl_down_sync(kFull, x, 1);  // count below level lane + 1
        const unsigned h = lane < 31 ? up - x : c32 - x;
        if (h) atomicAdd(&hist[lane], h);
        if (lane == 0 && nbound > c32) atomicAdd(&hist[32], nbound - c32);
    }
    __syncthreads();
    if (threadIdx.x < kAnsvLevels) {
        tile_first[threadIdx.x * tiles + blockIdx.x] = sfirst[threadIdx.x];
        tile_last[threadIdx.x * tiles + blockIdx.x] = slast[threadIdx.x];
    }
    // the next step's sort reads how many neighbouring codes share d digits
    if (threadIdx.x < 33 && hist[threadIdx.x]) atomicAdd(lcp_hist + threadIdx.x, hist[threadIdx.x]);
}

// One block per level v: tile_last becomes the last boundary of tiles 0..t
// with a level below v, tile_first the first of tiles t..tiles-1.
constexpr int kTileScanThreads = 1024;
__global__ void __launch_bounds__(kTileScanThreads)
tree_ansv_tiles(int tiles, int32_t* __restrict__ tile_first, int32_t* __restrict__ tile_last) {
    __shared__ int wagg[kTileScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t* last = tile_last + blockIdx.x * tiles;
    int32_t* first = tile_first + blockIdx.x * tiles;
    int carry = -1;
    for (int b = 0; b < tiles; b += kTileScanThreads) {
        const int t = b + threadIdx.x;
        int x = t < tiles ? last[t] : -1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x = max(x, y);
        }
        if (lane == 31) wagg[warp] = x;
        __syncthreads();
        int pre = carry, tot = carry;
        for (int w = 0; w < kTileScanThreads / 32; ++w) {
            if (w < warp) pre = max(pre, wagg[w]);
            tot = max(tot, wagg[w]);
        }
        if (t < tiles) last[t] = max(x, pre);
        carry = tot;
        __syncthreads();
    }
    carry = INT_MAX;
    for (int b = tiles - 1; b >= 0; b -= kTileScanThreads) {
        const int t = b - (int)threadIdx.x;  // descending: a prefix over the threads is a suffix over tiles
        int x = t >= 0 ? first[t] : INT_MAX;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x = min(x, y);
        }
        if (lane == 31) wagg[warp] = x;
        __syncthreads();
        int pre = carry, tot = carry;
        for (int w = 0; w < kTileScanThreads / 32; ++w) {
            if (w < warp) pre = min(pre, wagg[w]);
            tot = min(tot, wagg[w]);
        }
        if (t >= 0) first[t] = min(x, pre);
        carry = tot;
        __syncthreads();
    }
}

// Per boundary i below kMaxLevel: flag = 1 iff i is its cell's first
// separator (no equal level between it and the cell's start), which numbers
// the cells; bnd[i] = {first body of the cell, last body of the cell,
// previous separator of the cell or -1, next separator or -1}, the first two
// written for flagged boundaries only.  The cell's first body follows the
// nearest smaller level on the left, its last body is the nearest smaller on
// the right (or n - 1); a separator's neighbours are the nearest levels <= c_i
// when those equal c_i.
__global__ void __launch_bounds__(kThreads)
tree_ansv(const uint8_t* __restrict__ lcp8, int n, int tiles,
          const int32_t* __restrict__ tile_first, const int32_t* __restrict__ tile_last,
          int32_t* __restrict__ flag, int4* __restrict__ bnd) {
    // masks[r][v]: row r's ballot of "level < v" (v = 1..30; 0 elsewhere).
    // rlast[r][v]: after the scan, the last boundary with a level below v in
    // rows 8p..r of r's part p (-1 if none), rfirst[r][v] the first in rows
    // r..8p+7 (kAnsvTile if none); tile-local positions
    __shared__ unsigned masks[kAnsvRows][32];
    __shared__ int16_t rlast[kAnsvRows][kAnsvLevels];
    __shared__ int16_t rfirst[kAnsvRows][kAnsvLevels];
    __shared__ int16_t before[kThreads / 32][kAnsvLevels];  // last in the parts before p
    __shared__ int16_t after[kThreads / 32][kAnsvLevels];   // first in the parts after p
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tile = blockIdx.x, tbase = tile * kAnsvTile;
#pragma unroll 1
    for (int r = 0; r < kAnsvItems; ++r) {
        const int row = warp * kAnsvItems + r;
        const int i = tbase + 32 * row + lane;
        const int cap = i < n ? lcp8[i] : kNoLevel;
        // lane v: the row's mask of levels below v (lanes 0 and 31 unused: 0)
        unsigned mine = warp_transpose_bits(thermometer(cap));
        if (lane == 0 || lane > kMaxLevel) mine = 0u;
        masks[row][lane] = mine;
        rfirst[row][lane] = (int16_t)(mine ? 32 * row + __ffs(mine) - 1 : kAnsvTile);
        rlast[row][lane] = (int16_t)(mine ? 32 * row + 31 - __clz(mine) : -1);
    }
    __syncwarp();
    {   // scan the warp's own 8 rows, lane = level
        int run = -1;
        for (int r = 0; r < kAnsvItems; ++r) {
            const int row = warp * kAnsvItems + r;
            run = max(run, (int)rlast[row][lane]);
            rlast[row][lane] = (int16_t)run;
        }
        int runf = kAnsvTile;
        for (int r = kAnsvItems - 1; r >= 0; --r) {
            const int row = warp * kAnsvItems + r;
            runf = min(runf, (int)rfirst[row][lane]);
            rfirst[row][lane] = (int16_t)runf;
        }
    }
    __syncthreads();
    {
        int b = -1, a = kAnsvTile;
        for (int p = 0; p < kThreads / 32; ++p) {
            if (p < warp) b = max(b, (int)rlast[p * kAnsvItems + kAnsvItems - 1][lane]);
            if (p > warp) a = min(a, (int)rfirst[p * kAnsvItems][lane]);
        }
        before[warp][lane] = (int16_t)b;
        after[warp][lane] = (int16_t)a;
    }
    __syncthreads();
    const unsigned lt = lanemask_lt(), gt = ~lt & ~(1u << lane);
#pragma unroll 1
    for (int r = 0; r < kAnsvItems; ++r) {
        const int row = warp * kAnsvItems + r;
        const int i = tbase + 32 * row + lane;
        if (i >= n) continue;
        const int v = lcp8[i];
        if (i == n - 1 || v >= kMaxLevel) {
            flag[i] = 0;
            continue;
        }
        // nearest boundary on the left / right with a level below u
        auto left = [&](int u) {
            const unsigned m = masks[row][u] & lt;
            if (m) return tbase + 32 * row + 31 - __clz(m);
            int j = r > 0 ? (int)rlast[row - 1][u] : -1;
            if (j < 0) j = before[warp][u];
            if (j >= 0) return tbase + j;
            return tile > 0 ? tile_last[u * tiles + tile - 1] : -1;
        };
        auto right = [&](int u) {
            const unsigned m = masks[row][u] & gt;
            if (m) return tbase + 32 * row + __ffs(m) - 1;
            int j = r < kAnsvItems - 1 ? (int)rfirst[row + 1][u] : kAnsvTile;
            if (j >= kAnsvTile) j = after[warp][u];
            if (j < kAnsvTile) return tbase + j;
            const int g = tile + 1 < tiles ? tile_first[u * tiles + tile + 1] : INT_MAX;
            return g == INT_MAX ? n - 1 : g;
        };
        const int l_lt = left(v), l_le = left(v + 1);
        const int r_lt = right(v), r_le = right(v + 1);
        const bool first_sep = l_le == l_lt;
        flag[i] = first_sep ? 1 : 0;
        bnd[i] = make_int4(first_sep ? l_lt + 1 : -1, first_sep ? r_lt : -1,
                           first_sep ? -1 : l_le, r_le == r_lt ? -1 : r_le);
    }
}

// ---- exclusive scan of flag[] -> cell_of[], total -> scal->cells ----------
__device__ __forceinline__ int warp_inclusive(int v) {
    const int lane = threadIdx.x & 31;
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

template <int kBlock = kThreads>
__device__ int block_exclusive(int v, int* wsum, int* total) {
    static_assert(kBlock % 32 == 0 && kBlock <= 1024, "one warp scans the warp sums");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int inc = warp_inclusive(v);
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const int w = lane < kBlock / 32 ? wsum[lane] : 0;
        const int winc = warp_inclusive(w);
        if (lane < kBlock / 32) wsum[lane] = winc - w;
        if (lane == kBlock / 32 - 1 && total) *total = winc;
    }
    __syncthreads();
    const int r = wsum[warp] + inc - v;
    __syncthreads();
    return r;
}

// Items of a tile are read in coalesced rows: warp w takes the 32 *
// kScanItems items [w 32 kScanItems, (w + 1) 32 kScanItems) of the tile,
// lane l the items 32 k + l of them.
__global__ void __launch_bounds__(kThreads)
scan_reduce(const int32_t* __restrict__ in, int n, int32_t* __restrict__ block_sums) {
    __shared__ int wsum[kThreads / 32];
    __shared__ int total;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int base = blockIdx.x * kScanTile + warp * 32 * kScanItems + lane;
    int v = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int i = base + 32 * k;
        if (i < n) v += in[i];
    }
    block_exclusive(v, wsum, &total);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

// One block of kSumsThreads: the block sums of 4M entries (2,048) take two
// rounds instead of eight.
constexpr int kSumsThreads = 1024;
__global__ void __launch_bounds__(kSumsThreads)
scan_block_sums(int32_t* __restrict__ block_sums, int blocks, int32_t* __restrict__ total_out) {
    __shared__ int wsum[kSumsThreads / 32];
    __shared__ int total;
    int carry = 0;
    for (int b = 0; b < blocks; b += kSumsThreads) {
        const int t = b + threadIdx.x;
        const int v = t < blocks ? block_sums[t] : 0;
        const int ex = block_exclusive<kSumsThreads>(v, wsum, &total);
        if (t < blocks) block_sums[t] = carry + ex;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total_out = carry;
}

// Each row of 32 items is scanned with shuffles; the rows' totals carry
// within the warp, and the warps' totals (one barrier) within the tile.
__global__ void __launch_bounds__(kThreads)
scan_apply(const int32_t* __restrict__ in, int n, const int32_t* __restrict__ block_sums,
           int32_t* __restrict__ out, int32_t* __restrict__ index_of) {
    __shared__ int wsum[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int base = blockIdx.x * kScanTile + warp * 32 * kScanItems + lane;
    int v[kScanItems], ex[kScanItems];
    int carry = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int i = base + 32 * k;
        v[k] = i < n ? in[i] : 0;
        const int inc = warp_inclusive(v[k]);
        ex[k] = carry + inc - v[k];
        carry += __shfl_sync(kFull, inc, 31);
    }
    if (lane == 0) wsum[warp] = carry;
    __syncthreads();
    int off = block_sums[blockIdx.x];
    for (int w = 0; w < warp; ++w) off += wsum[w];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int i = base + 32 * k;
        if (i < n) {
            const int run = off + ex[k];
            out[i] = run;
            // with 0/1 inputs, index_of lists the flagged positions in order
            if (index_of && v[k]) index_of[run] = i;
        }
    }
}

// Moments of a multi-body leaf in the reference's summation order: 128
// strided partial sums, then a halving tree (CU:284-309).  The halving tree
// adds the partials as a balanced binary tree whose leaves, left to right, are
// the partials in 7-bit bit-reversed order, so a binary-counter pairwise sum
// over that sequence reproduces it with an 8-entry stack.  Such leaves only
// hold bodies whose codes agree in 60 bits, so they are rare and small.
__device__ void bucket_moments(const double2* __restrict__ pos, const double* __restrict__ mass,
                               int first, int last, double* out_m, double2* out_c) {
    double sm[8], sx[8], sy[8];
    for (int k = 0; k < 128; ++k) {
        const int tx = (int)(__brev((unsigned)k) >> 25);
        double M = 0.0, Rx = 0.0, Ry = 0.0;
        for (int i = first + tx; i <= last; i += 128) {
            const double m = mass[i];
            M += m;
            Rx = fma(m, pos[i].x, Rx);
            Ry = fma(m, pos[i].y, Ry);
        }
        int lvl = 0;
        while ((k >> lvl) & 1) {
            M = sm[lvl] + M;
            Rx = sx[lvl] + Rx;
            Ry = sy[lvl] + Ry;
            ++lvl;
        }
        sm[lvl] = M;
        sx[lvl] = Rx;
        sy[lvl] = Ry;
    }
    *out_m = sm[7];
    *out_c = make_double2(sx[7] / sm[7], sy[7] / sm[7]);
}

// Every cell (one thread each) writes its own record and its leaf children,
// and enters itself in its parent's child list: the parent is the cell of the
// deeper of the two boundaries around this cell's bodies (their levels are
// below the cell's; ties are two separators of the same parent), and the
// slot is the child's position among the parent's children in code order.
// Mass, COM and the packed FP32 record of cell id from two prefix sums
// (SPLIT monopoles; defined with the prefix kernels below, which run before
// the tree build).
__device__ void cell_from_prefix(const double4* __restrict__ prefix, const Tree& t,
                                 const DeviceScalars* __restrict__ s, const Batch& bt,
                                 const double2* __restrict__ pos, int id, int2 r, int level,
                                 float accept_scale);

// The SPLIT target groups of one cell (defined with tree_groups_write below).
template <bool kWrite>
__device__ int cell_groups(int2 rg, bool is_root, int nc, const int* ca, const int* cb,
                           const bool* leaf, int gsize, int fill, const Batch& bt,
                           const uint64_t* __restrict__ key, int2* __restrict__ out);

// Five blocks per SM (48 registers): more dependent load chains in flight
// than the 56-register build's four (tree phase 0.196 -> 0.192 ms at 4M).
// kMono (SPLIT monopoles): the prefix sums are ready, and each cell also
// writes its monopole record, which saves a pass over the cells.  gsize > 0
// (SPLIT): each cell also counts its target groups into gcount.
template <bool kMono>
__global__ void __launch_bounds__(kThreads, 5)
tree_link(const uint64_t* __restrict__ key, const uint8_t* __restrict__ lcp8, int n,
          const double2* __restrict__ pos, const double* __restrict__ mass, Tree t,
          DeviceScalars* __restrict__ s, const double4* __restrict__ prefix, Batch bt,
          float accept_scale, int gsize, int fill) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    const int cells = s->cells;
    if (id >= cells) {
        if (gsize > 0 && id < n) t.gcount[id] = 0;  // the group scan runs over n entries
        return;
    }
    const int i = t.rep_of[id];
    const int4 bi = t.bnd[i];
    const int c = lcp8[i];
    const int first = bi.x, last = bi.y;
    // the cell's separators: i, then the chain of next separators
    int sep[3] = {i, n - 1, n - 1};
    int ns = 1;
    for (int j = bi.w; j >= 0; j = t.bnd[j].w) {
        if (ns == 3) {  // a fifth child: the codes are inconsistent
            atomicOr(&s->error, kErrTree);
            break;
        }
        sep[ns++] = j;
    }
    int* child = reinterpret_cast<int*>(t.child + id);
    int nint = 0;
    int ca[4], cb[4];
    bool leaf[4];
    for (int q = 0; q <= ns; ++q) {
        const int a = q == 0 ? first : sep[q - 1] + 1;
        const int b = q == ns ? last : sep[q];
        ca[q] = a;
        cb[q] = b;
        leaf[q] = true;
        if (a == b) {
            child[q] = ~a;
            t.leaf_last[a] = a;
            t.leaf_plevel[a] = c;
        } else if (lcp8[a] == kMaxLevel && lcp_digits(key[a], key[b]) >= kMaxLevel) {
            // (a boundary below level 30 right after a makes the child a cell)
            child[q] = ~a;
            t.leaf_last[a] = b;
            t.leaf_plevel[a] = c;
            bucket_moments(pos, mass, a, b, t.bucket_mass + a, t.bucket_com + a);
        } else {
            leaf[q] = false;
            ++nint;  // a cell: it enters itself below
        }
    }
    if (gsize > 0)
        t.gcount[id] = cell_groups<false>(make_int2(first, last), first == 0 && last == n - 1,
                                          ns + 1, ca, cb, leaf, gsize, fill, bt, key, nullptr);
    for (int q = ns + 1; q < 4; ++q) child[q] = INT_MIN;
    t.range[id] = make_int2(first, last);
    t.level[id] = c;
    t.nint[id] = nint;
    t.ready[id] = 0;
    if (kMono) cell_from_prefix(prefix, t, s, bt, pos, id, make_int2(first, last), c, accept_scale);
    // cells whose children are all leaves start the bottom-up climb: listed
    // with one atomic per warp
    const unsigned active = __activemask();
    const unsigned starts = __ballot_sync(active, nint == 0);
    if (nint == 0) {
        const int leader = __ffs(starts) - 1;
        const int lane = threadIdx.x & 31;
        int base = 0;
        if (lane == leader) base = atomicAdd(&s->nstart, __popc(starts));
        base = __shfl_sync(starts, base, leader);
        t.start_list[base + __popc(starts & ((1u << lane) - 1u))] = id;
    }
    if (first == 0 && last == n - 1) {
        s->root = id;
        t.parent[id] = -1;
        return;
    }
    const int cl = first > 0 ? lcp8[first - 1] : -1;
    const int cr = last < n - 1 ? lcp8[last] : -1;
    const bool from_left = cl >= cr;
    int k = from_left ? first - 1 : last;  // a separator of the parent
    int rank = 0;  // its rank among the parent's separators; k ends at the first
    for (int p = t.bnd[k].z; p >= 0 && rank < 3; p = t.bnd[k].z) {
        k = p;
        ++rank;
    }
    const int slot = from_left ? rank + 1 : rank;
    if (slot > 3) {  // more than four children: the codes are inconsistent
        atomicOr(&s->error, kErrTree);
        return;
    }
    const int pid = t.cell_of[k];
    reinterpret_cast<int*>(t.child + pid)[slot] = id;
    t.parent[id] = pid;
}

// A tree without internal cells: one body, or all bodies in one level-30 leaf.
__global__ void tree_trivial_root(const double2* __restrict__ pos, const double* __restrict__ mass,
                                  int n, Tree t, DeviceScalars* __restrict__ s, int gsize) {
    if (s->cells != 0) return;
    if (gsize > 0) t.gcount[0] = (n + gsize - 1) / gsize;  // groups of the root leaf
    s->root = ~0;
    t.leaf_last[0] = n - 1;
    t.leaf_plevel[0] = -1;
    if (n > 1) bucket_moments(pos, mass, 0, n - 1, t.bucket_mass, t.bucket_com);
}

// Moments of one cell from its children, in quadrant order, with the
// reference's arithmetic (CU:329-343): M += m; R = fma(m, com, R); com = R / M.
// kSplit packs the FP32 records the group traversal reads.  kSecond (the
// quadrupole walk) also accumulates second moments
// about the COM by the parallel-axis rule, S = sum_c [S_c + m_c d_c d_c^T]
// with d_c = com_c - com, in FP64.  Leaves have S = 0 (a multi-body leaf
// spans less than width / 2^30, so its own S is negligible).
// Children are read with L2-coherent loads: other threads of this launch
// wrote them, published by the arrival counter's release/acquire.
// b_max^2 of a cell: squared distance from its COM to the farthest corner of
// its square.  The square is the cell's Morton prefix decoded in the box the
// codes were made in (the single box, or the cell's universe); forest cells
// above the universe roots are never accepted and get 0.
__device__ __forceinline__ double cell_bmax2(const DeviceScalars* s, const Batch& bt,
                                             const double2* __restrict__ pos, int first, int level,
                                             double2 com) {
    double2 lo;
    double w, scale;
    int bits, lvl = level;
    if (bt.nuni == 0) {
        lo = make_double2(s->box[0], s->box[2]);
        w = s->box[1] - s->box[0];
        scale = 4294967296.0;
        bits = 32;
    } else {
        if (level < kBatchUidDigits) return 0.0;
        const int u = bt.uid[first];
        lo = bt.lo[u];
        w = sqrt(bt.w2[u]);
        scale = (double)(1u << kBatchMortonBits);
        bits = kBatchMortonBits;
        lvl = level - kBatchUidDigits;
    }
    if (!(w > 0.0)) return 0.0;
    // the cell's column and row: the first body's grid coordinate, as the
    // Morton kernels compute it, cut to the cell's level
    const double inv_w = 1.0 / w, top = scale - 1.0;
    const double2 p = pos[first];
    const unsigned ix = __double2uint_rd(fmin(fmax((p.x - lo.x) * inv_w * scale, 0.0), top));
    const unsigned iy = __double2uint_rd(fmin(fmax((p.y - lo.y) * inv_w * scale, 0.0), top));
    const double wc = ldexp(w, -lvl);
    const double kx = lvl == 0 ? 0.0 : (double)(ix >> (bits - lvl));
    const double ky = lvl == 0 ? 0.0 : (double)(iy >> (bits - lvl));
    const double ax = fma(kx, wc, lo.x), ay = fma(ky, wc, lo.y);
    const double dx = fmax(fabs(ax - com.x), fabs(ax + wc - com.x));
    const double dy = fmax(fabs(ay - com.y), fabs(ay + wc - com.y));
    return dx * dx + dy * dy;
}

// The acceptance size the walk compares with theta^2 d^2: w^2, or with the
// b_max test max(w^2, b_max^2 theta^2 / ratio^2) (accept_scale =
// theta^2 / ratio^2), so that one comparison applies both tests.
__device__ __forceinline__ float accept_size2(const DeviceScalars* s, const Batch& bt,
                                              const double2* __restrict__ pos, int first,
                                              int level, double2 com, float accept_scale) {
    const double w2 = cell_width2(s, bt, first, level);
    if (accept_scale <= 0.f) return (float)w2;
    return (float)fmax(w2, cell_bmax2(s, bt, pos, first, level, com) * (double)accept_scale);
}

// Two floats rounded to BF16 (round to nearest even), lo in the low half.
__device__ __forceinline__ uint32_t bf16_pair(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

template <bool kSplit, bool kSecond>
__device__ __forceinline__ void cell_moments(int id, const DeviceScalars* __restrict__ s,
                                             const double2* __restrict__ pos,
                                             const double* __restrict__ mass, const Tree& t,
                                             const Batch& bt, float accept_scale) {
    const int4 ch = t.child[id];
    const int refs[4] = {ch.x, ch.y, ch.z, ch.w};
    double cm[4], cmx[4], cmy[4];
    double M = 0.0, Rx = 0.0, Ry = 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int r = refs[q];
        cm[q] = 0.0;
        cmx[q] = 0.0;
        cmy[q] = 0.0;
        if (r == INT_MIN) continue;
        double2 cc;
        if (r >= 0) {
            cm[q] = __ldcg(t.mass + r);
            cc = __ldcg(t.com + r);
        } else {
            const int b = ~r;
            if (t.leaf_last[b] == b) {
                cm[q] = mass[b];
                cc = pos[b];
            } else {
                cm[q] = t.bucket_mass[b];
                cc = t.bucket_com[b];
            }
        }
        cmx[q] = cc.x;
        cmy[q] = cc.y;
        M += cm[q];
        Rx = fma(cm[q], cc.x, Rx);
        Ry = fma(cm[q], cc.y, Ry);
    }
    const double2 com = make_double2(Rx / M, Ry / M);
    __stcg(t.mass + id, M);
    __stcg(t.com + id, com);
    if (kSplit && !kSecond) {
        const int first = t.range[id].x;
        const double2 fc = frame_center(s, bt, first);
        t.cell4[id] = make_float4((float)(com.x - fc.x), (float)(com.y - fc.y), (float)M,
                                  accept_size2(s, bt, pos, first, t.level[id], com, accept_scale));
    }
    if (kSplit && kSecond) {
        double sxx = 0.0, sxy = 0.0, syy = 0.0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = refs[q];
            if (r == INT_MIN) continue;
            if (r >= 0) {
                const double2* sc = reinterpret_cast<const double2*>(t.s64 + r);
                const double2 s01 = __ldcg(sc), s2 = __ldcg(sc + 1);
                sxx += s01.x;
                sxy += s01.y;
                syy += s2.x;
            }
            const double dx = cmx[q] - com.x, dy = cmy[q] - com.y;
            sxx += cm[q] * dx * dx;
            sxy += cm[q] * dx * dy;
            syy += cm[q] * dy * dy;
        }
        double2* so = reinterpret_cast<double2*>(t.s64 + id);
        __stcg(so, make_double2(sxx, sxy));
        __stcg(so + 1, make_double2(syy, 0.0));
        const int first = t.range[id].x;
        const double2 fc = frame_center(s, bt, first);
        t.cell4[id] = make_float4((float)(com.x - fc.x), (float)(com.y - fc.y), (float)M,
                                  accept_size2(s, bt, pos, first, t.level[id], com, accept_scale));
        // the walk's record carries 7.5 S, the factor of its (d.S.d) r^-7 term
        t.cellq[id] = make_float4((float)(7.5 * sxx), (float)(7.5 * sxy), (float)(7.5 * syy), 0.f);
    }
}

// Arrival at a parent: release publishes this cell's moments, acquire makes
// the siblings' moments visible to the thread that goes on to the parent.
__device__ __forceinline__ int arrive_acq_rel(int* counter) {
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;"
                 : "=r"(old)
                 : "l"(counter)
                 : "memory");
    return old;
}

// Bottom-up pass: threads start at cells without internal children and
// climb; the last child to arrive at a parent (atomic counter) computes it.
template <bool kSplit, bool kSecond>
__global__ void tree_moments(DeviceScalars* __restrict__ s, const double2* __restrict__ pos,
                             const double* __restrict__ mass, Tree t, Batch bt,
                             float accept_scale) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int cells = s->cells;
    if (k >= s->nstart) return;
    int id = t.start_list[k];
    // A path to the root crosses at most 30 cells; the bound only guards
    // against a malformed tree.
    for (int hop = 0;; ++hop) {
        if (hop > kMaxLevel + 1) {
            atomicOr(&s->error, kErrTree);
            return;
        }
        cell_moments<kSplit, kSecond>(id, s, pos, mass, t, bt, accept_scale);
        const int par = t.parent[id];
        if (par < 0) return;
        if (par >= cells) {
            atomicOr(&s->error, kErrTree);
            return;
        }
        const int arrived = arrive_acq_rel(t.ready + par);
        if (arrived != t.nint[par] - 1) return;
        id = par;
    }
}

// ---- SPLIT monopole moments from prefix sums ----------------------------
// A cell's bodies are one contiguous range of the sorted bodies, so its mass
// and first moment are differences of prefix sums over the bodies: one scan
// and one independent pass over the cells replace the bottom-up climb.  The
// sums are taken relative to each body's frame centre in FP64, so the
// cancellation in a difference stays far below the FP32 rounding of the cell
// records.  The FP64 parity mode (the reference's summation order) and the
// second and third moments (whose differences would cancel) keep the climb.
__device__ __forceinline__ double4 d4_add(double4 a, double4 b) {
    return make_double4(a.x + b.x, a.y + b.y, a.z + b.z, 0.0);
}

__device__ __forceinline__ double4 body_term(const double2* __restrict__ pos,
                                             const double* __restrict__ mass,
                                             const DeviceScalars* __restrict__ s, const Batch& bt,
                                             int i) {
    const double m = mass[i];
    const double2 p = pos[i], c = frame_center(s, bt, i);
    return make_double4(m, m * (p.x - c.x), m * (p.y - c.y), 0.0);
}

__device__ double4 block_sum_d4(double4 v, double4* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_down_sync(kFull, v.x, o);
        v.y += __shfl_down_sync(kFull, v.y, o);
        v.z += __shfl_down_sync(kFull, v.z, o);
    }
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double4 tot = make_double4(0.0, 0.0, 0.0, 0.0);
    if (threadIdx.x == 0)
        for (int w = 0; w < kThreads / 32; ++w) tot = d4_add(tot, red[w]);
    return tot;  // valid in thread 0
}

// Bodies of a tile are read in coalesced rows: warp w takes the kWarpItems
// bodies [w kWarpItems, (w + 1) kWarpItems) of the tile, lane l the bodies
// 32 k + l of them.
constexpr int kWarpItems = 32 * kScanItems;

// Phase 1: per tile of kScanTile bodies, the total.
__global__ void __launch_bounds__(kThreads)
prefix_reduce(const double2* __restrict__ pos, const double* __restrict__ mass, int n,
              const DeviceScalars* __restrict__ s, Batch bt, double4* __restrict__ tiles) {
    __shared__ double4 red[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int base = blockIdx.x * kScanTile + warp * kWarpItems + lane;
    double4 v = make_double4(0.0, 0.0, 0.0, 0.0);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + 32 * k < n) v = d4_add(v, body_term(pos, mass, s, bt, base + 32 * k));
    const double4 tot = block_sum_d4(v, red);
    if (threadIdx.x == 0) tiles[blockIdx.x] = tot;
}

// Inclusive scan across the warp of the three components body_term fills.
__device__ __forceinline__ double4 warp_inclusive_d4(double4 v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double x = __shfl_up_sync(kFull, v.x, o);
        const double y = __shfl_up_sync(kFull, v.y, o);
        const double z = __shfl_up_sync(kFull, v.z, o);
        if (lane >= o) {
            v.x += x;
            v.y += y;
            v.z += z;
        }
    }
    return v;
}

// Exclusive scan, in thread order, of one value per thread of the block.
__device__ double4 block_exclusive_d4(double4 v, double4* part, double4& total) {
    part[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < kThreads; o <<= 1) {
        const double4 t = threadIdx.x >= o ? part[threadIdx.x - o] : make_double4(0.0, 0.0, 0.0, 0.0);
        __syncthreads();
        part[threadIdx.x] = d4_add(part[threadIdx.x], t);
        __syncthreads();
    }
    total = part[kThreads - 1];
    const double4 ex = threadIdx.x > 0 ? part[threadIdx.x - 1] : make_double4(0.0, 0.0, 0.0, 0.0);
    __syncthreads();  // part[] is reused by the caller's next round
    return ex;
}

// Phase 2: exclusive scan of the tile totals (one block, chunks of
// kThreads * kScanItems tiles in order); tiles[ntiles] = the grand total.
__global__ void __launch_bounds__(kThreads) prefix_tiles_scan(double4* __restrict__ tiles, int ntiles) {
    __shared__ double4 part[kThreads];
    double4 carry = make_double4(0.0, 0.0, 0.0, 0.0);
    for (int c0 = 0; c0 < ntiles; c0 += kScanTile) {
        const int base = c0 + threadIdx.x * kScanItems;
        double4 v[kScanItems];
        double4 run = make_double4(0.0, 0.0, 0.0, 0.0);
        for (int k = 0; k < kScanItems; ++k) {
            v[k] = base + k < ntiles ? tiles[base + k] : make_double4(0.0, 0.0, 0.0, 0.0);
            run = d4_add(run, v[k]);
        }
        double4 total;
        double4 acc = d4_add(carry, block_exclusive_d4(run, part, total));
        for (int k = 0; k < kScanItems; ++k) {
            if (base + k < ntiles) tiles[base + k] = acc;
            acc = d4_add(acc, v[k]);
        }
        carry = d4_add(carry, total);
    }
    if (threadIdx.x == 0) tiles[ntiles] = carry;
}

// Phase 3: prefix[i] = sum over bodies before i; prefix[n] = the total.
// Each row of 32 bodies is scanned with shuffles; the rows' totals carry
// within the warp, and the warps' totals (one barrier) within the tile.
__global__ void __launch_bounds__(kThreads)
prefix_apply(const double2* __restrict__ pos, const double* __restrict__ mass, int n,
             const DeviceScalars* __restrict__ s, Batch bt, const double4* __restrict__ tiles,
             int ntiles, double4* __restrict__ prefix) {
    __shared__ double4 wtot[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int base = blockIdx.x * kScanTile + warp * kWarpItems + lane;
    const double4 zero = make_double4(0.0, 0.0, 0.0, 0.0);
    double4 ex[kScanItems];   // exclusive prefix within the row, then within the warp
    double4 carry = zero;     // total of the rows before
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int i = base + 32 * k;
        const double4 v = i < n ? body_term(pos, mass, s, bt, i) : zero;
        const double4 inc = warp_inclusive_d4(v);
        double4 e;
        e.x = __shfl_up_sync(kFull, inc.x, 1);
        e.y = __shfl_up_sync(kFull, inc.y, 1);
        e.z = __shfl_up_sync(kFull, inc.z, 1);
        e.w = 0.0;
        if (lane == 0) e = zero;
        ex[k] = d4_add(carry, e);
        const double4 row = make_double4(__shfl_sync(kFull, inc.x, 31), __shfl_sync(kFull, inc.y, 31),
                                         __shfl_sync(kFull, inc.z, 31), 0.0);
        carry = d4_add(carry, row);
    }
    if (lane == 0) wtot[warp] = carry;
    __syncthreads();
    double4 off = tiles[blockIdx.x];
    for (int w = 0; w < warp; ++w) off = d4_add(off, wtot[w]);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int i = base + 32 * k;
        if (i < n) prefix[i] = d4_add(off, ex[k]);
    }
    if (blockIdx.x == ntiles - 1 && threadIdx.x == 0) prefix[n] = tiles[ntiles];
}

__device__ void cell_from_prefix(const double4* __restrict__ prefix, const Tree& t,
                                 const DeviceScalars* __restrict__ s, const Batch& bt,
                                 const double2* __restrict__ pos, int id, int2 r, int level,
                                 float accept_scale) {
    const double4 a = prefix[r.x], b = prefix[r.y + 1];
    const double M = b.x - a.x;
    const double rx = (b.y - a.y) / M, ry = (b.z - a.z) / M;
    const double2 fc = frame_center(s, bt, r.x);
    const double2 com = make_double2(fc.x + rx, fc.y + ry);
    t.mass[id] = M;
    t.com[id] = com;
    t.cell4[id] = make_float4((float)rx, (float)ry, (float)M,
                              accept_size2(s, bt, pos, r.x, level, com, accept_scale));
}


// ---- learned features: second and third moments -------------------------
// The features need S and T about each cell's centre of mass, which the
// prefix pass has already written.  A cell with fewer than kDirectCell
// bodies, or with only leaf children, sums them directly over its bodies;
// a larger cell combines its children by the parallel-axis shift
//   S = sum_c [S_c + m_c d d^T]
//   T = sum_c [T_c + (d_i S_c,jk + d_j S_c,ik + d_k S_c,ij) + m_c d_i d_j d_k],
// bottom-up: a directly summed cell under a larger parent arrives at the
// parent's counter, and the last child to arrive computes the parent and
// climbs on.  Only the few cells above the direct size climb.  FP32: the
// moments only feed BF16 features.
constexpr int kDirectCell = 32;

__device__ __forceinline__ bool direct_cell(const Tree& t, int id) {
    const int2 r = t.range[id];
    return r.y - r.x < kDirectCell || t.nint[id] == 0;
}

__device__ __forceinline__ double child_mass(const Tree& t, const double* __restrict__ mass,
                                             int r) {
    if (r >= 0) return t.mass[r];
    const int b = ~r;
    return t.leaf_last[b] == b ? mass[b] : t.bucket_mass[b];
}

// The cell's feature record (the BF16 features, then COM, mass and width)
// and its S and T for the parent's shift.
__device__ void write_features(const Tree& t, const DeviceScalars* __restrict__ s,
                               const Batch& bt, const double* __restrict__ mass, int id,
                               const float* S, const float* T) {
    const int4 ch = t.child[id];
    const int refs[4] = {ch.x, ch.y, ch.z, ch.w};
    double mmax = 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q)
        if (refs[q] != INT_MIN) mmax = fmax(mmax, child_mass(t, mass, refs[q]));
    const double M = t.mass[id];
    const int first = t.range[id].x;
    const double w2 = cell_width2(s, bt, first, t.level[id]), w = sqrt(w2);
    const float im2 = (float)(1.0 / (M * w2)), im3 = (float)(1.0 / (M * w2 * w));
    __stcg(t.s32 + id, make_float4(S[0], S[1], S[2], 0.f));
    __stcg(t.t32 + id, make_float4(T[0], T[1], T[2], T[3]));
    const float4 c4 = t.cell4[id];
    t.cellh[2 * id] = make_uint4(bf16_pair((float)(mmax / M), S[0] * im2),
                                 bf16_pair(S[1] * im2, S[2] * im2),
                                 bf16_pair(T[0] * im3, T[1] * im3),
                                 bf16_pair(T[2] * im3, T[3] * im3));
    t.cellh[2 * id + 1] = make_uint4(__float_as_uint(c4.x), __float_as_uint(c4.y),
                                     __float_as_uint(c4.z), __float_as_uint((float)w));
}

// One mass point (or a child's moments) at offset (dx, dy) from the COM.
__device__ __forceinline__ void add_shifted(float m, float dx, float dy, const float4 cs,
                                            const float4 ct, float* S, float* T) {
    T[0] += ct.x + 3.f * dx * cs.x + m * dx * dx * dx;
    T[1] += ct.y + 2.f * dx * cs.y + dy * cs.x + m * dx * dx * dy;
    T[2] += ct.z + dx * cs.z + 2.f * dy * cs.y + m * dx * dy * dy;
    T[3] += ct.w + 3.f * dy * cs.z + m * dy * dy * dy;
    S[0] += cs.x + m * dx * dx;
    S[1] += cs.y + m * dx * dy;
    S[2] += cs.z + m * dy * dy;
}

__global__ void __launch_bounds__(kThreads)
learned_features(DeviceScalars* __restrict__ s, const double2* __restrict__ pos,
                 const double* __restrict__ mass, Tree t, Batch bt) {
    int id = blockIdx.x * blockDim.x + threadIdx.x;
    const int cells = s->cells;
    if (id >= cells || !direct_cell(t, id)) return;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    {
        const double2 com = t.com[id];
        const int2 r = t.range[id];
        float S[3] = {0.f, 0.f, 0.f}, T[4] = {0.f, 0.f, 0.f, 0.f};
        for (int j = r.x; j <= r.y; ++j) {
            const double2 p = pos[j];
            add_shifted((float)mass[j], (float)(p.x - com.x), (float)(p.y - com.y), zero, zero, S,
                        T);
        }
        write_features(t, s, bt, mass, id, S, T);
    }
    // A path to the root crosses at most 30 cells; the bound only guards
    // against a malformed tree.
    for (int hop = 0;; ++hop) {
        const int par = t.parent[id];
        if (par < 0) return;
        if (par >= cells || hop > kMaxLevel + 1) {
            atomicOr(&s->error, kErrTree);
            return;
        }
        if (direct_cell(t, par)) return;  // its own thread sums it
        const int arrived = arrive_acq_rel(t.ready + par);
        if (arrived != t.nint[par] - 1) return;
        id = par;
        const double2 com = t.com[id];
        const int4 ch = t.child[id];
        const int refs[4] = {ch.x, ch.y, ch.z, ch.w};
        float S[3] = {0.f, 0.f, 0.f}, T[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = refs[q];
            if (r == INT_MIN) continue;
            double2 cc;
            float4 cs = zero, ct = zero;
            if (r >= 0) {
                cc = t.com[r];
                cs = __ldcg(t.s32 + r);
                ct = __ldcg(t.t32 + r);
            } else {
                const int b = ~r;
                cc = t.leaf_last[b] == b ? pos[b] : t.bucket_com[b];
            }
            add_shifted((float)child_mass(t, mass, r), (float)(cc.x - com.x), (float)(cc.y - com.y),
                        cs, ct, S, T);
        }
        write_features(t, s, bt, mass, id, S, T);
    }
}

// ---- SPLIT target groups -----------------------------------------------
// A cell with more than gsize bodies hands its small children (cells or
// leaves with <= gsize bodies) to groups: consecutive small children are
// merged while the sum stays <= gsize, so a group never leaves its parent
// cell and its bounding box stays within one cell width.  With fill set, a
// child that would overflow the group is split instead: the group takes
// exactly gsize bodies and the child's rest starts the next group.  Multi-body
// leaves larger than a group are cut into chunks of gsize.  kWrite = false
// counts the groups of each cell, kWrite = true writes them at gbase[cell].
//
// Children in key order are quadrants 0..3; 0,1 and 2,3 are the two halves of
// the cell, while a run that takes quadrants from both halves has the whole
// cell as its bounding box.  When one child is large (it emits its own
// groups), such a box would cover that dense quadrant and the group's walk
// would open it down to its bodies: in a sparse disc tail, a group of outer
// bodies then walked the whole core on one warp (2.3 ms of a 65,536-body
// step).  So with a large child present, runs also end at the half boundary.
// The groups of one cell with body range rg and nc children in code order
// ([ca, cb], leaf marks the leaf children); returns their number and, with
// kWrite, writes them from out on.
template <bool kWrite>
__device__ int cell_groups(int2 rg, bool is_root, int nc, const int* ca, const int* cb,
                           const bool* leaf, int gsize, int fill, const Batch& bt,
                           const uint64_t* __restrict__ key, int2* __restrict__ out) {
    int emitted = 0;
    auto emit = [&](int a, int b) {
        if (kWrite) out[emitted] = make_int2(a, b);
        ++emitted;
    };
    // batched universes: a forest cell above the universe roots may hold few
    // bodies but never becomes a group; it hands its children on instead
    const bool spans = bt.nuni && bt.uid[rg.x] != bt.uid[rg.y];
    if (rg.y - rg.x + 1 <= gsize && !spans) {
        if (is_root) emit(rg.x, rg.y);  // the whole (small) tree is one group
        return emitted;
    }
    bool large = false;  // some child emits its own groups
    for (int q = 0; q < nc; ++q)
        large |= cb[q] - ca[q] + 1 > gsize || (bt.nuni && bt.uid[ca[q]] != bt.uid[cb[q]]);
    // the children differ in digit `level` of their codes; its high bit is
    // the half (read only when a large child makes it matter)
    const int level = large ? min(lcp_digits(key[rg.x], key[rg.y]), 31) : 0;
    int run_a = -1, run_b = -1, run_half = 0;
    for (int q = 0; q < nc; ++q) {
        const int a = ca[q], b = cb[q];
        const int cnt = b - a + 1;
        if (cnt > gsize || (bt.nuni && bt.uid[a] != bt.uid[b])) {  // the child emits
            if (run_a >= 0) emit(run_a, run_b);
            run_a = -1;
            if (leaf[q])  // oversized multi-body leaf: chunks of one group each
                for (int k = a; k <= b; k += gsize) emit(k, min(b, k + gsize - 1));
            continue;
        }
        const int half = large ? (int)(key[a] >> (63 - 2 * level)) & 1 : 0;
        // a group never spans two universes (a forest cell's children may),
        // nor both halves of a cell that has a large child
        if (run_a >= 0 && ((bt.nuni && bt.uid[a] != bt.uid[run_a]) ||
                           (large && half != run_half))) {
            emit(run_a, run_b);
            run_a = -1;
        } else if (run_a >= 0 && b - run_a + 1 > gsize) {
            if (fill) {
                // fill the group; the rest of this child starts the next one
                emit(run_a, run_a + gsize - 1);
                run_a += gsize;
                run_b = b;
                continue;
            }
            emit(run_a, run_b);
            run_a = -1;
        }
        if (run_a < 0) {
            run_a = a;
            run_half = half;
        }
        run_b = b;
    }
    if (run_a >= 0) emit(run_a, run_b);
    return emitted;
}

// Writes every cell's groups at gbase[cell] (the linking pass counted them).
__global__ void tree_groups_write(int n, int gsize, int fill, Tree t,
                                  const DeviceScalars* __restrict__ s, Batch bt,
                                  const uint64_t* __restrict__ key) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    const int cells = s->cells;
    if (id >= n) return;
    if (id >= cells) {
        if (cells == 0 && id == 0) {  // no cell: the root leaf holds all bodies
            const int ng = (n + gsize - 1) / gsize;
            for (int k = 0; k < ng; ++k)
                t.groups[k] = make_int2(k * gsize, min(n, (k + 1) * gsize) - 1);
        }
        return;
    }
    const int2 rg = t.range[id];
    const int4 ch = t.child[id];
    const int refs[4] = {ch.x, ch.y, ch.z, ch.w};
    int ca[4], cb[4], nc = 0;
    bool leaf[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int r = refs[q];
        if (r == INT_MIN) break;
        leaf[q] = r < 0;
        if (r >= 0) {
            const int2 cr = t.range[r];
            ca[q] = cr.x;
            cb[q] = cr.y;
        } else {
            ca[q] = ~r;
            cb[q] = t.leaf_last[ca[q]];
        }
        nc = q + 1;
    }
    cell_groups<true>(rg, id == s->root, nc, ca, cb, leaf, gsize, fill, bt, key,
                      t.groups + t.gbase[id]);
}

// Root reference of each universe: the cell whose body range is exactly the
// universe's (found like a child cell in tree_link), or its single leaf.
__global__ void batch_roots(const uint64_t* __restrict__ key, Tree t, Batch bt) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= bt.nuni) return;
    const int a = bt.off[u], b = bt.off[u + 1] - 1;
    if (b <= a) {
        bt.root[u] = ~a;
        return;
    }
    const int c = lcp_digits(key[a], key[b]);
    if (c >= kMaxLevel) {  // all bodies of the universe in one level-30 leaf
        bt.root[u] = ~a;
        return;
    }
    bt.root[u] = t.cell_of[gallop_right(key, a, b, c + 1)];
}

inline unsigned blocks_for(int64_t n, int threads) {
    return (unsigned)((n + threads - 1) / threads);
}

}  // namespace

void launch_batch_roots(nb_ctx* c) {
    if (c->batch.nuni == 0) return;
    c->launches += 1;
    batch_roots<<<blocks_for(c->batch.nuni, 128), 128, 0, c->stream>>>(c->sort.key[0], c->tree,
                                                                      c->batch);
}

void launch_groups(nb_ctx* c) {
    const int n = (int)c->n;
    const int sblocks = (int)blocks_for(n, kScanTile);
    c->launches += 4;
    const int gsize = split_group_size(c);
    // plain SPLIT fills groups to gsize bodies across sibling cells (fuller
    // warps, measured 2.6% off the walk at 4M with slightly lower errors); the
    // learned correction keeps groups of whole cells, whose residuals it fits.
    // The linking pass counted every cell's groups; scan, then write them.
    const int fill = (c->p.flags & NB_FLAG_LEARNED) ? 0 : 1;
    scan_reduce<<<sblocks, kThreads, 0, c->stream>>>(c->tree.gcount, n, c->scan.block_sums);
    scan_block_sums<<<1, kSumsThreads, 0, c->stream>>>(c->scan.block_sums, sblocks, &c->scal->groups);
    scan_apply<<<sblocks, kThreads, 0, c->stream>>>(c->tree.gcount, n, c->scan.block_sums,
                                                     c->tree.gbase, nullptr);
    tree_groups_write<<<blocks_for(n, kThreads), kThreads, 0, c->stream>>>(
        n, gsize, fill, c->tree, c->scal, c->batch, c->sort.key[0]);
}

// SPLIT without quadrupoles takes its monopoles from prefix sums over the
// sorted bodies, which the linking pass turns into cell records.
static bool mono_prefix(const nb_ctx* c) {
    return c->p.mode == NB_MODE_SPLIT && !(c->p.flags & NB_FLAG_QUADRUPOLE);
}

// The acceptance-size factor of the b_max test (0 = plain width test).
static float split_accept_scale(const nb_ctx* c) {
    const double ratio = c->p.bmax_ratio;
    return c->p.mode == NB_MODE_SPLIT && ratio > 0.0
               ? (float)(c->p.theta * c->p.theta / (ratio * ratio))
               : 0.f;
}

void launch_prefix_sums(nb_ctx* c, const BodyBuffers& b) {
    if (!mono_prefix(c)) return;
    const int n = (int)c->n;
    {  // the prefix sums need only the sorted bodies
        const int ptiles = (int)blocks_for(n, kScanTile);
        c->launches += 3;
        prefix_reduce<<<ptiles, kThreads, 0, c->stream>>>(b.pos, b.mass, n, c->scal, c->batch,
                                                          c->tree.prefix_tiles);
        prefix_tiles_scan<<<1, kThreads, 0, c->stream>>>(c->tree.prefix_tiles, ptiles);
        prefix_apply<<<ptiles, kThreads, 0, c->stream>>>(b.pos, b.mass, n, c->scal, c->batch,
                                                         c->tree.prefix_tiles, ptiles,
                                                         c->tree.prefix);
    }
}

void launch_tree(nb_ctx* c, const BodyBuffers& b, bool prefix_done) {
    const int n = (int)c->n;
    const bool mono = mono_prefix(c);
    if (mono && !prefix_done) launch_prefix_sums(c, b);
    const uint64_t* key = c->sort.key[0];
    Tree& t = c->tree;
    const int tiles = (int)blocks_for(n, kAnsvTile);
    c->launches += 8;
    tree_lcp<<<tiles, kThreads, 0, c->stream>>>(key, n, tiles, t.lcp8, t.ansv_first, t.ansv_last,
                                                c->scal->lcp_hist);
    tree_ansv_tiles<<<kAnsvLevels, kTileScanThreads, 0, c->stream>>>(tiles, t.ansv_first,
                                                                     t.ansv_last);
    tree_ansv<<<tiles, kThreads, 0, c->stream>>>(t.lcp8, n, tiles, t.ansv_first, t.ansv_last,
                                                 t.flag, t.bnd);
    const int sblocks = (int)blocks_for(n, kScanTile);
    scan_reduce<<<sblocks, kThreads, 0, c->stream>>>(t.flag, n, c->scan.block_sums);
    scan_block_sums<<<1, kSumsThreads, 0, c->stream>>>(c->scan.block_sums, sblocks, &c->scal->cells);
    scan_apply<<<sblocks, kThreads, 0, c->stream>>>(t.flag, n, c->scan.block_sums, t.cell_of,
                                                     t.rep_of);
    cudaMemsetAsync(&c->scal->nstart, 0, sizeof(int32_t), c->stream);
    // SPLIT: the cells count their target groups as they link
    const int gsize = c->p.mode == NB_MODE_SPLIT ? split_group_size(c) : 0;
    const int fill = (c->p.flags & NB_FLAG_LEARNED) ? 0 : 1;
    if (mono)
        tree_link<true><<<blocks_for(n, kThreads), kThreads, 0, c->stream>>>(
            key, t.lcp8, n, b.pos, b.mass, t, c->scal, t.prefix, c->batch, split_accept_scale(c),
            gsize, fill);
    else
        tree_link<false><<<blocks_for(n, kThreads), kThreads, 0, c->stream>>>(
            key, t.lcp8, n, b.pos, b.mass, t, c->scal, nullptr, c->batch, 0.f, gsize, fill);
    tree_trivial_root<<<1, 1, 0, c->stream>>>(b.pos, b.mass, n, t, c->scal, gsize);
}

void launch_features(nb_ctx* c, const BodyBuffers& b) {
    const int cap = (int)(c->n > 1 ? c->n - 1 : 1);
    c->launches += 1;
    learned_features<<<blocks_for(cap, kThreads), kThreads, 0, c->stream>>>(c->scal, b.pos, b.mass,
                                                                           c->tree, c->batch);
}

void launch_moments(nb_ctx* c, const BodyBuffers& b, bool split) {
    // Cells never exceed n - 1; threads beyond the live count exit at once.
    const int cap = (int)(c->n > 1 ? c->n - 1 : 1);
    const bool second = split && (c->p.flags & NB_FLAG_QUADRUPOLE);
    const double ratio = c->p.bmax_ratio;
    const float accept_scale =
        split && ratio > 0.0 ? (float)(c->p.theta * c->p.theta / (ratio * ratio)) : 0.f;
    const unsigned blocks = blocks_for(cap, kThreads);
    if (second) {
        c->launches += 1;
        tree_moments<true, true><<<blocks, kThreads, 0, c->stream>>>(c->scal, b.pos, b.mass, c->tree,
                                                                     c->batch, accept_scale);
    } else if (split) {
        // monopoles: the prefix sums ran before the tree, and the linking
        // pass wrote every cell's record from them
    } else {
        c->launches += 1;
        tree_moments<false, false><<<blocks, kThreads, 0, c->stream>>>(c->scal, b.pos, b.mass,
                                                                       c->tree, c->batch, 0.f);
    }
}

}  // namespace nb
