// k_force32.cu -- SPLIT mode: warp-cooperative group traversal in FP32 with
// shared-memory interaction lists, fused with the FP64 kick and drift.
//
// One warp owns a group of 32 Morton-consecutive bodies (one per lane) and
// walks the tree once for the whole group.  Each round the warp pops up to 32
// cells from its shared-memory stack, one per lane, and decides for each:
//   * accept: the cell does not hold a body of the group and
//     width^2 < theta^2 d^2, d = distance from the cell's centre of mass to
//     the group's bounding box (so every body of the group passes the
//     reference's per-body test width^2 < theta^2 d_i^2 of CU:463);
//     the cell joins the cell list;
//   * summed directly: a cell with at most leaf_size bodies, or a leaf; its
//     bodies join the body list;
//   * opened: its children are pushed.
// Whenever a list holds 32 entries, every lane sums them for its own body,
// reading entries by broadcast from shared memory.  Cells contribute their
// monopole (the reference's pair law, CU:427-431) and, with quadrupoles on,
// the second-moment term of the softened potential.  Accelerations
// accumulate in FP32; velocities and positions are updated in FP64.
#include <cfloat>
#include <climits>
#include <cuda_runtime.h>
#include <stdint.h>

#include "nb_internal.cuh"

namespace nb {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarpsPerBlock = 4;
constexpr int kStk = 256;              // stack bound kept by the batch size rule
constexpr int kStkAlloc = kStk + 96;   // + one depth-first descent (<= 3 x 30 + 1)
constexpr int kList = 64;
constexpr int kBodiesPerLane = 2;      // group of 64 bodies per warp
constexpr int kDefaultLeaf = 8;        // cells this small are summed body by body
constexpr int kMaxBPL = 4;             // largest group: 128 bodies per warp

// Interaction lists hold entries in pairs, so that one lane evaluates two
// entries with the packed FP32x2 instructions of sm_100 (FADD2/FMUL2/FFMA2):
// pair k is xy[k] = (x0, x1, y0, y1) and m[k] = (m0, m1), with the quadrupole
// (xx0, xx1, xy0, xy1) in qa[k] and (yy0, yy1) in qb[k].
struct WarpLists {
    int stack[kStkAlloc];
    float4 cxy[kList / 2];
    float2 cm[kList / 2];
    float4 qa[kList / 2];
    float2 qb[kList / 2];
    float4 bxy[kList / 2];
    float2 bm[kList / 2];
    float2 tot[2 * kMaxBPL][32];   // running {x, y} sums of each lane's bodies (halves kept apart)
};

// An entry that adds nothing: zero mass far away, so that d2 stays finite
// and positive whatever eps2 is (it completes a pair at an odd count).
constexpr float kPadCoord = 1e15f;

// 1/sqrt(x) on the special-function unit.  kExact keeps subnormal x (the
// eps2 = 0 variant, where d2 can be that small); otherwise x >= eps2 is a
// normal float and the flush-to-zero form saves the subnormal handling.
template <bool kExact>
__device__ __forceinline__ float rsq(float x) {
    if (kExact) return rsqrtf(x);
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void put_entry(float4* xy, float2* m, int slot, float x, float y,
                                          float mass) {
    float* f = reinterpret_cast<float*>(xy + (slot >> 1));
    f[slot & 1] = x;
    f[2 + (slot & 1)] = y;
    reinterpret_cast<float*>(m)[slot] = mass;
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ int warp_exclusive_sum(int v, int& total) {
    const int lane = threadIdx.x & 31;
    int inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc += t;
    }
    total = __shfl_sync(kFull, inc, 31);
    return inc - v;
}

__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(kFull, v, o));
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

// One pair of list entries against the lane's kBPL bodies.  nx/ny hold the
// negated body coordinates broadcast to both halves.  Each half follows the
// scalar law d2 = dx^2 + (dy^2 + eps2), a = (m / r^2) / r of the reference's
// pair term (CU:427-431) with the same rounding; the halves are separate
// partial sums.  kZeroSoft: eps2 = 0, where an entry at the body's own FP32
// coordinates (the body itself, or one that coincides with it at FP32
// resolution) adds nothing instead of 0 * inf, and 1/sqrt keeps subnormal
// arguments.  With eps2 > 0 the body's own entry has dx = dy = 0 exactly and
// adds 0 without a test.
template <bool kZeroSoft, int kBPL>
__device__ __forceinline__ void mono_pair(const float4 xy, const float2 m, const float2* nx,
                                          const float2* ny, const float2 e2, float2* ax,
                                          float2* ay) {
    const float2 ex = make_float2(xy.x, xy.y), ey = make_float2(xy.z, xy.w);
#pragma unroll
    for (int b = 0; b < kBPL; ++b) {
        const float2 dx = __fadd2_rn(ex, nx[b]);
        const float2 dy = __fadd2_rn(ey, ny[b]);
        const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, e2));
        const float2 inv = make_float2(rsq<kZeroSoft>(d2.x), rsq<kZeroSoft>(d2.y));
        float2 a = __fmul2_rn(__fmul2_rn(m, __fmul2_rn(inv, inv)), inv);
        if (kZeroSoft) {
            a.x = d2.x == 0.f ? 0.f : a.x;
            a.y = d2.y == 0.f ? 0.f : a.y;
        }
        ax[b] = __ffma2_rn(dx, a, ax[b]);
        ay[b] = __ffma2_rn(dy, a, ay[b]);
    }
}

// Monopole plus the second-moment term of the softened potential,
//   a = d [M r^-3 - 1.5 tr(S) r^-5 + 7.5 (d.S.d) r^-7] - 3 r^-5 S d,
// from the cell record Q = 7.5 S (the moments pass stores it so) as
//   a = d r^-3 [M + r^-2 (-0.2 tr(Q) + r^-2 (d.Q.d))] - 0.4 r^-3 r^-2 Q d:
// 21 packed FMA-pipe operations per body and pair (23 in the textbook order).
// The walk is FMA-pipe bound with quadrupoles, so the count is the cost.
template <bool kZeroSoft, int kBPL>
__device__ __forceinline__ void quad_pair(const float4 xy, const float2 m, const float4 qa,
                                          const float2 qb, const float2* nx, const float2* ny,
                                          const float2 e2, float2* ax, float2* ay) {
    const float2 ex = make_float2(xy.x, xy.y), ey = make_float2(xy.z, xy.w);
    const float2 qxx = make_float2(qa.x, qa.y), qxy = make_float2(qa.z, qa.w), qyy = qb;
    const float2 tr = __fmul2_rn(make_float2(-0.2f, -0.2f), __fadd2_rn(qxx, qyy));
    const float2 m04 = make_float2(-0.4f, -0.4f);
#pragma unroll
    for (int b = 0; b < kBPL; ++b) {
        const float2 dx = __fadd2_rn(ex, nx[b]);
        const float2 dy = __fadd2_rn(ey, ny[b]);
        const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, e2));
        const float2 inv = make_float2(rsq<kZeroSoft>(d2.x), rsq<kZeroSoft>(d2.y));
        const float2 inv2 = __fmul2_rn(inv, inv);
        const float2 inv3 = __fmul2_rn(inv, inv2);
        const float2 sdx = __ffma2_rn(qxx, dx, __fmul2_rn(qxy, dy));
        const float2 sdy = __ffma2_rn(qxy, dx, __fmul2_rn(qyy, dy));
        const float2 dsd = __ffma2_rn(dx, sdx, __fmul2_rn(dy, sdy));
        const float2 radial = __fmul2_rn(__ffma2_rn(__ffma2_rn(dsd, inv2, tr), inv2, m), inv3);
        const float2 k5 = __fmul2_rn(inv3, __fmul2_rn(m04, inv2));
        ax[b] = __ffma2_rn(dx, radial, __ffma2_rn(k5, sdx, ax[b]));
        ay[b] = __ffma2_rn(dy, radial, __ffma2_rn(k5, sdy, ay[b]));
    }
}

// Every kFoldFlushes list flushes, the lane's register sums are added to the
// body's running totals, kept in the warp's shared lists, and restart from
// zero (blocked summation): the FP32 rounding of a body's total then grows
// with the block length plus the number of blocks, not with the number of
// terms (a body's terms mostly share their sign, so a running sum's rounding
// adds up).  The totals live in shared memory so that the blocking costs no
// registers, and a block spans four flushes so that it costs few
// instructions.
constexpr int kFoldFlushes = 4;
template <int kBPL>
__device__ __forceinline__ void fold_block(WarpLists& L, float2* ax, float2* ay) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int b = 0; b < kBPL; ++b) {
        L.tot[2 * b][lane] = __fadd2_rn(L.tot[2 * b][lane], ax[b]);
        L.tot[2 * b + 1][lane] = __fadd2_rn(L.tot[2 * b + 1][lane], ay[b]);
        ax[b] = ay[b] = make_float2(0.f, 0.f);
    }
}

// Sum the first npairs pairs of the cell list.
template <bool kQuad, bool kZeroSoft, int kBPL>
__device__ __forceinline__ void sum_cells(WarpLists& L, int npairs, const float2* nx,
                                          const float2* ny, const float2 e2, float2* ax,
                                          float2* ay, bool fold) {
    if (npairs == 16) {
#pragma unroll 4
        for (int k = 0; k < 16; ++k) {
            if (kQuad)
                quad_pair<kZeroSoft, kBPL>(L.cxy[k], L.cm[k], L.qa[k], L.qb[k], nx, ny, e2, ax,
                                           ay);
            else
                mono_pair<kZeroSoft, kBPL>(L.cxy[k], L.cm[k], nx, ny, e2, ax, ay);
        }
    } else {
        for (int k = 0; k < npairs; ++k) {
            if (kQuad)
                quad_pair<kZeroSoft, kBPL>(L.cxy[k], L.cm[k], L.qa[k], L.qb[k], nx, ny, e2, ax,
                                           ay);
            else
                mono_pair<kZeroSoft, kBPL>(L.cxy[k], L.cm[k], nx, ny, e2, ax, ay);
        }
    }
    if (fold) fold_block<kBPL>(L, ax, ay);
}

template <bool kZeroSoft, int kBPL>
__device__ __forceinline__ void sum_bodies(WarpLists& L, int npairs, const float2* nx,
                                           const float2* ny, const float2 e2, float2* ax,
                                           float2* ay, bool fold) {
    if (npairs == 16) {
#pragma unroll 4
        for (int k = 0; k < 16; ++k)
            mono_pair<kZeroSoft, kBPL>(L.bxy[k], L.bm[k], nx, ny, e2, ax, ay);
    } else {
        for (int k = 0; k < npairs; ++k)
            mono_pair<kZeroSoft, kBPL>(L.bxy[k], L.bm[k], nx, ny, e2, ax, ay);
    }
    if (fold) fold_block<kBPL>(L, ax, ay);
}

// Walk the tree for one group [g0, g1] of <= 32 kBPL bodies (lane l owns
// g0 + l, g0 + 32 + l, ...) and accumulate the FP32 accelerations.
template <bool kQuad, int kBPL, bool kLearned, bool kZeroSoft>
__device__ __forceinline__ void walk_group(WarpLists& L, const Tree& t, int root, int n, int g0,
                                           int g1, const float* px, const float* py,
                                           const bool* act_body, float eps2, float theta2,
                                           int leaf_size, float* ax, float* ay,
                                           unsigned long long& ncell, unsigned long long& npair,
                                           unsigned* err, int* band, int& nband, int band_cap,
                                           float band2) {
    const int lane = threadIdx.x & 31;
    float bx0 = INFINITY, bx1 = -INFINITY, by0 = INFINITY, by1 = -INFINITY;
#pragma unroll
    for (int b = 0; b < kBPL; ++b)
        if (act_body[b]) {
            bx0 = fminf(bx0, px[b]);
            bx1 = fmaxf(bx1, px[b]);
            by0 = fminf(by0, py[b]);
            by1 = fmaxf(by1, py[b]);
        }
    bx0 = warp_min(bx0);
    bx1 = warp_max(bx1);
    by0 = warp_min(by0);
    by1 = warp_max(by1);
    const float gcx = 0.5f * (bx0 + bx1), gcy = 0.5f * (by0 + by1);
    const float ghx = 0.5f * (bx1 - bx0), ghy = 0.5f * (by1 - by0);
    const unsigned below = lanemask_lt();
    // packed operands: the body broadcast to both halves, negated
    float2 nx[kBPL], ny[kBPL], ax2[kBPL], ay2[kBPL];
#pragma unroll
    for (int b = 0; b < kBPL; ++b) {
        nx[b] = make_float2(-px[b], -px[b]);
        ny[b] = make_float2(-py[b], -py[b]);
        ax2[b] = make_float2(0.f, 0.f);
        ay2[b] = make_float2(0.f, 0.f);
    }
    const float2 e2 = make_float2(eps2, eps2);
    ncell = 0;
    npair = 0;
#pragma unroll
    for (int b = 0; b < kBPL; ++b) L.tot[2 * b][lane] = L.tot[2 * b + 1][lane] = make_float2(0.f, 0.f);
    int ccount = 0, bcount = 0, size = 1;
    int flushes = 0;  // warp-uniform: every lane takes part in every flush
    if (lane == 0) L.stack[0] = root;
    __syncwarp();

    while (size > 0) {
        int k = min(32, size);
        k = min(k, max(1, (kStk - size) / 3));
        const int ref = lane < k ? L.stack[size - k + lane] : 0;
        size -= k;
        __syncwarp();
        int act = 0;  // 1 accept, 2 bodies, 3 open
        int bfirst = 0, bcnt = 0;
        int4 ch = make_int4(INT_MIN, INT_MIN, INT_MIN, INT_MIN);
        float4 c4 = make_float4(0.f, 0.f, 0.f, 0.f);
        float band_d2 = 0.f;
        if (lane < k) {
            // the tree is read-only while the walk runs: non-coherent loads
            if (ref >= 0) {
                c4 = __ldg(t.cell4 + ref);
                const int2 rg = __ldg(t.range + ref);
                const bool overlap = !(rg.y < g0 || rg.x > g1);
                const float dx = fmaxf(fabsf(c4.x - gcx) - ghx, 0.f);
                const float dy = fmaxf(fabsf(c4.y - gcy) - ghy, 0.f);
                const float d2 = fmaf(dx, dx, dy * dy);
                band_d2 = d2;
                if (!overlap && c4.w < theta2 * d2) {
                    act = 1;
                } else if (rg.y - rg.x < leaf_size) {
                    act = 2;
                    bfirst = rg.x;
                    bcnt = rg.y - rg.x + 1;
                } else {
                    act = 3;
                    ch = __ldg(t.child + ref);
                }
            } else {
                const int b = ~ref;
                act = 2;
                bfirst = b;
                bcnt = max(0, min(t.leaf_last[b], n - 1) - b + 1);
            }
        }
        // accepted cells
        const unsigned acc_mask = __ballot_sync(kFull, act == 1);
        if (act == 1) {
            const int slot = ccount + __popc(acc_mask & below);
            put_entry(L.cxy, L.cm, slot, c4.x, c4.y, c4.z);
            if (kQuad) {
                const float4 q = t.cellq[ref];
                put_entry(L.qa, L.qb, slot, q.x, q.y, q.z);
            }
        }
        if (kLearned) {
            // band: accepted here but opened by the plain theta_B walk
            const bool in_band = act == 1 && c4.w >= band2 * band_d2;
            const unsigned bm = __ballot_sync(kFull, in_band);
            if (in_band) {
                const int slot = nband + __popc(bm & below);
                if (slot < band_cap) band[slot] = ref;
            }
            nband += __popc(bm);
        }
        ccount += __popc(acc_mask);
        __syncwarp();
        if (ccount >= 32) {
            sum_cells<kQuad, kZeroSoft, kBPL>(L, 16, nx, ny, e2, ax2, ay2,
                                              ++flushes % kFoldFlushes == 0);
            ncell += 32;
            __syncwarp();
            // pairs 16.. move down; source and destination never overlap
            if (lane < (ccount - 31) / 2) {
                L.cxy[lane] = L.cxy[16 + lane];
                L.cm[lane] = L.cm[16 + lane];
                if (kQuad) {
                    L.qa[lane] = L.qa[16 + lane];
                    L.qb[lane] = L.qb[16 + lane];
                }
            }
            ccount -= 32;
            __syncwarp();
        }
        // opened cells push their children
        const int nch = act == 3 ? (ch.y == INT_MIN ? 1 : ch.z == INT_MIN ? 2 : ch.w == INT_MIN ? 3 : 4)
                                 : 0;
        int pushed;
        const int off = warp_exclusive_sum(nch, pushed);
        if (size + pushed > kStkAlloc) {  // excluded by the batch rule; stop safely
            if (lane == 0) atomicOr(err, kErrStack);
            break;
        }
        if (act == 3) {
            int* dst = L.stack + size + off;
            dst[0] = ch.x;
            if (nch > 1) dst[1] = ch.y;
            if (nch > 2) dst[2] = ch.z;
            if (nch > 3) dst[3] = ch.w;
        }
        size += pushed;
        // bodies of directly summed cells and leaves, expanded 32 at a time
        int btot;
        const int boff = warp_exclusive_sum(bcnt, btot);
        for (int base = 0; base < btot; base += 32) {
            const int item = base + lane;
            int owner = 0;
#pragma unroll
            for (int st = 16; st > 0; st >>= 1) {
                const int cand = owner + st;
                const int o = __shfl_sync(kFull, boff, cand);
                if (item >= o) owner = cand;
            }
            const int j = __shfl_sync(kFull, bfirst, owner) + item - __shfl_sync(kFull, boff, owner);
            const int added = min(32, btot - base);
            __syncwarp();
            if (lane < added) {
                const float4 b4 = __ldg(t.body4 + j);
                put_entry(L.bxy, L.bm, bcount + lane, b4.x, b4.y, b4.z);
            }
            bcount += added;
            __syncwarp();
            if (bcount >= 32) {
                sum_bodies<kZeroSoft, kBPL>(L, 16, nx, ny, e2, ax2, ay2,
                                            ++flushes % kFoldFlushes == 0);
                npair += 32;
                __syncwarp();
                if (lane < (bcount - 31) / 2) {
                    L.bxy[lane] = L.bxy[16 + lane];
                    L.bm[lane] = L.bm[16 + lane];
                }
                bcount -= 32;
                __syncwarp();
            }
        }
    }
    // odd counts: a padding entry completes the last pair
    if (lane == 0) {
        if (ccount & 1) {
            put_entry(L.cxy, L.cm, ccount, kPadCoord, kPadCoord, 0.f);
            if (kQuad) put_entry(L.qa, L.qb, ccount, 0.f, 0.f, 0.f);
        }
        if (bcount & 1) put_entry(L.bxy, L.bm, bcount, kPadCoord, kPadCoord, 0.f);
    }
    __syncwarp();
    sum_cells<kQuad, kZeroSoft, kBPL>(L, (ccount + 1) >> 1, nx, ny, e2, ax2, ay2, false);
    sum_bodies<kZeroSoft, kBPL>(L, (bcount + 1) >> 1, nx, ny, e2, ax2, ay2, true);
    ncell += ccount;
    npair += bcount;
#pragma unroll
    for (int b = 0; b < kBPL; ++b) {
        const float2 tx = L.tot[2 * b][lane], ty = L.tot[2 * b + 1][lane];
        ax[b] = tx.x + tx.y;
        ay[b] = ty.x + ty.y;
    }
    __syncwarp();
}

// Persistent: each warp takes groups from a global ticket until none is left,
// which balances groups of very different cost.
template <bool kQuad, int kBPL, bool kLearned, bool kZeroSoft>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
force_split(double2* __restrict__ pos, double2* __restrict__ vel, double2* __restrict__ acc_out,
            float2* __restrict__ acc32, int n, Tree t, DeviceScalars* __restrict__ s, Batch bt,
            float eps2, float theta2, int leaf_size, double G_dt, double dt, int kick,
            float band2) {
    __shared__ WarpLists lists[kWarpsPerBlock];
    const int lane = threadIdx.x & 31;
    WarpLists& L = lists[threadIdx.x >> 5];
    const int ngroups = s->groups;
    unsigned long long cells_total = 0, pairs_total = 0;
    while (true) {
        int g = 0;
        if (lane == 0) g = (int)atomicAdd(&s->group_ticket, 1u);
        g = __shfl_sync(kFull, g, 0);
        if (g >= ngroups) break;
        const int2 gr = t.groups[g];
        const int g0 = gr.x, g1 = min(gr.y, n - 1);
        // batched universes: walk the group's own universe from its root
        const int root = bt.nuni ? bt.root[bt.uid[g0]] : s->root;
        const double2 fc = frame_center(s, bt, g0);
        const double cx = fc.x, cy = fc.y;
        int me[kBPL];
        bool on[kBPL];
        float px[kBPL], py[kBPL], ax[kBPL], ay[kBPL];
        double2 P[kBPL];
#pragma unroll
        for (int b = 0; b < kBPL; ++b) {
            on[b] = g0 + 32 * b + lane <= g1;
            me[b] = min(g0 + 32 * b + lane, g1);
            P[b] = pos[me[b]];
            px[b] = (float)(P[b].x - cx);
            py[b] = (float)(P[b].y - cy);
        }
        unsigned long long ncell, npair;
        int nband = 0;
        int* band = kLearned ? t.band + (int64_t)kBandPerBody * g0 : nullptr;
        walk_group<kQuad, kBPL, kLearned, kZeroSoft>(L, t, root, n, g0, g1, px, py, on, eps2, theta2,
                                          leaf_size, ax, ay, ncell, npair, &s->error, band, nband,
                                          kBandPerBody * (g1 - g0 + 1), band2);
        if (kLearned) {
            // the correction kernel adds the learned term, then kicks and drifts
            if (lane == 0) t.band_count[g] = nband;
#pragma unroll
            for (int b = 0; b < kBPL; ++b)
                if (on[b]) acc32[me[b]] = make_float2(ax[b], ay[b]);
        }
#pragma unroll
        for (int b = 0; b < kBPL; ++b) {
            if (kLearned || !on[b]) continue;
            const int i = me[b];
            if (acc_out) acc_out[i] = make_double2((double)ax[b], (double)ay[b]);
            if (kick) {
                double2 v = vel[i];
                v.x += (double)ax[b] * G_dt;
                v.y += (double)ay[b] * G_dt;
                vel[i] = v;
                double2 p = P[b];
                p.x += v.x * dt;
                p.y += v.y * dt;
                pos[i] = p;
            }
        }
        // every body of the group summed every entry and skipped itself once
        const unsigned long long bodies = (unsigned long long)(g1 - g0 + 1);
        cells_total += ncell * bodies;
        pairs_total += npair * bodies - bodies;
    }
    if (lane == 0) {
        atomicAdd(&s->cell_terms, cells_total);
        atomicAdd(&s->body_terms, pairs_total);
    }
}

template <bool kQuad, int kBPL, bool kLearned, bool kZeroSoft>
void launch_split_soft(nb_ctx* c, const BodyBuffers& b, bool kick, bool store_acc, float eps2) {
    int& grid = c->split_blocks[(kQuad ? 1 : 0) + (kLearned ? 2 : 0) + (kBPL == 1 ? 4 : 0) +
                                (kBPL == 4 ? 16 : 0) +
                                (kZeroSoft ? 8 : 0)];
    if (grid == 0) {
        int blocks = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &blocks, force_split<kQuad, kBPL, kLearned, kZeroSoft>, kWarpsPerBlock * 32, 0) !=
                    cudaSuccess ||
            blocks < 1)
            blocks = 4;
        grid = c->sm_count * blocks;
    }
    const float theta2 = (float)(c->p.theta * c->p.theta);
    const int leaf = c->p.leaf_size > 0 ? c->p.leaf_size : kDefaultLeaf;
    force_split<kQuad, kBPL, kLearned, kZeroSoft><<<grid, 32 * kWarpsPerBlock, 0, c->stream>>>(
        b.pos, b.vel, store_acc ? c->acc : nullptr, c->acc32, (int)c->n, c->tree, c->scal, c->batch,
        eps2, theta2, leaf, c->p.G * c->p.timestep, c->p.timestep, kick ? 1 : 0,
        band_theta(c) * band_theta(c));
}

// eps2 = 0 takes the variant whose terms skip coincident FP32 points
template <bool kQuad, int kBPL, bool kLearned>
void launch_split_kernel(nb_ctx* c, const BodyBuffers& b, bool kick, bool store_acc) {
    // eps2 below the smallest normal float is treated like eps2 = 0
    const float eps2 = (float)c->p.epsilon_squared;
    if (eps2 >= FLT_MIN)
        launch_split_soft<kQuad, kBPL, kLearned, false>(c, b, kick, store_acc, eps2);
    else
        launch_split_soft<kQuad, kBPL, kLearned, true>(c, b, kick, store_acc, eps2);
}

}  // namespace

int split_group_size(const nb_ctx* c) {
    // learned contexts keep groups of 64 (the correction kernel's layout)
    if (c->p.flags & NB_FLAG_LEARNED) return 32 * kBodiesPerLane;
    return 32 * (c->bpl == 1 ? 1 : c->bpl == 4 ? 4 : kBodiesPerLane);
}

void launch_force_split(nb_ctx* c, const BodyBuffers& b, bool kick, bool store_acc) {
    c->launches += 1;
    cudaMemsetAsync(&c->scal->group_ticket, 0, sizeof(unsigned), c->stream);
    if (c->p.flags & NB_FLAG_LEARNED) {  // the correction kernel assumes groups of 64
        if (c->p.flags & NB_FLAG_QUADRUPOLE)  // the network corrects the quadrupole walk
            launch_split_kernel<true, kBodiesPerLane, true>(c, b, kick, store_acc);
        else
            launch_split_kernel<false, kBodiesPerLane, true>(c, b, kick, store_acc);
    }
    else if (c->p.flags & NB_FLAG_QUADRUPOLE)
        c->bpl == 1   ? launch_split_kernel<true, 1, false>(c, b, kick, store_acc)
        : c->bpl == 4 ? launch_split_kernel<true, 4, false>(c, b, kick, store_acc)
                      : launch_split_kernel<true, kBodiesPerLane, false>(c, b, kick, store_acc);
    else
        c->bpl == 1   ? launch_split_kernel<false, 1, false>(c, b, kick, store_acc)
        : c->bpl == 4 ? launch_split_kernel<false, 4, false>(c, b, kick, store_acc)
                      : launch_split_kernel<false, kBodiesPerLane, false>(c, b, kick, store_acc);
}

}  // namespace nb
