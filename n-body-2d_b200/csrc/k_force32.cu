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

struct WarpLists {
    int stack[kStkAlloc];
    float4 cell[kList];
    float4 quad[kList];
    float4 body[kList];
};

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

// Sum cnt cell entries into the accelerations of the lane's kBPL bodies.
template <bool kQuad, int kBPL>
__device__ __forceinline__ void cell_terms(const float4 e, const float4 q, const float* px,
                                           const float* py, float eps2, float* ax, float* ay) {
#pragma unroll
    for (int b = 0; b < kBPL; ++b) {
        const float dx = e.x - px[b], dy = e.y - py[b];
        const float d2 = fmaf(dx, dx, fmaf(dy, dy, eps2));
        const float inv = rsqrtf(d2);
        const float inv2 = inv * inv;
        const float inv3 = inv * inv2;
        if (kQuad) {
            const float inv5 = inv3 * inv2;
            const float inv7 = inv5 * inv2;
            const float sdx = fmaf(q.x, dx, q.y * dy);
            const float sdy = fmaf(q.y, dx, q.z * dy);
            const float dsd = fmaf(dx, sdx, dy * sdy);
            // a = d [M r^-3 - 1.5 tr(S) r^-5 + 7.5 (d.S.d) r^-7] - 3 r^-5 S d
            const float radial =
                fmaf(7.5f * dsd, inv7, fmaf(-1.5f * (q.x + q.z), inv5, e.z * inv3));
            ax[b] = fmaf(dx, radial, fmaf(-3.f * inv5, sdx, ax[b]));
            ay[b] = fmaf(dy, radial, fmaf(-3.f * inv5, sdy, ay[b]));
        } else {
            const float a = e.z * inv3;
            ax[b] = fmaf(dx, a, ax[b]);
            ay[b] = fmaf(dy, a, ay[b]);
        }
    }
}

// A body's own entry has dx = dy = 0 exactly (body4 and px/py round the same
// double difference), so with eps2 > 0 it adds 0 * finite = 0 and needs no
// index test.  d2 == 0 (eps2 = 0 and the same FP32 coordinates: the body
// itself, or a body that coincides with it at FP32 resolution) contributes
// nothing instead of 0 * inf.
template <int kBPL>
__device__ __forceinline__ void body_terms(const float4 e, const float* px, const float* py,
                                           float eps2, float* ax, float* ay) {
#pragma unroll
    for (int b = 0; b < kBPL; ++b) {
        const float dx = e.x - px[b], dy = e.y - py[b];
        const float d2 = fmaf(dx, dx, fmaf(dy, dy, eps2));
        const float inv = rsqrtf(d2);
        const float a = d2 == 0.f ? 0.f : e.z * (inv * inv) * inv;
        ax[b] = fmaf(dx, a, ax[b]);
        ay[b] = fmaf(dy, a, ay[b]);
    }
}

template <bool kQuad, int kBPL>
__device__ __forceinline__ void sum_cells(const WarpLists& L, int cnt, const float* px,
                                          const float* py, float eps2, float* ax, float* ay) {
    if (cnt == 32) {
#pragma unroll 4
        for (int j = 0; j < 32; ++j)
            cell_terms<kQuad, kBPL>(L.cell[j], kQuad ? L.quad[j] : L.cell[j], px, py, eps2, ax, ay);
    } else {
        for (int j = 0; j < cnt; ++j)
            cell_terms<kQuad, kBPL>(L.cell[j], kQuad ? L.quad[j] : L.cell[j], px, py, eps2, ax, ay);
    }
}

template <int kBPL>
__device__ __forceinline__ void sum_bodies(const WarpLists& L, int cnt, const float* px,
                                           const float* py, float eps2, float* ax, float* ay) {
    if (cnt == 32) {
#pragma unroll 4
        for (int j = 0; j < 32; ++j) body_terms<kBPL>(L.body[j], px, py, eps2, ax, ay);
    } else {
        for (int j = 0; j < cnt; ++j) body_terms<kBPL>(L.body[j], px, py, eps2, ax, ay);
    }
}

// Walk the tree for one group [g0, g1] of <= 32 kBPL bodies (lane l owns
// g0 + l, g0 + 32 + l, ...) and accumulate the FP32 accelerations.
template <bool kQuad, int kBPL, bool kLearned>
__device__ __forceinline__ void walk_group(WarpLists& L, const Tree& t, int root, int n, int g0,
                                           int g1, const float* px, const float* py,
                                           const bool* act_body, float eps2, float theta2,
                                           int leaf_size, float* ax, float* ay,
                                           unsigned long long& ncell, unsigned long long& npair,
                                           unsigned* err, int* band, int& nband, int band_cap) {
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
#pragma unroll
    for (int b = 0; b < kBPL; ++b) {
        ax[b] = 0.f;
        ay[b] = 0.f;
    }
    ncell = 0;
    npair = 0;
    int ccount = 0, bcount = 0, size = 1;
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
            if (ref >= 0) {
                c4 = t.cell4[ref];
                const int2 rg = t.range[ref];
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
                    ch = t.child[ref];
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
            L.cell[slot] = c4;
            if (kQuad) L.quad[slot] = t.cellq[ref];
        }
        if (kLearned) {
            // band: accepted here but opened by the plain theta_B walk
            const bool in_band = act == 1 && c4.w >= kThetaBand * kThetaBand * band_d2;
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
            sum_cells<kQuad, kBPL>(L, 32, px, py, eps2, ax, ay);
            ncell += 32;
            __syncwarp();
            // entries 32.. move down; source and destination slots never overlap
            if (lane < ccount - 32) {
                L.cell[lane] = L.cell[32 + lane];
                if (kQuad) L.quad[lane] = L.quad[32 + lane];
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
            if (lane < added) L.body[bcount + lane] = t.body4[j];
            bcount += added;
            __syncwarp();
            if (bcount >= 32) {
                sum_bodies<kBPL>(L, 32, px, py, eps2, ax, ay);
                npair += 32;
                __syncwarp();
                if (lane < bcount - 32) L.body[lane] = L.body[32 + lane];
                bcount -= 32;
                __syncwarp();
            }
        }
    }
    sum_cells<kQuad, kBPL>(L, ccount, px, py, eps2, ax, ay);
    sum_bodies<kBPL>(L, bcount, px, py, eps2, ax, ay);
    ncell += ccount;
    npair += bcount;
    __syncwarp();
}

// Persistent: each warp takes groups from a global ticket until none is left,
// which balances groups of very different cost.
template <bool kQuad, int kBPL, bool kLearned>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
force_split(double2* __restrict__ pos, double2* __restrict__ vel, double2* __restrict__ acc_out,
            float2* __restrict__ acc32, int n, Tree t, DeviceScalars* __restrict__ s, Batch bt,
            float eps2, float theta2, int leaf_size, double G_dt, double dt, int kick) {
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
        walk_group<kQuad, kBPL, kLearned>(L, t, root, n, g0, g1, px, py, on, eps2, theta2,
                                          leaf_size, ax, ay, ncell, npair, &s->error, band, nband,
                                          kBandPerBody * (g1 - g0 + 1));
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

template <bool kQuad, int kBPL, bool kLearned>
void launch_split_kernel(nb_ctx* c, const BodyBuffers& b, bool kick, bool store_acc) {
    int& grid = c->split_blocks[(kQuad ? 1 : 0) + (kLearned ? 2 : 0) + (kBPL == 1 ? 4 : 0)];
    if (grid == 0) {
        int blocks = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &blocks, force_split<kQuad, kBPL, kLearned>, kWarpsPerBlock * 32, 0) != cudaSuccess ||
            blocks < 1)
            blocks = 4;
        grid = c->sm_count * blocks;
    }
    const float theta2 = (float)(c->p.theta * c->p.theta);
    const int leaf = c->p.leaf_size > 0 ? c->p.leaf_size : kDefaultLeaf;
    force_split<kQuad, kBPL, kLearned><<<grid, 32 * kWarpsPerBlock, 0, c->stream>>>(
        b.pos, b.vel, store_acc ? c->acc : nullptr, c->acc32, (int)c->n, c->tree, c->scal, c->batch,
        (float)c->p.epsilon_squared, theta2, leaf, c->p.G * c->p.timestep, c->p.timestep,
        kick ? 1 : 0);
}

}  // namespace

int split_group_size(const nb_ctx* c) { return 32 * (c->bpl == 1 ? 1 : kBodiesPerLane); }

void launch_force_split(nb_ctx* c, const BodyBuffers& b, bool kick, bool store_acc) {
    c->launches += 1;
    cudaMemsetAsync(&c->scal->group_ticket, 0, sizeof(unsigned), c->stream);
    if (c->p.flags & NB_FLAG_LEARNED)  // the correction kernel assumes groups of 64
        launch_split_kernel<false, kBodiesPerLane, true>(c, b, kick, store_acc);
    else if (c->p.flags & NB_FLAG_QUADRUPOLE)
        c->bpl == 1 ? launch_split_kernel<true, 1, false>(c, b, kick, store_acc)
                    : launch_split_kernel<true, kBodiesPerLane, false>(c, b, kick, store_acc);
    else
        c->bpl == 1 ? launch_split_kernel<false, 1, false>(c, b, kick, store_acc)
                    : launch_split_kernel<false, kBodiesPerLane, false>(c, b, kick, store_acc);
}

}  // namespace nb
