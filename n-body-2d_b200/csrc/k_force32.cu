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

// Sum cnt cell entries into (ax, ay).
template <bool kQuad>
__device__ __forceinline__ void sum_cells(const WarpLists& L, int cnt, float px, float py,
                                          float eps2, float& ax, float& ay) {
    for (int j = 0; j < cnt; ++j) {
        const float4 e = L.cell[j];
        const float dx = e.x - px, dy = e.y - py;
        const float d2 = fmaf(dx, dx, fmaf(dy, dy, eps2));
        const float inv = rsqrtf(d2);
        const float inv3 = inv * inv * inv;
        if (kQuad) {
            const float4 q = L.quad[j];
            const float inv2 = inv * inv;
            const float inv5 = inv3 * inv2;
            const float inv7 = inv5 * inv2;
            const float sdx = fmaf(q.x, dx, q.y * dy);
            const float sdy = fmaf(q.y, dx, q.z * dy);
            const float dsd = fmaf(dx, sdx, dy * sdy);
            // a = d [M r^-3 - 1.5 tr(S) r^-5 + 7.5 (d.S.d) r^-7] - 3 r^-5 S d
            const float radial = fmaf(7.5f * dsd, inv7, fmaf(-1.5f * (q.x + q.z), inv5, e.z * inv3));
            ax = fmaf(dx, radial, fmaf(-3.f * inv5, sdx, ax));
            ay = fmaf(dy, radial, fmaf(-3.f * inv5, sdy, ay));
        } else {
            const float a = e.z * inv3;
            ax = fmaf(dx, a, ax);
            ay = fmaf(dy, a, ay);
        }
    }
}

__device__ __forceinline__ void sum_bodies(const WarpLists& L, int cnt, float px, float py,
                                           float eps2, int me, float& ax, float& ay) {
    for (int j = 0; j < cnt; ++j) {
        const float4 e = L.body[j];
        const bool self = __float_as_int(e.w) == me;
        const float dx = e.x - px, dy = e.y - py;
        const float d2 = self ? 1.f : fmaf(dx, dx, fmaf(dy, dy, eps2));
        const float inv = rsqrtf(d2);
        const float a = (self ? 0.f : e.z) * inv * inv * inv;
        ax = fmaf(dx, a, ax);
        ay = fmaf(dy, a, ay);
    }
}

template <bool kQuad>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
force_split(double2* __restrict__ pos, double2* __restrict__ vel, double2* __restrict__ acc_out,
            int n, Tree t, DeviceScalars* __restrict__ s, float eps2, float theta2, int leaf_size,
            double G_dt, double dt, int kick) {
    __shared__ WarpLists lists[kWarpsPerBlock];
    const int lane = threadIdx.x & 31;
    WarpLists& L = lists[threadIdx.x >> 5];
    const int group = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    const int g0 = group * 32;
    if (g0 >= n) return;  // whole warp leaves together
    const int g1 = min(g0 + 31, n - 1);
    const int i = min(g0 + lane, g1);
    const bool valid = g0 + lane < n;
    const double cx = s->center[0], cy = s->center[1];
    const double2 P = pos[i];
    const float px = (float)(P.x - cx), py = (float)(P.y - cy);
    const float bx0 = warp_min(px), bx1 = warp_max(px);
    const float by0 = warp_min(py), by1 = warp_max(py);
    const float gcx = 0.5f * (bx0 + bx1), gcy = 0.5f * (by0 + by1);
    const float ghx = 0.5f * (bx1 - bx0), ghy = 0.5f * (by1 - by0);
    const unsigned below = lanemask_lt();

    float ax = 0.f, ay = 0.f;
    unsigned long long ncell = 0, npair = 0;
    int ccount = 0, bcount = 0, size = 1;
    if (lane == 0) L.stack[0] = s->root;
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
        if (lane < k) {
            if (ref >= 0) {
                c4 = t.cell4[ref];
                const int2 rg = t.range[ref];
                const bool overlap = !(rg.y < g0 || rg.x > g1);
                const float dx = fmaxf(fabsf(c4.x - gcx) - ghx, 0.f);
                const float dy = fmaxf(fabsf(c4.y - gcy) - ghy, 0.f);
                const float d2 = fmaf(dx, dx, dy * dy);
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
        ccount += __popc(acc_mask);
        __syncwarp();
        if (ccount >= 32) {
            sum_cells<kQuad>(L, 32, px, py, eps2, ax, ay);
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
            if (lane == 0) atomicOr(&s->error, kErrStack);
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
                sum_bodies(L, 32, px, py, eps2, i, ax, ay);
                npair += 32;
                __syncwarp();
                if (lane < bcount - 32) L.body[lane] = L.body[32 + lane];
                bcount -= 32;
                __syncwarp();
            }
        }
    }
    sum_cells<kQuad>(L, ccount, px, py, eps2, ax, ay);
    sum_bodies(L, bcount, px, py, eps2, i, ax, ay);
    ncell += ccount;
    npair += bcount;

    if (valid) {
        if (acc_out) acc_out[i] = make_double2((double)ax, (double)ay);
        if (kick) {
            double2 v = vel[i];
            v.x += (double)ax * G_dt;
            v.y += (double)ay * G_dt;
            vel[i] = v;
            double2 p = P;
            p.x += v.x * dt;
            p.y += v.y * dt;
            pos[i] = p;
        }
    }
    // interaction counts: every valid lane summed every entry (self excluded)
    if (lane == 0) {
        const unsigned long long lanes = (unsigned long long)(g1 - g0 + 1);
        atomicAdd(&s->cell_terms, ncell * lanes);
        atomicAdd(&s->body_terms, npair * lanes - lanes);  // each lane skips itself once
    }
}

inline unsigned blocks_for(int64_t n, int per) { return (unsigned)((n + per - 1) / per); }

}  // namespace

void launch_force_split(nb_ctx* c, const BodyBuffers& b, bool kick, bool store_acc) {
    const float theta2 = (float)(c->p.theta * c->p.theta);
    const int leaf = c->p.leaf_size > 0 ? c->p.leaf_size : 16;
    const unsigned blocks = blocks_for(c->n, 32 * kWarpsPerBlock);
    c->launches += 1;
    const bool quad = (c->p.flags & NB_FLAG_QUADRUPOLE) != 0;
    if (quad)
        force_split<true><<<blocks, 32 * kWarpsPerBlock, 0, c->stream>>>(
            b.pos, b.vel, store_acc ? c->acc : nullptr, (int)c->n, c->tree, c->scal,
            (float)c->p.epsilon_squared, theta2, leaf, c->p.G * c->p.timestep, c->p.timestep,
            kick ? 1 : 0);
    else
        force_split<false><<<blocks, 32 * kWarpsPerBlock, 0, c->stream>>>(
            b.pos, b.vel, store_acc ? c->acc : nullptr, (int)c->n, c->tree, c->scal,
            (float)c->p.epsilon_squared, theta2, leaf, c->p.G * c->p.timestep, c->p.timestep,
            kick ? 1 : 0);
}

}  // namespace nb
