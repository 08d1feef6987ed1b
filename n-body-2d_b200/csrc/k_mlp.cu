// k_mlp.cu -- learned far-field correction (SPLIT mode, NB_FLAG_LEARNED).
//
// A 12 -> 64 -> 64 -> 2 MLP (tanh hidden layers, BF16 weights and activations,
// FP32 accumulation) predicts, for a cell accepted at theta_L = theta but that
// plain theta_B = 0.5 would have opened, the residual between the cell's exact
// pull and its monopole, in units of M / d^2:
//   r = (sum_j m_j (x_j - p)(|x_j - p|^2 + eps^2)^-3/2
//        - M (c - p)(|c - p|^2 + eps^2)^-3/2) * d^2 / M,    d = |p - c|.
// Features of (point p, cell): u = (p - c) / d (2), w / d, the heaviest child's
// mass fraction, S / (M w^2) (3), T / (M w^3) (4), and eps^2 / (d^2 + eps^2):
// the softening ratio takes the last of the eight moment slots because near
// cells (d ~ eps) have residuals that depend on it far more than on any
// higher moment.
//
// Tensor-core layout: training (nb_mlp_train, nb_mlp_loss_grad) and bulk
// evaluation (nb_mlp_forward) run on tcgen05 in 128-row tiles with BF16
// operands in shared memory and FP32 accumulators in TMEM (mlp_grad_tc,
// mlp_forward_tc, further down).  The step's correction uses mma.sync
// m16n8k16: a 16-row tile (16 cells of one target group) runs through the
// three layers in registers, the accumulator fragment of one layer being,
// element for element, the A fragment of the next.
//
// Inference is per target group: the traversal lists each group's band cells;
// mlp_correct_kick evaluates the MLP at the group's centre for all of them in
// tiles of 16, adds the summed correction to every body's acceleration, and
// applies the FP64 kick and drift.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "nb_internal.cuh"

namespace nb {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kH = 64;
constexpr int kNin = 12;

// FP32 parameter vector layout (also the ABI layout of the weights).
constexpr int kW1 = 0;                    // [64][12]
constexpr int kB1 = kW1 + kH * kNin;      // [64]
constexpr int kW2 = kB1 + kH;             // [64][64]  (out, in)
constexpr int kB2 = kW2 + kH * kH;        // [64]
constexpr int kW3 = kB2 + kH;             // [2][64]
constexpr int kB3 = kW3 + 2 * kH;         // [2]
constexpr int kYS = kB3 + 2;              // output scale
constexpr int kParams = kYS + 1;
static_assert(kParams == NB_MLP_PARAMS, "weight layout and header disagree");

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// A fragment of a 16 x 16 tile of a row-major BF16 matrix.
__device__ __forceinline__ void load_a(const __nv_bfloat16* m, int ld, int kb, uint32_t a[4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    a[0] = *reinterpret_cast<const uint32_t*>(m + g * ld + kb + 2 * q);
    a[1] = *reinterpret_cast<const uint32_t*>(m + (g + 8) * ld + kb + 2 * q);
    a[2] = *reinterpret_cast<const uint32_t*>(m + g * ld + kb + 2 * q + 8);
    a[3] = *reinterpret_cast<const uint32_t*>(m + (g + 8) * ld + kb + 2 * q + 8);
}

__device__ __forceinline__ float bf16_round(float v) {
    return __bfloat162float(__float2bfloat16_rn(v));
}

// Hardware tanh (one MUFU op, relative error about 2^-11, below the BF16
// rounding the activations get next); training and inference both use it.
__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

constexpr int kWarps = 4;

// Adam on the FP32 master parameters (the output scale is not trained).
__global__ void mlp_adam_kernel(float* __restrict__ p, const float* __restrict__ g,
                                float* __restrict__ m, float* __restrict__ v, float lr, float b1,
                                float b2, float eps, float c1, float c2) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kYS) return;
    const float gk = g[k];
    const float mk = b1 * m[k] + (1.f - b1) * gk;
    const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    p[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
}

}  // namespace

namespace {

// ---- features shared by sampling and inference -------------------------
// The (point, cell) features: u = (p - c) / d (2), w / d and
// eps^2 / (d^2 + eps^2), plus the output scale M / d^2; the cell's eight
// moment features come from cellh.  Sampling and inference both call this,
// so training data and inference agree bit for bit.
struct PointFeatures {
    float x0, x1, x2, x11, scale;
};

__device__ __forceinline__ PointFeatures point_features(float ux, float uy, float w, float mass,
                                                        float eps2) {
    const float d2 = fmaxf(fmaf(ux, ux, uy * uy), 1e-30f);
    const float inv = rsqrtf(d2);
    PointFeatures f;
    f.x0 = ux * inv;
    f.x1 = uy * inv;
    f.x2 = w * inv;
    f.x11 = eps2 / (d2 + eps2);
    f.scale = mass * (inv * inv);
    return f;
}

__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }

// ---- residual samples (training data) ----------------------------------
// Samples are drawn exactly as inference uses the network: one warp per target
// group, the group's bounding box and acceptance tests in the traversal's FP32
// arithmetic (cell accepted when it holds no body of the group and
// w^2 < theta_L^2 d^2, band when also w^2 >= theta_B^2 d^2, d = distance from
// the cell's COM to the box), and for every band cell one sample: the features
// at the group's centre and, as target, the mean over the group's bodies of
// the exact-minus-monopole pull (FP64 sums over the cell's bodies), in units
// of M / d_c^2 with d_c the centre's distance.  That mean is the best single
// correction for the whole group, which is what inference applies.  When the
// walk adds quadrupoles (quad != 0) the target is exact minus monopole minus
// quadrupole, the residual the network then has to supply.
constexpr int kSampleStack = 128;

__global__ void __launch_bounds__(kWarps * 32)
mlp_samples_kernel(Tree t, const DeviceScalars* __restrict__ s, const double2* __restrict__ pos,
                   const double* __restrict__ mass, int n, const int* __restrict__ pick, int npick,
                   float thL2, float thB2, double eps2, int quad, float* __restrict__ X,
                   float* __restrict__ Y, unsigned* __restrict__ count, unsigned cap) {
    __shared__ int stacks[kWarps][kSampleStack];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int* stk = stacks[warp];
    const int cells = s->cells, ngroups = s->groups;
    const double cx = s->center[0], cy = s->center[1];
    for (int w = blockIdx.x * kWarps + warp; w < npick; w += gridDim.x * kWarps) {
        const int gi = pick[w] % max(ngroups, 1);
        if (gi >= ngroups) continue;
        const int2 gr = t.groups[gi];
        const int g0 = gr.x, g1 = min(gr.y, n - 1);
        const int nb = g1 - g0 + 1;
        double2 P[2];
        bool on[2];
        float bx0 = INFINITY, bx1 = -INFINITY, by0 = INFINITY, by1 = -INFINITY;
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int i = min(g0 + 32 * b + lane, g1);
            on[b] = g0 + 32 * b + lane <= g1;
            P[b] = pos[i];
            if (on[b]) {
                const float px = (float)(P[b].x - cx), py = (float)(P[b].y - cy);
                bx0 = fminf(bx0, px);
                bx1 = fmaxf(bx1, px);
                by0 = fminf(by0, py);
                by1 = fmaxf(by1, py);
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            bx0 = fminf(bx0, __shfl_xor_sync(kFull, bx0, o));
            bx1 = fmaxf(bx1, __shfl_xor_sync(kFull, bx1, o));
            by0 = fminf(by0, __shfl_xor_sync(kFull, by0, o));
            by1 = fmaxf(by1, __shfl_xor_sync(kFull, by1, o));
        }
        const float gcx = 0.5f * (bx0 + bx1), gcy = 0.5f * (by0 + by1);
        const float ghx = 0.5f * (bx1 - bx0), ghy = 0.5f * (by1 - by0);
        int top = 0;
        if (lane == 0) stk[0] = s->root;
        __syncwarp();
        while (top >= 0) {
            const int ref = stk[top];
            --top;
            __syncwarp();
            if (ref < 0 || ref >= cells) continue;  // leaves are summed exactly: no correction
            const float4 c4 = t.cell4[ref];
            const int2 rg = t.range[ref];
            const bool overlap = !(rg.y < g0 || rg.x > g1);
            const float dx = fmaxf(fabsf(c4.x - gcx) - ghx, 0.f);
            const float dy = fmaxf(fabsf(c4.y - gcy) - ghy, 0.f);
            const float d2 = fmaf(dx, dx, dy * dy);
            if (overlap || !(c4.w < thL2 * d2)) {
                const int4 ch = t.child[ref];
                const int refs[4] = {ch.x, ch.y, ch.z, ch.w};
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (refs[q] >= 0 && top + 1 < kSampleStack) {
                        ++top;
                        if (lane == 0) stk[top] = refs[q];
                    }
                __syncwarp();
                continue;
            }
            if (!(c4.w >= thB2 * d2)) continue;  // accepted by the plain theta_B walk too
            // mean over the group's bodies of (exact - monopole), FP64
            const double M = t.mass[ref];
            const double2 c = t.com[ref];
            double sxx = 0.0, sxy = 0.0, syy = 0.0;
            if (quad) {
                const float4 q = t.cellq[ref];  // 7.5 S
                sxx = q.x / 7.5;
                sxy = q.y / 7.5;
                syy = q.z / 7.5;
            }
            double rx = 0.0, ry = 0.0;
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                if (!on[b]) continue;
                double ax = 0.0, ay = 0.0;
                for (int j = rg.x; j <= rg.y; ++j) {
                    const double2 q = pos[j];
                    const double ex = q.x - P[b].x, ey = q.y - P[b].y;
                    const double r2 = ex * ex + ey * ey + eps2;
                    const double a = mass[j] / (r2 * sqrt(r2));
                    ax += ex * a;
                    ay += ey * a;
                }
                const double mx = c.x - P[b].x, my = c.y - P[b].y;
                const double r2 = mx * mx + my * my + eps2;
                const double am = M / (r2 * sqrt(r2));
                rx += ax - mx * am;
                ry += ay - my * am;
                if (quad) {
                    // the walk's second-moment term (the softened potential's):
                    // d [-1.5 tr(S) r^-5 + 7.5 (d.S.d) r^-7] - 3 r^-5 S d
                    const double ir2 = 1.0 / r2, ir5 = ir2 * ir2 / sqrt(r2), ir7 = ir5 * ir2;
                    const double sdx = sxx * mx + sxy * my, sdy = sxy * mx + syy * my;
                    const double radial = -1.5 * (sxx + syy) * ir5 + 7.5 * (mx * sdx + my * sdy) * ir7;
                    rx -= mx * radial - 3.0 * ir5 * sdx;
                    ry -= my * radial - 3.0 * ir5 * sdy;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                rx += __shfl_xor_sync(kFull, rx, o);
                ry += __shfl_xor_sync(kFull, ry, o);
            }
            if (lane == 0) {
                const float ux = gcx - c4.x, uy = gcy - c4.y;
                const float dc2 = fmaxf(ux * ux + uy * uy, 1e-30f);
                const double scale = (double)dc2 / (M * nb);
                const unsigned slot = atomicAdd(count, 1u);
                if (slot < cap) {
                    const float w = __uint_as_float(t.cellh[2 * ref + 1].w);
                    const PointFeatures pf = point_features(ux, uy, w, c4.z, (float)eps2);
                    const uint4 h = t.cellh[2 * ref];
                    const float x[kNin] = {pf.x0,       pf.x1,       pf.x2,       bf16_lo(h.x),
                                           bf16_hi(h.x), bf16_lo(h.y), bf16_hi(h.y), bf16_lo(h.z),
                                           bf16_hi(h.z), bf16_lo(h.w), bf16_hi(h.w), pf.x11};
#pragma unroll
                    for (int k = 0; k < kNin; ++k) X[(int64_t)slot * kNin + k] = x[k];
                    Y[2 * (int64_t)slot] = (float)(rx * scale);
                    Y[2 * (int64_t)slot + 1] = (float)(ry * scale);
                }
            }
            __syncwarp();
        }
    }
}

// ---- inference: per-group correction, then kick and drift --------------
// acc32 holds the traversal's FP32 accelerations (monopoles of every
// accepted cell and the direct sums); band[] lists, per group, the cells
// accepted at theta but not at theta_B (capacity kBandPerBody per body of the
// group, starting at kBandPerBody * first body).
//
// The weights sit in shared memory as per-lane B fragments, prepared once per
// nb_set_mlp_weights (mlp_prepare_infer), so each fragment (or pair of
// k-tiles) is one 64/128-bit shared load.  The input tile's columns are the
// features in the order 3..10 (the cell's BF16 record, copied as is), 0, 1,
// 2, 11, then zeros; the layer-1 image permutes W1's columns to match.  The
// hidden activations are tanh on packed BF16 pairs (one SFU op per two
// values), which is also the rounding the next layer's A fragment needs.
struct InferW {
    uint2 w1[8][32];      // layer 1, n-tile nt: {b0, b1}
    uint4 w2[8][2][32];   // layer 2, n-tile nt, k-tiles 2j and 2j + 1: {b0, b1, b0', b1'}
    uint4 w3[2][32];      // layer 3 (outputs padded to 8), k-tiles 2j and 2j + 1
    float2 b1[8][4];      // bias of columns 8 nt + 2q and 8 nt + 2q + 1
    float2 b2[8][4];
    float2 b3[4];
    float yscale;
};

constexpr int kCorrWarps = 4;

struct CorrSmem {
    InferW W;
    uint4 x[kCorrWarps][2][16][2];  // per warp: two 16-row input tiles, 32 bytes a row
    float scale[kCorrWarps][2][16];  // per row: M / d^2 (0 for padding rows)
};

// Input column of the inference tile -> feature index (-1: zero padding).
__device__ __forceinline__ int infer_feature(int col) {
    return col < 8 ? col + 3 : col < 11 ? col - 8 : col == 11 ? 11 : -1;
}

__global__ void mlp_prepare_infer(const float* __restrict__ p, InferW* __restrict__ W) {
    const int lane = threadIdx.x & 31, nt = threadIdx.x >> 5, g = lane >> 2, q = lane & 3;
    const int n = 8 * nt + g;
    auto w1 = [&](int col) {
        const int f = infer_feature(col);
        return f < 0 ? 0.f : p[kW1 + n * kNin + f];
    };
    W->w1[nt][lane] = make_uint2(pack_bf16(w1(2 * q), w1(2 * q + 1)),
                                 pack_bf16(w1(2 * q + 8), w1(2 * q + 9)));
    auto w2 = [&](int k) { return p[kW2 + n * kH + k]; };
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int k0 = 32 * j + 2 * q, k1 = k0 + 16;
        W->w2[nt][j][lane] = make_uint4(pack_bf16(w2(k0), w2(k0 + 1)), pack_bf16(w2(k0 + 8), w2(k0 + 9)),
                                        pack_bf16(w2(k1), w2(k1 + 1)), pack_bf16(w2(k1 + 8), w2(k1 + 9)));
    }
    if (nt == 0) {
        auto w3 = [&](int k) { return g < 2 ? p[kW3 + g * kH + k] : 0.f; };
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int k0 = 32 * j + 2 * q, k1 = k0 + 16;
            W->w3[j][lane] = make_uint4(pack_bf16(w3(k0), w3(k0 + 1)), pack_bf16(w3(k0 + 8), w3(k0 + 9)),
                                        pack_bf16(w3(k1), w3(k1 + 1)), pack_bf16(w3(k1 + 8), w3(k1 + 9)));
        }
        if (lane < 4)
            W->b3[lane] = lane == 0 ? make_float2(p[kB3], p[kB3 + 1]) : make_float2(0.f, 0.f);
        if (lane == 0) W->yscale = p[kYS];
    }
    if (lane < 4) {
        W->b1[nt][lane] = make_float2(p[kB1 + 8 * nt + 2 * lane], p[kB1 + 8 * nt + 2 * lane + 1]);
        W->b2[nt][lane] = make_float2(p[kB2 + 8 * nt + 2 * lane], p[kB2 + 8 * nt + 2 * lane + 1]);
    }
}

__device__ __forceinline__ uint32_t tanh_bf16x2(uint32_t x) {
    uint32_t y;
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(y) : "r"(x));
    return y;
}

// kT independent 16-row tiles through the network (their mma chains
// interleave); y[t] = output fragment of tile t (columns 2q, 2q+1 of rows g,
// g + 8; only q = 0 holds the two outputs).
template <int kT>
__device__ __forceinline__ void infer_tiles(const InferW& W, const uint32_t (*a)[4], float (*y)[4]) {
    const int lane = threadIdx.x & 31, q = lane & 3;
    uint32_t h1[kT][4][4], h2[kT][4][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const float2 b = W.b1[nt][q];
        const uint2 f = W.w1[nt][lane];
#pragma unroll
        for (int t = 0; t < kT; ++t) {
            float c[4] = {b.x, b.y, b.x, b.y};
            mma16816(c, a[t], f.x, f.y);
            h1[t][nt >> 1][(nt & 1) * 2] = tanh_bf16x2(pack_bf16(c[0], c[1]));
            h1[t][nt >> 1][(nt & 1) * 2 + 1] = tanh_bf16x2(pack_bf16(c[2], c[3]));
        }
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const float2 b = W.b2[nt][q];
        float c[kT][4];
#pragma unroll
        for (int t = 0; t < kT; ++t) {
            c[t][0] = b.x;
            c[t][1] = b.y;
            c[t][2] = b.x;
            c[t][3] = b.y;
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const uint4 f = W.w2[nt][j][lane];
#pragma unroll
            for (int t = 0; t < kT; ++t) {
                mma16816(c[t], h1[t][2 * j], f.x, f.y);
                mma16816(c[t], h1[t][2 * j + 1], f.z, f.w);
            }
        }
#pragma unroll
        for (int t = 0; t < kT; ++t) {
            h2[t][nt >> 1][(nt & 1) * 2] = tanh_bf16x2(pack_bf16(c[t][0], c[t][1]));
            h2[t][nt >> 1][(nt & 1) * 2 + 1] = tanh_bf16x2(pack_bf16(c[t][2], c[t][3]));
        }
    }
    const float2 b = W.b3[q];
#pragma unroll
    for (int t = 0; t < kT; ++t) {
        y[t][0] = b.x;
        y[t][1] = b.y;
        y[t][2] = b.x;
        y[t][3] = b.y;
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const uint4 f = W.w3[j][lane];
#pragma unroll
        for (int t = 0; t < kT; ++t) {
            mma16816(y[t], h2[t][2 * j], f.x, f.y);
            mma16816(y[t], h2[t][2 * j + 1], f.z, f.w);
        }
    }
}

// at most 102 registers: five blocks of four warps per SM (measured faster
// than four or six, despite a few spilled bytes)
__global__ void __launch_bounds__(kCorrWarps * 32, 5)
mlp_correct_kick(const InferW* __restrict__ Wg, Tree t, const DeviceScalars* __restrict__ s,
                 double2* __restrict__ pos, double2* __restrict__ vel,
                 const float2* __restrict__ acc32, double2* __restrict__ acc_out, int n,
                 float eps2, double G_dt, double dt, int kick) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CorrSmem& S = *reinterpret_cast<CorrSmem*>(smem_raw);
    {
        const uint4* src = reinterpret_cast<const uint4*>(Wg);
        uint4* dst = reinterpret_cast<uint4*>(&S.W);
        for (int k = threadIdx.x; k < (int)(sizeof(InferW) / 16); k += blockDim.x) dst[k] = src[k];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, q = lane & 3;
    const int row = lane & 15, half = lane >> 4;
    const double cx = s->center[0], cy = s->center[1];
    const int ngroups = s->groups;
    const float ys = S.W.yscale;
    for (int gi = blockIdx.x * kCorrWarps + warp; gi < ngroups; gi += gridDim.x * kCorrWarps) {
        const int2 gr = t.groups[gi];
        const int g0 = gr.x, g1 = min(gr.y, n - 1);
        double2 P[2];
        bool on[2];
        float bx0 = INFINITY, bx1 = -INFINITY, by0 = INFINITY, by1 = -INFINITY;
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int i = min(g0 + 32 * b + lane, g1);
            on[b] = g0 + 32 * b + lane <= g1;
            P[b] = pos[i];
            if (on[b]) {
                const float px = (float)(P[b].x - cx), py = (float)(P[b].y - cy);
                bx0 = fminf(bx0, px);
                bx1 = fmaxf(bx1, px);
                by0 = fminf(by0, py);
                by1 = fmaxf(by1, py);
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            bx0 = fminf(bx0, __shfl_xor_sync(kFull, bx0, o));
            bx1 = fmaxf(bx1, __shfl_xor_sync(kFull, bx1, o));
            by0 = fminf(by0, __shfl_xor_sync(kFull, by0, o));
            by1 = fmaxf(by1, __shfl_xor_sync(kFull, by1, o));
        }
        const float gx = 0.5f * (bx0 + bx1), gy = 0.5f * (by0 + by1);
        const int nband = min(t.band_count[gi], kBandPerBody * (g1 - g0 + 1));
        const int* band = t.band + (int64_t)kBandPerBody * g0;
        float cxs = 0.f, cys = 0.f;
        // the next batch's band index is loaded one batch ahead
        int ref_next = lane < nband ? band[lane] : 0;
        for (int base = 0; base < nband; base += 32) {
            // lane l builds row l % 16 of tile l / 16
            const int r = base + lane;
            const int ref = ref_next;
            ref_next = r + 32 < nband ? band[r + 32] : 0;
            uint4 lo = make_uint4(0u, 0u, 0u, 0u), hi = lo;
            float sc = 0.f;
            if (r < nband) {
                // one 32-byte record: the BF16 features, then COM, mass, width
                lo = t.cellh[2 * ref];
                const uint4 gb = t.cellh[2 * ref + 1];
                const PointFeatures pf =
                    point_features(gx - __uint_as_float(gb.x), gy - __uint_as_float(gb.y),
                                   __uint_as_float(gb.w), __uint_as_float(gb.z), eps2);
                hi = make_uint4(pack_bf16(pf.x0, pf.x1), pack_bf16(pf.x2, pf.x11), 0u, 0u);
                sc = pf.scale;
            }
            S.x[warp][half][row][0] = lo;
            S.x[warp][half][row][1] = hi;
            S.scale[warp][half][row] = sc;
            __syncwarp();
            uint32_t a[2][4];
            float y[2][4];
            load_a(reinterpret_cast<const __nv_bfloat16*>(&S.x[warp][0][0][0]), 16, 0, a[0]);
            if (nband - base > 16) {
                load_a(reinterpret_cast<const __nv_bfloat16*>(&S.x[warp][1][0][0]), 16, 0, a[1]);
                infer_tiles<2>(S.W, a, y);
            } else {
                infer_tiles<1>(S.W, a, y);
                y[1][0] = y[1][1] = y[1][2] = y[1][3] = 0.f;
            }
            if (q == 0) {
#pragma unroll
                for (int tt = 0; tt < 2; ++tt) {
                    const float s0 = S.scale[warp][tt][g], s1 = S.scale[warp][tt][g + 8];
                    cxs = fmaf(y[tt][0], s0, fmaf(y[tt][2], s1, cxs));
                    cys = fmaf(y[tt][1], s0, fmaf(y[tt][3], s1, cys));
                }
            }
            __syncwarp();
        }
        for (int o = 16; o > 0; o >>= 1) {
            cxs += __shfl_xor_sync(kFull, cxs, o);
            cys += __shfl_xor_sync(kFull, cys, o);
        }
        cxs *= ys;
        cys *= ys;
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            if (!on[b]) continue;
            const int i = g0 + 32 * b + lane;
            const float2 a32 = acc32[i];
            const double ax = (double)a32.x + (double)cxs, ay = (double)a32.y + (double)cys;
            if (acc_out) acc_out[i] = make_double2(ax, ay);
            if (kick) {
                double2 v = vel[i];
                v.x += ax * G_dt;
                v.y += ay * G_dt;
                vel[i] = v;
                double2 p = P[b];
                p.x += v.x * dt;
                p.y += v.y * dt;
                pos[i] = p;
            }
        }
    }
}

// ---- the network on the 5th-generation tensor cores (tcgen05) --------------
// 128-row tiles: row r of a tile is TMEM lane r, so warp w of a four-warp CTA
// writes rows 32w..32w+31 and reads back exactly those lanes.  One thread
// issues the three layers as tcgen05.mma (M = 128; N = 64, 64, 16; K = 16,
// 64, 64) with BF16 operands in shared memory and FP32 accumulators in TMEM.
// The step's correction (mlp_correct_kick) stays on mma.sync: there every
// warp feeds its own group's 32 band cells at a time, and the three MMA round
// trips and barriers a 128-row tile needs made it slower (0.83 against
// 0.64 ms at 4M bodies, measured; 1.04 ms with two tiles in flight per CTA),
// while bulk evaluation fills whole tiles.
//
// Shared-memory operands use the no-swizzle K-major layout of 8-row x 16-byte
// core matrices: element (row, k) of an operand with K columns sits at byte
//   (row / 8) * SBO + (k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2,
// SBO = 16 K bytes; a K step of 16 starts 256 bytes further on.
constexpr int kTcRows = 128;
constexpr int kTcWarps = kTcRows / 32;  // one warp per 32 rows (TMEM lanes)
constexpr uint32_t kTcCols = 64;    // TMEM columns a CTA allocates; the three layers share them
constexpr int kTcBlocksPerSm = 5;   // shared memory allows five CTAs per SM, TMEM eight
constexpr int kTcSpin = 1 << 20;    // bound on each wait for an MMA to complete

struct UmmaW {
    uint4 w1[kH * 16 / 8];     // B of layer 1: n = hidden (64) x k = input column (16)
    uint4 w2[kH * kH / 8];     // B of layer 2: n = out (64) x k = in (64)
    uint4 w3[16 * kH / 8];     // B of layer 3: n = out (2 used of 16) x k = hidden (64)
    float b1[kH], b2[kH], b3[2], yscale, pad;
};

__host__ __device__ constexpr int umma_off(int row, int k, int sbo) {
    return (row / 8) * sbo + (k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2;
}

__global__ void mlp_prepare_umma(const float* __restrict__ p, UmmaW* __restrict__ W) {
    auto put = [](uint4* img, int off, float v) {
        reinterpret_cast<__nv_bfloat16*>(img)[off / 2] = __float2bfloat16_rn(v);
    };
    for (int e = threadIdx.x; e < kH * 16; e += blockDim.x) {
        const int n = e / 16, k = e % 16, f = infer_feature(k);
        put(W->w1, umma_off(n, k, 256), f < 0 ? 0.f : p[kW1 + n * kNin + f]);
    }
    for (int e = threadIdx.x; e < kH * kH; e += blockDim.x) {
        const int n = e / kH, k = e % kH;
        put(W->w2, umma_off(n, k, 1024), p[kW2 + n * kH + k]);
    }
    for (int e = threadIdx.x; e < 16 * kH; e += blockDim.x) {
        const int n = e / kH, k = e % kH;
        put(W->w3, umma_off(n, k, 1024), n < 2 ? p[kW3 + n * kH + k] : 0.f);
    }
    for (int e = threadIdx.x; e < kH; e += blockDim.x) {
        W->b1[e] = p[kB1 + e];
        W->b2[e] = p[kB2 + e];
    }
    if (threadIdx.x == 0) {
        W->b3[0] = p[kB3];
        W->b3[1] = p[kB3 + 1];
        W->yscale = p[kYS];
        W->pad = 0.f;
    }
}

struct TcSmem {
    UmmaW W;
    alignas(128) uint4 a1[kTcRows * 16 / 8];   // layer-1 input rows (K = 16)
    alignas(128) uint4 a2[kTcRows * kH / 8];   // hidden rows (K = 64), both layers
    alignas(16) float xs[kTcRows * kNin];      // the next tile's FP32 features (bulk copy)
    alignas(8) uint64_t mbar;                  // MMA completion
    alignas(8) uint64_t xbar;                  // feature tile arrived
    uint32_t tmem;                             // TMEM base address from tcgen05.alloc
    int fail;                                  // a wait for an MMA ran out
};

__device__ __forceinline__ uint32_t smem_u32(const void* ptr) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(ptr));
}

// shared-memory matrix descriptor (sm_100 format): start, LBO and SBO in
// 16-byte units, version 1, no swizzle
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, M x N
constexpr uint32_t umma_idesc(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        :: "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate) : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// generic-proxy stores to shared memory become visible to the MMA's reads
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// waits for phase `parity` of the barrier; false when the bound ran out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (int i = 0; i < kTcSpin; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// 16 consecutive FP32 columns of this thread's TMEM lane; the wait is tied to
// the registers so that no use moves above it
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
          "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]),
                   "+r"(v[6]), "+r"(v[7]), "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]),
                   "+r"(v[12]), "+r"(v[13]), "+r"(v[14]), "+r"(v[15])
                 :: "memory");
}

__device__ __forceinline__ void tmem_ld2(uint32_t taddr, uint32_t& a, uint32_t& b) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];"
                 : "=r"(a), "=r"(b) : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(a), "+r"(b) :: "memory");
}

// Bias, tanh and BF16 packing of this thread's 64 hidden columns at TMEM
// column col0; the row is stored as the next layer's A operand.
__device__ __forceinline__ void tc_hidden_row(uint32_t tlane, uint32_t col0, const float* bias,
                                              uint4* a2, int row) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        uint32_t v[16];
        tmem_ld16(tlane + col0 + 16 * c, v);
        uint32_t h[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            h[j] = tanh_bf16x2(pack_bf16(__uint_as_float(v[2 * j]) + bias[16 * c + 2 * j],
                                         __uint_as_float(v[2 * j + 1]) + bias[16 * c + 2 * j + 1]));
        uint4* dst = a2 + umma_off(row, 16 * c, 1024) / 16;
        dst[0] = make_uint4(h[0], h[1], h[2], h[3]);
        dst[8] = make_uint4(h[4], h[5], h[6], h[7]);  // the next 8 columns: +128 bytes
    }
}

// Bulk evaluation of n independent feature rows (nb_mlp_forward): every tile
// is 128 rows, row r of the tile in TMEM lane r.  Per tile one thread issues
// the three layers as tcgen05.mma; between them every thread loads its row
// from TMEM, adds the bias, applies tanh to packed BF16 pairs and stores the
// row as the next layer's A operand.  The input columns are in the order of
// the correction's records (infer_feature), so the weight image is shared.
__global__ void __launch_bounds__(kTcWarps * 32, kTcBlocksPerSm)
mlp_forward_tc(const UmmaW* __restrict__ Wg, const float* __restrict__ X, int64_t n,
               float* __restrict__ Y, unsigned* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TcSmem& S = *reinterpret_cast<TcSmem*>(smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u));
    const int tid = threadIdx.x, warp = tid >> 5;
    {
        const uint4* src = reinterpret_cast<const uint4*>(Wg);
        uint4* dst = reinterpret_cast<uint4*>(&S.W);
        for (int k = tid; k < (int)(sizeof(UmmaW) / 16); k += blockDim.x) dst[k] = src[k];
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&S.mbar)) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&S.xbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        S.fail = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&S.tmem)), "r"(kTcCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();  // the weights, stored through the generic proxy, feed the MMAs
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem;
    const uint32_t tlane = tmem + ((uint32_t)(32 * warp) << 16);  // this warp's lanes
    const uint32_t a1_addr = smem_u32(S.a1), a2_addr = smem_u32(S.a2);
    const uint32_t w1_addr = smem_u32(S.W.w1), w2_addr = smem_u32(S.W.w2),
                   w3_addr = smem_u32(S.W.w3);
    const int row = tid;  // this thread's tile row and TMEM lane
    uint32_t phase = 0;
    // the features of the CTA's first tile; each later tile's are copied in
    // while the tile before it runs through the network
    auto fetch = [&](int64_t tile) {
        const int64_t rows = std::min<int64_t>(kTcRows, n - tile * kTcRows);
        const unsigned bytes = (unsigned)(rows * kNin * sizeof(float));  // 48 B a row
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                         smem_u32(&S.xbar)),
                     "r"(bytes)
                     : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
            "[%3];" ::"r"(smem_u32(S.xs)),
            "l"(X + tile * kTcRows * kNin), "r"(bytes), "r"(smem_u32(&S.xbar))
            : "memory");
    };
    if (tid == 0 && (int64_t)blockIdx.x * kTcRows < n) fetch(blockIdx.x);
    uint32_t xphase = 0;
    for (int64_t tile = blockIdx.x; tile * kTcRows < n; tile += gridDim.x) {
        if (S.fail) break;  // uniform: set before the barrier that ended the last tile
        const int64_t sr = tile * kTcRows + row;
        if (!mbar_wait(&S.xbar, xphase)) S.fail = 1;
        xphase ^= 1u;
        uint32_t x[8];
        {
            float v[kNin];
            const float4* src = reinterpret_cast<const float4*>(S.xs + row * kNin);
#pragma unroll
            for (int q = 0; q < kNin / 4; ++q) {
                const float4 f = sr < n ? src[q] : make_float4(0.f, 0.f, 0.f, 0.f);
                v[4 * q] = f.x;
                v[4 * q + 1] = f.y;
                v[4 * q + 2] = f.z;
                v[4 * q + 3] = f.w;
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int f0 = infer_feature(2 * k), f1 = infer_feature(2 * k + 1);
                x[k] = pack_bf16(f0 >= 0 ? v[f0] : 0.f, f1 >= 0 ? v[f1] : 0.f);
            }
        }
        {
            uint4* dst = S.a1 + umma_off(row, 0, 256) / 16;
            dst[0] = make_uint4(x[0], x[1], x[2], x[3]);
            dst[8] = make_uint4(x[4], x[5], x[6], x[7]);
        }
        fence_async_smem();
        __syncthreads();  // every row of xs has been read: the next tile may land there
        if (tid == 0) {
            if ((tile + gridDim.x) * kTcRows < n) fetch(tile + gridDim.x);
            tc_fence_after();
            umma_bf16(tmem, umma_desc(a1_addr, 128, 256), umma_desc(w1_addr, 128, 256),
                      umma_idesc(kTcRows, kH), 0u);
            umma_commit(&S.mbar);
        }
        if (!mbar_wait(&S.mbar, phase)) S.fail = 1;
        phase ^= 1u;
        tc_fence_after();
        tc_hidden_row(tlane, 0u, S.W.b1, S.a2, row);

        tc_fence_before();
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
#pragma unroll
            for (int j = 0; j < 4; ++j)
                umma_bf16(tmem, umma_desc(a2_addr + 256u * j, 128, 1024),
                          umma_desc(w2_addr + 256u * j, 128, 1024), umma_idesc(kTcRows, kH),
                          j > 0 ? 1u : 0u);
            umma_commit(&S.mbar);
        }
        if (!mbar_wait(&S.mbar, phase)) S.fail = 1;
        phase ^= 1u;
        tc_fence_after();
        tc_hidden_row(tlane, 0u, S.W.b2, S.a2, row);

        tc_fence_before();
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
#pragma unroll
            for (int j = 0; j < 4; ++j)
                umma_bf16(tmem, umma_desc(a2_addr + 256u * j, 128, 1024),
                          umma_desc(w3_addr + 256u * j, 128, 1024), umma_idesc(kTcRows, 16),
                          j > 0 ? 1u : 0u);
            umma_commit(&S.mbar);
        }
        if (!mbar_wait(&S.mbar, phase)) S.fail = 1;
        phase ^= 1u;
        tc_fence_after();
        uint32_t y0, y1;
        tmem_ld2(tlane, y0, y1);
        if (sr < n) {
            Y[2 * sr] = __uint_as_float(y0) + S.W.b3[0];
            Y[2 * sr + 1] = __uint_as_float(y1) + S.W.b3[1];
        }
        tc_fence_before();
        __syncthreads();  // TMEM columns and operand rows are free for the next tile
    }
    if (S.fail) {
        // the last MMAs may still run, and the feature tile fetched for the
        // tile not taken: wait for both (bounded) before TMEM and the CTA go
        mbar_wait(&S.mbar, phase ^ 1u);
        mbar_wait(&S.xbar, xphase);
        if (tid == 0) atomicOr(err, kErrTimeout);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(kTcCols) : "memory");
    }
}

// ---- training on tcgen05: loss and gradients of a batch -----------------
// One CTA of 128 threads per SM walks 128-row tiles of the batch; row r of a
// tile is thread r and TMEM lane r.  Per tile, one thread issues
//   L1  h1 = tanh(x W1^T + b1)        M 128, N 64, K 16
//   L2  h2 = tanh(h1 W2^T + b2)       M 128, N 64, K 64
//   L3  y  = h2 W3^T + b3             M 128, N 16 (2 used), K 64
//   L4  dh1 = dp2 W2                  M 128, N 64, K 64   (dp2 = dy W3 (1 - h2^2))
// and, with the batch as K, the weight gradients accumulated in TMEM across
// the CTA's tiles:
//   [dp2^T; dp1^T] [h1^T; x^T; 1]     M 128, N 80, K 128: dW2, db2 (rows 0-63),
//                                     dW1, db1 (rows 64-127)
//   [dy^T; 0]      [h2^T; 1; 0]       M 128, N 80, K 128: dW3, db3 (rows 0-1)
// The transposed operands are written K-major by the epilogue threads, each
// its own column.  BF16 rounding points are those of the mma.sync kernel
// (inputs, weights, h1, h2, dy, dp2, dp1 enter the products as BF16; the bias
// sums take the BF16 dp and dy here).
constexpr uint32_t kGtCols = 256;      // TMEM columns: weight-gradient sums + layer accumulator
constexpr uint32_t kGtDwg = 0;         // [dW2 | dW1 | db] accumulator, 80 columns
constexpr uint32_t kGtDw3 = 96;        // [dW3 | db3] accumulator, 80 columns
constexpr uint32_t kGtLayer = 192;     // L1..L4 accumulators, 64 columns, reused

struct GtW {                            // BF16 K-major images of the weights
    alignas(128) uint4 w1[kH * 16 / 8];     // n = hidden x k = input (natural order, 12 used)
    alignas(128) uint4 w2[kH * kH / 8];     // n = out x k = in
    alignas(128) uint4 w3[16 * kH / 8];     // n = out (2 used) x k = hidden
    alignas(128) uint4 w2t[kH * kH / 8];    // n = in x k = out
    float b1[kH], b2[kH], b3[2];
    float w3f[2][kH];                       // W3 rounded to BF16, for dp2 on the CUDA cores
};

struct GtSmem {
    GtW W;
    alignas(128) uint4 a1[kTcRows * 16 / 8];     // x rows (K = 16), column 12 = 1 on valid rows
    alignas(128) uint4 a2[kTcRows * kH / 8];     // h1, then h2, then dp2 rows (K = 64)
    alignas(128) uint4 at[kTcRows * kTcRows / 8];  // [dp2^T; dp1^T] (K = 128 rows of the tile)
    alignas(128) uint4 bt1[80 * kTcRows / 8];    // [h1^T; x^T with the ones row] (K = 128)
    alignas(128) uint4 bt3[80 * kTcRows / 8];    // [h2^T; ones row; 0]
    alignas(128) uint4 a5[kTcRows * kTcRows / 8];  // [dy^T; 0]
    alignas(8) uint64_t mbar;
    uint32_t tmem;
    int fail;
    float loss;
};

__global__ void mlp_prepare_train_tc(const float* __restrict__ p, GtW* __restrict__ W) {
    auto put = [](uint4* img, int off, float v) {
        reinterpret_cast<__nv_bfloat16*>(img)[off / 2] = __float2bfloat16_rn(v);
    };
    for (int e = threadIdx.x; e < kH * 16; e += blockDim.x) {
        const int n = e / 16, k = e % 16;
        put(W->w1, umma_off(n, k, 256), k < kNin ? p[kW1 + n * kNin + k] : 0.f);
    }
    for (int e = threadIdx.x; e < kH * kH; e += blockDim.x) {
        const int n = e / kH, k = e % kH;
        put(W->w2, umma_off(n, k, 1024), p[kW2 + n * kH + k]);
        put(W->w2t, umma_off(n, k, 1024), p[kW2 + k * kH + n]);
    }
    for (int e = threadIdx.x; e < 16 * kH; e += blockDim.x) {
        const int n = e / kH, k = e % kH;
        put(W->w3, umma_off(n, k, 1024), n < 2 ? p[kW3 + n * kH + k] : 0.f);
    }
    for (int e = threadIdx.x; e < kH; e += blockDim.x) {
        W->b1[e] = p[kB1 + e];
        W->b2[e] = p[kB2 + e];
        W->w3f[0][e] = bf16_round(p[kW3 + e]);
        W->w3f[1][e] = bf16_round(p[kW3 + kH + e]);
    }
    if (threadIdx.x < 2) W->b3[threadIdx.x] = p[kB3 + threadIdx.x];
}

// element (row, k) of a K-major operand with 128 columns of K
__device__ __forceinline__ void put_t(uint4* img, int row, int k, float v) {
    reinterpret_cast<__nv_bfloat16*>(img)[umma_off(row, k, 2048) / 2] = __float2bfloat16_rn(v);
}

// Issues one MMA group (thread 0) and waits for it (every thread, bounded).
template <typename F>
__device__ __forceinline__ void gt_mma(GtSmem& S, uint32_t& phase, F issue) {
    tc_fence_before();
    fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
        tc_fence_after();
        issue();
        umma_commit(&S.mbar);
    }
    if (!mbar_wait(&S.mbar, phase)) S.fail = 1;
    phase ^= 1u;
    tc_fence_after();
}

__global__ void __launch_bounds__(kTcRows, 1)
mlp_grad_tc(const GtW* __restrict__ Wg, const float* __restrict__ X, const float* __restrict__ Yt,
            const int64_t* __restrict__ idx, int64_t n, float inv_n, float* __restrict__ grad,
            float* __restrict__ loss, unsigned* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GtSmem& S = *reinterpret_cast<GtSmem*>(smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    {
        const uint4* src = reinterpret_cast<const uint4*>(Wg);
        uint4* dst = reinterpret_cast<uint4*>(&S.W);
        for (int k = tid; k < (int)(sizeof(GtW) / 16); k += blockDim.x) dst[k] = src[k];
        // operands whose other rows stay zero: [dy^T; 0], [h2^T; 1; 0], x^T's padding rows
        for (int k = tid; k < kTcRows * kTcRows / 8; k += blockDim.x) S.a5[k] = make_uint4(0, 0, 0, 0);
        for (int k = tid; k < 80 * kTcRows / 8; k += blockDim.x) {
            S.bt1[k] = make_uint4(0, 0, 0, 0);
            S.bt3[k] = make_uint4(0, 0, 0, 0);
        }
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&S.mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        S.fail = 0;
        S.loss = 0.f;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&S.tmem)), "r"(kGtCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem;
    const uint32_t tlane = tmem + ((uint32_t)(32 * warp) << 16);
    const uint32_t a1 = smem_u32(S.a1), a2 = smem_u32(S.a2), at = smem_u32(S.at),
                   bt1 = smem_u32(S.bt1), bt3 = smem_u32(S.bt3), a5 = smem_u32(S.a5);
    const uint32_t w1 = smem_u32(S.W.w1), w2 = smem_u32(S.W.w2), w3 = smem_u32(S.W.w3),
                   w2t = smem_u32(S.W.w2t);
    const int r = tid;
    uint32_t phase = 0;
    bool first = true;
    float my_loss = 0.f;
    for (int64_t tile = blockIdx.x; tile * kTcRows < n; tile += gridDim.x) {
        if (S.fail) break;  // uniform: written before the barrier that ended the last wait
        const int64_t s = tile * kTcRows + r;
        const bool valid = s < n;
        const int64_t src = valid ? (idx ? idx[s] : s) : 0;
        // x: the row (A of L1) and its column of x^T (B of the weight gradients)
        {
            float x[16];
#pragma unroll
            for (int k = 0; k < 16; ++k)
                x[k] = valid && k < kNin ? X[src * kNin + k] : (valid && k == kNin ? 1.f : 0.f);
            uint32_t w[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) w[k] = pack_bf16(x[2 * k], x[2 * k + 1]);
            uint4* dst = S.a1 + umma_off(r, 0, 256) / 16;
            dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
            dst[8] = make_uint4(w[4], w[5], w[6], w[7]);
#pragma unroll
            for (int k = 0; k < 13; ++k) put_t(S.bt1, kH + k, r, x[k]);
        }
        const float t0 = valid ? Yt[2 * src] : 0.f, t1 = valid ? Yt[2 * src + 1] : 0.f;
        gt_mma(S, phase, [&] {
            umma_bf16(tmem + kGtLayer, umma_desc(a1, 128, 256), umma_desc(w1, 128, 256),
                      umma_idesc(kTcRows, kH), 0u);
        });
        // h1 = bf16(tanh(. + b1)): row of L2's A, column of h1^T, kept for dp1
        uint32_t h1p[32];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            uint32_t v[16];
            tmem_ld16(tlane + kGtLayer + 16 * c, v);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int o = 16 * c + 2 * j;
                h1p[8 * c + j] = pack_bf16(tanh_fast(__uint_as_float(v[2 * j]) + S.W.b1[o]),
                                           tanh_fast(__uint_as_float(v[2 * j + 1]) + S.W.b1[o + 1]));
            }
            uint4* dst = S.a2 + umma_off(r, 16 * c, 1024) / 16;
            dst[0] = make_uint4(h1p[8 * c], h1p[8 * c + 1], h1p[8 * c + 2], h1p[8 * c + 3]);
            dst[8] = make_uint4(h1p[8 * c + 4], h1p[8 * c + 5], h1p[8 * c + 6], h1p[8 * c + 7]);
        }
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            put_t(S.bt1, 2 * j, r, bf16_lo(h1p[j]));
            put_t(S.bt1, 2 * j + 1, r, bf16_hi(h1p[j]));
        }
        gt_mma(S, phase, [&] {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                umma_bf16(tmem + kGtLayer, umma_desc(a2 + 256u * j, 128, 1024),
                          umma_desc(w2 + 256u * j, 128, 1024), umma_idesc(kTcRows, kH),
                          j > 0 ? 1u : 0u);
        });
        uint32_t h2p[32];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            uint32_t v[16];
            tmem_ld16(tlane + kGtLayer + 16 * c, v);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int o = 16 * c + 2 * j;
                h2p[8 * c + j] = pack_bf16(tanh_fast(__uint_as_float(v[2 * j]) + S.W.b2[o]),
                                           tanh_fast(__uint_as_float(v[2 * j + 1]) + S.W.b2[o + 1]));
            }
            uint4* dst = S.a2 + umma_off(r, 16 * c, 1024) / 16;
            dst[0] = make_uint4(h2p[8 * c], h2p[8 * c + 1], h2p[8 * c + 2], h2p[8 * c + 3]);
            dst[8] = make_uint4(h2p[8 * c + 4], h2p[8 * c + 5], h2p[8 * c + 6], h2p[8 * c + 7]);
        }
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            put_t(S.bt3, 2 * j, r, bf16_lo(h2p[j]));
            put_t(S.bt3, 2 * j + 1, r, bf16_hi(h2p[j]));
        }
        put_t(S.bt3, kH, r, valid ? 1.f : 0.f);
        gt_mma(S, phase, [&] {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                umma_bf16(tmem + kGtLayer, umma_desc(a2 + 256u * j, 128, 1024),
                          umma_desc(w3 + 256u * j, 128, 1024), umma_idesc(kTcRows, 16),
                          j > 0 ? 1u : 0u);
        });
        float dy0 = 0.f, dy1 = 0.f;
        {
            uint32_t y0, y1;
            tmem_ld2(tlane + kGtLayer, y0, y1);
            if (valid) {
                const float d0 = __uint_as_float(y0) + S.W.b3[0] - t0;
                const float d1 = __uint_as_float(y1) + S.W.b3[1] - t1;
                my_loss += d0 * d0 + d1 * d1;
                dy0 = bf16_round(2.f * d0 * inv_n);
                dy1 = bf16_round(2.f * d1 * inv_n);
            }
        }
        put_t(S.a5, 0, r, dy0);
        put_t(S.a5, 1, r, dy1);
        // dp2 = (dy W3) (1 - h2^2): a row of L4's A and a column of dp2^T
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            uint32_t w[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int o = 16 * c + 2 * j;
                const float ha = bf16_lo(h2p[8 * c + j]), hb = bf16_hi(h2p[8 * c + j]);
                const float pa = fmaf(dy0, S.W.w3f[0][o], dy1 * S.W.w3f[1][o]) * (1.f - ha * ha);
                const float pb =
                    fmaf(dy0, S.W.w3f[0][o + 1], dy1 * S.W.w3f[1][o + 1]) * (1.f - hb * hb);
                w[j] = pack_bf16(pa, pb);
                put_t(S.at, o, r, pa);
                put_t(S.at, o + 1, r, pb);
            }
            uint4* dst = S.a2 + umma_off(r, 16 * c, 1024) / 16;
            dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
            dst[8] = make_uint4(w[4], w[5], w[6], w[7]);
        }
        gt_mma(S, phase, [&] {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                umma_bf16(tmem + kGtLayer, umma_desc(a2 + 256u * j, 128, 1024),
                          umma_desc(w2t + 256u * j, 128, 1024), umma_idesc(kTcRows, kH),
                          j > 0 ? 1u : 0u);
        });
        // dp1 = dh1 (1 - h1^2): a column of dp1^T
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            uint32_t v[16];
            tmem_ld16(tlane + kGtLayer + 16 * c, v);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int o = 16 * c + 2 * j;
                const float ha = bf16_lo(h1p[8 * c + j]), hb = bf16_hi(h1p[8 * c + j]);
                put_t(S.at, kH + o, r, valid ? __uint_as_float(v[2 * j]) * (1.f - ha * ha) : 0.f);
                put_t(S.at, kH + o + 1, r,
                      valid ? __uint_as_float(v[2 * j + 1]) * (1.f - hb * hb) : 0.f);
            }
        }
        // weight and bias gradients of the tile, added to the CTA's sums
        const uint32_t acc = first ? 0u : 1u;
        gt_mma(S, phase, [&] {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                umma_bf16(tmem + kGtDwg, umma_desc(at + 256u * j, 128, 2048),
                          umma_desc(bt1 + 256u * j, 128, 2048), umma_idesc(kTcRows, 80),
                          j > 0 ? 1u : acc);
                umma_bf16(tmem + kGtDw3, umma_desc(a5 + 256u * j, 128, 2048),
                          umma_desc(bt3 + 256u * j, 128, 2048), umma_idesc(kTcRows, 80),
                          j > 0 ? 1u : acc);
            }
        });
        first = false;
        __syncthreads();  // S.fail is read by every thread at the top of the loop
    }
    for (int o = 16; o > 0; o >>= 1) my_loss += __shfl_xor_sync(kFull, my_loss, o);
    if (lane == 0) atomicAdd(&S.loss, my_loss);
    if (S.fail) {
        mbar_wait(&S.mbar, phase ^ 1u);  // let an MMA in flight finish before TMEM is freed
        if (tid == 0) atomicOr(err, kErrTimeout);
    } else if (!first) {
        // row r of the sums: dW2[r] and db2[r] (r < 64) or dW1[r - 64] and db1[r - 64]
        uint32_t v[16];
        for (int c = 0; c < 5; ++c) {
            tmem_ld16(tlane + kGtDwg + 16 * c, v);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int col = 16 * c + j;
                const float g = __uint_as_float(v[j]);
                if (r < kH) {
                    if (col < kH) atomicAdd(grad + kW2 + r * kH + col, g);
                    else if (col == kH + kNin) atomicAdd(grad + kB2 + r, g);
                } else {
                    if (col >= kH && col < kH + kNin)
                        atomicAdd(grad + kW1 + (r - kH) * kNin + (col - kH), g);
                    else if (col == kH + kNin)
                        atomicAdd(grad + kB1 + (r - kH), g);
                }
            }
        }
        // rows 0 and 1 of the second sum: dW3 and db3
        for (int c = 0; c < 5; ++c) {
            tmem_ld16(tlane + kGtDw3 + 16 * c, v);
            if (r < 2) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = 16 * c + j;
                    const float g = __uint_as_float(v[j]);
                    if (col < kH) atomicAdd(grad + kW3 + r * kH + col, g);
                    else if (col == kH) atomicAdd(grad + kB3 + r, g);
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (tid == 0) atomicAdd(loss, S.loss * inv_n);
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(kGtCols) : "memory");
    }
}

inline unsigned blocks_for(int64_t n, int per) { return (unsigned)((n + per - 1) / per); }

}  // namespace

size_t mlp_infer_bytes() { return sizeof(InferW); }

void mlp_prepare_inference(nb_ctx* c) {
    mlp_prepare_infer<<<1, 256, 0, c->stream>>>(c->mlp_params, static_cast<InferW*>(c->mlp_infer));
}

void launch_mlp_correct(nb_ctx* c, const BodyBuffers& b, bool kick, bool store_acc) {
    c->launches += 1;
    const int smem = (int)sizeof(CorrSmem);
    // per context, so per device: the shared-memory attribute is a property
    // of the kernel on the current device
    if (c->corr_blocks_per_sm == 0) {
        cudaFuncSetAttribute(mlp_correct_kick, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        int blocks = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, mlp_correct_kick,
                                                          kCorrWarps * 32, smem) != cudaSuccess ||
            blocks < 1)
            blocks = 2;
        c->corr_blocks_per_sm = blocks;
    }
    mlp_correct_kick<<<c->sm_count * c->corr_blocks_per_sm, kCorrWarps * 32, smem, c->stream>>>(
        static_cast<const InferW*>(c->mlp_infer), c->tree, c->scal, b.pos, b.vel, c->acc32,
        store_acc ? c->acc : nullptr, (int)c->n, (float)c->p.epsilon_squared,
        c->p.G * c->p.timestep, c->p.timestep, kick ? 1 : 0);
}

void launch_mlp_samples(nb_ctx* c, const BodyBuffers& b, const int* pick, int npick, float* X,
                        float* Y, unsigned* count, unsigned cap) {
    const float thL = (float)c->p.theta, thB = band_theta(c);
    mlp_samples_kernel<<<c->sm_count * 8, kWarps * 32, 0, c->stream>>>(
        c->tree, c->scal, b.pos, b.mass, (int)c->n, pick, npick, thL * thL, thB * thB,
        c->p.epsilon_squared, (c->p.flags & NB_FLAG_QUADRUPOLE) ? 1 : 0, X, Y, count, cap);
}

size_t mlp_forward_image_bytes() { return sizeof(UmmaW); }

int mlp_forward_device(const float* params, const float* X, int64_t n, float* Y, void* image,
                       unsigned* err, int sm_count, cudaStream_t st) {
    UmmaW* W = static_cast<UmmaW*>(image);
    mlp_prepare_umma<<<1, 256, 0, st>>>(params, W);
    // 1 KB of slack to align the operands to 1024 bytes
    const int smem = (int)(sizeof(TcSmem) + 1024);
    cudaFuncSetAttribute(mlp_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    const int64_t tiles = (n + kTcRows - 1) / kTcRows;
    const int grid = (int)std::min<int64_t>(tiles, (int64_t)sm_count * kTcBlocksPerSm);
    mlp_forward_tc<<<grid, kTcWarps * 32, smem, st>>>(W, X, n, Y, err);
    return cudaGetLastError() == cudaSuccess ? NB_OK : NB_ERR_CUDA;
}

size_t mlp_train_image_bytes() { return sizeof(GtW); }

int mlp_grad_tc_device(const float* params, const float* X, const float* Yt, const int64_t* idx,
                       int64_t n, float* grad, float* loss, void* image, unsigned* err,
                       int sm_count, cudaStream_t st) {
    GtW* W = static_cast<GtW*>(image);
    mlp_prepare_train_tc<<<1, 256, 0, st>>>(params, W);
    const int smem = (int)(sizeof(GtSmem) + 1024);
    cudaFuncSetAttribute(mlp_grad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    const int64_t tiles = (n + kTcRows - 1) / kTcRows;
    const int grid = (int)std::min<int64_t>(tiles, (int64_t)sm_count);
    mlp_grad_tc<<<grid, kTcRows, smem, st>>>(W, X, Yt, idx, n, 1.f / (float)n, grad, loss, err);
    return cudaGetLastError() == cudaSuccess ? NB_OK : NB_ERR_CUDA;
}

int mlp_adam_device(float* p, const float* g, float* m, float* v, float lr, int step,
                    cudaStream_t st) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    mlp_adam_kernel<<<blocks_for(kYS, 256), 256, 0, st>>>(p, g, m, v, lr, b1, b2, 1e-8f, c1, c2);
    return cudaGetLastError() == cudaSuccess ? NB_OK : NB_ERR_CUDA;
}

}  // namespace nb
