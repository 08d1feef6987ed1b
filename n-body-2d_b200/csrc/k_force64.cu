// k_force64.cu -- FP64 parity traversal, kick, drift and the original-order
// scatter.
//
// The traversal keeps the reference's semantics (BarnesHutCuda.cu:382-486):
// one target body per thread, a depth-first walk that visits children in
// quadrant order, the per-body opening test width^2 < theta^2 d^2 against the
// cell's centre of mass, the Plummer pair law a += d m (d^2 + eps^2)^-3/2, no
// opening test for a multi-body leaf that does not hold the target, and the
// kick v += a G dt.  On the compressed tree a cell is tested at its own
// (deepest-chain) level, which decides exactly as the reference's chain does;
// a multi-body leaf that holds the target is first tested at level 29 when the
// reference reaches it through a chain of single-child cells, because the
// reference may accept such a chain (and so the target's own mass) when
// theta > 1/sqrt(2).
#include <climits>
#include <cuda_runtime.h>
#include <stdint.h>

#include "nb_internal.cuh"

namespace nb {
namespace {

constexpr int kThreads = 128;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ void plummer(double dx, double dy, double m, double eps2, double& ax,
                                        double& ay) {
    const double d2 = dx * dx + dy * dy + eps2;
    const double inv_r = rsqrt(d2);
    const double inv_r3 = inv_r * inv_r * inv_r;
    const double a = m * inv_r3;
    ax += dx * a;
    ay += dy * a;
}

__global__ void __launch_bounds__(kThreads)
force_fp64(const double2* __restrict__ pos, const double* __restrict__ mass, double2* __restrict__ vel,
           double2* __restrict__ acc_out, int n, Tree t, DeviceScalars* __restrict__ s, double eps2,
           double theta_sq, double G_dt, int kick, uint2* __restrict__ terms_out) {
    __shared__ double wsq[kMaxLevel + 1];
    if (threadIdx.x <= kMaxLevel) wsq[threadIdx.x] = s->wsq[threadIdx.x];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int cells = s->cells;
    unsigned long long ncell = 0, pairs = 0;
    int deepest = 0;  // stack entries in use after the fullest push
    if (i < n) {
        const double2 me = pos[i];
        double ax = 0.0, ay = 0.0;
        int stack[kStackDepth];
        int top = 0;
        deepest = 1;
        stack[0] = s->root;
        while (top >= 0) {
            const int ref = stack[top--];
            if (ref >= 0) {
                const int lv = ref < cells ? t.level[ref] : -1;
                if (lv < 0 || lv >= kMaxLevel) {
                    atomicOr(&s->error, kErrTree);
                    break;
                }
                const double m = t.mass[ref];
                const double2 cc = t.com[ref];
                const double dx = cc.x - me.x;
                const double dy = cc.y - me.y;
                const double dist_sq = dx * dx + dy * dy;
                if (wsq[lv] < theta_sq * dist_sq) {
                    plummer(dx, dy, m, eps2, ax, ay);
                    ++ncell;
                    continue;
                }
                const int4 ch = t.child[ref];
                if (top + 4 >= kStackDepth) {
                    atomicOr(&s->error, kErrStack);
                    break;
                }
                // push in reverse so child 0 is walked first (CU:474-481)
                if (ch.w != INT_MIN) stack[++top] = ch.w;
                if (ch.z != INT_MIN) stack[++top] = ch.z;
                if (ch.y != INT_MIN) stack[++top] = ch.y;
                stack[++top] = ch.x;
                deepest = max(deepest, top + 1);
                continue;
            }
            const int b = ~ref;
            const int e = t.leaf_last[b];
            if (e < b || e >= n) {
                atomicOr(&s->error, kErrTree);
                break;
            }
            if (b == e) {  // single-body leaf, CU:424-433
                if (b != i) {
                    const double2 p = pos[b];
                    plummer(p.x - me.x, p.y - me.y, mass[b], eps2, ax, ay);
                    ++pairs;
                }
                continue;
            }
            const double m = t.bucket_mass[b];
            const double2 cc = t.bucket_com[b];
            const double dx = cc.x - me.x;
            const double dy = cc.y - me.y;
            if (i < b || i > e) {  // CU:434-442
                plummer(dx, dy, m, eps2, ax, ay);
                ++ncell;
                continue;
            }
            const int plevel = t.leaf_plevel[b];
            if (plevel < kMaxLevel - 1 && wsq[kMaxLevel - 1] < theta_sq * (dx * dx + dy * dy)) {
                plummer(dx, dy, m, eps2, ax, ay);
                ++ncell;
                continue;
            }
            for (int j = b; j <= e; ++j) {  // CU:443-457
                if (j == i) continue;
                const double2 p = pos[j];
                plummer(p.x - me.x, p.y - me.y, mass[j], eps2, ax, ay);
                ++pairs;
            }
        }
        if (acc_out) acc_out[i] = make_double2(ax, ay);
        if (terms_out) terms_out[i] = make_uint2((unsigned)ncell, (unsigned)pairs);
        if (kick) {
            double2 v = vel[i];
            v.x += ax * G_dt;
            v.y += ay * G_dt;
            vel[i] = v;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        ncell += __shfl_xor_sync(kFull, ncell, o);
        pairs += __shfl_xor_sync(kFull, pairs, o);
        deepest = max(deepest, __shfl_xor_sync(kFull, deepest, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&s->cell_terms, ncell);
        atomicAdd(&s->body_terms, pairs);
        atomicMax(&s->stack_hw, deepest);
    }
}

// Drift, CU:489-495.
__global__ void drift_kernel(double2* __restrict__ pos, const double2* __restrict__ vel, int64_t n,
                             double dt) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double2 p = pos[i];
    const double2 v = vel[i];
    p.x += v.x * dt;
    p.y += v.y * dt;
    pos[i] = p;
}

// CU:498-506, plus the optional accelerations.
__global__ void scatter_kernel(const double2* __restrict__ pos, const double2* __restrict__ vel,
                               const int32_t* __restrict__ orig, int64_t n, double2* out_pos,
                               double2* out_vel, const double2* __restrict__ acc,
                               double2* out_acc) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t o = orig[i];
    if (out_pos) out_pos[o] = pos[i];
    if (out_vel) out_vel[o] = vel[i];
    if (out_acc) out_acc[o] = acc[i];
}

// Uploaded bodies: orig = identity, and the checks nb_upload promises
// (finite positions and velocities, positive finite masses) done on the
// device: bit 0 of *bad for a non-finite value, bit 1 for a mass <= 0.
__global__ void upload_kernel(int32_t* __restrict__ orig, const double* __restrict__ mass,
                              const double2* __restrict__ pos, const double2* __restrict__ vel,
                              int64_t n, unsigned* __restrict__ bad) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (orig) orig[i] = (int32_t)i;
    const double m = mass[i];
    const double2 p = pos[i], v = vel[i];
    unsigned f = 0;
    if (!(isfinite(m) && isfinite(p.x) && isfinite(p.y) && isfinite(v.x) && isfinite(v.y))) f |= 1u;
    if (!(m > 0.0)) f |= 2u;
    if (__any_sync(__activemask(), f != 0) && f) atomicOr(bad, f);
}

// Moves checked staged bodies into the state in original order.  After a
// rejected check the state keeps its bodies: when they live in another
// buffer (keep != dst) they are copied over, since the next step reads dst.
__global__ void upload_commit(const double* __restrict__ sm, const double2* __restrict__ sp,
                              const double2* __restrict__ sv, BodyBuffers keep, BodyBuffers dst,
                              int64_t n, const unsigned* __restrict__ bad,
                              unsigned* __restrict__ err) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (*bad) {
        if (i == 0) atomicOr(err, kErrUpload);
        if (keep.mass == dst.mass) return;
        dst.orig[i] = keep.orig[i];
        dst.mass[i] = keep.mass[i];
        dst.pos[i] = keep.pos[i];
        dst.vel[i] = keep.vel[i];
        return;
    }
    dst.orig[i] = (int32_t)i;
    dst.mass[i] = sm[i];
    dst.pos[i] = sp[i];
    dst.vel[i] = sv[i];
}

__global__ void identity_kernel(int32_t* orig, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) orig[i] = (int32_t)i;
}

inline unsigned blocks_for(int64_t n, int threads) {
    return (unsigned)((n + threads - 1) / threads);
}

}  // namespace

void launch_force_fp64(nb_ctx* c, const BodyBuffers& b, bool kick, bool store_acc) {
    const double theta_sq = c->p.theta * c->p.theta;
    const double G_dt = c->p.G * c->p.timestep;
    c->launches += 1;
    force_fp64<<<blocks_for(c->n, kThreads), kThreads, 0, c->stream>>>(
        b.pos, b.mass, b.vel, store_acc ? c->acc : nullptr, (int)c->n, c->tree, c->scal,
        c->p.epsilon_squared, theta_sq, G_dt, kick ? 1 : 0, c->want_terms ? c->dbg_terms : nullptr);
}

void launch_drift(nb_ctx* c, const BodyBuffers& b) {
    c->launches += 1;
    drift_kernel<<<blocks_for(c->n, 256), 256, 0, c->stream>>>(b.pos, b.vel, c->n, c->p.timestep);
}

void launch_scatter(nb_ctx* c, const BodyBuffers& b, double2* out_pos, double2* out_vel,
                    const double2* acc, double2* out_acc) {
    c->launches += 1;
    scatter_kernel<<<blocks_for(c->n, 256), 256, 0, c->stream>>>(b.pos, b.vel, b.orig, c->n, out_pos,
                                                                 out_vel, acc, out_acc);
}

void launch_identity(nb_ctx* c, int32_t* orig) {
    c->launches += 1;
    identity_kernel<<<blocks_for(c->n, 256), 256, 0, c->stream>>>(orig, c->n);
}

void launch_upload_commit(nb_ctx* c, const double* m, const double2* p, const double2* v,
                          const BodyBuffers& keep, const BodyBuffers& dst, unsigned* bad) {
    c->launches += 2;
    cudaMemsetAsync(bad, 0, sizeof(unsigned), c->stream);
    upload_kernel<<<blocks_for(c->n, 256), 256, 0, c->stream>>>(nullptr, m, p, v, c->n, bad);
    upload_commit<<<blocks_for(c->n, 256), 256, 0, c->stream>>>(m, p, v, keep, dst, c->n, bad,
                                                                 &c->scal->error);
}

void launch_upload_check(nb_ctx* c, const BodyBuffers& b, unsigned* bad) {
    c->launches += 1;
    upload_kernel<<<blocks_for(c->n, 256), 256, 0, c->stream>>>(b.orig, b.mass, b.pos, b.vel, c->n,
                                                                 bad);
}

}  // namespace nb
