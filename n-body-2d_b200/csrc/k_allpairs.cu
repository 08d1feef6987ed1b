// k_allpairs.cu -- FP64 all-pairs accelerations on the GPU: the error oracle
// (nb_allpairs_accelerations) and the NB_MODE_ALLPAIRS step.
//
// a_i = sum_{j != i} m_j d_ij (|d_ij|^2 + eps2)^-3/2, the pair law of the
// reference GPU backend (BarnesHutCuda.cu:427-431) without any tree.  Used to
// state p50/p99 force errors at full size, where a CPU all-pairs sum is too
// slow.  Sources are staged through shared memory in tiles; each thread owns
// one target.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "nb_internal.cuh"
#include "nbody_b200.h"

namespace {

constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads)
allpairs_fp64(const double2* __restrict__ pos, const double* __restrict__ mass, int64_t n,
              const int64_t* __restrict__ targets, int64_t k, double eps2, double2* __restrict__ acc) {
    __shared__ double2 sp[kThreads];
    __shared__ double sm[kThreads];
    const int64_t t = blockIdx.x * (int64_t)kThreads + threadIdx.x;
    const int64_t me = t < k ? targets[t] : -1;
    const double2 p = me >= 0 ? pos[me] : make_double2(0.0, 0.0);
    double ax = 0.0, ay = 0.0;
    for (int64_t base = 0; base < n; base += kThreads) {
        const int64_t j = base + threadIdx.x;
        sp[threadIdx.x] = j < n ? pos[j] : make_double2(0.0, 0.0);
        sm[threadIdx.x] = j < n ? mass[j] : 0.0;
        __syncthreads();
        const int lim = (int)min((int64_t)kThreads, n - base);
        for (int q = 0; q < lim; ++q) {
            if (base + q == me) continue;
            const double dx = sp[q].x - p.x;
            const double dy = sp[q].y - p.y;
            const double d2 = dx * dx + dy * dy + eps2;
            const double inv_r = 1.0 / sqrt(d2);
            const double a = sm[q] * inv_r * inv_r * inv_r;
            ax += dx * a;
            ay += dy * a;
        }
        __syncthreads();
    }
    if (t < k) acc[t] = make_double2(ax, ay);
}

// NB_MODE_ALLPAIRS, stage 1 (AllPairs.cpp:31-35): b = a with x += v dt (or a
// plain copy when only accelerations are wanted).
__global__ void allpairs_drift(nb::BodyBuffers a, nb::BodyBuffers b, int64_t n, double dt) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double2 p = a.pos[i], v = a.vel[i];
    // x + v dt rounded twice, as the reference's `pos += vel * timestep`
    b.pos[i] = make_double2(__dadd_rn(p.x, __dmul_rn(v.x, dt)), __dadd_rn(p.y, __dmul_rn(v.y, dt)));
    b.vel[i] = v;
    b.mass[i] = a.mass[i];
    b.orig[i] = a.orig[i];
}

// Stage 2 (AllPairs.cpp:38-49): every body sums all others (each pair is
// evaluated from both sides: twice the reference's pair evaluations, no
// atomics).  kCpuLaw: the law of Simulation::force,
// a = m (p_j - p_i) / (d (d^2 + eps2)) (Simulation.cpp:74-80, G applied with
// the kick); otherwise Plummer's a = m (p_j - p_i) (d^2 + eps2)^-3/2.  Block
// (x, y) sums targets x*256.. over source chunk y; small systems split the
// sources into chunks so that the grid fills the GPU, and the partial sums
// are added in chunk order by the kick (deterministic).
template <bool kCpuLaw>
__global__ void __launch_bounds__(kThreads)
allpairs_partial(const double2* __restrict__ pos, const double* __restrict__ mass, int64_t n,
                 int64_t chunk, double eps2, double2* __restrict__ partial) {
    __shared__ double2 sp[kThreads];
    __shared__ double sm[kThreads];
    const int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
    const double2 p = i < n ? pos[i] : make_double2(0.0, 0.0);
    const int64_t s0 = blockIdx.y * chunk, s1 = min(n, s0 + chunk);
    double ax = 0.0, ay = 0.0;
    for (int64_t base = s0; base < s1; base += kThreads) {
        const int64_t j = base + threadIdx.x;
        sp[threadIdx.x] = j < s1 ? pos[j] : make_double2(0.0, 0.0);
        sm[threadIdx.x] = j < s1 ? mass[j] : 0.0;
        __syncthreads();
        const int lim = (int)min((int64_t)kThreads, s1 - base);
        for (int q = 0; q < lim; ++q) {
            if (base + q == i) continue;
            const double dx = sp[q].x - p.x;
            const double dy = sp[q].y - p.y;
            const double r2 = dx * dx + dy * dy;
            double a;
            if (kCpuLaw) {
                a = sm[q] / (sqrt(r2) * (r2 + eps2));
            } else {
                const double inv_r = 1.0 / sqrt(r2 + eps2);
                a = sm[q] * inv_r * inv_r * inv_r;
            }
            ax += dx * a;
            ay += dy * a;
        }
        __syncthreads();
    }
    if (i < n) partial[blockIdx.y * n + i] = make_double2(ax, ay);
}

__global__ void allpairs_kick(const double2* __restrict__ partial, int chunks, int64_t n,
                              double2* __restrict__ vel, double2* __restrict__ acc_out,
                              double G_dt, int kick, unsigned long long* __restrict__ body_terms) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double ax = 0.0, ay = 0.0;
    for (int c = 0; c < chunks; ++c) {
        const double2 a = partial[c * n + i];
        ax += a.x;
        ay += a.y;
    }
    if (acc_out) acc_out[i] = make_double2(ax, ay);
    if (kick) {
        double2 v = vel[i];
        v.x += ax * G_dt;
        v.y += ay * G_dt;
        vel[i] = v;
    }
    if (threadIdx.x == 0)
        atomicAdd(body_terms, (unsigned long long)min((int64_t)blockDim.x, n - i) * (n - 1));
}

}  // namespace

int nb::allpairs_chunks(int64_t n, int sm_count) {
    const int64_t xblocks = (n + kThreads - 1) / kThreads;
    const int64_t want = (int64_t)sm_count * 8;  // blocks to fill the GPU a few times over
    int64_t chunks = (want + xblocks - 1) / xblocks;
    chunks = std::min<int64_t>(chunks, std::max<int64_t>(1, n / kThreads));
    return (int)std::max<int64_t>(1, std::min<int64_t>(chunks, 64));
}

void nb::launch_allpairs_step(nb_ctx* c, const BodyBuffers& a, const BodyBuffers& b, bool integrate,
                              bool store_acc) {
    const unsigned blocks = (unsigned)((c->n + kThreads - 1) / kThreads);
    const int chunks = allpairs_chunks(c->n, c->sm_count);
    const int64_t chunk = (c->n + chunks - 1) / chunks;
    c->launches += 3;
    allpairs_drift<<<blocks, kThreads, 0, c->stream>>>(a, b, c->n, integrate ? c->p.timestep : 0.0);
    const dim3 grid(blocks, (unsigned)chunks);
    if (c->p.flags & NB_FLAG_CPU_LAW)
        allpairs_partial<true><<<grid, kThreads, 0, c->stream>>>(b.pos, b.mass, c->n, chunk,
                                                                c->p.epsilon_squared, c->ap_partial);
    else
        allpairs_partial<false><<<grid, kThreads, 0, c->stream>>>(b.pos, b.mass, c->n, chunk,
                                                                 c->p.epsilon_squared, c->ap_partial);
    allpairs_kick<<<blocks, kThreads, 0, c->stream>>>(c->ap_partial, chunks, c->n, b.vel,
                                                       store_acc ? c->acc : nullptr,
                                                       c->p.G * c->p.timestep, integrate ? 1 : 0,
                                                       &c->scal->body_terms);
}

extern "C" int nb_allpairs_accelerations(int32_t device, uint64_t n, const double* mass,
                                         const double* pos_xy, uint64_t k, const int64_t* targets,
                                         double epsilon_squared, double* acc_xy) {
    if (!mass || !pos_xy || !targets || !acc_xy || n == 0 || k == 0) return NB_ERR_INVALID;
    if (!std::isfinite(epsilon_squared) || epsilon_squared < 0.0) return NB_ERR_INVALID;
    for (uint64_t i = 0; i < k; ++i)
        if (targets[i] < 0 || (uint64_t)targets[i] >= n) return NB_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return NB_ERR_NOTFOUND;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    double2 *dpos = nullptr, *dacc = nullptr;
    double* dmass = nullptr;
    int64_t* dtgt = nullptr;
    cudaStream_t st = nullptr;
    int rc = NB_OK;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&dpos, n * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&dmass, n * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&dtgt, k * sizeof(int64_t)) != cudaSuccess ||
        cudaMalloc(&dacc, k * sizeof(double2)) != cudaSuccess) {
        rc = NB_ERR_NOMEM;
    }
    if (rc == NB_OK) {
        cudaMemcpyAsync(dpos, pos_xy, n * sizeof(double2), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(dmass, mass, n * sizeof(double), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(dtgt, targets, k * sizeof(int64_t), cudaMemcpyHostToDevice, st);
        const unsigned blocks = (unsigned)((k + kThreads - 1) / kThreads);
        allpairs_fp64<<<blocks, kThreads, 0, st>>>(dpos, dmass, (int64_t)n, dtgt, (int64_t)k,
                                                   epsilon_squared, dacc);
        cudaMemcpyAsync(acc_xy, dacc, k * sizeof(double2), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess)
            rc = NB_ERR_CUDA;
    }
    cudaFree(dpos);
    cudaFree(dmass);
    cudaFree(dtgt);
    cudaFree(dacc);
    if (st) cudaStreamDestroy(st);
    cudaSetDevice(prev);
    return rc;
}
