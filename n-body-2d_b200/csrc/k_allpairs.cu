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

// Stage 2 (AllPairs.cpp:38-49): every body sums all others (the sum runs over
// j in order, each pair evaluated from both sides: twice the reference's pair
// evaluations, no atomics), then v += a G dt.  kCpuLaw: the law of
// Simulation::force, a = m (p_j - p_i) / (d (d^2 + eps2)) (Simulation.cpp:
// 74-80, G applied with the kick); otherwise Plummer's
// a = m (p_j - p_i) (d^2 + eps2)^-3/2.
template <bool kCpuLaw>
__global__ void __launch_bounds__(kThreads)
allpairs_kick(double2* __restrict__ pos, const double* __restrict__ mass, double2* __restrict__ vel,
              double2* __restrict__ acc_out, int64_t n, double eps2, double G_dt, int kick,
              unsigned long long* __restrict__ body_terms) {
    __shared__ double2 sp[kThreads];
    __shared__ double sm[kThreads];
    const int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
    const double2 p = i < n ? pos[i] : make_double2(0.0, 0.0);
    double ax = 0.0, ay = 0.0;
    for (int64_t base = 0; base < n; base += kThreads) {
        const int64_t j = base + threadIdx.x;
        sp[threadIdx.x] = j < n ? pos[j] : make_double2(0.0, 0.0);
        sm[threadIdx.x] = j < n ? mass[j] : 0.0;
        __syncthreads();
        const int lim = (int)min((int64_t)kThreads, n - base);
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
    if (i >= n) return;
    if (acc_out) acc_out[i] = make_double2(ax, ay);
    if (kick) {
        double2 v = vel[i];
        v.x += ax * G_dt;
        v.y += ay * G_dt;
        vel[i] = v;
    }
    if (threadIdx.x == 0) atomicAdd(body_terms, (unsigned long long)min((int64_t)kThreads, n - i) * (n - 1));
}

}  // namespace

void nb::launch_allpairs_step(nb_ctx* c, const BodyBuffers& a, const BodyBuffers& b, bool integrate,
                              bool store_acc) {
    const unsigned blocks = (unsigned)((c->n + kThreads - 1) / kThreads);
    c->launches += 2;
    allpairs_drift<<<blocks, kThreads, 0, c->stream>>>(a, b, c->n, integrate ? c->p.timestep : 0.0);
    const double G_dt = c->p.G * c->p.timestep;
    double2* acc = store_acc ? c->acc : nullptr;
    if (c->p.flags & NB_FLAG_CPU_LAW)
        allpairs_kick<true><<<blocks, kThreads, 0, c->stream>>>(b.pos, b.mass, b.vel, acc, c->n,
                                                                c->p.epsilon_squared, G_dt,
                                                                integrate ? 1 : 0,
                                                                &c->scal->body_terms);
    else
        allpairs_kick<false><<<blocks, kThreads, 0, c->stream>>>(b.pos, b.mass, b.vel, acc, c->n,
                                                                 c->p.epsilon_squared, G_dt,
                                                                 integrate ? 1 : 0,
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
