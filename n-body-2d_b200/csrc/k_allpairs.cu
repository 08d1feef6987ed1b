// k_allpairs.cu -- FP64 all-pairs accelerations on the GPU (error oracle).
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

}  // namespace

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
