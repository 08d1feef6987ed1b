// nb_static.cu -- the one entry point that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc: a renderer that steps
// the simulation once per frame cannot afford the device-wide
// synchronisation cudaMalloc/cudaFree may cause in the middle of its frame,
// and host programs that own all device memory through their own pool
// (fixed budgets, custom allocators) hand libraries buffers instead of
// letting them allocate.  For those callers nb_morton_sort_static runs the
// bounding-box, Morton-code and radix-sort stage of the step on buffers the
// caller owns, with its scratch in the file-scope device array below instead
// of cudaMalloc'd memory.
//
// The array is part of the library image, so every GPU that loads the library
// holds it (NB_STATIC_SORT_MAX_BODIES x 24 bytes plus about 100 KB of per-tile
// digit counts and reduction partials: 6.4 MB in all) until the process
// exits.  All calls on a device share it and it keeps the contents of
// the last call; calls that overlap on the GPU (two streams, or two host
// threads) race on it and must be serialised by the caller.
#include <cuda_runtime.h>
#include <stdint.h>

#include "nb_internal.cuh"

namespace {

constexpr int64_t kMaxBodies = NB_STATIC_SORT_MAX_BODIES;
constexpr int kMaxTiles = (int)((kMaxBodies + nb::kSortTile - 1) / nb::kSortTile);
constexpr int kBoxBlocks = 256;

// Scratch layout (all offsets multiples of 256 bytes).
constexpr size_t kKeyBytes = sizeof(uint64_t) * kMaxBodies;
constexpr size_t kValBytes = sizeof(uint32_t) * kMaxBodies;
constexpr size_t kOffKey0 = 0;
constexpr size_t kOffKey1 = kOffKey0 + kKeyBytes;
constexpr size_t kOffVal0 = kOffKey1 + kKeyBytes;
constexpr size_t kOffVal1 = kOffVal0 + kValBytes;
constexpr size_t kOffCounts = kOffVal1 + kValBytes;
constexpr size_t kOffTotals = kOffCounts + sizeof(uint32_t) * 256 * kMaxTiles;
constexpr size_t kOffPartials = kOffTotals + sizeof(uint32_t) * 256;
constexpr size_t kOffScalars = kOffPartials + sizeof(double) * 4 * kBoxBlocks;
constexpr size_t kScratchBytes = kOffScalars + ((sizeof(nb::DeviceScalars) + 255) / 256) * 256;
static_assert(kScratchBytes - kOffCounts < 100 * 1024 && kScratchBytes < 6400 * 1000,
              "the documented size of the scratch array (6.4 MB, ~100 KB beyond the keys) is stale");
static_assert(kOffKey1 % 256 == 0 && kOffVal0 % 256 == 0 && kOffVal1 % 256 == 0 &&
                  kOffCounts % 256 == 0 && kOffTotals % 256 == 0 && kOffPartials % 256 == 0 &&
                  kOffScalars % 256 == 0,
              "scratch regions must stay 256-byte aligned");

static __device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

// Device address of the scratch array in the current device's context.  Host
// code only holds a host-side stand-in for the symbol, so the address is
// asked for on every call: a cached value would go stale after
// cudaDeviceReset or under another context, and the lookup is cheap once the
// library's device image is loaded (the first call on a device loads it).
int scratch_for_current_device(unsigned char** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return NB_ERR_NOTFOUND;
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_sort_scratch) != cudaSuccess || !p) return NB_ERR_CUDA;
    *out = static_cast<unsigned char*>(p);
    return NB_OK;
}

}  // namespace

extern "C" int nb_morton_sort_static(const double* pos_xy, uint64_t n, uint64_t* codes,
                                     int32_t* order, double* box, void* stream) {
    if (!pos_xy || !codes || !order || n == 0) return NB_ERR_INVALID;
    if (n > (uint64_t)kMaxBodies) return NB_ERR_CAPACITY;
    unsigned char* base = nullptr;
    const int rc = scratch_for_current_device(&base);
    if (rc != NB_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint64_t* const key[2] = {reinterpret_cast<uint64_t*>(base + kOffKey0),
                              reinterpret_cast<uint64_t*>(base + kOffKey1)};
    uint32_t* const val[2] = {reinterpret_cast<uint32_t*>(base + kOffVal0),
                              reinterpret_cast<uint32_t*>(base + kOffVal1)};
    auto* scal = reinterpret_cast<nb::DeviceScalars*>(base + kOffScalars);
    // The scratch keeps the previous call's contents: the bounding-box
    // reduction's block counter must start at zero.
    if (cudaMemsetAsync(&scal->bbox_ticket, 0, sizeof(unsigned), st) != cudaSuccess)
        return NB_ERR_CUDA;
    nb::launch_morton_sort_raw(reinterpret_cast<const double2*>(pos_xy), (int64_t)n, key, val,
                               codes, reinterpret_cast<uint32_t*>(order),
                               reinterpret_cast<uint32_t*>(base + kOffCounts),
                               reinterpret_cast<uint32_t*>(base + kOffTotals),
                               reinterpret_cast<double*>(base + kOffPartials), kBoxBlocks, scal, st);
    if (cudaGetLastError() != cudaSuccess) return NB_ERR_CUDA;
    if (box && cudaMemcpyAsync(box, scal->box, 4 * sizeof(double), cudaMemcpyDeviceToDevice, st) !=
                   cudaSuccess)
        return NB_ERR_CUDA;
    return NB_OK;
}
