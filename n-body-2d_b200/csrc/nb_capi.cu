// nb_capi.cu -- the extern "C" surface of libnbody_b200.so (include/nbody_b200.h).
//
// Owns the context: device buffers (allocated once, as init_device_resources
// does at BarnesHutCuda.cu:550-606), the stream, and one captured CUDA graph
// per buffer parity that holds a whole step, so a step costs one graph launch
// and no host synchronisation (the reference synchronises ~40 times per step).
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>
#include <algorithm>

#include "nb_internal.cuh"

namespace {

int fail(nb_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

#define NB_CUDA(ctx, call)                                                                     \
    do {                                                                                       \
        const cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                                 \
            return fail((ctx), NB_ERR_CUDA,                                                    \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                   \
    } while (0)

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
    return cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * (count ? count : 1));
}


int check_params(const nb_params* p) {
    if (!p) return NB_ERR_INVALID;
    if (!std::isfinite(p->G) || !std::isfinite(p->timestep) || !std::isfinite(p->theta) ||
        !std::isfinite(p->epsilon_squared) || !std::isfinite(p->bmax_ratio) ||
        !std::isfinite(p->band_theta))
        return NB_ERR_INVALID;
    if (p->theta < 0.0 || p->epsilon_squared < 0.0 || p->bmax_ratio < 0.0 || p->band_theta < 0.0)
        return NB_ERR_INVALID;
    if (p->mode != NB_MODE_FP64 && p->mode != NB_MODE_SPLIT && p->mode != NB_MODE_ALLPAIRS)
        return NB_ERR_INVALID;
    if (p->bodies_per_lane != 0 && p->bodies_per_lane != 1 && p->bodies_per_lane != 2 &&
        p->bodies_per_lane != 4)
        return NB_ERR_INVALID;
    if (p->reserved != 0) return NB_ERR_INVALID;
    if (p->leaf_size < 0 ||
        (p->flags & ~(int32_t)(NB_FLAG_QUADRUPOLE | NB_FLAG_LEARNED | NB_FLAG_CPU_LAW)) != 0)
        return NB_ERR_INVALID;
    if ((p->flags & (NB_FLAG_LEARNED | NB_FLAG_QUADRUPOLE)) && p->mode != NB_MODE_SPLIT)
        return NB_ERR_INVALID;
    if ((p->flags & NB_FLAG_CPU_LAW) && p->mode != NB_MODE_ALLPAIRS) return NB_ERR_INVALID;
    return NB_OK;
}

int alloc_all(nb_ctx* c) {
    const size_t n = (size_t)c->n;
    for (int k = 0; k < 2; ++k) {
        NB_CUDA(c, dalloc(&c->buf[k].pos, n));
        NB_CUDA(c, dalloc(&c->buf[k].vel, n));
        NB_CUDA(c, dalloc(&c->buf[k].mass, n));
        NB_CUDA(c, dalloc(&c->buf[k].orig, n));
        NB_CUDA(c, dalloc(&c->sort.key[k], n));
        NB_CUDA(c, dalloc(&c->sort.val[k], n));
    }
    c->sort.tiles = (int)((n + nb::kSortTile - 1) / nb::kSortTile);
    NB_CUDA(c, dalloc(&c->sort.counts, (size_t)256 * c->sort.tiles));
    NB_CUDA(c, dalloc(&c->sort.totals, 256));
    NB_CUDA(c, dalloc(&c->sort.hist, 8 * 256));
    NB_CUDA(c, dalloc(&c->sort.status, (size_t)8 * 256 * c->sort.tiles));
    NB_CUDA(c, dalloc(&c->sort.tile_counter, 8));
    NB_CUDA(c, dalloc(&c->sort.ties_small, n / 2 + 1));
    NB_CUDA(c, dalloc(&c->sort.ties_big, n / 33 + 1));
    c->scan.blocks = (int)((n + 2047) / 2048);
    NB_CUDA(c, dalloc(&c->scan.block_sums, (size_t)c->scan.blocks));
    nb::Tree& t = c->tree;
    NB_CUDA(c, dalloc(&t.level, n));
    NB_CUDA(c, dalloc(&t.child, n));
    NB_CUDA(c, dalloc(&t.parent, n));
    NB_CUDA(c, dalloc(&t.nint, n));
    NB_CUDA(c, dalloc(&t.ready, n));
    NB_CUDA(c, dalloc(&t.mass, n));
    NB_CUDA(c, dalloc(&t.com, n));
    NB_CUDA(c, dalloc(&t.range, n));
    NB_CUDA(c, dalloc(&t.start_list, n));
    if (c->p.mode == NB_MODE_ALLPAIRS)
        NB_CUDA(c, dalloc(&c->ap_partial, n * (size_t)nb::allpairs_chunks((int64_t)n, c->sm_count)));
    if (c->p.mode == NB_MODE_SPLIT) {
        NB_CUDA(c, dalloc(&t.s64, n));
        NB_CUDA(c, dalloc(&t.cell4, n));
        NB_CUDA(c, dalloc(&t.cellq, n));
        NB_CUDA(c, dalloc(&t.s32, n));
        NB_CUDA(c, dalloc(&t.body4, n));
        NB_CUDA(c, dalloc(&t.gcount, n));
        NB_CUDA(c, dalloc(&t.gbase, n));
        NB_CUDA(c, dalloc(&t.groups, n));
        NB_CUDA(c, dalloc(&t.prefix, n + 1));
        NB_CUDA(c, dalloc(&t.prefix_tiles, (n + 2047) / 2048 + 1));
    }
    if (c->p.flags & NB_FLAG_LEARNED) {
        NB_CUDA(c, dalloc(&t.t32, n));
        NB_CUDA(c, dalloc(&t.cellh, 2 * n));
        NB_CUDA(c, dalloc(&t.band, (size_t)nb::kBandPerBody * n));
        NB_CUDA(c, dalloc(&t.band_count, n));
        NB_CUDA(c, dalloc(&c->acc32, n));
        NB_CUDA(c, dalloc(&c->mlp_params, NB_MLP_PARAMS));
        NB_CUDA(c, cudaMalloc(&c->mlp_infer, nb::mlp_infer_bytes()));
    }
    NB_CUDA(c, dalloc(&t.leaf_last, n));
    NB_CUDA(c, dalloc(&t.leaf_plevel, n));
    NB_CUDA(c, dalloc(&t.bucket_mass, n));
    NB_CUDA(c, dalloc(&t.bucket_com, n));
    NB_CUDA(c, dalloc(&t.flag, n));
    NB_CUDA(c, dalloc(&t.cell_of, n));
    NB_CUDA(c, dalloc(&t.rep_of, n));
    NB_CUDA(c, dalloc(&t.bnd, n));
    NB_CUDA(c, dalloc(&t.lcp8, n));
    {
        const size_t tiles = (n + nb::kAnsvTile - 1) / nb::kAnsvTile;
        NB_CUDA(c, dalloc(&t.ansv_first, tiles * nb::kAnsvLevels));
        NB_CUDA(c, dalloc(&t.ansv_last, tiles * nb::kAnsvLevels));
    }
    NB_CUDA(c, dalloc(&c->scal, 1));
    NB_CUDA(c, cudaMemset(c->scal, 0, sizeof(nb::DeviceScalars)));
    c->bbox_blocks = 2 * c->sm_count;
    NB_CUDA(c, dalloc(&c->bbox_partials, (size_t)4 * c->bbox_blocks));
    NB_CUDA(c, dalloc(&c->acc, n));
    NB_CUDA(c, dalloc(&c->stage_pos, n));
    NB_CUDA(c, dalloc(&c->stage_vel, n));
    return NB_OK;
}

void free_all(nb_ctx* c) {
    for (int k = 0; k < 2; ++k) {
        cudaFree(c->buf[k].pos);
        cudaFree(c->buf[k].vel);
        cudaFree(c->buf[k].mass);
        cudaFree(c->buf[k].orig);
        cudaFree(c->sort.key[k]);
        cudaFree(c->sort.val[k]);
    }
    cudaFree(c->sort.counts);
    cudaFree(c->sort.totals);
    cudaFree(c->sort.hist);
    cudaFree(c->sort.status);
    cudaFree(c->sort.tile_counter);
    cudaFree(c->sort.ties_small);
    cudaFree(c->sort.ties_big);
    cudaFree(c->scan.block_sums);
    nb::Tree& t = c->tree;
    void* tree_ptrs[] = {t.level,       t.child,      t.parent,
                         t.nint,      t.ready,       t.mass,        t.com,        t.leaf_last,
                         t.leaf_plevel, t.bucket_mass, t.bucket_com, t.flag,      t.cell_of,
                         t.bnd,       t.range,       t.s64,         t.cell4,      t.cellq,      t.s32,
                         t.body4,     t.gcount,      t.gbase,       t.groups,     t.rep_of,
                         t.t32,       t.cellh,       t.band,        t.band_count,
                         t.start_list, t.prefix, t.prefix_tiles, t.lcp8, t.ansv_first,
                         t.ansv_last};
    for (void* q : tree_ptrs) cudaFree(q);
    cudaFree(c->scal);
    cudaFree(c->bbox_partials);
    cudaFree(c->acc);
    cudaFree(c->dbg_terms);
    cudaFree(c->stage_pos);
    cudaFree(c->stage_vel);
    for (auto& u : c->up) {
        cudaFree(u.mass);
        cudaFree(u.pos);
        cudaFree(u.vel);
    }
    cudaFree(c->ap_partial);
    cudaFree(c->render_count);
    cudaFree(c->render_rgba);
    cudaFree(c->render_table);
    cudaFree(c->acc32);
    cudaFree(c->mlp_params);
    cudaFree(c->mlp_infer);
}

int alloc_batch(nb_ctx* c, uint32_t nuni, const uint64_t* counts) {
    nb::Batch& b = c->batch;
    std::vector<int32_t> off(nuni + 1), uid((size_t)c->n);
    off[0] = 0;
    for (uint32_t u = 0; u < nuni; ++u) {
        off[u + 1] = off[u] + (int32_t)counts[u];
        for (int32_t i = off[u]; i < off[u + 1]; ++i) uid[i] = (int32_t)u;
    }
    int32_t *doff = nullptr, *duid = nullptr;
    NB_CUDA(c, dalloc(&doff, nuni + 1));
    NB_CUDA(c, dalloc(&duid, (size_t)c->n));
    b.off = doff;
    b.uid = duid;
    NB_CUDA(c, dalloc(&b.boxbits, 4 * (size_t)nuni));
    NB_CUDA(c, dalloc(&b.center, nuni));
    NB_CUDA(c, dalloc(&b.w2, nuni));
    NB_CUDA(c, dalloc(&b.lo, nuni));
    NB_CUDA(c, dalloc(&b.root, nuni));
    NB_CUDA(c, cudaMemcpy(doff, off.data(), sizeof(int32_t) * (nuni + 1), cudaMemcpyHostToDevice));
    NB_CUDA(c, cudaMemcpy(duid, uid.data(), sizeof(int32_t) * c->n, cudaMemcpyHostToDevice));
    NB_CUDA(c, cudaMemset(b.boxbits, 0xff, sizeof(unsigned long long) * 4 * nuni));
    b.nuni = (int)nuni;
    return NB_OK;
}

void free_batch(nb_ctx* c) {
    nb::Batch& b = c->batch;
    cudaFree(const_cast<int32_t*>(b.off));
    cudaFree(const_cast<int32_t*>(b.uid));
    cudaFree(b.boxbits);
    cudaFree(b.center);
    cudaFree(b.w2);
    cudaFree(b.lo);
    cudaFree(b.root);
    b = nb::Batch();
}

void drop_graphs(nb_ctx* c) {
    for (auto& g : c->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

// "drift": the FP64 drift kernel; in learned mode the correction kernel, which
// also kicks and drifts (plain SPLIT fuses both into the force kernel).
const char* const kPhaseNames[nb::kPhases] = {"bbox+morton", "sort", "gather", "prefix", "tree",
                                              "moments", "groups", "force", "drift"};

// Enqueues one step reading the state from buf[parity]; leaves it in the
// other buffer.  integrate=false stops after the force pass (no kick/drift).
// timed=true records the phase events between stages.
void enqueue_step(nb_ctx* c, int parity, bool integrate, bool store_acc, bool timed = false) {
    const nb::BodyBuffers& A = c->buf[parity];
    const nb::BodyBuffers& B = c->buf[parity ^ 1];
    // External records become event nodes of the captured graph, so the
    // events carry timestamps from every replay of the step.
    auto mark = [&](int k) {
        if (timed) cudaEventRecordWithFlags(c->phase_ev[k], c->stream, cudaEventRecordExternal);
    };
    mark(0);
    // cell_terms, body_terms and stack_hw start every force pass at zero
    cudaMemsetAsync(&c->scal->cell_terms, 0, 3 * sizeof(unsigned long long), c->stream);
    if (c->p.mode == NB_MODE_ALLPAIRS) {
        // AllPairsSim: drift into the other buffer, then the all-pairs kick there
        for (int k = 1; k < 8; ++k) mark(k);
        nb::launch_allpairs_step(c, A, B, integrate, store_acc);
        mark(8);
        mark(9);
        return;
    }
    nb::launch_bbox(c, A.pos);
    nb::launch_morton(c, A.pos);
    mark(1);
    nb::launch_sort(c);
    mark(2);
    const bool split = c->p.mode == NB_MODE_SPLIT;
    nb::launch_gather(c, A, B, split ? c->tree.body4 : nullptr);
    mark(3);
    nb::launch_prefix_sums(c, B);  // SPLIT monopoles only
    mark(4);
    nb::launch_tree(c, B, true);
    nb::launch_batch_roots(c);
    mark(5);
    // the target groups need only the tree: they are built on the side stream
    // while the moments run (two branches of the captured graph)
    if (split) {
        cudaEventRecord(c->fork_ev, c->stream);
        cudaStreamWaitEvent(c->side_stream, c->fork_ev, 0);
        cudaStream_t main_stream = c->stream;
        c->stream = c->side_stream;
        nb::launch_groups(c);
        c->stream = main_stream;
        cudaEventRecord(c->join_ev, c->side_stream);
    }
    nb::launch_moments(c, B, split);
    mark(6);
    if (split) cudaStreamWaitEvent(c->stream, c->join_ev, 0);
    mark(7);
    if (split && (c->p.flags & NB_FLAG_LEARNED)) {
        // the features need only the monopoles, and only the correction reads
        // them: they are built on the side stream while the walk runs
        cudaEventRecord(c->feat_fork_ev, c->stream);
        cudaStreamWaitEvent(c->side_stream, c->feat_fork_ev, 0);
        cudaStream_t main_stream = c->stream;
        c->stream = c->side_stream;
        nb::launch_features(c, B);
        c->stream = main_stream;
        cudaEventRecord(c->feat_join_ev, c->side_stream);
        nb::launch_force_split(c, B, integrate, store_acc);  // FP32 accelerations + band lists
        mark(8);
        cudaStreamWaitEvent(c->stream, c->feat_join_ev, 0);
        nb::launch_mlp_correct(c, B, integrate, store_acc);  // learned term, kick, drift
    } else if (split) {
        nb::launch_force_split(c, B, integrate, store_acc);  // kick and drift fused
        mark(8);
    } else {
        nb::launch_force_fp64(c, B, integrate, store_acc);
        mark(8);
        if (integrate) nb::launch_drift(c, B);
    }
    mark(9);
}

int capture_graph(nb_ctx* c, int parity) {
    cudaGraph_t g = nullptr;
    NB_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const uint64_t before = c->launches;
    enqueue_step(c, parity, true, false, true);
    c->kernels_per_step = c->launches - before;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (e != cudaSuccess) return fail(c, NB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    const cudaError_t e2 = cudaGraphInstantiate(&c->graph[parity], g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess)
        return fail(c, NB_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e2));
    return NB_OK;
}

int read_device_error(nb_ctx* c) {
    unsigned flags = 0;
    NB_CUDA(c, cudaMemcpyAsync(&flags, &c->scal->error, sizeof(unsigned), cudaMemcpyDeviceToHost,
                               c->stream));
    NB_CUDA(c, cudaStreamSynchronize(c->stream));
    if (!flags) return NB_OK;
    NB_CUDA(c, cudaMemsetAsync(&c->scal->error, 0, sizeof(unsigned), c->stream));
    if (flags & nb::kErrTimeout) return fail(c, NB_ERR_TIMEOUT, "a bounded device wait gave up");
    if (flags & nb::kErrStack) return fail(c, NB_ERR_CAPACITY, "traversal stack bound exceeded");
    if (flags & nb::kErrUpload)
        return fail(c, NB_ERR_INVALID,
                    "asynchronous upload rejected (non-finite value or mass <= 0); state unchanged");
    return fail(c, NB_ERR_CAPACITY, "tree build saw more than four children in a cell");
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

namespace {

struct DeviceScope {
    int prev = -1;
    int rc = NB_OK;
    explicit DeviceScope(int dev) {
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || dev < 0 || dev >= ndev) {
            rc = NB_ERR_NOTFOUND;
            return;
        }
        cudaGetDevice(&prev);
        cudaSetDevice(dev);
    }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

template <typename T>
struct DBuf {
    T* p = nullptr;
    explicit DBuf(size_t count) {
        if (cudaMalloc(&p, sizeof(T) * (count ? count : 1)) != cudaSuccess) p = nullptr;
    }
    ~DBuf() { cudaFree(p); }
};

}  // namespace

extern "C" {

int nb_params_default(nb_params* p) {
    if (!p) return NB_ERR_INVALID;
    std::memset(p, 0, sizeof(*p));
    p->G = 1.0;
    p->timestep = 1e-4;
    p->theta = 0.5;
    p->epsilon_squared = 1e-4;
    p->mode = NB_MODE_FP64;
    p->band_theta = 0.5;
    return NB_OK;
}

const char* nb_status_string(int s) {
    switch (s) {
        case NB_OK: return "ok";
        case NB_ERR_INVALID: return "invalid argument";
        case NB_ERR_CUDA: return "CUDA error";
        case NB_ERR_CAPACITY: return "device capacity exceeded";
        case NB_ERR_TIMEOUT: return "device wait timed out";
        case NB_ERR_NOMEM: return "out of memory";
        case NB_ERR_NOTFOUND: return "no such CUDA device";
        default: return "unknown status";
    }
}

const char* nb_last_error(const nb_ctx* c) { return c ? c->err.c_str() : "null context"; }

}  // extern "C"

namespace {

// nb_create and nb_batch_create: counts == nullptr for a single universe.
int create_context(const nb_params* p, uint64_t n, const double* mass, const double* pos_xy,
                   const double* vel_xy, uint32_t nuni, const uint64_t* counts, nb_ctx** out) {
    if (!out) return NB_ERR_INVALID;
    *out = nullptr;
    if (check_params(p) != NB_OK) return NB_ERR_INVALID;
    if (n == 0 || n > (uint64_t)INT32_MAX - 1 || !mass || !pos_xy || !vel_xy) return NB_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || p->device < 0 || p->device >= ndev)
        return NB_ERR_NOTFOUND;
    nb_ctx* c = new (std::nothrow) nb_ctx();
    if (!c) return NB_ERR_NOMEM;
    c->p = *p;
    // default group size: 32 bodies below 131,072 bodies (too few groups of 64
    // to fill the GPU; 16,384- and 65,536-body discs step 7-8% faster), else 64
    c->bpl = p->bodies_per_lane > 0 ? p->bodies_per_lane : (n < 131072 ? 1 : 2);
    c->n = (int64_t)n;
    c->device = p->device;
    DeviceGuard guard(c->device);
    int rc = NB_OK;
    if (cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->side_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->join_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->feat_fork_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->feat_join_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->staged, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->copied, cudaEventDisableTiming) != cudaSuccess) {
        rc = NB_ERR_CUDA;
    }
    for (auto& e : c->phase_ev)
        if (rc == NB_OK && cudaEventCreate(&e) != cudaSuccess) rc = NB_ERR_CUDA;
    if (rc == NB_OK) rc = alloc_all(c);
    if (rc == NB_OK && counts) rc = alloc_batch(c, nuni, counts);
    if (rc == NB_OK) rc = nb_upload(c, mass, pos_xy, vel_xy);
    if (rc != NB_OK) {
        nb_destroy(c);
        return rc == NB_ERR_CUDA ? NB_ERR_NOMEM : rc;
    }
    *out = c;
    return NB_OK;
}

}  // namespace

extern "C" {

int nb_create(const nb_params* p, uint64_t n, const double* mass, const double* pos_xy,
              const double* vel_xy, nb_ctx** out) {
    return create_context(p, n, mass, pos_xy, vel_xy, 0, nullptr, out);
}

int nb_batch_create(const nb_params* p, uint32_t nuniverses, const uint64_t* counts,
                    const double* mass, const double* pos_xy, const double* vel_xy, nb_ctx** out) {
    if (!out || !counts || !p || nuniverses == 0 || nuniverses > (uint32_t)nb::kBatchMaxUniverses)
        return NB_ERR_INVALID;
    if (p->mode != NB_MODE_SPLIT || (p->flags & NB_FLAG_LEARNED)) return NB_ERR_INVALID;
    uint64_t n = 0;
    for (uint32_t u = 0; u < nuniverses; ++u) {
        if (counts[u] == 0) return NB_ERR_INVALID;
        n += counts[u];
    }
    return create_context(p, n, mass, pos_xy, vel_xy, nuniverses, counts, out);
}

int nb_destroy(nb_ctx* c) {
    if (!c) return NB_OK;
    DeviceGuard guard(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    if (c->side_stream) cudaStreamSynchronize(c->side_stream);
    if (c->up_stream) cudaStreamSynchronize(c->up_stream);
    drop_graphs(c);
    free_all(c);
    free_batch(c);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->staged) cudaEventDestroy(c->staged);
    if (c->copied) cudaEventDestroy(c->copied);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->fork_ev) cudaEventDestroy(c->fork_ev);
    if (c->join_ev) cudaEventDestroy(c->join_ev);
    if (c->feat_fork_ev) cudaEventDestroy(c->feat_fork_ev);
    if (c->feat_join_ev) cudaEventDestroy(c->feat_join_ev);
    if (c->side_stream) cudaStreamDestroy(c->side_stream);
    for (auto& u : c->up) {
        if (u.ready) cudaEventDestroy(u.ready);
        if (u.used) cudaEventDestroy(u.used);
    }
    if (c->up_stream) cudaStreamDestroy(c->up_stream);
    for (auto& e : c->phase_ev)
        if (e) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return NB_OK;
}

// The bodies are checked on the device after the copy (a host loop over 5n
// doubles costs more than the copy itself).  A rejected upload has already
// replaced the state: upload valid bodies before stepping again.
int nb_upload(nb_ctx* c, const double* mass, const double* pos_xy, const double* vel_xy) {
    if (!c || !mass || !pos_xy || !vel_xy) return NB_ERR_INVALID;
    const size_t n = (size_t)c->n;
    DeviceGuard guard(c->device);
    c->parity = 0;
    const nb::BodyBuffers& A = c->buf[0];
    NB_CUDA(c, cudaMemsetAsync(&c->scal->upload_bad, 0, sizeof(unsigned), c->stream));
    NB_CUDA(c, cudaMemcpyAsync(A.mass, mass, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    NB_CUDA(c, cudaMemcpyAsync(A.pos, pos_xy, n * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    NB_CUDA(c, cudaMemcpyAsync(A.vel, vel_xy, n * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    nb::launch_upload_check(c, A, &c->scal->upload_bad);
    NB_CUDA(c, cudaGetLastError());
    unsigned bad = 0;
    NB_CUDA(c, cudaMemcpyAsync(&bad, &c->scal->upload_bad, sizeof(unsigned), cudaMemcpyDeviceToHost,
                               c->stream));
    NB_CUDA(c, cudaStreamSynchronize(c->stream));
    if (bad & 1u) return fail(c, NB_ERR_INVALID, "non-finite mass, position or velocity");
    if (bad & 2u) return fail(c, NB_ERR_INVALID, "masses must be positive");
    return NB_OK;
}

// Staging areas and stream are made on first use; a failed set-up leaves the
// context as it was and nb_upload still works.  Two areas are used in turn, so
// an upload's copy can start while the previous one waits for the step before
// it to finish.
int nb_upload_async(nb_ctx* c, const double* mass, const double* pos_xy, const double* vel_xy) {
    if (!c || !mass || !pos_xy || !vel_xy) return NB_ERR_INVALID;
    const size_t n = (size_t)c->n;
    DeviceGuard guard(c->device);
    if (!c->up_stream) {
        cudaStream_t st = nullptr;
        nb_ctx::UploadSlot slot[2];
        bool ok = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess;
        for (auto& u : slot)
            ok = ok && cudaEventCreateWithFlags(&u.ready, cudaEventDisableTiming) == cudaSuccess &&
                 cudaEventCreateWithFlags(&u.used, cudaEventDisableTiming) == cudaSuccess &&
                 dalloc(&u.mass, n) == cudaSuccess && dalloc(&u.pos, n) == cudaSuccess &&
                 dalloc(&u.vel, n) == cudaSuccess;
        if (!ok) {
            for (auto& u : slot) {
                cudaFree(u.mass);
                cudaFree(u.pos);
                cudaFree(u.vel);
                if (u.ready) cudaEventDestroy(u.ready);
                if (u.used) cudaEventDestroy(u.used);
            }
            if (st) cudaStreamDestroy(st);
            cudaGetLastError();
            return fail(c, NB_ERR_NOMEM, "no device memory for the upload staging areas");
        }
        c->up_stream = st;
        c->up[0] = slot[0];
        c->up[1] = slot[1];
        c->up_next = 0;
    }
    nb_ctx::UploadSlot& u = c->up[c->up_next];
    c->up_next ^= 1;
    // the area is free once the upload that used it before has been moved
    // into the state
    NB_CUDA(c, cudaStreamWaitEvent(c->up_stream, u.used, 0));
    NB_CUDA(c, cudaMemcpyAsync(u.mass, mass, n * sizeof(double), cudaMemcpyHostToDevice,
                               c->up_stream));
    NB_CUDA(c, cudaMemcpyAsync(u.pos, pos_xy, n * sizeof(double2), cudaMemcpyHostToDevice,
                               c->up_stream));
    NB_CUDA(c, cudaMemcpyAsync(u.vel, vel_xy, n * sizeof(double2), cudaMemcpyHostToDevice,
                               c->up_stream));
    NB_CUDA(c, cudaEventRecord(u.ready, c->up_stream));
    // everything enqueued before this call still sees the old state
    NB_CUDA(c, cudaStreamWaitEvent(c->stream, u.ready, 0));
    const nb::BodyBuffers keep = c->buf[c->parity];
    c->parity = 0;
    nb::launch_upload_commit(c, u.mass, u.pos, u.vel, keep, c->buf[0], &c->scal->upload_bad);
    NB_CUDA(c, cudaGetLastError());
    NB_CUDA(c, cudaEventRecord(u.used, c->stream));
    return NB_OK;
}

int nb_set_timestep(nb_ctx* c, double dt) {
    if (!c || !std::isfinite(dt)) return NB_ERR_INVALID;
    if (dt != c->p.timestep) {
        DeviceGuard guard(c->device);
        NB_CUDA(c, cudaStreamSynchronize(c->stream));
        c->p.timestep = dt;
        drop_graphs(c);
    }
    return NB_OK;
}

int nb_step(nb_ctx* c, uint32_t nsteps) {
    if (!c) return NB_ERR_INVALID;
    if (nsteps == 0) return NB_OK;
    if ((c->p.flags & NB_FLAG_LEARNED) && !c->mlp_ready)
        return fail(c, NB_ERR_INVALID, "learned mode: call nb_set_mlp_weights first");
    DeviceGuard guard(c->device);
    for (int par = 0; par < 2; ++par)
        if (!c->graph[par]) {
            const int rc = capture_graph(c, par);
            if (rc != NB_OK) return rc;
        }
    NB_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    for (uint32_t k = 0; k < nsteps; ++k) {
        NB_CUDA(c, cudaGraphLaunch(c->graph[c->parity], c->stream));
        c->parity ^= 1;
    }
    NB_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    c->steps += nsteps;
    c->batch_steps = nsteps;
    return NB_OK;
}

int nb_sync(nb_ctx* c) {
    if (!c) return NB_ERR_INVALID;
    DeviceGuard guard(c->device);
    NB_CUDA(c, cudaStreamSynchronize(c->stream));
    NB_CUDA(c, cudaStreamSynchronize(c->copy_stream));
    float ms = 0.f;
    if (c->batch_steps && cudaEventElapsedTime(&ms, c->ev0, c->ev1) == cudaSuccess)
        c->ms_last = ms / c->batch_steps;
    c->batch_steps = 0;
    return read_device_error(c);
}

int nb_debug_wait_timeout(int32_t device) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return NB_ERR_NOTFOUND;
    DeviceGuard guard(device);
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return NB_ERR_CUDA;
    const unsigned flags = nb::sort_timeout_probe(st);
    cudaStreamDestroy(st);
    if (flags == ~0u) return NB_ERR_CUDA;
    return (flags & nb::kErrTimeout) ? NB_ERR_TIMEOUT : NB_OK;
}

int nb_download_async(nb_ctx* c, double* pos_xy, double* vel_xy) {
    if (!c) return NB_ERR_INVALID;
    if (!pos_xy && !vel_xy) return NB_OK;
    DeviceGuard guard(c->device);
    const nb::BodyBuffers& A = c->buf[c->parity];
    const size_t bytes = (size_t)c->n * sizeof(double2);
    // the staging buffers are reused: the previous copy-out must be done
    NB_CUDA(c, cudaStreamWaitEvent(c->stream, c->copied, 0));
    nb::launch_scatter(c, A, pos_xy ? c->stage_pos : nullptr, vel_xy ? c->stage_vel : nullptr,
                       nullptr, nullptr);
    NB_CUDA(c, cudaGetLastError());
    NB_CUDA(c, cudaEventRecord(c->staged, c->stream));
    NB_CUDA(c, cudaStreamWaitEvent(c->copy_stream, c->staged, 0));
    if (pos_xy)
        NB_CUDA(c, cudaMemcpyAsync(pos_xy, c->stage_pos, bytes, cudaMemcpyDeviceToHost,
                                   c->copy_stream));
    if (vel_xy)
        NB_CUDA(c, cudaMemcpyAsync(vel_xy, c->stage_vel, bytes, cudaMemcpyDeviceToHost,
                                   c->copy_stream));
    NB_CUDA(c, cudaEventRecord(c->copied, c->copy_stream));
    return NB_OK;
}

int nb_download_wait(nb_ctx* c) {
    if (!c) return NB_ERR_INVALID;
    DeviceGuard guard(c->device);
    NB_CUDA(c, cudaStreamSynchronize(c->copy_stream));
    return read_device_error(c);
}

int nb_download(nb_ctx* c, double* pos_xy, double* vel_xy) {
    if (!c) return NB_ERR_INVALID;
    if (!pos_xy && !vel_xy) return NB_OK;
    DeviceGuard guard(c->device);
    const nb::BodyBuffers& A = c->buf[c->parity];
    const size_t bytes = (size_t)c->n * sizeof(double2);
    NB_CUDA(c, cudaStreamWaitEvent(c->stream, c->copied, 0));
    nb::launch_scatter(c, A, pos_xy ? c->stage_pos : nullptr, vel_xy ? c->stage_vel : nullptr,
                       nullptr, nullptr);
    NB_CUDA(c, cudaGetLastError());
    if (pos_xy)
        NB_CUDA(c, cudaMemcpyAsync(pos_xy, c->stage_pos, bytes, cudaMemcpyDeviceToHost, c->stream));
    if (vel_xy)
        NB_CUDA(c, cudaMemcpyAsync(vel_xy, c->stage_vel, bytes, cudaMemcpyDeviceToHost, c->stream));
    NB_CUDA(c, cudaStreamSynchronize(c->stream));
    return read_device_error(c);
}

int nb_accelerations(nb_ctx* c, double* acc_xy) {
    if (!c || !acc_xy) return NB_ERR_INVALID;
    if ((c->p.flags & NB_FLAG_LEARNED) && !c->mlp_ready)
        return fail(c, NB_ERR_INVALID, "learned mode: call nb_set_mlp_weights first");
    DeviceGuard guard(c->device);
    enqueue_step(c, c->parity, false, true);
    NB_CUDA(c, cudaGetLastError());
    c->parity ^= 1;
    const nb::BodyBuffers& A = c->buf[c->parity];
    nb::launch_scatter(c, A, nullptr, nullptr, c->acc, c->stage_pos);
    NB_CUDA(c, cudaGetLastError());
    NB_CUDA(c, cudaMemcpyAsync(acc_xy, c->stage_pos, (size_t)c->n * sizeof(double2),
                               cudaMemcpyDeviceToHost, c->stream));
    NB_CUDA(c, cudaStreamSynchronize(c->stream));
    return read_device_error(c);
}

int nb_debug_morton(nb_ctx* c, uint64_t* codes, int32_t* order, double* box_out) {
    if (!c) return NB_ERR_INVALID;
    DeviceGuard guard(c->device);
    const nb::BodyBuffers& A = c->buf[c->parity];
    nb::launch_bbox(c, A.pos);
    nb::launch_morton(c, A.pos);
    nb::launch_sort(c);
    NB_CUDA(c, cudaGetLastError());
    const size_t n = (size_t)c->n;
    if (codes)
        NB_CUDA(c, cudaMemcpyAsync(codes, c->sort.key[0], n * 8, cudaMemcpyDeviceToHost, c->stream));
    if (order)
        NB_CUDA(c, cudaMemcpyAsync(order, c->sort.val[0], n * 4, cudaMemcpyDeviceToHost, c->stream));
    if (box_out)
        NB_CUDA(c, cudaMemcpyAsync(box_out, c->scal->box, 4 * sizeof(double), cudaMemcpyDeviceToHost,
                                   c->stream));
    NB_CUDA(c, cudaStreamSynchronize(c->stream));
    return read_device_error(c);
}

int nb_debug_interactions(nb_ctx* c, uint32_t* cell_terms, uint32_t* body_terms,
                          int32_t* stack_high_water) {
    if (!c) return NB_ERR_INVALID;
    if (c->p.mode != NB_MODE_FP64)
        return fail(c, NB_ERR_INVALID, "per-body interaction counts come from the FP64 walk");
    DeviceGuard guard(c->device);
    const size_t n = (size_t)c->n;
    if (!c->dbg_terms) NB_CUDA(c, dalloc(&c->dbg_terms, n));
    c->want_terms = true;
    enqueue_step(c, c->parity, false, false);
    c->want_terms = false;
    NB_CUDA(c, cudaGetLastError());
    c->parity ^= 1;
    std::vector<uint2> terms(n);
    std::vector<int32_t> orig(n);
    NB_CUDA(c, cudaMemcpyAsync(terms.data(), c->dbg_terms, n * sizeof(uint2), cudaMemcpyDeviceToHost,
                               c->stream));
    NB_CUDA(c, cudaMemcpyAsync(orig.data(), c->buf[c->parity].orig, n * sizeof(int32_t),
                               cudaMemcpyDeviceToHost, c->stream));
    nb::DeviceScalars s;
    NB_CUDA(c, cudaMemcpyAsync(&s, c->scal, sizeof(s), cudaMemcpyDeviceToHost, c->stream));
    NB_CUDA(c, cudaStreamSynchronize(c->stream));
    for (size_t i = 0; i < n; ++i) {
        const int32_t o = orig[i];
        if (o < 0 || (size_t)o >= n) return fail(c, NB_ERR_CUDA, "corrupt body permutation");
        if (cell_terms) cell_terms[o] = terms[i].x;
        if (body_terms) body_terms[o] = terms[i].y;
    }
    if (stack_high_water) *stack_high_water = s.stack_hw;
    return read_device_error(c);
}

int nb_debug_sort_passes(nb_ctx* c, int32_t passes, int32_t* last_passes) {
    if (!c || passes < -1 || passes > 8) return NB_ERR_INVALID;
    DeviceGuard guard(c->device);
    nb::DeviceScalars s;
    NB_CUDA(c, cudaMemcpyAsync(&s, c->scal, sizeof(s), cudaMemcpyDeviceToHost, c->stream));
    if (passes >= 0)
        NB_CUDA(c, cudaMemcpyAsync(&c->scal->sort_passes_forced, &passes, sizeof(int32_t),
                                   cudaMemcpyHostToDevice, c->stream));
    NB_CUDA(c, cudaStreamSynchronize(c->stream));
    if (last_passes) *last_passes = s.sort_passes;
    return NB_OK;
}

int nb_debug_groups(nb_ctx* c, int32_t* first_body, int32_t* last_body, uint64_t capacity,
                    uint64_t* count) {
    if (!c || !count) return NB_ERR_INVALID;
    if (c->p.mode != NB_MODE_SPLIT)
        return fail(c, NB_ERR_INVALID, "target groups exist only in SPLIT mode");
    DeviceGuard guard(c->device);
    NB_CUDA(c, cudaStreamSynchronize(c->stream));
    nb::DeviceScalars s;
    NB_CUDA(c, cudaMemcpy(&s, c->scal, sizeof(s), cudaMemcpyDeviceToHost));
    *count = (uint64_t)(s.groups > 0 ? s.groups : 0);
    const size_t m = (size_t)std::min<uint64_t>(*count, capacity);
    if (m && (first_body || last_body)) {
        std::vector<int2> g(m);
        NB_CUDA(c, cudaMemcpy(g.data(), c->tree.groups, m * sizeof(int2), cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < m; ++k) {
            if (first_body) first_body[k] = g[k].x;
            if (last_body) last_body[k] = g[k].y;
        }
    }
    return NB_OK;
}

int nb_debug_state(nb_ctx* c, double* mass, double* pos_xy, double* vel_xy, int32_t* orig) {
    if (!c) return NB_ERR_INVALID;
    DeviceGuard guard(c->device);
    const nb::BodyBuffers& A = c->buf[c->parity];
    const size_t n = (size_t)c->n;
    if (mass) NB_CUDA(c, cudaMemcpyAsync(mass, A.mass, n * 8, cudaMemcpyDeviceToHost, c->stream));
    if (pos_xy) NB_CUDA(c, cudaMemcpyAsync(pos_xy, A.pos, n * 16, cudaMemcpyDeviceToHost, c->stream));
    if (vel_xy) NB_CUDA(c, cudaMemcpyAsync(vel_xy, A.vel, n * 16, cudaMemcpyDeviceToHost, c->stream));
    if (orig) NB_CUDA(c, cudaMemcpyAsync(orig, A.orig, n * 4, cudaMemcpyDeviceToHost, c->stream));
    NB_CUDA(c, cudaStreamSynchronize(c->stream));
    return NB_OK;
}

int nb_debug_tree(nb_ctx* c, double* cell_mass, double* cell_com_xy, int32_t* level,
                  int32_t* first_body, int32_t* last_body, int32_t* root_ref) {
    if (!c) return NB_ERR_INVALID;
    DeviceGuard guard(c->device);
    NB_CUDA(c, cudaStreamSynchronize(c->stream));
    nb::DeviceScalars s;
    NB_CUDA(c, cudaMemcpy(&s, c->scal, sizeof(s), cudaMemcpyDeviceToHost));
    const size_t m = (size_t)s.cells;
    const nb::Tree& t = c->tree;
    if (cell_mass && m) NB_CUDA(c, cudaMemcpy(cell_mass, t.mass, m * 8, cudaMemcpyDeviceToHost));
    if (cell_com_xy && m) NB_CUDA(c, cudaMemcpy(cell_com_xy, t.com, m * 16, cudaMemcpyDeviceToHost));
    if (level && m) NB_CUDA(c, cudaMemcpy(level, t.level, m * 4, cudaMemcpyDeviceToHost));
    // the body ranges are {first, last} pairs: copy each half with a pitch of 8 bytes
    if (first_body && m)
        NB_CUDA(c, cudaMemcpy2D(first_body, 4, t.range, 8, 4, m, cudaMemcpyDeviceToHost));
    if (last_body && m)
        NB_CUDA(c, cudaMemcpy2D(last_body, 4, reinterpret_cast<const char*>(t.range) + 4, 8, 4, m,
                                cudaMemcpyDeviceToHost));
    if (root_ref) *root_ref = s.root;
    return NB_OK;
}

int nb_get_stats(nb_ctx* c, nb_stats* out) {
    if (!c || !out) return NB_ERR_INVALID;
    DeviceGuard guard(c->device);
    NB_CUDA(c, cudaStreamSynchronize(c->stream));
    nb::DeviceScalars s;
    NB_CUDA(c, cudaMemcpy(&s, c->scal, sizeof(s), cudaMemcpyDeviceToHost));
    std::memset(out, 0, sizeof(*out));
    out->steps = c->steps;
    out->n = (uint64_t)c->n;
    out->tree_nodes = (uint64_t)s.cells;
    out->cell_interactions = s.cell_terms;
    out->body_interactions = s.body_terms;
    out->ms_last_step = c->ms_last;
    out->root_width = s.box[1] - s.box[0];
    out->kernels_per_step = c->kernels_per_step;
    return NB_OK;
}

int nb_phase_times(nb_ctx* c, double* ms, int max) {
    if (!c || (!ms && max > 0)) return -NB_ERR_INVALID;
    DeviceGuard guard(c->device);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return -NB_ERR_CUDA;
    for (int k = 0; k < nb::kPhases && k < max; ++k) {
        float t = 0.f;
        ms[k] = cudaEventElapsedTime(&t, c->phase_ev[k], c->phase_ev[k + 1]) == cudaSuccess ? t : -1.0;
    }
    cudaGetLastError();
    return nb::kPhases;
}

const char* nb_phase_name(int k) { return k >= 0 && k < nb::kPhases ? kPhaseNames[k] : ""; }

int nb_render(nb_ctx* c, const nb_view* v, uint8_t* rgba_out) {
    if (!c || !v || !rgba_out) return NB_ERR_INVALID;
    if (v->res_x == 0 || v->res_y == 0 || v->res_x > 16384 || v->res_y > 16384 || v->reserved)
        return fail(c, NB_ERR_INVALID, "resolution must be 1..16384 pixels per side");
    if (!std::isfinite(v->x) || !std::isfinite(v->y) || !(v->width > 0.0) || !(v->height > 0.0) ||
        !std::isfinite(v->width) || !std::isfinite(v->height))
        return fail(c, NB_ERR_INVALID, "view rectangle must be finite with positive size");
    if (!(v->point_diameter >= 1.f && v->point_diameter <= 50.f))
        return fail(c, NB_ERR_INVALID, "point diameter must be 1..50 pixels");
    DeviceGuard guard(c->device);
    const int64_t pixels = (int64_t)v->res_x * v->res_y;
    if (!c->render_table) {
        // k successive blends of white at alpha 120/255 over black, 8 bits each
        uint8_t table[256];
        double cv = 0.0;
        for (int k = 0; k < 256; ++k) {
            table[k] = (uint8_t)cv;
            cv = std::floor(120.0 + cv * 135.0 / 255.0 + 0.5);
        }
        NB_CUDA(c, dalloc(&c->render_table, 256));
        NB_CUDA(c, cudaMemcpy(c->render_table, table, 256, cudaMemcpyHostToDevice));
    }
    if (c->render_pixels < pixels) {
        NB_CUDA(c, cudaStreamSynchronize(c->stream));
        cudaFree(c->render_count);
        cudaFree(c->render_rgba);
        c->render_count = nullptr;
        c->render_rgba = nullptr;
        c->render_pixels = 0;
        NB_CUDA(c, dalloc(&c->render_count, pixels));
        NB_CUDA(c, dalloc(&c->render_rgba, pixels));
        c->render_pixels = pixels;
    }
    nb::launch_render(c, c->buf[c->parity].pos, *v, c->render_count, c->render_table,
                      c->render_rgba);
    NB_CUDA(c, cudaGetLastError());
    NB_CUDA(c, cudaMemcpyAsync(rgba_out, c->render_rgba, (size_t)pixels * 4, cudaMemcpyDeviceToHost,
                               c->stream));
    NB_CUDA(c, cudaStreamSynchronize(c->stream));
    return read_device_error(c);
}

int nb_autotune(nb_ctx* c, uint32_t steps, int32_t* leaf_out, int32_t* bpl_out) {
    if (!c || steps == 0) return NB_ERR_INVALID;
    if (c->p.mode != NB_MODE_SPLIT)
        return fail(c, NB_ERR_INVALID, "autotuning applies to NB_MODE_SPLIT");
    if ((c->p.flags & NB_FLAG_LEARNED) && !c->mlp_ready)
        return fail(c, NB_ERR_INVALID, "learned mode: call nb_set_mlp_weights first");
    DeviceGuard guard(c->device);
    NB_CUDA(c, cudaStreamSynchronize(c->stream));
    // the trials run on a copy of the bodies, restored afterwards
    const size_t n = (size_t)c->n;
    const int parity0 = c->parity;
    const uint64_t steps0 = c->steps;
    nb::BodyBuffers save;
    NB_CUDA(c, dalloc(&save.pos, n));
    NB_CUDA(c, dalloc(&save.vel, n));
    NB_CUDA(c, dalloc(&save.mass, n));
    NB_CUDA(c, dalloc(&save.orig, n));
    const nb::BodyBuffers& A = c->buf[parity0];
    cudaMemcpyAsync(save.pos, A.pos, n * 16, cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(save.vel, A.vel, n * 16, cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(save.mass, A.mass, n * 8, cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(save.orig, A.orig, n * 4, cudaMemcpyDeviceToDevice, c->stream);
    const bool learned = (c->p.flags & NB_FLAG_LEARNED) != 0;
    const int bpls[3] = {2, 1, 4};
    const int leaves[4] = {4, 8, 16, 32};
    double best = 1e300;
    int best_leaf = c->p.leaf_size, best_bpl = c->bpl;
    int rc = NB_OK;
    for (int bi = 0; bi < (learned ? 1 : 3) && rc == NB_OK; ++bi)
        for (int li = 0; li < 4 && rc == NB_OK; ++li) {
            c->bpl = bpls[bi];
            c->p.leaf_size = leaves[li];
            drop_graphs(c);
            rc = nb_step(c, 1);  // warm-up (captures the graphs)
            if (rc == NB_OK) rc = nb_step(c, steps);
            if (rc == NB_OK) rc = nb_sync(c);
            if (rc == NB_OK && c->ms_last < best) {
                best = c->ms_last;
                best_leaf = leaves[li];
                best_bpl = bpls[bi];
            }
        }
    c->bpl = best_bpl;
    c->p.leaf_size = best_leaf;
    drop_graphs(c);
    c->parity = parity0;
    c->steps = steps0;
    const nb::BodyBuffers& R = c->buf[parity0];
    cudaMemcpyAsync(R.pos, save.pos, n * 16, cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(R.vel, save.vel, n * 16, cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(R.mass, save.mass, n * 8, cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(R.orig, save.orig, n * 4, cudaMemcpyDeviceToDevice, c->stream);
    cudaStreamSynchronize(c->stream);
    cudaFree(save.pos);
    cudaFree(save.vel);
    cudaFree(save.mass);
    cudaFree(save.orig);
    if (leaf_out) *leaf_out = best_leaf;
    if (bpl_out) *bpl_out = best_bpl;
    return rc;
}

int nb_set_mlp_weights(nb_ctx* c, const float* params) {
    if (!c || !params) return NB_ERR_INVALID;
    if (!(c->p.flags & NB_FLAG_LEARNED))
        return fail(c, NB_ERR_INVALID, "context was not created with NB_FLAG_LEARNED");
    for (int k = 0; k < NB_MLP_PARAMS; ++k)
        if (!std::isfinite(params[k])) return fail(c, NB_ERR_INVALID, "non-finite MLP parameter");
    DeviceGuard guard(c->device);
    NB_CUDA(c, cudaMemcpyAsync(c->mlp_params, params, sizeof(float) * NB_MLP_PARAMS,
                               cudaMemcpyHostToDevice, c->stream));
    nb::mlp_prepare_inference(c);
    NB_CUDA(c, cudaGetLastError());
    NB_CUDA(c, cudaStreamSynchronize(c->stream));
    c->mlp_ready = true;
    return NB_OK;
}

int nb_mlp_samples(nb_ctx* c, uint64_t ntargets, uint64_t seed, uint64_t capacity, float* features,
                   float* residuals, uint64_t* count) {
    if (!c || !features || !residuals || !count || ntargets == 0 || capacity == 0)
        return NB_ERR_INVALID;
    if (!(c->p.flags & NB_FLAG_LEARNED))
        return fail(c, NB_ERR_INVALID, "context was not created with NB_FLAG_LEARNED");
    if (capacity > 0xffffffffull || ntargets > (uint64_t)INT32_MAX) return NB_ERR_INVALID;
    DeviceGuard guard(c->device);
    // sorted bodies, tree and moments of the current state, without integrating
    const nb::BodyBuffers& A = c->buf[c->parity];
    const nb::BodyBuffers& B = c->buf[c->parity ^ 1];
    nb::launch_bbox(c, A.pos);
    nb::launch_morton(c, A.pos);
    nb::launch_sort(c);
    nb::launch_gather(c, A, B, c->tree.body4);
    nb::launch_tree(c, B);
    nb::launch_moments(c, B, true);
    nb::launch_features(c, B);
    nb::launch_groups(c);
    NB_CUDA(c, cudaGetLastError());
    c->parity ^= 1;
    // target groups: a seeded uniform choice (splitmix64), reduced modulo the
    // group count on the device
    std::vector<int> slots(ntargets);
    uint64_t z = seed + 0x9e3779b97f4a7c15ull;
    for (auto& sl : slots) {
        z += 0x9e3779b97f4a7c15ull;
        uint64_t x = z;
        x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
        x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
        x ^= x >> 31;
        sl = (int)(x & 0x7fffffff);
    }
    int* dslots = nullptr;
    float *dX = nullptr, *dY = nullptr;
    unsigned* dcount = nullptr;
    int rc = NB_OK;
    if (cudaMalloc(&dslots, sizeof(int) * ntargets) != cudaSuccess ||
        cudaMalloc(&dX, sizeof(float) * 12 * capacity) != cudaSuccess ||
        cudaMalloc(&dY, sizeof(float) * 2 * capacity) != cudaSuccess ||
        cudaMalloc(&dcount, sizeof(unsigned)) != cudaSuccess)
        rc = fail(c, NB_ERR_NOMEM, "sample buffers");
    unsigned hcount = 0;
    if (rc == NB_OK) {
        cudaMemcpyAsync(dslots, slots.data(), sizeof(int) * ntargets, cudaMemcpyHostToDevice,
                        c->stream);
        cudaMemsetAsync(dcount, 0, sizeof(unsigned), c->stream);
        nb::launch_mlp_samples(c, B, dslots, (int)ntargets, dX, dY, dcount, (unsigned)capacity);
        cudaMemcpyAsync(&hcount, dcount, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream);
        if (cudaStreamSynchronize(c->stream) != cudaSuccess)
            rc = fail(c, NB_ERR_CUDA, "sample kernel failed");
    }
    if (rc == NB_OK) {
        const uint64_t rows = hcount < capacity ? hcount : capacity;
        cudaMemcpy(features, dX, sizeof(float) * 12 * rows, cudaMemcpyDeviceToHost);
        cudaMemcpy(residuals, dY, sizeof(float) * 2 * rows, cudaMemcpyDeviceToHost);
        *count = rows;
    }
    cudaFree(dslots);
    cudaFree(dX);
    cudaFree(dY);
    cudaFree(dcount);
    if (rc == NB_OK) rc = read_device_error(c);
    return rc;
}

int nb_mlp_forward(int32_t device, const float* params, uint64_t n, const float* features,
                   float* out) {
    if (!params || !features || !out || n == 0) return NB_ERR_INVALID;
    DeviceScope scope(device);
    if (scope.rc != NB_OK) return scope.rc;
    DBuf<float> p(NB_MLP_PARAMS), x(12 * n), y(2 * n);
    DBuf<unsigned char> image(nb::mlp_forward_image_bytes());
    DBuf<unsigned> err(1);
    if (!p.p || !x.p || !y.p || !image.p || !err.p) return NB_ERR_NOMEM;
    int sm_count = 0;
    if (cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return NB_ERR_CUDA;
    cudaMemcpy(p.p, params, sizeof(float) * NB_MLP_PARAMS, cudaMemcpyHostToDevice);
    cudaMemcpy(x.p, features, sizeof(float) * 12 * n, cudaMemcpyHostToDevice);
    cudaMemset(err.p, 0, sizeof(unsigned));
    if (nb::mlp_forward_device(p.p, x.p, (int64_t)n, y.p, image.p, err.p, sm_count, nullptr) !=
        NB_OK)
        return NB_ERR_CUDA;
    unsigned flags = 0;
    if (cudaMemcpy(out, y.p, sizeof(float) * 2 * n, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&flags, err.p, sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess)
        return NB_ERR_CUDA;
    return (flags & nb::kErrTimeout) ? NB_ERR_TIMEOUT : NB_OK;
}

int nb_mlp_loss_grad(int32_t device, const float* params, uint64_t n, const float* features,
                     const float* targets, float* grad, float* loss) {
    if (!params || !features || !targets || !grad || !loss || n == 0) return NB_ERR_INVALID;
    DeviceScope scope(device);
    if (scope.rc != NB_OK) return scope.rc;
    DBuf<float> p(NB_MLP_PARAMS), x(12 * n), y(2 * n), g(NB_MLP_PARAMS), l(1);
    DBuf<unsigned char> image(nb::mlp_train_image_bytes());
    DBuf<unsigned> err(1);
    if (!p.p || !x.p || !y.p || !g.p || !l.p || !image.p || !err.p) return NB_ERR_NOMEM;
    cudaMemcpy(p.p, params, sizeof(float) * NB_MLP_PARAMS, cudaMemcpyHostToDevice);
    cudaMemcpy(x.p, features, sizeof(float) * 12 * n, cudaMemcpyHostToDevice);
    cudaMemcpy(y.p, targets, sizeof(float) * 2 * n, cudaMemcpyHostToDevice);
    cudaMemset(g.p, 0, sizeof(float) * NB_MLP_PARAMS);
    cudaMemset(l.p, 0, sizeof(float));
    cudaMemset(err.p, 0, sizeof(unsigned));
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (nb::mlp_grad_tc_device(p.p, x.p, y.p, nullptr, (int64_t)n, g.p, l.p, image.p, err.p,
                               sms > 0 ? sms : 1, nullptr) != NB_OK)
        return NB_ERR_CUDA;
    unsigned flags = 0;
    if (cudaMemcpy(grad, g.p, sizeof(float) * NB_MLP_PARAMS, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(loss, l.p, sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&flags, err.p, sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess)
        return NB_ERR_CUDA;
    return flags ? NB_ERR_TIMEOUT : NB_OK;
}

int nb_mlp_train(int32_t device, uint64_t n, const float* features, const float* residuals,
                 const nb_mlp_train_params* tp, float* params, float* loss_per_epoch) {
    if (!features || !residuals || !tp || !params || n == 0 || tp->batch == 0 || tp->epochs == 0 ||
        !(tp->lr > 0.f))
        return NB_ERR_INVALID;
    DeviceScope scope(device);
    if (scope.rc != NB_OK) return scope.rc;
    // host-side set-up: output scale and seeded initialisation
    std::vector<float> P(params, params + NB_MLP_PARAMS);
    bool all_zero = true;
    for (int k = 0; k < NB_MLP_PARAMS - 1; ++k) all_zero = all_zero && P[k] == 0.f;
    uint64_t z = tp->seed * 0x9e3779b97f4a7c15ull + 1;
    auto uniform = [&z]() {
        z += 0x9e3779b97f4a7c15ull;
        uint64_t x = z;
        x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
        x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
        x ^= x >> 31;
        return (double)(x >> 11) * (1.0 / 9007199254740992.0);
    };
    if (all_zero) {  // uniform(-a, a), a = sqrt(6 / (fan_in + fan_out))
        const int w1 = 0, w2 = 64 * 12 + 64, w3 = w2 + 64 * 64 + 64;
        const double a1 = std::sqrt(6.0 / (12 + 64)), a2 = std::sqrt(6.0 / 128.0),
                     a3 = std::sqrt(6.0 / 66.0);
        for (int k = 0; k < 64 * 12; ++k) P[w1 + k] = (float)((2 * uniform() - 1) * a1);
        for (int k = 0; k < 64 * 64; ++k) P[w2 + k] = (float)((2 * uniform() - 1) * a2);
        for (int k = 0; k < 2 * 64; ++k) P[w3 + k] = (float)((2 * uniform() - 1) * a3);
    }
    if (!(P[NB_MLP_PARAMS - 1] > 0.f)) {
        double ss = 0.0;
        for (uint64_t k = 0; k < 2 * n; ++k) ss += (double)residuals[k] * residuals[k];
        P[NB_MLP_PARAMS - 1] = (float)std::sqrt(ss / (2.0 * n) + 1e-30);
    }
    const float inv_scale = 1.f / P[NB_MLP_PARAMS - 1];
    std::vector<float> T(2 * n);
    for (uint64_t k = 0; k < 2 * n; ++k) T[k] = residuals[k] * inv_scale;
    DBuf<float> p(NB_MLP_PARAMS), x(12 * n), y(2 * n), g(NB_MLP_PARAMS), m(NB_MLP_PARAMS),
        v(NB_MLP_PARAMS), l(1);
    DBuf<int64_t> idx(n);
    DBuf<unsigned char> image(nb::mlp_train_image_bytes());
    DBuf<unsigned> err(1);
    if (!p.p || !x.p || !y.p || !g.p || !m.p || !v.p || !l.p || !idx.p || !image.p || !err.p)
        return NB_ERR_NOMEM;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return NB_ERR_CUDA;
    cudaMemcpyAsync(p.p, P.data(), sizeof(float) * NB_MLP_PARAMS, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(x.p, features, sizeof(float) * 12 * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(y.p, T.data(), sizeof(float) * 2 * n, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(m.p, 0, sizeof(float) * NB_MLP_PARAMS, st);
    cudaMemsetAsync(v.p, 0, sizeof(float) * NB_MLP_PARAMS, st);
    cudaMemsetAsync(err.p, 0, sizeof(unsigned), st);
    std::vector<int64_t> perm(n);
    for (uint64_t k = 0; k < n; ++k) perm[k] = (int64_t)k;
    int rc = NB_OK;
    int step = 0;
    const uint64_t B = tp->batch;
    for (uint32_t e = 0; e < tp->epochs && rc == NB_OK; ++e) {
        for (uint64_t k = n - 1; k > 0; --k) {  // Fisher-Yates
            const uint64_t j = (uint64_t)(uniform() * (double)(k + 1)) % (k + 1);
            std::swap(perm[k], perm[j]);
        }
        cudaMemcpyAsync(idx.p, perm.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(l.p, 0, sizeof(float), st);
        uint64_t nbatches = 0;
        for (uint64_t b0 = 0; b0 < n; b0 += B, ++nbatches) {
            const uint64_t cnt = std::min<uint64_t>(B, n - b0);
            cudaMemsetAsync(g.p, 0, sizeof(float) * NB_MLP_PARAMS, st);
            if (nb::mlp_grad_tc_device(p.p, x.p, y.p, idx.p + b0, (int64_t)cnt, g.p, l.p, image.p,
                                       err.p, sms > 0 ? sms : 1, st) != NB_OK ||
                nb::mlp_adam_device(p.p, g.p, m.p, v.p, tp->lr, ++step, st) != NB_OK) {
                rc = NB_ERR_CUDA;
                break;
            }
        }
        float lsum = 0.f;
        cudaMemcpyAsync(&lsum, l.p, sizeof(float), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = NB_ERR_CUDA;
        if (loss_per_epoch) loss_per_epoch[e] = lsum / (float)nbatches;
    }
    unsigned flags = 0;
    if (rc == NB_OK) {
        cudaMemcpyAsync(P.data(), p.p, sizeof(float) * (NB_MLP_PARAMS - 1), cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(&flags, err.p, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = NB_ERR_CUDA;
        else if (flags) rc = NB_ERR_TIMEOUT;
        else std::memcpy(params, P.data(), sizeof(float) * NB_MLP_PARAMS);
    }
    cudaStreamDestroy(st);
    return rc;
}

}  // extern "C"
