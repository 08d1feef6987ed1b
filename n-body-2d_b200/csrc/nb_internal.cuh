// nb_internal.cuh -- device data layout and kernel entry points of the B200
// Barnes-Hut step.  Everything here is private to libnbody_b200.so; the public
// surface is include/nbody_b200.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "nbody_b200.h"

namespace nb {

constexpr int kMaxLevel = 30;     // level-30 cells are leaves (BarnesHutCuda.cu:182)
constexpr int kStackDepth = 96;   // >= 1 + 3 * 30 pending cells of a DFS
constexpr int kSortTileItems = 12; // keys per thread in a radix tile
constexpr int kSortThreads = 256;
constexpr int kSortTile = kSortTileItems * kSortThreads;  // 3072 keys
constexpr int kAnsvTile = 2048;   // boundaries per tile of the tree build's level scans
constexpr int kAnsvLevels = 32;   // table width per tile: levels 0..30 and one spare
constexpr int kPhases = 9;        // morton, sort, gather, prefix, tree, moments, groups, force, drift
constexpr float kThetaBand = 0.5f; // learned mode: the default plain walk the MLP stands in for
constexpr int kBandPerBody = 16;   // learned mode: band-list capacity per body of a group

// Device error flags (bit mask in DeviceScalars::error).
constexpr unsigned kErrStack = 1u;      // DFS stack bound exceeded
constexpr unsigned kErrTree = 2u;       // tree build saw an impossible range
constexpr unsigned kErrTimeout = 4u;    // a bounded wait gave up
constexpr unsigned kErrUpload = 8u;     // nb_upload_async rejected its bodies

// Small device-resident values written and read by kernels of one step.
struct DeviceScalars {
    double box[4];            // squared root box: x_min, x_max, y_min, y_max
    double center[2];         // box centre: origin of the FP32 coordinates
    double inv_wh[2];         // 1 / (x_max - x_min), 1 / (y_max - y_min): the Morton scaling
    double wsq[kMaxLevel + 1];// squared cell width per level (root * 0.25^L)
    int32_t root;             // >= 0 cell id, < 0 leaf ~first_body
    int32_t cells;            // internal cells of the current tree
    int32_t groups;           // SPLIT: target groups of the current tree
    unsigned group_ticket;    // SPLIT: next group for the persistent traversal
    unsigned error;           // kErr* bits, sticky until read by the host
    unsigned bbox_ticket;     // last-block-done counter of the bbox reduction
    unsigned long long cell_terms;
    unsigned long long body_terms;
    int32_t stack_hw;         // FP64 walk: deepest stack (entries) of the last force pass
    int32_t stack_pad_;
    int32_t nstart;           // cells whose children are all leaves (climb starts)
    unsigned upload_bad;      // nb_upload's checks: bit 0 non-finite, bit 1 mass <= 0
    // Radix sort over the top sort_passes bytes of the keys only (1..8), chosen
    // per step from the previous tree's histogram of shared leading digits of
    // neighbouring codes; keys that agree in those bytes are then put in order
    // of their low bytes by the tie pass, so the order stays the full stable
    // sort.  sort_passes_forced != 0 overrides the choice (tests).
    int32_t sort_passes;
    int32_t sort_passes_forced;
    unsigned lcp_hist[33];    // neighbouring codes sharing d leading 2-bit digits (d = 32: equal)
    unsigned tie_count[2];    // tie groups of <= 32 keys / of more keys, this step
};

// Batched universes (nb_batch_create): bodies of universe u occupy the fixed
// slot range [off[u], off[u+1]) in every step, because the sort key puts the
// universe id above a 54-bit Morton code of the body in its own universe's
// squared box.  The id takes the top kBatchUidDigits 2-bit digits, so a
// universe's spatial level L is tree level L + kBatchUidDigits, and cells
// above that level mix universes ("forest" cells, never accepted).
constexpr int kBatchUidDigits = 5;               // 10 bits: up to 1024 universes
constexpr int kBatchMortonBits = 27;             // per axis
constexpr int kBatchMaxUniverses = 1 << (2 * kBatchUidDigits);

struct Batch {
    int nuni = 0;                        // 0: a single universe (the default path)
    const int32_t* off = nullptr;        // [nuni + 1]
    const int32_t* uid = nullptr;        // [n] universe of each body slot
    unsigned long long* boxbits = nullptr;  // [nuni][4] order-preserving min/max of x, y
    double2* center = nullptr;           // [nuni] squared-box centre
    double* w2 = nullptr;                // [nuni] squared root width
    double2* lo = nullptr;               // [nuni] squared-box lower corner
    int32_t* root = nullptr;             // [nuni] root ref (cell, or ~first body of a leaf)
};

// Body state; two copies so the Morton gather can ping-pong.
struct BodyBuffers {
    double2* pos = nullptr;
    double2* vel = nullptr;
    double* mass = nullptr;
    int32_t* orig = nullptr;
};

// Compressed quadtree, one entry per internal cell (capacity n).
struct Tree {
    int32_t* level = nullptr;    // depth in the reference's uncompressed tree
    int4* child = nullptr;       // child refs: >= 0 cell, < 0 leaf ~first_body, INT_MIN none
    int32_t* parent = nullptr;   // parent cell, -1 at the root
    int32_t* nint = nullptr;     // children that are internal cells
    int32_t* ready = nullptr;    // bottom-up arrival counter
    double* mass = nullptr;      // FP64 monopole
    double2* com = nullptr;
    int2* range = nullptr;       // {first, last} body of the cell (one 8-byte load)
    // SPLIT mode: FP64 second moments about the COM for the bottom-up pass and
    // the packed FP32 records the traversal reads
    double4* s64 = nullptr;      // {Sxx, Sxy, Syy, 0}
    float4* cell4 = nullptr;     // {com_x - cx, com_y - cy, mass, width^2}
    float4* cellq = nullptr;     // the walk's quadrupole record {7.5 Sxx, 7.5 Sxy, 7.5 Syy, 0}
    float4* body4 = nullptr;     // per body {x - cx, y - cy, mass, index bits}
    // learned correction: third moments (FP64, bottom-up) and the per-cell
    // MLP features (see k_mlp.cu): the eight moment features as BF16 and the
    // cell width
    float4* t32 = nullptr;       // {Txxx, Txxy, Txyy, Tyyy} (FP32: they only feed BF16 features)
    float4* s32 = nullptr;       // {Sxx, Sxy, Syy, 0} of the feature pass (FP32, its own copy:
                                 // it runs beside the walk, which reads cellq)
    // two uint4 per cell (one 32-byte sector for the correction's gathers):
    // BF16 pairs {f3 f4, f5 f6, f7 f8, f9 f10}, then the float bits of
    // {com_x - cx, com_y - cy, mass, width}
    uint4* cellh = nullptr;
    int32_t* band = nullptr;       // per group: band cells, kBandPerBody x first body onwards
    int32_t* band_count = nullptr; // per group: band cells found
    int32_t* start_list = nullptr; // cells without internal children, in any order
    // SPLIT monopole moments: exclusive prefix sums over the sorted bodies of
    // {m, m (x - frame centre), m (y - frame centre), 0}, n + 1 entries, and
    // the per-tile totals of the scan that builds them
    double4* prefix = nullptr;
    double4* prefix_tiles = nullptr;
    // SPLIT target groups: <= split_group_size() Morton-consecutive bodies in one
    // parent cell (merged sibling cells/leaves), stored as body ranges
    int32_t* gcount = nullptr;   // groups each cell emits
    int32_t* gbase = nullptr;    // exclusive scan of gcount
    int2* groups = nullptr;      // {first, last} body of each group
    // per-body side tables, only meaningful at leaf starts
    int32_t* leaf_last = nullptr;   // last body of the leaf starting here
    int32_t* leaf_plevel = nullptr; // level of the leaf's parent cell (-1: root leaf)
    double* bucket_mass = nullptr;  // moments of multi-body leaves
    double2* bucket_com = nullptr;
    // build scratch (per boundary i between bodies i and i+1)
    uint8_t* lcp8 = nullptr;        // level of boundary i: shared leading digits, capped at 30
    int32_t* flag = nullptr;
    int32_t* cell_of = nullptr;     // exclusive scan of flag
    int32_t* rep_of = nullptr;      // cell id -> the boundary that creates it
    int4* bnd = nullptr;            // per boundary: {first body, last body} of the cell it
                                    // creates (flagged boundaries only), {previous, next}
                                    // separator of its cell or -1
    int32_t* ansv_first = nullptr;  // [kAnsvLevels][tiles] per level v and tile: first /
    int32_t* ansv_last = nullptr;   //   last boundary with a level below v (then scanned)
};

struct SortBuffers {
    uint64_t* key[2] = {nullptr, nullptr};
    uint32_t* val[2] = {nullptr, nullptr};
    uint32_t* counts = nullptr;   // [256][tiles]
    uint32_t* totals = nullptr;   // [256]
    uint32_t* hist = nullptr;     // [8][256] digit histograms -> exclusive bin offsets
    uint32_t* status = nullptr;   // [8][tiles][256] look-back status words
    unsigned* tile_counter = nullptr;  // [8]
    uint2* ties_small = nullptr;  // tie groups of 2..32 keys: {first, size}, n / 2 + 1
    uint2* ties_big = nullptr;    // tie groups of more than 32 keys, n / 33 + 1
    int tiles = 0;
};

struct ScanBuffers {
    int32_t* block_sums = nullptr;
    int blocks = 0;
};

}  // namespace nb

struct nb_ctx {
    nb_params p{};
    int64_t n = 0;
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaStream_t copy_stream = nullptr;  // nb_download_async: device-to-host copies
    cudaStream_t side_stream = nullptr;  // the target groups, built while the moments run
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    cudaEvent_t feat_fork_ev = nullptr, feat_join_ev = nullptr;  // learned features beside the walk
    cudaEvent_t staged = nullptr;        // the download's scatter into the staging buffers is done
    cudaEvent_t copied = nullptr;        // the staging buffers have been copied out (free again)
    cudaStream_t up_stream = nullptr;    // nb_upload_async: host-to-device copies
    cudaEvent_t phase_ev[nb::kPhases + 1] = {};
    int parity = 0;                 // which BodyBuffers holds the state
    nb::BodyBuffers buf[2];
    nb::SortBuffers sort;
    nb::ScanBuffers scan;
    nb::Tree tree;
    nb::DeviceScalars* scal = nullptr;   // device
    double* bbox_partials = nullptr;     // [blocks][4]
    int bbox_blocks = 0;
    int split_blocks[32] = {};            // persistent grids of the SPLIT traversal variants
    int corr_blocks_per_sm = 0;          // learned correction kernel occupancy (0 = not set up)
    float* mlp_params = nullptr;         // learned mode: FP32 MLP parameters (device)
    void* mlp_infer = nullptr;           // learned mode: BF16 fragment images for inference
    double2* ap_partial = nullptr;       // NB_MODE_ALLPAIRS: per-source-chunk partial sums
    uint32_t* render_count = nullptr;    // nb_render: coverings per pixel
    uchar4* render_rgba = nullptr;       // nb_render: the image
    uint8_t* render_table = nullptr;     // nb_render: covering count -> 8-bit value
    int64_t render_pixels = 0;
    bool mlp_ready = false;
    float2* acc32 = nullptr;             // learned mode: traversal accelerations
    nb::Batch batch;                     // batched universes (nuni > 0)
    int bpl = 2;                         // SPLIT: bodies per lane, 1, 2 or 4 (groups of 32 x bpl)
    double2* acc = nullptr;              // optional FP64 accelerations (sorted order)
    uint2* dbg_terms = nullptr;          // nb_debug_interactions: per-body {cell, body} terms
    bool want_terms = false;             // the force pass writes dbg_terms
    double2* stage_pos = nullptr;        // original-order staging for downloads
    double2* stage_vel = nullptr;
    // nb_upload_async staging, two areas used in turn (allocated on first use)
    struct UploadSlot {
        double* mass = nullptr;
        double2* pos = nullptr;
        double2* vel = nullptr;
        cudaEvent_t ready = nullptr;     // the staged bodies have arrived on the device
        cudaEvent_t used = nullptr;      // they have been moved into the state (area free again)
    } up[2];
    int up_next = 0;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};  // one step from parity 0 / 1
    double graph_dt = 0.0;
    uint64_t steps = 0;
    uint32_t batch_steps = 0;       // steps of the last nb_step batch
    double ms_last = 0.0;
    uint64_t launches = 0;          // kernel launches enqueued (counted by launchers)
    uint64_t kernels_per_step = 0;
    std::string err;
};

namespace nb {

// Learned mode: opening angle of the plain walk whose extra openings the
// network replaces (band cells: accepted at theta, opened at this angle).
inline float band_theta(const nb_ctx* c) {
    return c->p.band_theta > 0.0 ? (float)c->p.band_theta : kThetaBand;
}

// Centre of the FP32 frame of body slot i, and the squared width of a cell at
// tree level `level` whose first body is slot i.
__device__ __forceinline__ double2 frame_center(const DeviceScalars* s, const Batch& b, int i) {
    if (b.nuni == 0) return make_double2(s->center[0], s->center[1]);
    return b.center[b.uid[i]];
}
__device__ __forceinline__ double cell_width2(const DeviceScalars* s, const Batch& b, int i,
                                              int level) {
    if (b.nuni == 0) return s->wsq[level];
    if (level < kBatchUidDigits) return __longlong_as_double(0x7ff0000000000000ll);  // +inf
    return ldexp(b.w2[b.uid[i]], -2 * (level - kBatchUidDigits));
}

// Number of radix passes (top bytes of the key) a sort should take, from the
// histogram of shared leading digits of neighbouring sorted codes: the fewest
// passes that leave at most n / 32 neighbouring pairs tied; 8 without data.
__device__ __forceinline__ int choose_sort_passes(const unsigned* hist, int64_t n) {
    unsigned long long total = 0;
    for (int d = 0; d <= 32; ++d) total += hist[d];
    if (total == 0) return 8;
    for (int p = 1; p < 8; ++p) {
        unsigned long long tied = 0;  // pairs that agree in p bytes but are not equal
        for (int d = 4 * p; d < 32; ++d) tied += hist[d];
        if (tied * 32 <= (unsigned long long)n) return p;
    }
    return 8;
}

// Kernel launchers (all enqueue on ctx->stream, no host synchronisation).
void launch_bbox(nb_ctx* c, const double2* pos);
void launch_morton(nb_ctx* c, const double2* pos);
void launch_batch_roots(nb_ctx* c);   // per-universe root cells after the tree build
void launch_sort(nb_ctx* c);
unsigned sort_timeout_probe(cudaStream_t st);                                   // result in key[0]/val[0]
void launch_gather(nb_ctx* c, const BodyBuffers& src, const BodyBuffers& dst, float4* body4);
// SPLIT monopoles: the prefix sums over the sorted bodies (nothing in other
// modes); launch_tree runs them itself unless prefix_done.
void launch_prefix_sums(nb_ctx* c, const BodyBuffers& b);
void launch_tree(nb_ctx* c, const BodyBuffers& b, bool prefix_done = false);
void launch_moments(nb_ctx* c, const BodyBuffers& b, bool split);
// learned mode: second and third moments and the BF16 feature records
void launch_features(nb_ctx* c, const BodyBuffers& b);
int split_group_size(const nb_ctx* c);   // bodies per SPLIT traversal group
void launch_mlp_correct(nb_ctx* c, const BodyBuffers& b, bool kick, bool store_acc);
size_t mlp_infer_bytes();
void mlp_prepare_inference(nb_ctx* c);
void launch_mlp_samples(nb_ctx* c, const BodyBuffers& b, const int* slots, int nslots, float* X,
                        float* Y, unsigned* count, unsigned cap);
// bulk forward on tcgen05: image = mlp_forward_image_bytes() of device scratch
size_t mlp_forward_image_bytes();
int mlp_forward_device(const float* params, const float* X, int64_t n, float* Y, void* image,
                       unsigned* err, int sm_count, cudaStream_t st);
int mlp_adam_device(float* p, const float* g, float* m, float* v, float lr, int step,
                    cudaStream_t st);
// training loss and gradients on tcgen05 (image = mlp_train_image_bytes() of
// device scratch for the BF16 weight images; err receives kErrTimeout)
size_t mlp_train_image_bytes();
int mlp_grad_tc_device(const float* params, const float* X, const float* Yt, const int64_t* idx,
                       int64_t n, float* grad, float* loss, void* image, unsigned* err,
                       int sm_count, cudaStream_t st);
void launch_groups(nb_ctx* c);
void launch_force_split(nb_ctx* c, const BodyBuffers& b, bool kick, bool store_acc);
void launch_force_fp64(nb_ctx* c, const BodyBuffers& b, bool kick, bool store_acc);
void launch_drift(nb_ctx* c, const BodyBuffers& b);
void launch_upload_check(nb_ctx* c, const BodyBuffers& b, unsigned* bad);
// Checks the staged bodies (m, p, v) into *bad, then copies them into dst;
// a rejected set leaves dst holding `keep` (or untouched when keep is dst)
// and raises kErrUpload.
void launch_upload_commit(nb_ctx* c, const double* m, const double2* p, const double2* v,
                          const BodyBuffers& keep, const BodyBuffers& dst, unsigned* bad);
void launch_render(nb_ctx* c, const double2* pos, const nb_view& v, uint32_t* count,
                   const uint8_t* table, uchar4* rgba);
void launch_allpairs_step(nb_ctx* c, const BodyBuffers& a, const BodyBuffers& b, bool integrate,
                          bool store_acc);
int allpairs_chunks(int64_t n, int sm_count);
void launch_scatter(nb_ctx* c, const BodyBuffers& b, double2* out_pos, double2* out_vel,
                    const double2* acc, double2* out_acc);
void launch_identity(nb_ctx* c, int32_t* orig);

// The bounding-box, Morton and radix-sort stage on caller-provided buffers
// (no context): key/val ping-pong scratch of n entries each, counts of
// 256 x ceil(n / kSortTile), totals of 256, partials of 4 x bbox_blocks.  The
// last pass writes the sorted codes and permutation to key_out / val_out.
void launch_morton_sort_raw(const double2* pos, int64_t n, uint64_t* const key[2],
                            uint32_t* const val[2], uint64_t* key_out, uint32_t* val_out,
                            uint32_t* counts, uint32_t* totals, double* partials, int bbox_blocks,
                            DeviceScalars* scal, cudaStream_t st);

}  // namespace nb
