/*
 * nbody_b200.h -- C ABI of the B200 Barnes-Hut step.
 *
 * This is the drop-in boundary for the GPU backend of PhivPap/n-body-2d.  The
 * reference backend is the C++ class BarnesHutCuda
 * (src/Simulation/include/Simulation/BarnesHutCuda.hpp:44-112), created by
 * create_sim() (src/main.cpp:26-38) behind the abstract Simulation interface
 * (src/Simulation/include/Simulation/Simulation.hpp:13-67).  Its device work
 * lives in private member functions with no C entry points; each function
 * below replaces one of them and is cited with the member it stands in for.
 *
 * Plain pointers and sizes only.  Host arrays use the reference's Bodies
 * layout (src/common_lib/Body/include/Body/Body.hpp:26-31): mass is double[n],
 * positions and velocities are interleaved {x, y} doubles (double[2n]), all in
 * the caller's original body order.
 *
 * Threading: one context per host thread at a time; the library keeps no
 * global mutable state.  Every call returns an NB_* status; on failure
 * nb_last_error() describes the cause (the reference calls exit(1) instead,
 * src/Simulation/src/BarnesHutCuda.cu:12-19).
 */
#ifndef NBODY_B200_H
#define NBODY_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define NB_API __attribute__((visibility("default")))
#else
#define NB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define NB_OK 0
#define NB_ERR_INVALID 1   /* bad argument, NaN/Inf input, n out of range      */
#define NB_ERR_CUDA 2      /* a CUDA runtime call failed                       */
#define NB_ERR_CAPACITY 3  /* a device-side capacity bound was hit             */
#define NB_ERR_TIMEOUT 4   /* a bounded device-side wait gave up               */
#define NB_ERR_NOMEM 5     /* device or host allocation failed                 */
#define NB_ERR_NOTFOUND 6  /* no CUDA device / bad device ordinal              */

/* ---- traversal modes --------------------------------------------------- */
/* NB_MODE_FP64: the reference's semantics (per-body DFS, per-body opening
 * test, leaf size 1, FP64 throughout), for parity with
 * src/Simulation/src/BarnesHutCuda.cu:382-486.
 * NB_MODE_SPLIT: warp-cooperative group traversal with FP32 cell moments and
 * interactions; FP64 kept for the bounding box, the tree's centre-of-mass sums
 * and the integrator's position/velocity accumulation. */
#define NB_MODE_FP64 0
#define NB_MODE_SPLIT 1
/* NB_MODE_ALLPAIRS: the reference's AllPairsSim backend
 * (src/Simulation/src/AllPairs.cpp:24-49): drift x += v dt, then the kick
 * with the exact FP64 sum over all other bodies; no tree, no sort.  The pair
 * law is Plummer's (CU:427-431), or with NB_FLAG_CPU_LAW the law of
 * Simulation::force (src/Simulation/src/Simulation.cpp:74-80),
 * |a| = G m / (d^2 + eps^2) along the unit vector, which AllPairsSim uses. */
#define NB_MODE_ALLPAIRS 2

/* nb_params.flags bits */
#define NB_FLAG_QUADRUPOLE 1u  /* SPLIT: add the cells' second-moment term */
#define NB_FLAG_LEARNED 2u     /* SPLIT: learned far-field correction (set weights first) */
#define NB_FLAG_CPU_LAW 4u     /* ALLPAIRS: the reference CPU backends' pair law        */

/* Learned correction: parameters of the 12 -> 64 -> 64 -> 2 MLP as one FP32
 * vector: W1[64][12], b1[64], W2[64][64], b2[64], W3[2][64], b3[2], then the
 * output scale (residuals are predicted in units of that scale). */
#define NB_MLP_PARAMS 5123

typedef struct nb_params {
    double G;               /* gravitational constant (Constants::Simulation::G)    */
    double timestep;        /* dt (Config::Simulation::timestep)                    */
    double theta;           /* opening angle (Config::Simulation::theta)            */
    double epsilon_squared; /* Plummer softening squared (Simulation::epsilon_squared) */
    int32_t mode;           /* NB_MODE_*                                            */
    int32_t leaf_size;      /* SPLIT: bodies a cell may hold and still be summed
                               body by body instead of opened (0 = default)         */
    int32_t device;         /* CUDA device ordinal                                  */
    int32_t flags;          /* NB_FLAG_* bits; others must be 0                     */
    double bmax_ratio;      /* SPLIT: a cell is accepted only if also b_max < bmax_ratio * d,
                               b_max = distance from its COM to its farthest corner
                               (Barnes' b_max test); 0 = off.  FP64 mode ignores it */
    double band_theta;      /* learned mode: the opening angle of the plain walk the
                               correction stands in for; cells accepted at theta that
                               this angle would open get the network's term (0 = 0.5) */
    int32_t bodies_per_lane;/* SPLIT: target group size 32 x this, 1, 2 or 4 (0 = 1 below
                               131,072 bodies, else 2; learned contexts always use 2);
                               nb_autotune may change it */
    int32_t reserved;       /* must be 0 */
} nb_params;

typedef struct nb_stats {
    uint64_t steps;              /* steps taken since nb_create                       */
    uint64_t n;                  /* bodies                                            */
    uint64_t tree_nodes;         /* internal cells of the last tree built             */
    uint64_t cell_interactions;  /* body-cell terms of the last force pass            */
    uint64_t body_interactions;  /* body-body terms of the last force pass            */
    double ms_last_step;         /* device ms per step of the last synced nb_step batch */
    double root_width;           /* width of the squared root box of the last step    */
    uint64_t kernels_per_step;   /* kernel launches one step makes                    */
} nb_stats;

typedef struct nb_ctx nb_ctx;

/* Fills *p with G=1, dt=1e-4, theta=0.5, epsilon_squared=1e-4, FP64 mode,
 * band_theta=0.5, everything else 0. */
NB_API int nb_params_default(nb_params* p);

/* Replaces BarnesHutCuda::BarnesHutCuda + init_device_resources
 * (src/Simulation/src/BarnesHutCuda.cpp:7-11, BarnesHutCuda.cu:550-606):
 * allocates every device buffer once and uploads the bodies. */
NB_API int nb_create(const nb_params* p, uint64_t n, const double* mass, const double* pos_xy,
              const double* vel_xy, nb_ctx** out);

/* Failure-detection check (no counterpart in the reference, which has no
 * device-side waits): runs one radix-sort pass whose look-back waits on a
 * tile that never publishes.  The wait is bounded (about a second), so the
 * kernel gives up, raises its timeout flag and returns; the call then
 * returns NB_ERR_TIMEOUT, and the device stays usable.  NB_OK would mean the
 * bound did not trigger.  For tests. */
NB_API int nb_debug_wait_timeout(int32_t device);

/* Asynchronous form of nb_download: enqueues the same copy after the steps
 * enqueued so far and returns at once.  The device-to-host copy runs on the
 * context's copy stream, so it overlaps whatever is enqueued next (an
 * nb_upload's host-to-device copy, the next nb_step).  pos_xy / vel_xy must
 * stay valid, and be pinned for the copy to be asynchronous, until
 * nb_download_wait (or nb_sync) returns.  No counterpart in the reference,
 * which copies the bodies back synchronously every step (CU:632-646). */
NB_API int nb_download_async(nb_ctx* ctx, double* pos_xy, double* vel_xy);
NB_API int nb_download_wait(nb_ctx* ctx);

/* Headless rendering of the current bodies into an RGBA8 image: the frame
 * the reference draws (src/Graphics/src/Graphics.cpp:122-128) through
 * SFML/OpenGL, without a graphics stack.  The view is the reference's
 * ViewPort rectangle (src/Graphics/lib/ViewPort/src/ViewPort.cpp): world
 * coordinates (x, y) of the top-left corner, world extent width x height
 * (resolution x pixel_scale), and the window resolution.  Bodies are points
 * of point_diameter pixels (1..50, Constants.hpp:40-41) clipped to circles as
 * the body shader does (Graphics.cpp:20-26), white with alpha 120/255 over
 * black (Constants.hpp:39); the exact coverage and blending rules are in
 * csrc/k_render.cu.  rgba_out receives res_y rows of res_x pixels, row 0 at
 * the top.  The first call at a resolution allocates the image buffers. */
typedef struct nb_view {
    double x, y;
    double width, height;
    uint32_t res_x, res_y;
    float point_diameter;
    uint32_t reserved;  /* must be 0 */
} nb_view;

NB_API int nb_render(nb_ctx* ctx, const nb_view* view, uint8_t* rgba_out);

/* Batched universes (no counterpart in the reference, which holds one
 * universe per process): nuniverses independent universes of counts[u]
 * bodies each, concatenated in universe order in mass/pos_xy/vel_xy.  They
 * are advanced together: one sort, one tree (a universe never sees
 * another's bodies) and one persistent traversal launch per step, in one
 * captured graph.  NB_MODE_SPLIT only (no learned correction); at most 1024
 * universes.  Every other call works on the batch as one body array in the
 * concatenated order. */
NB_API int nb_batch_create(const nb_params* p, uint32_t nuniverses, const uint64_t* counts,
                           const double* mass, const double* pos_xy, const double* vel_xy,
                           nb_ctx** out);

/* Picks the SPLIT traversal's bodies per lane (1, 2 or 4: target groups of
 * 32, 64 or 128) and leaf size (4, 8, 16, 32) by timing `steps` steps of each on a
 * copy of the bodies, which are restored afterwards; the choice stays set.
 * Either output pointer may be NULL. */
NB_API int nb_autotune(nb_ctx* ctx, uint32_t steps, int32_t* leaf_out, int32_t* bpl_out);

/* Replaces ~BarnesHutCuda + release_device_resources (BarnesHutCuda.cpp:13-18,
 * BarnesHutCuda.cu:608-630). Accepts NULL. */
NB_API int nb_destroy(nb_ctx* ctx);

/* Replaces nsteps iterations of the body of BarnesHutCuda::simulate
 * (src/Simulation/src/BarnesHutCuda.cpp:30-40) minus the per-step download:
 * bounding box, Morton sort, tree, force + kick, drift.  Enqueued on the
 * context's stream as captured CUDA graphs; returns once enqueued. */
NB_API int nb_step(nb_ctx* ctx, uint32_t nsteps);

/* Waits for enqueued work and reports any device-side error flag. */
NB_API int nb_sync(nb_ctx* ctx);

/* Replaces the timestep hot-swap of Simulation::post_iteration
 * (src/Simulation/src/Simulation.cpp:68-72); takes effect at the next step. */
NB_API int nb_set_timestep(nb_ctx* ctx, double dt);

/* Overwrites the device state with host bodies in original order (the upload
 * half of init_device_resources, BarnesHutCuda.cu:596-605). */
NB_API int nb_upload(nb_ctx* ctx, const double* mass, const double* pos_xy, const double* vel_xy);

/* Asynchronous form of nb_upload: enqueues the host-to-device copy into a
 * device staging area on the context's upload stream and returns at once,
 * so the copy overlaps the steps and downloads enqueued before it.  Work
 * enqueued before the call sees the old state, work enqueued after it the
 * new one.  The bodies are checked on the device as they are moved into the
 * state; a rejected set leaves the state unchanged and the next nb_sync or
 * nb_download_wait returns NB_ERR_INVALID.  Two staging areas (40 bytes per
 * body each, used in turn) are allocated by the first call.  mass / pos_xy / vel_xy must stay
 * valid and unchanged, and be pinned for the copy to be asynchronous, until
 * nb_sync returns.  No counterpart in the reference, which uploads once at
 * start-up (BarnesHutCuda.cu:596-605). */
NB_API int nb_upload_async(nb_ctx* ctx, const double* mass, const double* pos_xy,
                           const double* vel_xy);

/* Replaces sync_from_gpu_bodies (BarnesHutCuda.cu:632-646): scatters the
 * state back to original order and copies it to the host.  Either pointer
 * may be NULL.  Blocks until the copy is done. */
NB_API int nb_download(nb_ctx* ctx, double* pos_xy, double* vel_xy);

/* Accelerations (without G) of the current state, original order, as the
 * force pass would apply them (BarnesHutCuda.cu:382-486); no integration.
 * Re-sorts the device state, which does not change the bodies. */
NB_API int nb_accelerations(nb_ctx* ctx, double* acc_xy);

/* Debug view of the sort stage (BarnesHutCuda.cu:648-711) on the current
 * state without changing it: sorted 64-bit Morton codes and the permutation
 * (order[r] = device slot of the body ranked r); box_out (nullable) receives
 * the squared root box {x_min, x_max, y_min, y_max}. */
NB_API int nb_debug_morton(nb_ctx* ctx, uint64_t* codes, int32_t* order, double* box_out);

/* Debug view of the raw device state in device (sorted) order. Any pointer
 * may be NULL. orig[i] is the original index of device slot i. */
NB_API int nb_debug_state(nb_ctx* ctx, double* mass, double* pos_xy, double* vel_xy, int32_t* orig);

/* Debug view of the last tree: per-cell mass and centre of mass (FP64),
 * level, body range, and the root reference.  Arrays sized by
 * nb_stats.tree_nodes; any pointer may be NULL. root_ref >= 0 is a cell,
 * < 0 is the leaf starting at body ~root_ref. */
NB_API int nb_debug_tree(nb_ctx* ctx, double* cell_mass, double* cell_com_xy, int32_t* level,
                  int32_t* first_body, int32_t* last_body, int32_t* root_ref);

/* Debug view of the FP64 force pass (NB_MODE_FP64 only): runs the force pass
 * of the current state without integrating, as nb_accelerations does, and
 * writes each body's interaction counts in original order -- cell_terms[i]
 * monopole terms of cells and multi-body leaves, body_terms[i] body-body terms
 * (the per-body counterparts of the counters the reference keeps implicitly in
 * its DFS, BarnesHutCuda.cu:382-486) -- and the deepest traversal stack any
 * body used (entries; the bound is 96, the reference's is 32, CU:400).  Any
 * pointer may be NULL.  The first call allocates 8 bytes per body. */
NB_API int nb_debug_interactions(nb_ctx* ctx, uint32_t* cell_terms, uint32_t* body_terms,
                                 int32_t* stack_high_water);

/* Debug control of the sort stage (no counterpart in the reference, whose CUB
 * sort always orders all 64 bits, BarnesHutCuda.cu:692): each step's radix
 * sort orders the top P bytes of the keys, P chosen from the previous tree's
 * neighbouring codes, and a tie pass then orders keys that agree in those
 * bytes by their low bytes, so the permutation is the full stable sort's for
 * any P.  passes = 1..8 forces P for the following sorts, 0 returns to the
 * automatic choice, -1 changes nothing.  *last_passes (nullable) receives the
 * P of the last sort (0 before the first). */
NB_API int nb_debug_sort_passes(nb_ctx* ctx, int32_t passes, int32_t* last_passes);

/* Debug view of the SPLIT traversal's target groups of the last step (no
 * counterpart in the reference, which walks the tree once per body): *count
 * receives the number of groups, and the first min(count, capacity) groups'
 * first and last body slots (device order) go to first_body / last_body
 * (either may be NULL).  NB_MODE_SPLIT only. */
NB_API int nb_debug_groups(nb_ctx* ctx, int32_t* first_body, int32_t* last_body, uint64_t capacity,
                           uint64_t* count);

NB_API int nb_get_stats(nb_ctx* ctx, nb_stats* out);

/* Device time of each phase of the most recent graph-launched step, from CUDA
 * events recorded inside the step graph (the GPU counterpart of the phase
 * StopWatches of the reference CPU backend, src/Simulation/src/BarnesHut.cpp:
 * 22-25, 52-64).  Writes up to max values to ms and returns the number of
 * phases (>= 0) or a negative NB_* status.  Phase k is named by
 * nb_phase_name(k). */
NB_API int nb_phase_times(nb_ctx* ctx, double* ms, int max);
NB_API const char* nb_phase_name(int phase);

/* Last error text of this context (never NULL). */
NB_API const char* nb_last_error(const nb_ctx* ctx);
NB_API const char* nb_status_string(int status);

/* FP64 all-pairs accelerations on the GPU with the reference pair law
 * (BarnesHutCuda.cu:427-431): a_i = sum_{j != i} m_j d_ij (|d_ij|^2+eps2)^-1.5
 * for k targets (indices into the n sources).  Host arrays in, host array out.
 * This is the error oracle for p50/p99 force errors at full size. */
NB_API int nb_allpairs_accelerations(int32_t device, uint64_t n, const double* mass,
                              const double* pos_xy, uint64_t k, const int64_t* targets,
                              double epsilon_squared, double* acc_xy);

/* ---- learned far-field correction (no counterpart in the reference: the
 * reference's force pass is the plain monopole walk, BarnesHutCuda.cu:382-486).
 * A context created with NB_MODE_SPLIT | NB_FLAG_LEARNED accepts cells at
 * theta; for each cell that plain theta = 0.5 would have opened, a small MLP
 * predicts the residual between the cell's exact pull and its monopole. */

typedef struct nb_mlp_train_params {
    uint32_t epochs;      /* passes over the samples                           */
    uint32_t batch;       /* samples per Adam step                             */
    float lr;             /* Adam learning rate                                */
    uint64_t seed;        /* shuffling and (when params is zero) initialisation */
} nb_mlp_train_params;

/* Installs the MLP parameters (NB_MLP_PARAMS floats) into a learned context. */
NB_API int nb_set_mlp_weights(nb_ctx* ctx, const float* params);

/* Residual samples from the context's current bodies, drawn the way the
 * traversal uses the network: for ntargets random target groups, every cell
 * the group accepts at the context's theta but would open at 0.5 gives
 * features[12] at the group's centre and, as residual[2], the mean over the
 * group's bodies of the exact-minus-monopole pull (FP64 sums over the cell's
 * bodies) in units of M / d^2, d the centre's distance to the cell's COM.
 * Features: (p - c)/d (2), w/d, heaviest child's mass fraction,
 * S/(M w^2) (3), T/(M w^3) (4), eps^2/(d^2 + eps^2).  Host arrays of capacity rows;
 * *count receives the rows written. Does not change the bodies. */
NB_API int nb_mlp_samples(nb_ctx* ctx, uint64_t ntargets, uint64_t seed, uint64_t capacity,
                          float* features, float* residuals, uint64_t* count);

/* Batched MLP on the GPU: out[n][2] = network(features[n][12]) (without the
 * output scale).  Host arrays.  Runs on the tcgen05 tensor cores in 128-row
 * tiles (BF16 operands, FP32 accumulation, tanh on BF16 pairs as the step's
 * correction applies it); NB_ERR_TIMEOUT if a bounded wait for an MMA ran out. */
NB_API int nb_mlp_forward(int32_t device, const float* params, uint64_t n, const float* features,
                          float* out);

/* Mean squared error of network(features) against targets[n][2] and its
 * gradient with respect to the parameters (grad has NB_MLP_PARAMS entries; the
 * output-scale entry is zero).  Host arrays. */
NB_API int nb_mlp_loss_grad(int32_t device, const float* params, uint64_t n, const float* features,
                            const float* targets, float* grad, float* loss);

/* Trains on the GPU with Adam on BF16 tensor-core forward/backward kernels.
 * residuals are raw (units of M / d^2); params[NB_MLP_PARAMS - 1] <= 0 asks
 * for the output scale to be set to the residuals' RMS, and all-zero params
 * ask for a seeded initialisation.  loss_per_epoch (nullable) gets one mean
 * loss per epoch. */
NB_API int nb_mlp_train(int32_t device, uint64_t n, const float* features, const float* residuals,
                        const nb_mlp_train_params* tp, float* params, float* loss_per_epoch);

/* Largest n nb_morton_sort_static accepts (its scratch is sized for it). */
#define NB_STATIC_SORT_MAX_BODIES 262144

/* The sort stage without any allocation.  No counterpart in the reference:
 * for callers that cannot let a library allocate device memory -- a renderer
 * stepping once per frame cannot take the device-wide synchronisation that
 * cudaMalloc/cudaFree may cause, and host programs that own all device memory
 * through their own pool hand libraries buffers instead.
 *
 * Computes, on the current device and on `stream` (a cudaStream_t; NULL is
 * the legacy default stream), what nb_debug_morton computes: the squared root
 * box, the 64-bit Morton codes sorted stably, and the permutation.  All
 * pointers are DEVICE pointers owned by the caller: pos_xy holds n
 * interleaved {x, y} doubles; codes receives n uint64, order n int32
 * (order[r] = input index of the body ranked r); box (nullable) receives
 * {x_min, x_max, y_min, y_max}.  Returns once the work is enqueued.
 *
 * Calls no cudaMalloc/cudaFree: the scratch is a static device array in the
 * library (NB_STATIC_SORT_MAX_BODIES x 24 bytes + about 100 KB, 6.4 MB in all,
 * on every GPU that loads it, held until exit).  n above NB_STATIC_SORT_MAX_BODIES is
 * rejected with NB_ERR_CAPACITY, n == 0 or a NULL pointer with
 * NB_ERR_INVALID.  Every call looks up the array's device address in the
 * current context (so a cudaDeviceReset in between is harmless); the first
 * call on a device also loads the library's device image, so make it before
 * any stream capture.  All calls on a device share
 * the scratch: calls that overlap on the GPU race and must be serialised by
 * the caller. */
NB_API int nb_morton_sort_static(const double* pos_xy, uint64_t n, uint64_t* codes,
                                 int32_t* order, double* box, void* stream);

#ifdef __cplusplus
}
#endif
#endif
