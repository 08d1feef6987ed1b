/*
 * nbody_oracle.h -- CPU oracle for the Barnes-Hut step (TEST INFRASTRUCTURE ONLY).
 *
 * This library restates, in plain C and FP64, the algorithm of the reference
 * GPU backend of PhivPap/n-body-2d (src/Simulation/src/BarnesHutCuda.cu, "CU"
 * below) so that tests can check the CUDA product path against it.  Only the
 * test suite, the smoke check and the CPU-baseline leg of the benchmark may
 * load it; the product library never links or calls it.
 *
 * Every entry point cites the reference lines whose behaviour it follows.
 * The state arrays are kept in "device order" exactly as the reference keeps
 * its device buffers: after each step the bodies stay sorted by the Morton
 * order computed at the start of that step (CU:701-708), and orig[] maps each
 * slot back to the caller's original body index (CU:498-506).
 */
#ifndef NBODY_ORACLE_H
#define NBODY_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    double x_min, x_max, y_min, y_max;
} orc_box;

typedef struct {
    int64_t nodes_allocated;     /* node-pool high-water mark (root + 4 per split)   */
    int64_t nodes_nonempty;      /* sum of the per-level work-list lengths           */
    int64_t levels;              /* number of non-empty levels                       */
    int64_t max_stack;           /* deepest DFS stack (entries) over all targets     */
    int64_t cell_interactions;   /* monopole terms from internal/multi-body cells    */
    int64_t body_interactions;   /* body-body terms                                  */
    int64_t multi_leaves;        /* leaves holding more than one body                */
    int64_t max_level;           /* deepest level holding a leaf                     */
} orc_stats;

/* CU:78-114 + CU:648-680: exact FP64 min/max, then the host-side squaring. */
void orc_bbox_squared(int64_t n, const double* pos_xy, orc_box* out);

/* CU:54-69 + CU:117-132: 64-bit Morton code per body in the squared box. */
void orc_morton(int64_t n, const double* pos_xy, const orc_box* box, uint64_t* codes);

/* CU:591-594,692-693: stable LSD sort of (code, current index).
 * keys_out: sorted codes; order_out[r] = index of the body ranked r. */
void orc_stable_sort(int64_t n, const uint64_t* keys, uint64_t* keys_out, int32_t* order_out);

/*
 * One full reference step (CU:648-830 via BarnesHutCuda::simulate,
 * src/Simulation/src/BarnesHutCuda.cpp:30-40), in place on device-order
 * arrays: bbox -> Morton -> stable sort -> gather -> level-wise quadtree ->
 * bottom-up COM -> per-body DFS force + kick -> drift.
 *
 * acc_out (nullable): FP64 accelerations (without G) of the sorted bodies,
 *   i.e. the value the reference adds to vel/(G*dt) at CU:484-485.
 * codes_out / order_out (nullable): the sorted codes and the permutation
 *   used for the gather (order_out[r] = previous slot of the body now at r).
 * do_integrate == 0: stop after the force pass (velocities and positions
 *   unchanged apart from the sort permutation).
 * Returns 0 on success, -1 on allocation failure.
 */
int orc_ref_step(int64_t n, double* mass, double* pos_xy, double* vel_xy, int32_t* orig,
                 double G, double dt, double eps2, double theta, int do_integrate,
                 double* acc_out, uint64_t* codes_out, int32_t* order_out, int nthreads,
                 orc_stats* stats);

/*
 * The force pass of orc_ref_step for chosen targets only: stages 1-4 of the
 * step (bbox, Morton, stable sort + gather, tree, COM; CU:648-809) run in
 * place on the device-order arrays exactly as in orc_ref_step with
 * do_integrate == 0, then the per-body DFS of CU:382-486 walks only the k
 * bodies whose ORIGINAL indices are targets[0..k).  Per target q: the
 * acceleration (without G) in acc_out[2q..2q+1], the monopole terms of cells
 * and multi-body leaves in cells_out[q], the body-body terms in pairs_out[q],
 * and the deepest DFS stack in stack_out[q] (entries, the quantity bounded
 * by CU:400's int32_t stack[32]).  Output pointers may be NULL.  Returns 0,
 * -1 on allocation failure, -2 for a target outside [0, n).
 */
int orc_ref_walk_targets(int64_t n, double* mass, double* pos_xy, double* vel_xy, int32_t* orig,
                         double eps2, double theta, int64_t k, const int64_t* targets,
                         double* acc_out, int64_t* cells_out, int64_t* pairs_out,
                         int64_t* stack_out, int nthreads, orc_stats* stats);

/*
 * FP64 all-pairs accelerations with the reference GPU pair law
 * (CU:427-431): a_i = sum_{j != i} m_j d_ij (|d_ij|^2 + eps2)^(-3/2),
 * evaluated for the k targets tgt[0..k) against all n sources.
 */
void orc_allpairs_plummer(int64_t n, const double* mass, const double* pos_xy, int64_t k,
                          const int64_t* tgt, double eps2, double* acc_xy, int nthreads);

/* Sum of the magnitudes of the pair terms of orc_allpairs_plummer, per target:
 * the scale that bounds the rounding error of any order of summation. */
void orc_allpairs_plummer_abs(int64_t n, const double* mass, const double* pos_xy, int64_t k,
                              const int64_t* tgt, double eps2, double* out, int nthreads);

/* A per-target bound on the error of an FP32 pair sum whose coordinates are
 * rounded to FP32 relative to (cx, cy): sum_j |a_ij| (16 u + 3 u (|x_i-c| +
 * |x_j-c|)_1 / |d_ij|) + 8 sqrt(n) u sum_j |a_ij|, u = 2^-24 (the last term
 * covers accumulation rounding, taken as a random walk). */
void orc_allpairs_fp32_bound(int64_t n, const double* mass, const double* pos_xy, int64_t k,
                             const int64_t* tgt, double eps2, double cx, double cy, double* out,
                             int nthreads);

/*
 * FP64 all-pairs accelerations with the reference CPU pair law
 * (src/Simulation/src/Simulation.cpp:74-80, BarnesHut.cpp:130-135):
 * a_i = sum_j G m_j (x_j - x_i) / (|d| (|d|^2 + eps2)), skipping j whose
 * position equals x_i (BarnesHut.cpp:108).
 */
void orc_allpairs_cpulaw(int64_t n, const double* mass, const double* pos_xy, int64_t k,
                         const int64_t* tgt, double G, double eps2, double* acc_xy, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
