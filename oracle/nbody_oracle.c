/*
 * nbody_oracle.c -- CPU oracle for the Barnes-Hut step (TEST INFRASTRUCTURE ONLY).
 *
 * A plain-C FP64 restatement of the reference GPU backend
 * (src/Simulation/src/BarnesHutCuda.cu, cited as CU:<line>).  It is the
 * checker for the CUDA product path: only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg may load it.
 *
 * Arithmetic follows the reference statement by statement.  Where nvcc
 * contracts a multiply-add of the reference into one FMA (its default, and
 * implied by --use_fast_math in src/Simulation/CMakeLists.txt), this file
 * calls fma() so the accumulation rounds the same way; the double-precision
 * rsqrt() of CU:428 is restated as 1/sqrt(), which agrees to about one ulp.
 */
#include "nbody_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Bounding box, CU:78-114 (kernel) and CU:648-680 (host squaring).          */
/* ------------------------------------------------------------------------ */
void orc_bbox_squared(int64_t n, const double* pos, orc_box* out) {
    /* CU:649-654 seeds the box with +-DBL_MAX; the kernel folds fmin/fmax. */
    double xmin = 1.7976931348623157e308, xmax = -1.7976931348623157e308;
    double ymin = 1.7976931348623157e308, ymax = -1.7976931348623157e308;
    for (int64_t i = 0; i < n; ++i) {
        const double x = pos[2 * i], y = pos[2 * i + 1];
        xmin = fmin(xmin, x);
        xmax = fmax(xmax, x);
        ymin = fmin(ymin, y);
        ymax = fmax(ymax, y);
    }
    /* CU:666-677: grow the shorter side about its midpoint. */
    const double x_range = xmax - xmin;
    const double y_range = ymax - ymin;
    if (x_range > y_range) {
        const double mid = (ymin + ymax) * 0.5;
        ymin = mid - x_range * 0.5;
        ymax = mid + x_range * 0.5;
    } else {
        const double mid = (xmin + xmax) * 0.5;
        xmin = mid - y_range * 0.5;
        xmax = mid + y_range * 0.5;
    }
    out->x_min = xmin;
    out->x_max = xmax;
    out->y_min = ymin;
    out->y_max = ymax;
}

/* ------------------------------------------------------------------------ */
/* Morton codes, CU:54-69 and CU:117-132.                                    */
/* ------------------------------------------------------------------------ */
static uint64_t expand_bits_2d(uint32_t v) {
    uint64_t x = v;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x;
}

static uint32_t quantise(double t) {
    /* __double2uint_rd(fmin(fmax(t * 2^32, 0), 2^32 - 1)) */
    const double c = fmin(fmax(t * 4294967296.0, 0.0), 4294967295.0);
    return (uint32_t)floor(c);
}

void orc_morton(int64_t n, const double* pos, const orc_box* b, uint64_t* codes) {
    const double inv_w = 1.0 / (b->x_max - b->x_min);
    const double inv_h = 1.0 / (b->y_max - b->y_min);
    for (int64_t i = 0; i < n; ++i) {
        const double nx = (pos[2 * i] - b->x_min) * inv_w;
        const double ny = (pos[2 * i + 1] - b->y_min) * inv_h;
        codes[i] = (expand_bits_2d(quantise(nx)) << 1) | expand_bits_2d(quantise(ny));
    }
}

/* ------------------------------------------------------------------------ */
/* Stable sort by key (the contract of cub::DeviceRadixSort::SortPairs used  */
/* at CU:692 with values = current index).  LSD radix, 16-bit digits.       */
/* ------------------------------------------------------------------------ */
void orc_stable_sort(int64_t n, const uint64_t* keys, uint64_t* keys_out, int32_t* order_out) {
    uint64_t* ka = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n > 0 ? n : 1));
    uint64_t* kb = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n > 0 ? n : 1));
    int32_t* va = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int32_t* vb = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    size_t* cnt = (size_t*)malloc(sizeof(size_t) * 65536);
    for (int64_t i = 0; i < n; ++i) {
        ka[i] = keys[i];
        va[i] = (int32_t)i;
    }
    for (int pass = 0; pass < 4; ++pass) {
        const int shift = 16 * pass;
        memset(cnt, 0, sizeof(size_t) * 65536);
        for (int64_t i = 0; i < n; ++i) cnt[(ka[i] >> shift) & 0xFFFF]++;
        size_t run = 0;
        for (int d = 0; d < 65536; ++d) {
            const size_t c = cnt[d];
            cnt[d] = run;
            run += c;
        }
        for (int64_t i = 0; i < n; ++i) {
            const size_t p = cnt[(ka[i] >> shift) & 0xFFFF]++;
            kb[p] = ka[i];
            vb[p] = va[i];
        }
        uint64_t* tk = ka; ka = kb; kb = tk;
        int32_t* tv = va; va = vb; vb = tv;
    }
    memcpy(keys_out, ka, sizeof(uint64_t) * (size_t)n);
    memcpy(order_out, va, sizeof(int32_t) * (size_t)n);
    free(ka); free(kb); free(va); free(vb); free(cnt);
}

/* ------------------------------------------------------------------------ */
/* Level-wise quadtree, CU:153-240 (topology) and CU:713-777 (level loop).   */
/* ------------------------------------------------------------------------ */
typedef struct {
    double* wsq;
    int32_t* c0;
    int32_t* bs;
    int32_t* be;
    double* mass;
    double* cx;
    double* cy;
    int64_t cap;     /* max_quads = 5 n (src/Simulation/src/BarnesHutCuda.cpp:9) */
    int64_t alloc;   /* node_alloc counter                                       */
} orc_tree;

/* CU:153-163 */
static int32_t lower_bound_quadrant(const uint64_t* morton, int32_t lo, int32_t hi,
                                    uint64_t target, int shift) {
    while (lo < hi) {
        const int32_t mid = lo + (hi - lo) / 2;
        if (((morton[mid] >> shift) & 3ull) < target)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

/* Per-node body of build_tree_topology, CU:165-240; returns the number of
 * children appended to next[]. */
static int split_node(orc_tree* t, const uint64_t* morton, int32_t nid, int level, int32_t* next,
                      int64_t* next_count) {
    const int32_t start = t->bs[nid];
    const int32_t end = t->be[nid];
    if ((end - start) < 1 || level >= 30) return 0; /* LEAF_THRESHOLD = 1, CU:10,182 */
    const int shift = 62 - level * 2;
    int32_t b[5];
    b[0] = lower_bound_quadrant(morton, start, end + 1, 0ull, shift);
    b[1] = lower_bound_quadrant(morton, start, end + 1, 1ull, shift);
    b[2] = lower_bound_quadrant(morton, start, end + 1, 2ull, shift);
    b[3] = lower_bound_quadrant(morton, start, end + 1, 3ull, shift);
    b[4] = end + 1;
    int nch = 0;
    for (int q = 0; q < 4; ++q)
        if (b[q] <= b[q + 1] - 1) ++nch;
    if (nch == 0) return 0;
    const int64_t base = t->alloc;
    t->alloc += 4; /* atomicAdd(node_alloc, 4) happens before the capacity check */
    if (base + 3 >= t->cap) return 0;
    const double child_wsq = t->wsq[nid] * 0.25;
    t->c0[nid] = (int32_t)base;
    int added = 0;
    for (int q = 0; q < 4; ++q) {
        const int64_t cid = base + q;
        t->wsq[cid] = child_wsq;
        t->c0[cid] = -1;
        if (b[q] <= b[q + 1] - 1) {
            t->bs[cid] = b[q];
            t->be[cid] = b[q + 1] - 1;
            next[(*next_count)++] = (int32_t)cid;
            ++added;
        } else {
            t->bs[cid] = -1;
            t->be[cid] = -1;
        }
    }
    return added;
}

/* ------------------------------------------------------------------------ */
/* Bottom-up COM, CU:251-344, levels deepest first (CU:787-807).             */
/* ------------------------------------------------------------------------ */
static void leaf_com(orc_tree* t, const double* pos, const double* mass, int32_t nid,
                     int64_t* multi_leaves) {
    const int32_t start = t->bs[nid];
    const int32_t end = t->be[nid];
    if (start == end) { /* CU:268-275 */
        t->mass[nid] = mass[start];
        t->cx[nid] = pos[2 * start];
        t->cy[nid] = pos[2 * start + 1];
        return;
    }
    ++*multi_leaves;
    /* CU:284-309: 128 strided partial sums, then a shared-memory tree. */
    double sM[128], sX[128], sY[128];
    for (int tx = 0; tx < 128; ++tx) {
        double M = 0.0, Rx = 0.0, Ry = 0.0;
        for (int32_t i = start + tx; i <= end; i += 128) {
            const double m = mass[i];
            M += m;
            Rx = fma(m, pos[2 * i], Rx);
            Ry = fma(m, pos[2 * i + 1], Ry);
        }
        sM[tx] = M;
        sX[tx] = Rx;
        sY[tx] = Ry;
    }
    for (int s = 64; s > 0; s >>= 1)
        for (int tx = 0; tx < s; ++tx) {
            sM[tx] += sM[tx + s];
            sX[tx] += sX[tx + s];
            sY[tx] += sY[tx + s];
        }
    t->mass[nid] = sM[0];
    t->cx[nid] = sX[0] / sM[0];
    t->cy[nid] = sY[0] / sM[0];
}

static void internal_com(orc_tree* t, int32_t nid) {
    /* CU:329-343 */
    const int32_t c0 = t->c0[nid];
    double M = 0.0, Rx = 0.0, Ry = 0.0;
    for (int q = 0; q < 4; ++q) {
        const int32_t cid = c0 + q;
        if (t->bs[cid] < 0) continue;
        const double cm = t->mass[cid];
        M += cm;
        Rx = fma(cm, t->cx[cid], Rx);
        Ry = fma(cm, t->cy[cid], Ry);
    }
    t->mass[nid] = M;
    t->cx[nid] = Rx / M;
    t->cy[nid] = Ry / M;
}

/* ------------------------------------------------------------------------ */
/* Force pass, CU:382-486 (per-body DFS, pushes c0+3 .. c0).                 */
/* ------------------------------------------------------------------------ */
#define ORC_STACK 256

static void pair_term(double dx, double dy, double m, double eps2, double* ax, double* ay) {
    const double d2 = fma(dx, dx, dy * dy) + eps2;
    const double inv_r = 1.0 / sqrt(d2);
    const double inv_r3 = inv_r * inv_r * inv_r;
    const double a = m * inv_r3;
    *ax = fma(dx, a, *ax);
    *ay = fma(dy, a, *ay);
}

static void body_force(const orc_tree* t, const double* pos, const double* mass, int32_t i,
                       double eps2, double theta_sq, double* out_ax, double* out_ay,
                       int64_t* cells, int64_t* pairs, int64_t* max_stack) {
    const double bx = pos[2 * i], by = pos[2 * i + 1];
    double ax = 0.0, ay = 0.0;
    int32_t stack[ORC_STACK];
    int top = 0;
    stack[0] = 0;
    int64_t ncell = 0, npair = 0;
    int deepest = 1;
    while (top >= 0) {
        const int32_t nid = stack[top--];
        const int32_t bs = t->bs[nid];
        if (bs < 0) continue;
        const double dx = t->cx[nid] - bx;
        const double dy = t->cy[nid] - by;
        const double dist_sq = fma(dx, dx, dy * dy);
        const int32_t c0 = t->c0[nid];
        if (c0 < 0) {
            const int32_t be = t->be[nid];
            if (bs == be) {
                if (bs != i) {
                    pair_term(dx, dy, t->mass[nid], eps2, &ax, &ay);
                    ++npair;
                }
            } else if (i < bs || i > be) {
                pair_term(dx, dy, t->mass[nid], eps2, &ax, &ay);
                ++ncell;
            } else {
                for (int32_t j = bs; j <= be; ++j) {
                    if (j == i) continue;
                    pair_term(pos[2 * j] - bx, pos[2 * j + 1] - by, mass[j], eps2, &ax, &ay);
                    ++npair;
                }
            }
            continue;
        }
        if (t->wsq[nid] < theta_sq * dist_sq) {
            pair_term(dx, dy, t->mass[nid], eps2, &ax, &ay);
            ++ncell;
            continue;
        }
        for (int q = 3; q >= 0; --q)
            if (t->bs[c0 + q] >= 0) {
                if (top + 1 >= ORC_STACK) abort(); /* depth <= 31 levels x 3 pending */
                stack[++top] = c0 + q;
            }
        if (top + 1 > deepest) deepest = top + 1;
    }
    *out_ax = ax;
    *out_ay = ay;
    *cells += ncell;
    *pairs += npair;
    if (deepest > *max_stack) *max_stack = deepest;
}

/* ------------------------------------------------------------------------ */
/* One step, in the order of BarnesHutCuda::simulate                          */
/* (src/Simulation/src/BarnesHutCuda.cpp:30-40).                              */
/* ------------------------------------------------------------------------ */
static void free_tree(orc_tree* t) {
    free(t->wsq); free(t->c0); free(t->bs); free(t->be); free(t->mass); free(t->cx); free(t->cy);
}

/* Stages 1-4 of a step, in place on device-order arrays: bbox, Morton codes,
 * stable sort and gather (CU:648-711), the level-wise tree (CU:713-777) and
 * the bottom-up COM (CU:787-807).  On success *t holds the tree (free it
 * with free_tree). */
static int build_ref_tree(int64_t n, double* mass, double* pos, double* vel, int32_t* orig,
                          uint64_t* codes_out, int32_t* order_out, orc_tree* t, orc_stats* local) {
    /* 1. bounding box (CU:648-680) */
    orc_box box;
    orc_bbox_squared(n, pos, &box);

    /* 2. Morton codes + stable sort + gather (CU:682-711) */
    uint64_t* codes = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    uint64_t* sorted = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    int32_t* order = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    double* tmp = (double*)malloc(sizeof(double) * 2 * (size_t)n);
    int32_t* itmp = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    if (!codes || !sorted || !order || !tmp || !itmp) return -1;
    orc_morton(n, pos, &box, codes);
    orc_stable_sort(n, codes, sorted, order);
    free(codes);
    for (int64_t r = 0; r < n; ++r) { tmp[2 * r] = pos[2 * order[r]]; tmp[2 * r + 1] = pos[2 * order[r] + 1]; }
    memcpy(pos, tmp, sizeof(double) * 2 * (size_t)n);
    for (int64_t r = 0; r < n; ++r) { tmp[2 * r] = vel[2 * order[r]]; tmp[2 * r + 1] = vel[2 * order[r] + 1]; }
    memcpy(vel, tmp, sizeof(double) * 2 * (size_t)n);
    for (int64_t r = 0; r < n; ++r) tmp[r] = mass[order[r]];
    memcpy(mass, tmp, sizeof(double) * (size_t)n);
    for (int64_t r = 0; r < n; ++r) itmp[r] = orig[order[r]];
    memcpy(orig, itmp, sizeof(int32_t) * (size_t)n);
    free(tmp);
    free(itmp);
    if (codes_out) memcpy(codes_out, sorted, sizeof(uint64_t) * (size_t)n);
    if (order_out) memcpy(order_out, order, sizeof(int32_t) * (size_t)n);
    free(order);

    /* 3. tree (CU:713-777) in a 5n node pool; the level lists live in one array */
    t->cap = 5 * n;
    t->wsq = (double*)malloc(sizeof(double) * (size_t)t->cap);
    t->c0 = (int32_t*)malloc(sizeof(int32_t) * (size_t)t->cap);
    t->bs = (int32_t*)malloc(sizeof(int32_t) * (size_t)t->cap);
    t->be = (int32_t*)malloc(sizeof(int32_t) * (size_t)t->cap);
    t->mass = (double*)malloc(sizeof(double) * (size_t)t->cap);
    t->cx = (double*)malloc(sizeof(double) * (size_t)t->cap);
    t->cy = (double*)malloc(sizeof(double) * (size_t)t->cap);
    int32_t* lists = (int32_t*)malloc(sizeof(int32_t) * (size_t)t->cap);
    if (!t->wsq || !t->c0 || !t->bs || !t->be || !t->mass || !t->cx || !t->cy || !lists) return -1;
    const double w = box.x_max - box.x_min;
    t->wsq[0] = pow(w, 2.0); /* CU:717 */
    t->c0[0] = -1;
    t->bs[0] = 0;
    t->be[0] = (int32_t)(n - 1);
    t->alloc = 1;
    int64_t level_off[32], level_cnt[32];
    int nlev = 0;
    lists[0] = 0;
    int64_t cur = 0, cnt = 1;
    for (int level = 0; level < 31; ++level) {
        if (cnt == 0) break;
        level_off[nlev] = cur;
        level_cnt[nlev] = cnt;
        ++nlev;
        const int64_t next_off = cur + cnt;
        int64_t next_cnt = 0;
        for (int64_t k = 0; k < cnt; ++k)
            split_node(t, sorted, lists[cur + k], level, lists + next_off, &next_cnt);
        cur = next_off;
        cnt = next_cnt;
    }
    free(sorted);
    local->levels = nlev;
    local->nodes_allocated = t->alloc;
    local->nodes_nonempty = cur;

    /* 4. COM bottom-up (CU:787-807) */
    for (int lvl = nlev - 1; lvl >= 0; --lvl) {
        for (int64_t k = 0; k < level_cnt[lvl]; ++k) {
            const int32_t nid = lists[level_off[lvl] + k];
            if (t->c0[nid] < 0) {
                leaf_com(t, pos, mass, nid, &local->multi_leaves);
                if (lvl > local->max_level) local->max_level = lvl;
            }
        }
        for (int64_t k = 0; k < level_cnt[lvl]; ++k) {
            const int32_t nid = lists[level_off[lvl] + k];
            if (t->c0[nid] >= 0) internal_com(t, nid);
        }
    }
    free(lists);
    return 0;
}

int orc_ref_step(int64_t n, double* mass, double* pos, double* vel, int32_t* orig, double G,
                 double dt, double eps2, double theta, int do_integrate, double* acc_out,
                 uint64_t* codes_out, int32_t* order_out, int nthreads, orc_stats* st) {
    if (n <= 0) return -1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    orc_stats local;
    memset(&local, 0, sizeof(local));
    orc_tree t;
    memset(&t, 0, sizeof(t));
    if (build_ref_tree(n, mass, pos, vel, orig, codes_out, order_out, &t, &local) != 0) return -1;

    /* 5. force + kick (CU:812-822, CU:484-485) */
    const double theta_sq = theta * theta;
    const double G_dt = G * dt;
    int64_t cells = 0, pairs = 0, max_stack = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : cells, pairs) reduction(max : max_stack)
    for (int64_t i = 0; i < n; ++i) {
        double ax, ay;
        int64_t ms = 0;
        body_force(&t, pos, mass, (int32_t)i, eps2, theta_sq, &ax, &ay, &cells, &pairs, &ms);
        if (ms > max_stack) max_stack = ms;
        if (acc_out) {
            acc_out[2 * i] = ax;
            acc_out[2 * i + 1] = ay;
        }
        if (do_integrate) {
            vel[2 * i] = fma(ax, G_dt, vel[2 * i]);
            vel[2 * i + 1] = fma(ay, G_dt, vel[2 * i + 1]);
        }
    }
    local.cell_interactions = cells;
    local.body_interactions = pairs;
    local.max_stack = max_stack;

    /* 6. drift (CU:489-495) */
    if (do_integrate)
        for (int64_t i = 0; i < n; ++i) {
            pos[2 * i] = fma(vel[2 * i], dt, pos[2 * i]);
            pos[2 * i + 1] = fma(vel[2 * i + 1], dt, pos[2 * i + 1]);
        }

    free_tree(&t);
    if (st) *st = local;
    return 0;
}

int orc_ref_walk_targets(int64_t n, double* mass, double* pos, double* vel, int32_t* orig,
                         double eps2, double theta, int64_t k, const int64_t* targets,
                         double* acc_out, int64_t* cells_out, int64_t* pairs_out,
                         int64_t* stack_out, int nthreads, orc_stats* st) {
    if (n <= 0 || k < 0) return -1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    for (int64_t q = 0; q < k; ++q)
        if (targets[q] < 0 || targets[q] >= n) return -2;
    orc_stats local;
    memset(&local, 0, sizeof(local));
    orc_tree t;
    memset(&t, 0, sizeof(t));
    if (build_ref_tree(n, mass, pos, vel, orig, NULL, NULL, &t, &local) != 0) return -1;
    int32_t* slot = (int32_t*)malloc(sizeof(int32_t) * (size_t)n); /* original index -> slot */
    if (!slot) return -1;
    for (int64_t i = 0; i < n; ++i) slot[orig[i]] = (int32_t)i;
    const double theta_sq = theta * theta;
    int64_t cells = 0, pairs = 0, max_stack = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : cells, pairs) reduction(max : max_stack)
    for (int64_t q = 0; q < k; ++q) {
        double ax, ay;
        int64_t c = 0, p = 0, ms = 0;
        body_force(&t, pos, mass, slot[targets[q]], eps2, theta_sq, &ax, &ay, &c, &p, &ms);
        if (acc_out) {
            acc_out[2 * q] = ax;
            acc_out[2 * q + 1] = ay;
        }
        if (cells_out) cells_out[q] = c;
        if (pairs_out) pairs_out[q] = p;
        if (stack_out) stack_out[q] = ms;
        cells += c;
        pairs += p;
        if (ms > max_stack) max_stack = ms;
    }
    local.cell_interactions = cells;
    local.body_interactions = pairs;
    local.max_stack = max_stack;
    free(slot);
    free_tree(&t);
    if (st) *st = local;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* All-pairs oracles.                                                         */
/* ------------------------------------------------------------------------ */
void orc_allpairs_plummer(int64_t n, const double* mass, const double* pos, int64_t k,
                          const int64_t* tgt, double eps2, double* acc, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t t = 0; t < k; ++t) {
        const int64_t i = tgt[t];
        const double bx = pos[2 * i], by = pos[2 * i + 1];
        double ax = 0.0, ay = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            if (j == i) continue;
            const double dx = pos[2 * j] - bx, dy = pos[2 * j + 1] - by;
            const double d2 = dx * dx + dy * dy + eps2;
            const double inv_r = 1.0 / sqrt(d2);
            const double a = mass[j] * inv_r * inv_r * inv_r;
            ax += dx * a;
            ay += dy * a;
        }
        acc[2 * t] = ax;
        acc[2 * t + 1] = ay;
    }
}

void orc_allpairs_plummer_abs(int64_t n, const double* mass, const double* pos, int64_t k,
                              const int64_t* tgt, double eps2, double* out, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t t = 0; t < k; ++t) {
        const int64_t i = tgt[t];
        const double bx = pos[2 * i], by = pos[2 * i + 1];
        double s = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            if (j == i) continue;
            const double dx = pos[2 * j] - bx, dy = pos[2 * j + 1] - by;
            const double r2 = dx * dx + dy * dy;
            const double d2 = r2 + eps2;
            s += mass[j] * sqrt(r2) / (d2 * sqrt(d2));
        }
        out[t] = s;
    }
}

void orc_allpairs_fp32_bound(int64_t n, const double* mass, const double* pos, int64_t k,
                             const int64_t* tgt, double eps2, double cx, double cy, double* out,
                             int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    const double u = 5.9604644775390625e-08; /* 2^-24, FP32 unit roundoff */
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t t = 0; t < k; ++t) {
        const int64_t i = tgt[t];
        const double bx = pos[2 * i], by = pos[2 * i + 1];
        const double ri = fabs(bx - cx) + fabs(by - cy);
        double s = 0.0, abs_sum = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            if (j == i) continue;
            const double dx = pos[2 * j] - bx, dy = pos[2 * j + 1] - by;
            const double r2 = dx * dx + dy * dy;
            const double r = sqrt(r2);
            const double d2 = r2 + eps2;
            const double term = mass[j] * r / (d2 * sqrt(d2));
            const double rj = fabs(pos[2 * j] - cx) + fabs(pos[2 * j + 1] - cy);
            /* rounding of the two coordinates shifts d by up to u (ri + rj);
             * the term moves by at most 3 of that relative to r, plus 16 u of
             * per-term arithmetic */
            s += term * (16.0 * u + (r > 0.0 ? 3.0 * u * (ri + rj) / r : 0.0));
            abs_sum += term;
        }
        /* accumulation: each addition rounds by at most u |partial sum| <=
         * u abs_sum; independent roundings grow like sqrt(terms), taken with a
         * margin of 8 */
        out[t] = s + 8.0 * sqrt((double)n) * u * abs_sum;
    }
}

void orc_allpairs_cpulaw(int64_t n, const double* mass, const double* pos, int64_t k,
                         const int64_t* tgt, double G, double eps2, double* acc, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t t = 0; t < k; ++t) {
        const int64_t i = tgt[t];
        const double bx = pos[2 * i], by = pos[2 * i + 1];
        double ax = 0.0, ay = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            const double dx = pos[2 * j] - bx, dy = pos[2 * j + 1] - by;
            if (dx == 0.0 && dy == 0.0) continue;
            const double d = sqrt(dx * dx + dy * dy);
            const double f = G * mass[j] / (d * d + eps2);
            ax += dx / d * f;
            ay += dy / d * f;
        }
        acc[2 * t] = ax;
        acc[2 * t + 1] = ay;
    }
}
