// ref_gpu_harness.cu -- runs the reference's CUDA kernels to produce golden
// vectors for the oracle.  TEST INFRASTRUCTURE.
//
// The reference's kernels (src/Simulation/src/BarnesHutCuda.cu) are compiled
// unmodified from the reference checkout by including that file.  This
// harness supplies its own host driver instead of BarnesHutCuda's member
// functions, for one reason: the reference sizes its level work list for n+1
// cells (CU:585) but appends every level of the tree to it (CU:763,770), about
// 1.7 n entries, so its own driver writes past that allocation.  Here the work
// list holds the whole 5n node pool.  Everything else keeps the reference's
// sequence: box reduction, host squaring, Morton codes, CUB SortPairs, reorder,
// level-by-level topology, bottom-up COM, force + kick, drift.
//
// The force kernel keeps a 32-entry stack (CU:400); the script that calls this
// harness first has the oracle replay the same steps and refuses inputs whose
// walk would need more than 28 entries.
//
// Usage: ref_gpu_harness <input> <output>
// input : int64 n, steps, pad, pad; double theta, epsilon_squared, dt, G;
//         mass[n]; pos[2n]; vel[2n]
// output: int64 n, nodes_allocated, levels, ns per step (steps 1.. on the host
//         clock, 0 for one step); double box[4] (squared, first
//         step); uint64 sorted codes[n]; int32 permutation[n]; int32 orig[n];
//         double acc[2n] (first step, sorted order, without G);
//         double pos[2n], vel[2n] (after all steps, original order)
#include "BarnesHutCuda.cu"

#include <cfloat>
#include <chrono>
#include <cstdio>
#include <vector>

namespace harness {

template <typename T>
T* dmalloc(size_t count) {
    T* p = nullptr;
    CUDA_CHECK(cudaMalloc(&p, sizeof(T) * (count ? count : 1)));
    return p;
}

struct State {
    int32_t n = 0;
    int32_t max_nodes = 0;
    double *mass = nullptr, *mass_alt = nullptr;
    Vector2 *pos = nullptr, *pos_alt = nullptr, *vel = nullptr, *vel_alt = nullptr, *vel_zero = nullptr;
    int32_t *idx = nullptr, *idx_alt = nullptr, *sort_idx = nullptr, *sort_idx_alt = nullptr;
    uint64_t *morton = nullptr, *morton_alt = nullptr;
    BarnesHutCuda::Box* box_d = nullptr;
    TreeNodesSoA tree;
    int32_t *node_count = nullptr, *work_list = nullptr, *work_count = nullptr;
    void* cub_temp = nullptr;
    size_t cub_bytes = 0;
    BarnesHutCuda::Box box{};
    int32_t nodes_allocated = 0, levels = 0;
};

void squared_box(State& s) {
    s.box = BarnesHutCuda::Box{DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX};
    CUDA_CHECK(cudaMemcpy(s.box_d, &s.box, sizeof(s.box), cudaMemcpyHostToDevice));
    const uint32_t grid = (s.n + BLOCK_SIZE - 1) / BLOCK_SIZE;
    Kernel::compute_bounding_box<<<grid, BLOCK_SIZE, 4 * BLOCK_SIZE * sizeof(double)>>>(
        s.pos, (uint32_t)s.n, s.box_d);
    CUDA_CHECK(cudaGetLastError());
    CUDA_CHECK(cudaMemcpy(&s.box, s.box_d, sizeof(s.box), cudaMemcpyDeviceToHost));
    const double xr = s.box.x_max - s.box.x_min, yr = s.box.y_max - s.box.y_min;
    if (xr > yr) {
        const double mid = (s.box.y_min + s.box.y_max) * 0.5;
        s.box.y_min = mid - xr * 0.5;
        s.box.y_max = mid + xr * 0.5;
    } else {
        const double mid = (s.box.x_min + s.box.x_max) * 0.5;
        s.box.x_min = mid - yr * 0.5;
        s.box.x_max = mid + yr * 0.5;
    }
    CUDA_CHECK(cudaMemcpy(s.box_d, &s.box, sizeof(s.box), cudaMemcpyHostToDevice));
}

void sort_and_reorder(State& s) {
    const uint32_t grid = (s.n + BLOCK_SIZE - 1) / BLOCK_SIZE;
    Kernel::compute_morton_codes<<<grid, BLOCK_SIZE>>>(s.pos, (uint32_t)s.n, s.box_d, s.morton,
                                                       s.sort_idx);
    CUDA_CHECK(cudaGetLastError());
    CUDA_CHECK(cub::DeviceRadixSort::SortPairs(s.cub_temp, s.cub_bytes, s.morton, s.morton_alt,
                                               s.sort_idx, s.sort_idx_alt, s.n));
    Kernel::reorder_bodies<<<grid, BLOCK_SIZE>>>(s.sort_idx_alt, s.pos, s.vel, s.mass, s.idx,
                                                 s.pos_alt, s.vel_alt, s.mass_alt, s.idx_alt, s.n);
    CUDA_CHECK(cudaGetLastError());
    std::swap(s.pos, s.pos_alt);
    std::swap(s.vel, s.vel_alt);
    std::swap(s.mass, s.mass_alt);
    std::swap(s.idx, s.idx_alt);
    std::swap(s.morton, s.morton_alt);
    CUDA_CHECK(cudaDeviceSynchronize());
}

void build_tree(State& s) {
    const double root_wsq = std::pow(s.box.x_max - s.box.x_min, 2.0);
    const int32_t one = 1, zero = 0, none = -1, last = s.n - 1;
    CUDA_CHECK(cudaMemcpy(s.node_count, &one, 4, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(s.tree.width_sq, &root_wsq, 8, cudaMemcpyHostToDevice));
    for (int32_t* c : {s.tree.child0, s.tree.child1, s.tree.child2, s.tree.child3})
        CUDA_CHECK(cudaMemcpy(c, &none, 4, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(s.tree.body_start, &zero, 4, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(s.tree.body_end, &last, 4, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(s.work_list, &zero, 4, cudaMemcpyHostToDevice));
    std::vector<int32_t> offs, cnts;
    int32_t cur = 0, count = 1;
    for (int32_t level = 0; level < 31 && count > 0; ++level) {
        offs.push_back(cur);
        cnts.push_back(count);
        const int32_t next = cur + count;
        CUDA_CHECK(cudaMemset(s.work_count, 0, 4));
        Kernel::build_tree_topology<<<(count + BLOCK_SIZE - 1) / BLOCK_SIZE, BLOCK_SIZE>>>(
            s.morton, s.tree.width_sq, s.tree.child0, s.tree.child1, s.tree.child2, s.tree.child3,
            s.tree.body_start, s.tree.body_end, s.work_list + cur, count, s.work_list + next,
            s.work_count, s.node_count, s.max_nodes, level);
        CUDA_CHECK(cudaGetLastError());
        CUDA_CHECK(cudaMemcpy(&count, s.work_count, 4, cudaMemcpyDeviceToHost));
        cur = next;
        if (cur + count > s.max_nodes) {  // cannot happen: every listed cell is a pool slot
            std::fprintf(stderr, "work list overflow\n");
            std::exit(7);
        }
    }
    s.levels = (int32_t)offs.size();
    CUDA_CHECK(cudaMemcpy(&s.nodes_allocated, s.node_count, 4, cudaMemcpyDeviceToHost));
    for (int32_t l = s.levels - 1; l >= 0; --l) {
        const int32_t* nodes = s.work_list + offs[l];
        Kernel::compute_leaf_com<<<cnts[l], 128, 3 * 128 * sizeof(double)>>>(
            s.pos, s.mass, s.tree.mass, s.tree.com_x, s.tree.com_y, nodes, cnts[l],
            s.tree.body_start, s.tree.body_end, s.tree.child0);
        Kernel::propagate_com_up<<<(cnts[l] + BLOCK_SIZE - 1) / BLOCK_SIZE, BLOCK_SIZE>>>(
            s.tree.mass, s.tree.com_x, s.tree.com_y, s.tree.child0, s.tree.child1, s.tree.child2,
            s.tree.child3, s.tree.body_start, nodes, cnts[l]);
        CUDA_CHECK(cudaGetLastError());
    }
    CUDA_CHECK(cudaDeviceSynchronize());
}

void force(State& s, Vector2* vel, double eps2, double G_dt, double theta_sq) {
    const uint32_t grid = (s.n + BLOCK_SIZE - 1) / BLOCK_SIZE;
    Kernel::compute_force<<<grid, BLOCK_SIZE>>>(s.tree.mass, s.tree.com_x, s.tree.com_y,
                                                s.tree.width_sq, s.tree.child0, s.tree.body_start,
                                                s.tree.body_end, s.pos, s.mass, vel, s.n, eps2,
                                                G_dt, theta_sq);
    CUDA_CHECK(cudaGetLastError());
    CUDA_CHECK(cudaDeviceSynchronize());
}

}  // namespace harness

int main(int argc, char** argv) {
    using namespace harness;
    if (argc != 3) return 2;
    std::FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 3;
    int64_t hdr[4];
    double par[4];
    if (std::fread(hdr, 8, 4, in) != 4 || std::fread(par, 8, 4, in) != 4) return 4;
    const int32_t n = (int32_t)hdr[0];
    const int64_t steps = hdr[1];
    // header word 2, bit 0: end every step as BarnesHutCuda::simulate does,
    // with the scatter to original order and the download of positions and
    // velocities into host memory (CU:498-506, 632-646)
    const bool download = (hdr[2] & 1) != 0;
    const double theta = par[0], eps2 = par[1], dt = par[2], G = par[3];
    std::vector<double> m(n), p(2 * n), v(2 * n);
    if (std::fread(m.data(), 8, n, in) != (size_t)n || std::fread(p.data(), 8, 2 * n, in) != (size_t)(2 * n) ||
        std::fread(v.data(), 8, 2 * n, in) != (size_t)(2 * n))
        return 5;
    std::fclose(in);

    State s;
    s.n = n;
    s.max_nodes = 5 * n;  // max_quads, BarnesHutCuda.cpp:9
    s.mass = dmalloc<double>(n);
    s.mass_alt = dmalloc<double>(n);
    s.pos = dmalloc<Vector2>(n);
    s.pos_alt = dmalloc<Vector2>(n);
    s.vel = dmalloc<Vector2>(n);
    s.vel_alt = dmalloc<Vector2>(n);
    s.vel_zero = dmalloc<Vector2>(n);
    s.idx = dmalloc<int32_t>(n);
    s.idx_alt = dmalloc<int32_t>(n);
    s.sort_idx = dmalloc<int32_t>(n);
    s.sort_idx_alt = dmalloc<int32_t>(n);
    s.morton = dmalloc<uint64_t>(n);
    s.morton_alt = dmalloc<uint64_t>(n);
    s.box_d = dmalloc<BarnesHutCuda::Box>(1);
    alloc_tree_soa(s.tree, s.max_nodes);
    s.node_count = dmalloc<int32_t>(1);
    s.work_list = dmalloc<int32_t>((size_t)s.max_nodes + 1);
    s.work_count = dmalloc<int32_t>(1);
    CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, s.cub_bytes, s.morton, s.morton_alt,
                                               s.sort_idx, s.sort_idx_alt, n));
    s.cub_temp = dmalloc<char>(s.cub_bytes);
    CUDA_CHECK(cudaMemcpy(s.mass, m.data(), 8 * n, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(s.pos, p.data(), 16 * n, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(s.vel, v.data(), 16 * n, cudaMemcpyHostToDevice));
    Kernel::init_indices<<<(n + BLOCK_SIZE - 1) / BLOCK_SIZE, BLOCK_SIZE>>>(s.idx, n);
    CUDA_CHECK(cudaDeviceSynchronize());

    std::vector<uint64_t> codes(n);
    std::vector<int32_t> perm(n), orig(n);
    std::vector<double> acc(2 * n);
    BarnesHutCuda::Box box0{};
    int32_t nodes0 = 0, levels0 = 0;
    // steps after the first are timed on the host clock: the reference's step
    // is host-driven (a D2H count per tree level), so its cost is wall time
    std::chrono::steady_clock::time_point t1;
    for (int64_t step = 0; step < steps; ++step) {
        if (step == 1) t1 = std::chrono::steady_clock::now();
        squared_box(s);
        sort_and_reorder(s);
        build_tree(s);
        if (step == 0) {
            box0 = s.box;
            nodes0 = s.nodes_allocated;
            levels0 = s.levels;
            CUDA_CHECK(cudaMemcpy(codes.data(), s.morton, 8 * n, cudaMemcpyDeviceToHost));
            CUDA_CHECK(cudaMemcpy(perm.data(), s.sort_idx_alt, 4 * n, cudaMemcpyDeviceToHost));
            CUDA_CHECK(cudaMemcpy(orig.data(), s.idx, 4 * n, cudaMemcpyDeviceToHost));
            // the kick with zero velocities and G dt = 1 leaves the acceleration
            CUDA_CHECK(cudaMemset(s.vel_zero, 0, 16 * n));
            force(s, s.vel_zero, eps2, 1.0, theta * theta);
            CUDA_CHECK(cudaMemcpy(acc.data(), s.vel_zero, 16 * n, cudaMemcpyDeviceToHost));
        }
        force(s, s.vel, eps2, G * dt, theta * theta);
        Kernel::update_positions<<<(n + BLOCK_SIZE - 1) / BLOCK_SIZE, BLOCK_SIZE>>>(s.pos, s.vel, n, dt);
        if (download) {
            Kernel::scatter_to_original_order<<<(n + BLOCK_SIZE - 1) / BLOCK_SIZE, BLOCK_SIZE>>>(
                s.pos, s.vel, s.idx, s.pos_alt, s.vel_alt, n);
            CUDA_CHECK(cudaMemcpy(p.data(), s.pos_alt, 16 * n, cudaMemcpyDeviceToHost));
            CUDA_CHECK(cudaMemcpy(v.data(), s.vel_alt, 16 * n, cudaMemcpyDeviceToHost));
        }
        CUDA_CHECK(cudaDeviceSynchronize());
    }
    const double timed = steps > 1 ? std::chrono::duration<double>(
                                         std::chrono::steady_clock::now() - t1).count()
                                   : 0.0;
    Kernel::scatter_to_original_order<<<(n + BLOCK_SIZE - 1) / BLOCK_SIZE, BLOCK_SIZE>>>(
        s.pos, s.vel, s.idx, s.pos_alt, s.vel_alt, n);
    CUDA_CHECK(cudaDeviceSynchronize());
    CUDA_CHECK(cudaMemcpy(p.data(), s.pos_alt, 16 * n, cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(v.data(), s.vel_alt, 16 * n, cudaMemcpyDeviceToHost));

    std::FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 6;
    // header word 3: nanoseconds per step over steps 1.. (0 for a single step)
    const int64_t ns_per_step = steps > 1 ? (int64_t)(timed * 1e9 / (double)(steps - 1)) : 0;
    const int64_t oh[4] = {n, nodes0, levels0, ns_per_step};
    std::fwrite(oh, 8, 4, out);
    std::fwrite(&box0, 8, 4, out);
    std::fwrite(codes.data(), 8, n, out);
    std::fwrite(perm.data(), 4, n, out);
    std::fwrite(orig.data(), 4, n, out);
    std::fwrite(acc.data(), 8, 2 * n, out);
    std::fwrite(p.data(), 8, 2 * n, out);
    std::fwrite(v.data(), 8, 2 * n, out);
    std::fclose(out);
    return 0;
}
