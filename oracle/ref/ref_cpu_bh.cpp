// ref_cpu_bh.cpp -- drives the reference's threaded CPU Barnes-Hut backend
// (src/Simulation/src/BarnesHut.cpp, compiled unmodified from the reference
// sources) through its public Simulation interface, for timing and for
// checking it against its own pair law.  TEST / BASELINE INFRASTRUCTURE.
//
// Usage: ref_cpu_bh <input> <output>
// input  (binary, little endian): int64 n, steps, threads, warmup;
//        double theta, epsilon_squared, dt, G; mass[n]; pos[2n]; vel[2n]
// output: double seconds (wall time of the `steps` timed steps); pos[2n]; vel[2n]
// The `warmup` steps run first, untimed, on the same bodies.
//
// The reference hard-wires G = 6.67430e-11 (Constants.hpp:17); masses are
// scaled by G / 6.67430e-11 so the dynamics are those of the requested G.
// Its softening is estimated from random pair samples (Simulation.cpp:82-126);
// the harness builds it with softening_factor 0 and then sets the requested
// epsilon^2 on the constructed object.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <string>
#include <thread>
#include <vector>

#include "Constants/Constants.hpp"
#include "Logger/Logger.hpp"
#include "Simulation/BarnesHut.hpp"

namespace {

struct HarnessBarnesHut : BarnesHut {
    using BarnesHut::BarnesHut;
    void set_epsilon_squared(double e2) { const_cast<double&>(epsilon_squared) = e2; }
};

template <typename T>
bool read_all(std::FILE* f, T* p, size_t count) {
    return std::fread(p, sizeof(T), count, f) == count;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s <input> <output>\n", argv[0]);
        return 2;
    }
    Log::verbosity = Log::Verbosity::ERROR;
    std::FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 3;
    int64_t hdr[4];
    double par[4];
    if (!read_all(in, hdr, 4) || !read_all(in, par, 4)) return 4;
    const int64_t n = hdr[0], steps = hdr[1], threads = hdr[2], warmup = hdr[3];
    const double theta = par[0], eps2 = par[1], dt = par[2], G = par[3];
    std::vector<double> m(n), p(2 * n), v(2 * n);
    if (!read_all(in, m.data(), n) || !read_all(in, p.data(), 2 * n) ||
        !read_all(in, v.data(), 2 * n))
        return 5;
    std::fclose(in);

    const double scale = G / Constants::Simulation::G;
    std::vector<std::string> ids(n);
    std::vector<double> mass(n);
    std::vector<sf::Vector2<double>> pos(n), vel(n);
    for (int64_t i = 0; i < n; ++i) {
        ids[i] = std::to_string(i);
        mass[i] = m[i] * scale;
        pos[i] = {p[2 * i], p[2 * i + 1]};
        vel[i] = {v[2 * i], v[2 * i + 1]};
    }
    Bodies bodies(std::move(ids), std::move(mass), std::move(pos), std::move(vel));

    // One Simulation per phase: `warmup` steps untimed, then `steps` timed;
    // the backend advances `bodies` in place, so the second continues the first.
    auto advance = [&](int64_t iterations) {
        Config::Simulation cfg{};
        cfg.timestep = dt;
        cfg.iterations = static_cast<uint64_t>(iterations);
        cfg.simtype = Config::Simulation::SimType::BARNES_HUT;
        cfg.theta = theta;
        cfg.softening_factor = 0.0;
        cfg.threads = static_cast<uint16_t>(threads);
        HarnessBarnesHut sim(cfg, bodies);
        sim.set_epsilon_squared(eps2);
        const auto t0 = std::chrono::steady_clock::now();
        sim.run();
        while (!sim.is_finished()) std::this_thread::sleep_for(std::chrono::microseconds(200));
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    };  // each Simulation's destructor stops and joins its worker threads
    if (warmup > 0) advance(warmup);
    const double seconds = steps > 0 ? advance(steps) : 0.0;

    std::FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 6;
    std::fwrite(&seconds, sizeof(double), 1, out);
    std::fwrite(bodies.pos_data(), sizeof(double), 2 * n, out);
    std::fwrite(bodies.vel_data(), sizeof(double), 2 * n, out);
    std::fclose(out);
    return 0;
}
