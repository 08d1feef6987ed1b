// adapter_demo.cpp -- runs the BarnesHutB200 adapter (n-body-2d_b200/host)
// through the reference's own Simulation base class (src/Simulation/src/
// Simulation.cpp, compiled unmodified): construction, run(), is_finished(),
// destruction, exactly as the reference's Controller drives a backend.
// INTEGRATION CHECK, built with the reference sources into oracle/_ref/.
//
// Usage: adapter_demo <input> <output>; formats as ref_cpu_bh.cpp (the
// header's "warmup" word selects the mode: 0 FP64, 1 SPLIT).  The reference
// hard-wires G; masses are scaled by G / Constants::Simulation::G.  The
// second parameter word is the reference's softening_factor; the base class
// turns it into epsilon^2 (sampled mean pair distance x factor, squared),
// which the output carries after the run time: seconds, eps2, pos, vel.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <string>
#include <thread>
#include <vector>

#include "BarnesHutB200.hpp"
#include "Constants/Constants.hpp"
#include "Logger/Logger.hpp"

int main(int argc, char** argv) {
    if (argc != 3) return 2;
    Log::verbosity = Log::Verbosity::ERROR;
    std::FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 3;
    int64_t hdr[4];
    double par[4];
    if (std::fread(hdr, 8, 4, in) != 4 || std::fread(par, 8, 4, in) != 4) return 4;
    const int64_t n = hdr[0], steps = hdr[1], mode = hdr[3];
    std::vector<double> m(n), p(2 * n), v(2 * n);
    if (std::fread(m.data(), 8, n, in) != (size_t)n || std::fread(p.data(), 8, 2 * n, in) != (size_t)(2 * n) ||
        std::fread(v.data(), 8, 2 * n, in) != (size_t)(2 * n))
        return 5;
    std::fclose(in);
    const double scale = par[3] / Constants::Simulation::G;
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
    Config::Simulation cfg{};
    cfg.timestep = par[2];
    cfg.iterations = (uint64_t)steps;
    cfg.theta = par[0];
    cfg.softening_factor = par[1];
    cfg.threads = 1;
    double seconds = 0.0, eps2 = 0.0;
    {
        BarnesHutB200 sim(cfg, bodies, mode ? NB_MODE_SPLIT : NB_MODE_FP64, 1);
        eps2 = sim.softening_squared();
        const auto t0 = std::chrono::steady_clock::now();
        sim.run();
        while (!sim.is_finished()) std::this_thread::sleep_for(std::chrono::microseconds(100));
        seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    std::FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 6;
    std::fwrite(&seconds, 8, 1, out);
    std::fwrite(&eps2, 8, 1, out);
    std::fwrite(bodies.pos_data(), 8, 2 * n, out);
    std::fwrite(bodies.vel_data(), 8, 2 * n, out);
    std::fclose(out);
    return 0;
}
