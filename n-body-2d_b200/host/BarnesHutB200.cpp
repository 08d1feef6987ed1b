// BarnesHutB200.cpp -- see BarnesHutB200.hpp.
#include "BarnesHutB200.hpp"

#include <algorithm>
#include <stdexcept>
#include <string>

#include "Constants/Constants.hpp"
#include "Logger/Logger.hpp"

BarnesHutB200::BarnesHutB200(const Config::Simulation& sim_cfg, Bodies& bodies, int32_t mode,
                             uint32_t download_every_)
        : Simulation(sim_cfg, bodies), download_every(std::max<uint32_t>(1, download_every_)) {
    nb_params p;
    nb_params_default(&p);
    p.G = Constants::Simulation::G;
    p.timestep = sim_cfg.timestep;
    p.theta = sim_cfg.theta;
    p.epsilon_squared = epsilon_squared;
    p.mode = mode;
    // sf::Vector2<double> is two packed doubles: pos_data()/vel_data() are the
    // interleaved {x, y} arrays the ABI takes (as the reference's own uploads,
    // BarnesHutCuda.cu:597-599).
    const int rc = nb_create(&p, bodies.n, bodies.mass_data(),
                             reinterpret_cast<const double*>(bodies.pos_data()),
                             reinterpret_cast<const double*>(bodies.vel_data()), &ctx);
    if (rc != NB_OK)
        throw std::runtime_error(std::string("nb_create failed: ") + nb_status_string(rc));
}

BarnesHutB200::~BarnesHutB200() {
    if (sim_thread.joinable()) {
        on_pause();
    }
    nb_destroy(ctx);
}

void BarnesHutB200::on_run() {
    stop = false;
    sim_thread = std::thread(&BarnesHutB200::simulate, this);
}

void BarnesHutB200::on_pause() {
    stop = true;
    sim_thread.join();
}

// BarnesHutCuda::simulate (BarnesHutCuda.cpp:30-40) with the step on the GPU
// and the per-step download made optional.
void BarnesHutB200::simulate() {
    uint32_t since_download = 0;
    auto download = [&]() {
        return nb_download(ctx, reinterpret_cast<double*>(bodies.pos_data()),
                           reinterpret_cast<double*>(bodies.vel_data()));
    };
    while (!should_stop()) {
        int rc = nb_set_timestep(ctx, timestep);
        if (rc == NB_OK) rc = nb_step(ctx, 1);
        if (rc == NB_OK && ++since_download >= download_every) {
            rc = download();
            since_download = 0;
        } else if (rc == NB_OK) {
            rc = nb_sync(ctx);
        }
        if (rc != NB_OK) {
            Log::error("B200 step failed: {} ({})", nb_last_error(ctx), nb_status_string(rc));
            break;
        }
        post_iteration();
    }
    if (since_download > 0 && download() != NB_OK)
        Log::error("B200 download failed: {}", nb_last_error(ctx));
}
