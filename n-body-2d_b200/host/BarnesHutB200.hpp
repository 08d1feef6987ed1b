// BarnesHutB200.hpp -- Simulation backend of PhivPap/n-body-2d on the B200
// library.  Drop-in next to BarnesHutCuda
// (src/Simulation/include/Simulation/BarnesHutCuda.hpp:44-112): same base
// class, same constructor signature, same run/pause threading contract; the
// device work goes through the C ABI in include/nbody_b200.h.
#pragma once

#include <cstdint>
#include <thread>

#include "Simulation/Simulation.hpp"
#include "nbody_b200.h"

class BarnesHutB200 : public Simulation {
public:
    // mode: NB_MODE_SPLIT (default, fast) or NB_MODE_FP64 (the reference's
    // forces).  download_every: copy the bodies back every that many steps
    // (1 = after every step, as the reference does).
    BarnesHutB200(const Config::Simulation& sim_cfg, Bodies& bodies, int32_t mode = NB_MODE_SPLIT,
                  uint32_t download_every = 1);
    ~BarnesHutB200() override;

    // The Plummer epsilon^2 the base class derived from softening_factor
    // (Simulation.cpp:11-15), as passed to the library.
    double softening_squared() const { return epsilon_squared; }

private:
    nb_ctx* ctx = nullptr;
    std::thread sim_thread;
    const uint32_t download_every;

    void on_run() override;
    void on_pause() override;
    void simulate();
};
