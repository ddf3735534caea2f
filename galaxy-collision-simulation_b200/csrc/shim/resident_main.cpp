// resident_main.cpp -- the reference's simulation loop (cpp/core/main.cpp:140-184) for the
// cuda-direct solvers, run on the engine's resident session (include/gx_session.hpp).
//
// The reference calls cuda_direct_leapfrog_step once per step (main.cpp:172-174), and every
// call copies the whole particle vector to the device and back.  This program keeps the
// state on the device: it uploads the generated galaxies once, advances with
// gx_session_step in runs of steps that end at the snapshot steps (CUDA-graph launches, no
// host copies in between), and downloads the state only to write a snapshot.  Everything
// else is the reference's own code, compiled from its sources: the command line (--config,
// --output), load_config / default_config, generate_galaxies, SnapshotWriter (metadata,
// snapshots, diagnostics.csv) and the snapshot schedule (every snapshot_every steps and at
// the last step).
//
// GX_PRECISION = f64 (default) | mixed | f64-exact selects the arithmetic form, as in the
// drop-in shim; with f64-exact the snapshots are bit-identical to the reference CLI running
// the shim.  GX_DIAGNOSTICS = device (default: FP64 reductions on the device) | host (the
// reference's compute_diagnostics on the downloaded particles, O(N^2) on the CPU).
#include "core/config.hpp"
#include "core/diagnostics.hpp"
#include "core/initial_conditions.hpp"
#include "io/snapshot_writer.hpp"

#include "gx_session.hpp"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <filesystem>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

bool uses_cuda_direct_solver(const std::string& solver) {
    return solver == "cuda" || solver == "cuda-direct" || solver == "gpu-direct";
}

int precision_from_env() {
    const char* p = std::getenv("GX_PRECISION");
    if (!p || !*p || std::strcmp(p, "f64") == 0) return GX_PRECISION_F64;
    if (std::strcmp(p, "mixed") == 0) return GX_PRECISION_MIXED;
    if (std::strcmp(p, "f64-exact") == 0) return GX_PRECISION_F64_EXACT;
    throw std::runtime_error(std::string("GX_PRECISION must be f64, mixed or f64-exact, got ") + p);
}

bool host_diagnostics() {
    const char* d = std::getenv("GX_DIAGNOSTICS");
    if (!d || !*d || std::strcmp(d, "device") == 0) return false;
    if (std::strcmp(d, "host") == 0) return true;
    throw std::runtime_error(std::string("GX_DIAGNOSTICS must be device or host, got ") + d);
}

fmmgalaxy::Diagnostics from_gx(const gx_diagnostics& g) {
    fmmgalaxy::Diagnostics d;
    d.kinetic_energy = g.kinetic_energy;
    d.potential_energy = g.potential_energy;
    d.total_energy = g.total_energy;
    d.total_mass = g.total_mass;
    d.momentum = {g.momentum[0], g.momentum[1], g.momentum[2]};
    d.center_of_mass = {g.center_of_mass[0], g.center_of_mass[1], g.center_of_mass[2]};
    d.angular_momentum = {g.angular_momentum[0], g.angular_momentum[1], g.angular_momentum[2]};
    return d;
}

void run_resident(const fmmgalaxy::SimulationConfig& config) {
    if (!uses_cuda_direct_solver(config.solver))
        throw std::runtime_error("solver '" + config.solver +
                                 "': this program runs the cuda-direct solvers; use the reference CLI for the others");
    const int precision = precision_from_env();
    const bool host_diag = host_diagnostics();
    std::cout << "Simulation: " << config.name << '\n';
    std::cout << "Solver:     " << config.solver << " (resident session)\n";

    std::vector<fmmgalaxy::Particle> particles =
        fmmgalaxy::generate_galaxies(config.galaxies, config.physics, config.seed);
    if (particles.empty()) throw std::runtime_error("No particles were generated. Check galaxy n_particles values.");

    fmmgalaxy::SnapshotWriter writer(config);
    writer.write_metadata(config, particles.size());

    gx::ResidentSession sim((int64_t)particles.size(), config.physics.gravitational_constant,
                            config.physics.softening);
    sim.upload(particles);
    sim.compute_accelerations(precision);

    auto write_outputs = [&](int step, double time) {
        sim.download(particles);  // the only device-to-host copy of the state
        const fmmgalaxy::Diagnostics diagnostics =
            host_diag ? fmmgalaxy::compute_diagnostics(particles, config.physics) : from_gx(sim.diagnostics());
        writer.write_snapshot(step, time, particles);
        writer.write_diagnostics(step, time, diagnostics, particles.size());
        std::cout << "step " << step << " time " << time << " total_energy " << diagnostics.total_energy << '\n';
    };

    write_outputs(0, 0.0);
    const int every = std::max(1, config.snapshot_every);
    int step = 0;
    while (step < config.steps) {
        const int next = std::min(config.steps, (step / every + 1) * every);
        sim.step(next - step, config.dt, precision);
        step = next;
        write_outputs(step, static_cast<double>(step) * config.dt);
    }
    std::cout << "Wrote snapshots to " << config.output.directory.string() << '\n';
}

}  // namespace

int main(int argc, char** argv) {
    try {
        std::filesystem::path config_path, output;
        bool has_config = false, has_output = false;
        for (int i = 1; i < argc; ++i) {
            const std::string arg = argv[i];
            if (arg == "--help" || arg == "-h") {
                std::cout << "Usage: " << argv[0] << " [--config path] [--output directory]\n";
                return 0;
            } else if (arg == "--config" && i + 1 < argc) {
                config_path = argv[++i];
                has_config = true;
            } else if (arg == "--output" && i + 1 < argc) {
                output = argv[++i];
                has_output = true;
            } else {
                throw std::runtime_error("Unknown or incomplete argument: " + arg);
            }
        }
        fmmgalaxy::SimulationConfig config =
            has_config ? fmmgalaxy::load_config(config_path) : fmmgalaxy::default_config();
        if (has_output) config.output.directory = output;
        run_resident(config);
    } catch (const std::exception& error) {
        std::cerr << "error: " << error.what() << '\n';
        return 1;
    }
    return 0;
}
