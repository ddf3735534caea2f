// ref_wrap.cpp -- TEST INFRASTRUCTURE ONLY.
//
// extern "C" entry points over the reference's own, unmodified C++ sources (compiled
// where they lie by oracle/Makefile into oracle/_ref/libgxref.so).  Tests and the
// bench's reference arm call the real reference through these; the product never
// loads this library.
//
// The FMM tree of FastMultipoleSolver is private; to read its leaf lists and far-field
// moments (to split the reference FMM into "far field on the CPU" and "near field on the
// GPU" exactly as the drop-in does) this translation unit alone re-opens the class with
// `#define private public` before including the reference header.  Nothing in the
// reference is changed or copied.
#include <cstdint>
#include <cstring>
#include <random>
#include <thread>
#include <vector>

#define private public
#include "fmm/fmm_solver.hpp"
#undef private

#include "core/diagnostics.hpp"
#include "core/initial_conditions.hpp"
#include "core/integrator.hpp"
#include "direct/direct_solver.hpp"
#include "fmm/multipole.hpp"
#include "mpi/distributed_solver.hpp"

using fmmgalaxy::Particle;
using fmmgalaxy::PhysicsParams;

namespace {

std::vector<Particle> to_particles(int64_t n, const double* x, const double* y, const double* z,
                                   const double* m, const double* vx = nullptr,
                                   const double* vy = nullptr, const double* vz = nullptr,
                                   const double* ax = nullptr, const double* ay = nullptr,
                                   const double* az = nullptr) {
    std::vector<Particle> p(static_cast<std::size_t>(n));
    for (int64_t i = 0; i < n; ++i) {
        p[i].position = {x[i], y[i], z[i]};
        p[i].mass = m[i];
        if (vx) p[i].velocity = {vx[i], vy[i], vz[i]};
        if (ax) p[i].acceleration = {ax[i], ay[i], az[i]};
    }
    return p;
}

PhysicsParams physics(double G, double eps) {
    PhysicsParams p;
    p.gravitational_constant = G;
    p.softening = eps;
    return p;
}

}  // namespace

extern "C" {

// compute_direct_accelerations (direct_solver.cpp:38-57), the CLI's "direct" solver.
void ref_direct(int64_t n, const double* x, const double* y, const double* z, const double* m,
                double G, double eps, double* ax, double* ay, double* az) {
    auto p = to_particles(n, x, y, z, m);
    fmmgalaxy::compute_direct_accelerations(p, physics(G, eps));
    for (int64_t i = 0; i < n; ++i) {
        ax[i] = p[i].acceleration.x; ay[i] = p[i].acceleration.y; az[i] = p[i].acceleration.z;
    }
}

// compute_direct_accelerations_for_targets (direct_solver.cpp:59-83) over [begin,end),
// split across `threads` host threads by ownership_for_rank ranges (distributed_solver.cpp:68-79).
void ref_direct_targets_mt(int64_t n, const double* x, const double* y, const double* z,
                           const double* m, double G, double eps, int64_t begin, int64_t end,
                           double* ax, double* ay, double* az, int threads) {
    auto p = to_particles(n, x, y, z, m);
    const PhysicsParams ph = physics(G, eps);
    if (threads < 1) threads = 1;
    const std::size_t count = static_cast<std::size_t>(end - begin);
    std::vector<std::thread> pool;
    for (int r = 0; r < threads; ++r) {
        const auto own = fmmgalaxy::ownership_for_rank(count, r, threads);
        pool.emplace_back([&, own] {
            fmmgalaxy::compute_direct_accelerations_for_targets(p, ph, begin + own.begin, begin + own.end);
        });
    }
    for (auto& t : pool) t.join();
    for (int64_t i = begin; i < end; ++i) {
        ax[i - begin] = p[i].acceleration.x; ay[i - begin] = p[i].acceleration.y;
        az[i - begin] = p[i].acceleration.z;
    }
}

// `steps` reference leapfrog_step calls (integrator.cpp:33-42) with the symmetric direct force.
void ref_leapfrog_direct(int64_t n, double* x, double* y, double* z, double* vx, double* vy,
                         double* vz, double* ax, double* ay, double* az, const double* m, double G,
                         double eps, double dt, int steps) {
    auto p = to_particles(n, x, y, z, m, vx, vy, vz, ax, ay, az);
    const PhysicsParams ph = physics(G, eps);
    auto force = [&ph](std::vector<Particle>& s) { fmmgalaxy::compute_direct_accelerations(s, ph); };
    for (int s = 0; s < steps; ++s) fmmgalaxy::leapfrog_step(p, dt, force);
    for (int64_t i = 0; i < n; ++i) {
        x[i] = p[i].position.x; y[i] = p[i].position.y; z[i] = p[i].position.z;
        vx[i] = p[i].velocity.x; vy[i] = p[i].velocity.y; vz[i] = p[i].velocity.z;
        ax[i] = p[i].acceleration.x; ay[i] = p[i].acceleration.y; az[i] = p[i].acceleration.z;
    }
}

// `steps` reference leapfrog_step calls with the FMM force (compute_fmm_accelerations,
// fmm_solver.cpp:315-322), the CLI's "fmm" solver.
void ref_leapfrog_fmm(int64_t n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                      double* ax, double* ay, double* az, const double* m, double G, double eps, double dt,
                      int steps, double theta, int64_t leaf_capacity, int order) {
    auto p = to_particles(n, x, y, z, m, vx, vy, vz, ax, ay, az);
    const PhysicsParams ph = physics(G, eps);
    fmmgalaxy::FmmOptions o;
    o.theta = theta;
    o.leaf_capacity = static_cast<std::size_t>(leaf_capacity);
    o.expansion_order = order;
    auto force = [&ph, &o](std::vector<Particle>& s) { fmmgalaxy::compute_fmm_accelerations(s, ph, o); };
    for (int s = 0; s < steps; ++s) fmmgalaxy::leapfrog_step(p, dt, force);
    for (int64_t i = 0; i < n; ++i) {
        x[i] = p[i].position.x; y[i] = p[i].position.y; z[i] = p[i].position.z;
        vx[i] = p[i].velocity.x; vy[i] = p[i].velocity.y; vz[i] = p[i].velocity.z;
        ax[i] = p[i].acceleration.x; ay[i] = p[i].acceleration.y; az[i] = p[i].acceleration.z;
    }
}

// compute_diagnostics (diagnostics.cpp:7-37) -> 13 doubles in diagnostics.csv column order.
void ref_diagnostics(int64_t n, const double* x, const double* y, const double* z,
                     const double* vx, const double* vy, const double* vz, const double* m,
                     double G, double eps, double* out) {
    auto p = to_particles(n, x, y, z, m, vx, vy, vz);
    const auto d = fmmgalaxy::compute_diagnostics(p, physics(G, eps));
    const double v[13] = {d.total_mass, d.kinetic_energy, d.potential_energy, d.total_energy,
                          d.momentum.x, d.momentum.y, d.momentum.z,
                          d.center_of_mass.x, d.center_of_mass.y, d.center_of_mass.z,
                          d.angular_momentum.x, d.angular_momentum.y, d.angular_momentum.z};
    std::memcpy(out, v, sizeof(v));
}

// compute_fmm_accelerations (fmm_solver.cpp:315-322).
void ref_fmm(int64_t n, const double* x, const double* y, const double* z, const double* m,
             double G, double eps, double theta, int64_t leaf_capacity, int order, double* ax,
             double* ay, double* az) {
    auto p = to_particles(n, x, y, z, m);
    fmmgalaxy::FmmOptions o;
    o.theta = theta;
    o.leaf_capacity = static_cast<std::size_t>(leaf_capacity);
    o.expansion_order = order;
    fmmgalaxy::compute_fmm_accelerations(p, physics(G, eps), o);
    for (int64_t i = 0; i < n; ++i) {
        ax[i] = p[i].acceleration.x; ay[i] = p[i].acceleration.y; az[i] = p[i].acceleration.z;
    }
}

// Splits one reference FMM evaluation into its parts: the leaf lists as CSR (leaf order of
// collect_leaves, near lists in build_leaf_interactions order, near entries given as leaf
// ordinals) and the far-field-only acceleration of every body, summed over far_nodes in the
// order of evaluate_particle (fmm_solver.cpp:283-293).  Sizes first: call with null arrays
// to get n_leaves / n_near, then again with buffers.
int ref_fmm_split(int64_t n, const double* x, const double* y, const double* z, const double* m,
                  double G, double eps, double theta, int64_t leaf_capacity, int order,
                  int32_t* n_leaves, int64_t* n_near, int32_t* leaf_offsets, int32_t* leaf_particles,
                  int32_t* near_offsets, int32_t* near_leaves, double* far_ax, double* far_ay,
                  double* far_az) {
    auto p = to_particles(n, x, y, z, m);
    fmmgalaxy::FmmOptions o;
    o.theta = theta;
    o.leaf_capacity = static_cast<std::size_t>(leaf_capacity);
    o.expansion_order = order;
    fmmgalaxy::FastMultipoleSolver solver(physics(G, eps), o);
    solver.build(p);
    const auto& nodes = solver.nodes_;
    const auto& leaves = solver.leaf_indices_;
    std::vector<int> ordinal(nodes.size(), -1);
    for (std::size_t l = 0; l < leaves.size(); ++l) ordinal[leaves[l]] = static_cast<int>(l);
    int64_t nn = 0;
    for (int li : leaves) nn += static_cast<int64_t>(nodes[li].near_leaves.size());
    *n_leaves = static_cast<int32_t>(leaves.size());
    *n_near = nn;
    if (!leaf_offsets) return 0;
    int32_t run = 0, nrun = 0;
    for (std::size_t l = 0; l < leaves.size(); ++l) {
        const auto& L = nodes[leaves[l]];
        leaf_offsets[l] = run;
        near_offsets[l] = nrun;
        for (std::size_t q : L.particle_indices) leaf_particles[run++] = static_cast<int32_t>(q);
        for (int s : L.near_leaves) near_leaves[nrun++] = ordinal[s];
    }
    leaf_offsets[leaves.size()] = run;
    near_offsets[leaves.size()] = nrun;
    const PhysicsParams ph = physics(G, eps);
    for (int64_t i = 0; i < n; ++i) { far_ax[i] = 0.0; far_ay[i] = 0.0; far_az[i] = 0.0; }
    for (int li : leaves) {
        const auto& L = nodes[li];
        for (std::size_t q : L.particle_indices) {
            fmmgalaxy::Vec3 acc{};
            for (int s : L.far_nodes) {
                const auto& S = nodes[s];
                acc += fmmgalaxy::multipole_acceleration(p[q].position, S.center_of_mass, S.mass,
                                                         S.moments, ph, solver.options_.expansion_order);
            }
            far_ax[q] = acc.x; far_ay[q] = acc.y; far_az[q] = acc.z;
        }
    }
    return 0;
}

// The inputs of the reference smoke test's solver-agreement case (smoke_tests.cpp:83-89):
// 80 bodies at U(-1,1)^3 drawn from mt19937_64(7), mass 1/80.
void ref_smoke80_inputs(double* x, double* y, double* z, double* m) {
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> uniform(-1.0, 1.0);
    for (int i = 0; i < 80; ++i) {
        x[i] = uniform(rng); y[i] = uniform(rng); z[i] = uniform(rng);
        m[i] = 1.0 / 80.0;
    }
}

}  // extern "C"
