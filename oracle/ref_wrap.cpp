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
#include <chrono>
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
#include "io/snapshot_writer.hpp"
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

// Node data of the reference tree after FastMultipoleSolver::build: every node with
// mass > 0, breadth-first from the root with children in octant order, 35 doubles each
// (centre of mass, mass, moments.values[4..34]); stats = FmmStats (fmm_solver.hpp:22-27).
int ref_fmm_moments(int64_t n, const double* x, const double* y, const double* z, const double* m, double G,
                    double eps, double theta, int64_t leaf_capacity, int order, int64_t capacity, double* records,
                    int64_t* n_nodes, int64_t* stats) {
    auto p = to_particles(n, x, y, z, m);
    fmmgalaxy::FmmOptions o;
    o.theta = theta;
    o.leaf_capacity = static_cast<std::size_t>(leaf_capacity);
    o.expansion_order = order;
    fmmgalaxy::FastMultipoleSolver solver(physics(G, eps), o);
    solver.build(p);
    const auto& nodes = solver.nodes_;
    std::vector<int> bfs;
    if (!nodes.empty() && nodes[0].mass > 0.0) bfs.push_back(0);
    for (std::size_t k = 0; k < bfs.size(); ++k)
        for (int c : nodes[bfs[k]].children)
            if (c >= 0 && nodes[c].mass > 0.0) bfs.push_back(c);
    *n_nodes = static_cast<int64_t>(bfs.size());
    const auto& s = solver.stats();
    stats[0] = static_cast<int64_t>(s.node_count);
    stats[1] = static_cast<int64_t>(s.leaf_count);
    stats[2] = static_cast<int64_t>(s.far_interactions);
    stats[3] = static_cast<int64_t>(s.near_interactions);
    if (!records || capacity < static_cast<int64_t>(bfs.size())) return 0;
    for (std::size_t k = 0; k < bfs.size(); ++k) {
        const auto& nd = nodes[bfs[k]];
        double* r = records + k * 35;
        r[0] = nd.center_of_mass.x; r[1] = nd.center_of_mass.y; r[2] = nd.center_of_mass.z;
        r[3] = nd.mass;
        for (int j = 4; j < 35; ++j) r[j] = nd.moments.values[j];
    }
    return 0;
}

// Times the reference FMM on the host: FastMultipoleSolver::build once, then
// evaluate_particle (fmm_solver.cpp:279-310, a const method) for every stride-th body in
// leaf order, those bodies split over `threads` host threads.  The evaluated
// accelerations are written to (ax, ay, az) (others are left untouched) so a caller can
// check them.
void ref_fmm_timed(int64_t n, const double* x, const double* y, const double* z, const double* m, double G,
                   double eps, double theta, int64_t leaf_capacity, int order, int64_t stride, int threads,
                   double* ax, double* ay, double* az, double* build_s, double* eval_s, int64_t* n_eval) {
    auto p = to_particles(n, x, y, z, m);
    fmmgalaxy::FmmOptions o;
    o.theta = theta;
    o.leaf_capacity = static_cast<std::size_t>(leaf_capacity);
    o.expansion_order = order;
    fmmgalaxy::FastMultipoleSolver solver(physics(G, eps), o);
    const auto t0 = std::chrono::steady_clock::now();
    solver.build(p);
    const auto t1 = std::chrono::steady_clock::now();
    std::vector<std::pair<std::size_t, int>> work;  // (body, leaf node)
    int64_t k = 0;
    for (int li : solver.leaf_indices_)
        for (std::size_t q : solver.nodes_[li].particle_indices)
            if (k++ % stride == 0) work.emplace_back(q, li);
    if (threads < 1) threads = 1;
    std::vector<std::thread> pool;
    const auto t2 = std::chrono::steady_clock::now();
    for (int r = 0; r < threads; ++r) {
        const auto own = fmmgalaxy::ownership_for_rank(work.size(), r, threads);
        pool.emplace_back([&, own] {
            for (std::size_t w = own.begin; w < own.end; ++w) {
                const auto a = solver.evaluate_particle(work[w].first, solver.nodes_[work[w].second]);
                ax[work[w].first] = a.x;
                ay[work[w].first] = a.y;
                az[work[w].first] = a.z;
            }
        });
    }
    for (auto& t : pool) t.join();
    const auto t3 = std::chrono::steady_clock::now();
    *build_s = std::chrono::duration<double>(t1 - t0).count();
    *eval_s = std::chrono::duration<double>(t3 - t2).count();
    *n_eval = static_cast<int64_t>(work.size());
}

// SnapshotWriter (snapshot_writer.cpp:38-128) on one state: diagnostics.csv header, one
// snapshot file and one diagnostics row (diag: 13 doubles in the row's column order).
int ref_write_outputs(const char* directory, int64_t n, const double* x, const double* y, const double* z,
                      const double* vx, const double* vy, const double* vz, const double* ax, const double* ay,
                      const double* az, const double* m, const uint32_t* group, int step, double time,
                      const double* diag) {
    auto p = to_particles(n, x, y, z, m, vx, vy, vz, ax, ay, az);
    for (int64_t i = 0; i < n; ++i) p[i].group_id = group ? group[i] : 0u;
    fmmgalaxy::SimulationConfig cfg;
    cfg.output.directory = directory;
    cfg.output.format = "csv";
    fmmgalaxy::SnapshotWriter w(cfg);
    w.write_snapshot(step, time, p);
    fmmgalaxy::Diagnostics d;
    d.total_mass = diag[0];
    d.kinetic_energy = diag[1];
    d.potential_energy = diag[2];
    d.total_energy = diag[3];
    d.momentum = {diag[4], diag[5], diag[6]};
    d.center_of_mass = {diag[7], diag[8], diag[9]};
    d.angular_momentum = {diag[10], diag[11], diag[12]};
    w.write_diagnostics(step, time, d, static_cast<std::size_t>(n));
    return 0;
}

// SnapshotWriter::write_metadata (snapshot_writer.cpp:49-69) of a SimulationConfig holding
// these values.
int ref_write_metadata(const char* directory, const char* name, const char* solver, int64_t particle_count,
                       int steps, double dt, int snapshot_every, int dim, double G, double eps, double theta,
                       int64_t leaf_capacity, int order) {
    fmmgalaxy::SimulationConfig cfg;
    cfg.output.directory = directory;
    cfg.output.format = "csv";
    cfg.name = name;
    cfg.solver = solver;
    cfg.steps = steps;
    cfg.dt = dt;
    cfg.snapshot_every = snapshot_every;
    cfg.dim = dim;
    cfg.physics.gravitational_constant = G;
    cfg.physics.softening = eps;
    cfg.tree_theta = theta;
    cfg.tree_leaf_capacity = static_cast<std::size_t>(leaf_capacity);
    cfg.fmm_expansion_order = order;
    fmmgalaxy::SnapshotWriter w(cfg);
    w.write_metadata(cfg, static_cast<std::size_t>(particle_count));
    return 0;
}

// generate_galaxies (initial_conditions.cpp:92-114).  Galaxy g is cfg[13 g .. 13 g + 12] =
// n, mass, radius, position xyz, velocity xyz, orientation, group id, thickness, inclination.
int64_t ref_generate_galaxies(int n_gal, const double* cfg, double G, double eps, uint64_t seed, double* x, double* y,
                              double* z, double* vx, double* vy, double* vz, double* m, uint32_t* group) {
    std::vector<fmmgalaxy::GalaxyConfig> gs((size_t)n_gal);
    for (int g = 0; g < n_gal; ++g) {
        const double* c = cfg + 13 * g;
        gs[g].n_particles = (std::size_t)c[0];
        gs[g].mass = c[1];
        gs[g].radius = c[2];
        gs[g].position = {c[3], c[4], c[5]};
        gs[g].velocity = {c[6], c[7], c[8]};
        gs[g].orientation = c[9];
        gs[g].group_id = (std::uint32_t)c[10];
        gs[g].thickness = c[11];
        gs[g].inclination = c[12];
    }
    const auto p = fmmgalaxy::generate_galaxies(gs, physics(G, eps), seed);
    if (x)
        for (size_t i = 0; i < p.size(); ++i) {
            x[i] = p[i].position.x; y[i] = p[i].position.y; z[i] = p[i].position.z;
            vx[i] = p[i].velocity.x; vy[i] = p[i].velocity.y; vz[i] = p[i].velocity.z;
            m[i] = p[i].mass;
            group[i] = p[i].group_id;
        }
    return (int64_t)p.size();
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
