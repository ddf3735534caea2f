// cuda_solver_b200.cpp -- drop-in replacement for the reference's cpp/cuda/cuda_solver.cu.
//
// Compiled inside the reference tree in place of cuda_solver.cu (and instead of
// cuda_solver_stub.cpp), it implements the three functions of cpp/cuda/cuda_solver.hpp:10-12
// on top of the C ABI (include/gx.h), so cpp/core/main.cpp, its solver dispatch
// (main.cpp:62-139) and the `solver = "cuda-direct"` config key stay unchanged.
//
// Behaviour kept from the reference: the caller owns the particle vector, accelerations
// (and for the step, positions and velocities) are overwritten in place, the step reuses
// the stored accelerations for its first kick, empty input is a no-op and errors throw
// std::runtime_error.  Changed on purpose: there is no CPU fallback -- without a usable
// device both compute functions throw.  GX_PRECISION=f64 (default), mixed or f64-exact
// selects the arithmetic form (f64-exact is bit-identical to
// compute_direct_accelerations_for_targets).
#include "cuda/cuda_solver.hpp"
#include "gx.h"

#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace fmmgalaxy {
namespace {

void throw_on_gx(int status, const char* what) {
    if (status != GX_OK) throw std::runtime_error(std::string(what) + ": " + gx_last_error());
}

int precision_from_env() {
    const char* p = std::getenv("GX_PRECISION");
    if (!p || !*p || std::strcmp(p, "f64") == 0) return GX_PRECISION_F64;
    if (std::strcmp(p, "mixed") == 0) return GX_PRECISION_MIXED;
    if (std::strcmp(p, "f64-exact") == 0) return GX_PRECISION_F64_EXACT;
    throw std::runtime_error(std::string("GX_PRECISION must be f64, mixed or f64-exact, got ") + p);
}

gx_physics to_gx(const PhysicsParams& p) { return gx_physics{p.gravitational_constant, p.softening}; }

// Structure-of-arrays copy of the AoS particle vector.
struct Soa {
    std::vector<double> x, y, z, vx, vy, vz, ax, ay, az, m;
    explicit Soa(const std::vector<Particle>& p) {
        const std::size_t n = p.size();
        for (auto* v : {&x, &y, &z, &vx, &vy, &vz, &ax, &ay, &az, &m}) v->resize(n);
        for (std::size_t i = 0; i < n; ++i) {
            x[i] = p[i].position.x; y[i] = p[i].position.y; z[i] = p[i].position.z;
            vx[i] = p[i].velocity.x; vy[i] = p[i].velocity.y; vz[i] = p[i].velocity.z;
            ax[i] = p[i].acceleration.x; ay[i] = p[i].acceleration.y; az[i] = p[i].acceleration.z;
            m[i] = p[i].mass;
        }
    }
};

}  // namespace

bool cuda_solver_available() {
    int available = 0;
    return gx_device_available(&available) == GX_OK && available != 0;
}

void compute_cuda_direct_accelerations(std::vector<Particle>& particles, const PhysicsParams& params) {
    if (particles.empty()) return;
    Soa s(particles);
    throw_on_gx(gx_direct_accel((int64_t)particles.size(), s.x.data(), s.y.data(), s.z.data(), s.m.data(),
                                to_gx(params), precision_from_env(), s.ax.data(), s.ay.data(), s.az.data(),
                                nullptr),
                "gx_direct_accel");
    for (std::size_t i = 0; i < particles.size(); ++i) particles[i].acceleration = {s.ax[i], s.ay[i], s.az[i]};
}

void cuda_direct_leapfrog_step(std::vector<Particle>& particles, double dt, const PhysicsParams& params) {
    if (particles.empty()) return;
    Soa s(particles);
    throw_on_gx(gx_leapfrog_step((int64_t)particles.size(), s.x.data(), s.y.data(), s.z.data(), s.vx.data(),
                                 s.vy.data(), s.vz.data(), s.ax.data(), s.ay.data(), s.az.data(), s.m.data(), dt,
                                 to_gx(params), precision_from_env(), nullptr),
                "gx_leapfrog_step");
    for (std::size_t i = 0; i < particles.size(); ++i) {
        particles[i].position = {s.x[i], s.y[i], s.z[i]};
        particles[i].velocity = {s.vx[i], s.vy[i], s.vz[i]};
        particles[i].acceleration = {s.ax[i], s.ay[i], s.az[i]};
    }
}

}  // namespace fmmgalaxy
