// gx_session.hpp -- header-only C++ wrapper of the resident session of gx.h for the
// reference's step loop (cpp/core/main.cpp:172-184): upload once, step on the device with
// no per-step host copies, download only at snapshot steps.
//
// ParticleVec is any std::vector of records with Vec3-like `position`, `velocity`,
// `acceleration` members (fields x, y, z) and a double `mass` -- the reference's Particle
// (cpp/core/particle.hpp:8-14).  Errors throw std::runtime_error, as in the reference.
#pragma once

#include "gx.h"

#include <stdexcept>
#include <string>
#include <vector>

namespace gx {

inline void check(int status, const char* what) {
    if (status != GX_OK) throw std::runtime_error(std::string(what) + ": " + gx_last_error());
}

class ResidentSession {
public:
    ResidentSession(int64_t n, double G, double softening, int device = 0) : n_(n) {
        check(gx_session_create(n, gx_physics{G, softening}, device, &s_), "gx_session_create");
    }
    ~ResidentSession() { gx_session_destroy(s_); }
    ResidentSession(const ResidentSession&) = delete;
    ResidentSession& operator=(const ResidentSession&) = delete;

    template <class ParticleVec>
    void upload(const ParticleVec& p) {
        std::vector<double> a[10];
        for (auto& v : a) v.resize(p.size());
        for (std::size_t i = 0; i < p.size(); ++i) {
            a[0][i] = p[i].position.x; a[1][i] = p[i].position.y; a[2][i] = p[i].position.z;
            a[3][i] = p[i].velocity.x; a[4][i] = p[i].velocity.y; a[5][i] = p[i].velocity.z;
            a[6][i] = p[i].acceleration.x; a[7][i] = p[i].acceleration.y; a[8][i] = p[i].acceleration.z;
            a[9][i] = p[i].mass;
        }
        check(gx_session_set_state(s_, a[0].data(), a[1].data(), a[2].data(), a[3].data(), a[4].data(),
                                   a[5].data(), a[9].data(), a[6].data(), a[7].data(), a[8].data()),
              "gx_session_set_state");
    }

    template <class ParticleVec>
    void download(ParticleVec& p) {
        std::vector<double> a[9];
        for (auto& v : a) v.resize(p.size());
        check(gx_session_get_state(s_, a[0].data(), a[1].data(), a[2].data(), a[3].data(), a[4].data(),
                                   a[5].data(), a[6].data(), a[7].data(), a[8].data()),
              "gx_session_get_state");
        for (std::size_t i = 0; i < p.size(); ++i) {
            p[i].position = {a[0][i], a[1][i], a[2][i]};
            p[i].velocity = {a[3][i], a[4][i], a[5][i]};
            p[i].acceleration = {a[6][i], a[7][i], a[8][i]};
        }
    }

    void compute_accelerations(int precision = GX_PRECISION_F64) {
        check(gx_session_compute_accelerations(s_, precision), "gx_session_compute_accelerations");
    }
    void step(int64_t n_steps, double dt, int precision = GX_PRECISION_F64) {
        check(gx_session_step(s_, n_steps, dt, precision), "gx_session_step");
    }
    gx_diagnostics diagnostics() {
        gx_diagnostics d;
        check(gx_session_diagnostics(s_, &d), "gx_session_diagnostics");
        return d;
    }
    gx_session* handle() { return s_; }

private:
    int64_t n_;
    gx_session* s_ = nullptr;
};

}  // namespace gx
