// ics.cu -- disk-galaxy initial conditions generated on the device.
//
// The model is the reference's generate_disk_galaxy / generate_galaxies
// (cpp/core/initial_conditions.cpp:37-114): radius from the exponential disk of scale
// radius/3 truncated at radius (inverse CDF, u clamped to [1e-12, 1 - 1e-12], :28-33), angle
// uniform, height thickness * N(0,1), tangential circular speed from the uniform-disk
// enclosed mass max(M min(1, r^2/R^2), m) with the softened kernel (:66-72), a velocity
// dispersion of 0.025 sqrt(G M / R) (1/4 of it vertically, :54, 75-79), then rotation about x
// by the inclination and about z by the orientation, and the galaxy's position / velocity
// (:17-26, 81-86).
//
// The random numbers differ: the reference draws everything from one sequential mt19937_64
// (its normal_distribution rejects samples, so the draws per body vary).  Here each body
// draws from Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), a counter-based generator
// keyed by the seed, with the counter (galaxy, body, block): bodies are independent and a
// galaxy's bodies do not depend on the other galaxies.  Normals by Box-Muller.
#include "gx.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

extern "C" int gxi_fail(int code, const char* msg);

namespace {

struct Philox {
    uint32_t c0, c1, c2, c3;
};

__host__ __device__ inline void philox_round(uint32_t& c0, uint32_t& c1, uint32_t& c2, uint32_t& c3, uint32_t k0,
                                             uint32_t k1) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
}

// Philox4x32-10 of counter (c0..c3) under key (k0, k1).
__host__ __device__ inline Philox philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                                uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        philox_round(c0, c1, c2, c3, k0, k1);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return {c0, c1, c2, c3};
}

// Uniform double in [0, 1) from 53 bits of two 32-bit words.
__host__ __device__ inline double u53(uint32_t hi, uint32_t lo) {
    return (double)((((uint64_t)hi << 32) | lo) >> 11) * (1.0 / 9007199254740992.0);
}

struct Galaxy {
    int64_t first;  // index of the galaxy's first body in the output
    int64_t n;
    double mass, radius, thickness, orientation, inclination;
    double px, py, pz, vx, vy, vz;
    uint32_t group;
    uint32_t index;  // position among all configured galaxies (the counter's galaxy word)
};

struct IcArgs {
    const Galaxy* gal;
    int n_gal;
    int64_t total;
    double G, eps;
    uint32_t k0, k1;
    double *x, *y, *z, *vx, *vy, *vz, *m;
    uint32_t* group;
};

__global__ void __launch_bounds__(256) disk_kernel(const IcArgs a) {
    const int64_t k = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (k >= a.total) return;
    int lo = 0, hi = a.n_gal;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (a.gal[mid].first <= k) lo = mid;
        else hi = mid;
    }
    const Galaxy g = a.gal[lo];
    const int64_t i = k - g.first;
    const uint32_t ci = (uint32_t)i, cg = g.index, ch = (uint32_t)((uint64_t)i >> 32);
    const Philox r0 = philox4x32_10(ci, ch, cg, 0u, a.k0, a.k1);
    const Philox r1 = philox4x32_10(ci, ch, cg, 1u, a.k0, a.k1);
    const Philox r2 = philox4x32_10(ci, ch, cg, 2u, a.k0, a.k1);
    const double u_r = u53(r0.c0, r0.c1), u_t = u53(r0.c2, r0.c3);
    // Box-Muller: two normals from each pair (1 - u avoids log(0))
    const double b1 = sqrt(-2.0 * log(1.0 - u53(r1.c0, r1.c1))), a1 = 2.0 * M_PI * u53(r1.c2, r1.c3);
    const double b2 = sqrt(-2.0 * log(1.0 - u53(r2.c0, r2.c1))), a2 = 2.0 * M_PI * u53(r2.c2, r2.c3);
    const double nz = b1 * cos(a1), nvx = b1 * sin(a1), nvy = b2 * cos(a2), nvz = b2 * sin(a2);

    const double pm = g.mass / (double)g.n;
    const double vscale = sqrt(a.G * g.mass / g.radius);
    const double disp = 0.025 * vscale;
    const double scale = g.radius / 3.0;
    const double max_cdf = 1.0 - exp(-g.radius / scale);
    const double u = fmin(fmax(u_r, 1.0e-12), 1.0 - 1.0e-12);
    const double r = -scale * log(1.0 - u * max_cdf);
    const double th = 2.0 * M_PI * u_t;
    const double ct = cos(th), st = sin(th);
    const double lx = r * ct, ly = r * st, lz = g.thickness > 0.0 ? g.thickness * nz : 0.0;
    const double frac = fmin(1.0, (r * r) / (g.radius * g.radius));
    const double menc = fmax(g.mass * frac, pm);
    const double sr2 = r * r + a.eps * a.eps;
    const double vc = sqrt(a.G * menc * r * r / pow(sr2, 1.5));
    const double lvx = -st * vc + disp * nvx, lvy = ct * vc + disp * nvy, lvz = 0.25 * disp * nvz;
    // rotate_x(inclination) then rotate_z(orientation)
    const double ci_ = cos(g.inclination), si_ = sin(g.inclination), co = cos(g.orientation), so = sin(g.orientation);
    auto orient = [&](double ux, double uy, double uz, double& ox, double& oy, double& oz) {
        const double y1 = ci_ * uy - si_ * uz, z1 = si_ * uy + ci_ * uz;
        ox = co * ux - so * y1;
        oy = so * ux + co * y1;
        oz = z1;
    };
    double ox, oy, oz;
    orient(lx, ly, lz, ox, oy, oz);
    a.x[k] = g.px + ox;
    a.y[k] = g.py + oy;
    a.z[k] = g.pz + oz;
    orient(lvx, lvy, lvz, ox, oy, oz);
    a.vx[k] = g.vx + ox;
    a.vy[k] = g.vy + oy;
    a.vz[k] = g.vz + oz;
    a.m[k] = pm;
    if (a.group) a.group[k] = g.group;
}

bool device_ptr(const void* p) {
    cudaPointerAttributes at;
    if (!p || cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" int64_t gx_galaxies_body_count(int32_t n_galaxies, const gx_galaxy* galaxies) {
    int64_t t = 0;
    for (int32_t g = 0; g < n_galaxies && galaxies; ++g)
        if (galaxies[g].n_particles > 0 && galaxies[g].mass > 0.0 && galaxies[g].radius > 0.0)
            t += galaxies[g].n_particles;
    return t;
}

extern "C" int gx_generate_galaxies(int32_t n_galaxies, const gx_galaxy* galaxies, gx_physics phys, uint64_t seed,
                                    double* x, double* y, double* z, double* vx, double* vy, double* vz, double* m,
                                    uint32_t* group_id, void* stream) {
    if (n_galaxies < 0 || (n_galaxies > 0 && !galaxies))
        return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_generate_galaxies: bad galaxy list");
    std::vector<Galaxy> gal;
    int64_t total = 0;
    for (int32_t g = 0; g < n_galaxies; ++g) {
        const gx_galaxy& c = galaxies[g];
        // generate_disk_galaxy returns no bodies for these (initial_conditions.cpp:46-48)
        if (c.n_particles <= 0 || !(c.mass > 0.0) || !(c.radius > 0.0)) continue;
        Galaxy q;
        q.first = total;
        q.n = c.n_particles;
        q.mass = c.mass;
        q.radius = c.radius;
        q.thickness = c.thickness;
        q.orientation = c.orientation;
        q.inclination = c.inclination;
        q.px = c.position[0];
        q.py = c.position[1];
        q.pz = c.position[2];
        q.vx = c.velocity[0];
        q.vy = c.velocity[1];
        q.vz = c.velocity[2];
        q.group = c.group_id;
        q.index = (uint32_t)g;
        gal.push_back(q);
        total += c.n_particles;
    }
    if (total == 0) return GX_OK;
    if (!x || !y || !z || !vx || !vy || !vz || !m) return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_generate_galaxies: null array");
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0) {
        cudaGetLastError();
        return gxi_fail(GX_ERR_NO_DEVICE, "gx_generate_galaxies: no CUDA device");
    }
    const bool dev = device_ptr(x);
    const double* outs[7] = {x, y, z, vx, vy, vz, m};
    for (const double* p : outs)
        if (device_ptr(p) != dev) return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_generate_galaxies: mix of host and device arrays");
    if (group_id && device_ptr(group_id) != dev)
        return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_generate_galaxies: mix of host and device arrays");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t bytes = (size_t)total * sizeof(double);
    std::vector<void*> owned;
    auto cleanup = [&] {
        for (void* p : owned) cudaFreeAsync(p, st);
        cudaGetLastError();
    };
    auto cuda_fail = [&](cudaError_t e) {
        cleanup();
        return gxi_fail(GX_ERR_CUDA, (std::string("gx_generate_galaxies: ") + cudaGetErrorString(e)).c_str());
    };
    IcArgs a;
    a.n_gal = (int)gal.size();
    a.total = total;
    a.G = phys.G;
    a.eps = phys.softening;
    a.k0 = (uint32_t)seed;
    a.k1 = (uint32_t)(seed >> 32);
    double* d[7];
    cudaError_t e;
    void* g_dev = nullptr;
    if ((e = cudaMallocAsync(&g_dev, gal.size() * sizeof(Galaxy), st)) != cudaSuccess) return cuda_fail(e);
    owned.push_back(g_dev);
    if ((e = cudaMemcpyAsync(g_dev, gal.data(), gal.size() * sizeof(Galaxy), cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return cuda_fail(e);
    a.gal = (const Galaxy*)g_dev;
    for (int k = 0; k < 7; ++k) {
        if (dev) {
            d[k] = const_cast<double*>(outs[k]);
        } else {
            if ((e = cudaMallocAsync((void**)&d[k], bytes, st)) != cudaSuccess) return cuda_fail(e);
            owned.push_back(d[k]);
        }
    }
    uint32_t* dg = group_id;
    if (group_id && !dev) {
        if ((e = cudaMallocAsync((void**)&dg, (size_t)total * 4, st)) != cudaSuccess) return cuda_fail(e);
        owned.push_back(dg);
    }
    a.x = d[0]; a.y = d[1]; a.z = d[2]; a.vx = d[3]; a.vy = d[4]; a.vz = d[5]; a.m = d[6];
    a.group = dg;
    disk_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e);
    if (!dev) {
        for (int k = 0; k < 7; ++k)
            if ((e = cudaMemcpyAsync(const_cast<double*>(outs[k]), d[k], bytes, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
                return cuda_fail(e);
        if (group_id && (e = cudaMemcpyAsync(group_id, dg, (size_t)total * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return cuda_fail(e);
    }
    cleanup();
    if (!dev && (e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e);
    return GX_OK;
}
