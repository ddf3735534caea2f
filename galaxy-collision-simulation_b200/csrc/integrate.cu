// integrate.cu -- kick / drift kernels and the FP64 diagnostics reductions.
//
// Kick and drift follow cpp/core/integrator.cpp:7-17 operation by operation
// (v = v + a*dt, x = x + v*dt, no FMA contraction), so a device step reproduces the
// reference's rounding given the same accelerations.
//
// Diagnostics follow cpp/core/diagnostics.cpp:7-37 in FP64: the O(N) moments are block
// partial sums reduced in block order (deterministic); the potential energy
//     PE = -G sum_{i<j} m_i m_j / sqrt(|x_j - x_i|^2 + eps^2)
// is evaluated as -G/2 sum_i m_i sum_{j != i} m_j / s_ij with the same tiling as the force
// kernel (self pairs skipped by index, s == 0 pairs skipped as in the reference).
#include "gx_device.cuh"
#include "integrate.cuh"

namespace gx {
namespace {

__global__ void kick_kernel(int64_t n, double* vx, double* vy, double* vz, const double* ax,
                            const double* ay, const double* az, double dt) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        vx[i] = dadd(vx[i], dmul(ax[i], dt));
        vy[i] = dadd(vy[i], dmul(ay[i], dt));
        vz[i] = dadd(vz[i], dmul(az[i], dt));
    }
}

__global__ void drift_kernel(int64_t n, double* x, double* y, double* z, const double* vx,
                             const double* vy, const double* vz, double dt) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        x[i] = dadd(x[i], dmul(vx[i], dt));
        y[i] = dadd(y[i], dmul(vy[i], dt));
        z[i] = dadd(z[i], dmul(vz[i], dt));
    }
}

// Opening half of a KDK step: kick(kick_dt) then drift(drift_dt), fused per body.
__global__ void kick_drift_kernel(int64_t n, double* x, double* y, double* z, double* vx,
                                  double* vy, double* vz, const double* ax, const double* ay,
                                  const double* az, double kdt, double ddt) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double ux = dadd(vx[i], dmul(ax[i], kdt));
        const double uy = dadd(vy[i], dmul(ay[i], kdt));
        const double uz = dadd(vz[i], dmul(az[i], kdt));
        vx[i] = ux;
        vy[i] = uy;
        vz[i] = uz;
        x[i] = dadd(x[i], dmul(ux, ddt));
        y[i] = dadd(y[i], dmul(uy, ddt));
        z[i] = dadd(z[i], dmul(uz, ddt));
    }
}

constexpr int kMomBlock = 256;

// Block partial sums of the 11 O(N) moments:
// [M, KE, Px, Py, Pz, Cx, Cy, Cz, Lx, Ly, Lz] (C = sum m x before the division by M).
__global__ void __launch_bounds__(kMomBlock) moments_kernel(int64_t n, const double* x,
                                                            const double* y, const double* z,
                                                            const double* vx, const double* vy,
                                                            const double* vz, const double* m,
                                                            double* part) {
    double acc[11];
#pragma unroll
    for (int c = 0; c < 11; ++c) acc[c] = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * kMomBlock + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * kMomBlock) {
        const double mi = m[i], X = x[i], Y = y[i], Z = z[i], U = vx[i], V = vy[i], W = vz[i];
        acc[0] += mi;
        acc[1] += 0.5 * mi * (U * U + V * V + W * W);
        acc[2] += U * mi;
        acc[3] += V * mi;
        acc[4] += W * mi;
        acc[5] += X * mi;
        acc[6] += Y * mi;
        acc[7] += Z * mi;
        acc[8] += (Y * W - Z * V) * mi;
        acc[9] += (Z * U - X * W) * mi;
        acc[10] += (X * V - Y * U) * mi;
    }
    __shared__ double red[11][kMomBlock / 32];
#pragma unroll
    for (int c = 0; c < 11; ++c) {
        const double v = warp_sum(acc[c]);
        if ((threadIdx.x & 31) == 0) red[c][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 11) {
        double s = 0.0;
        for (int w = 0; w < kMomBlock / 32; ++w) s += red[threadIdx.x][w];
        part[(size_t)blockIdx.x * 11 + threadIdx.x] = s;
    }
}

// Potential: per target body i, pot_i = sum_{j != i} m_j / sqrt(s_ij); block partial of
// m_i * pot_i.  FP64 with the refined rsqrt.
template <int BLOCK, int JT, bool EPS0>
__global__ void __launch_bounds__(BLOCK) potential_kernel(int64_t n, const double* x,
                                                          const double* y, const double* z,
                                                          const double* m, double eps2,
                                                          double* part) {
    __shared__ __align__(16) double sx[JT];
    __shared__ __align__(16) double sy[JT];
    __shared__ __align__(16) double sz[JT];
    __shared__ __align__(16) double sm[JT];
    const int tid = threadIdx.x;
    const int64_t i = (int64_t)blockIdx.x * BLOCK + tid;
    const bool ok = i < n;
    const int64_t bi = ok ? i : 0;
    const double xi = x[bi], yi = y[bi], zi = z[bi];
    double pot = 0.0;
    for (int64_t j0 = 0; j0 < n; j0 += JT) {
#pragma unroll
        for (int r = 0; r < JT / BLOCK; ++r) {
            const int jj = r * BLOCK + tid;
            const int64_t j = j0 + jj;
            const bool in = j < n;
            sx[jj] = in ? x[j] : 0.0;
            sy[jj] = in ? y[j] : 0.0;
            sz[jj] = in ? z[j] : 0.0;
            sm[jj] = in ? m[j] : 0.0;
        }
        __syncthreads();
#pragma unroll 4
        for (int jj = 0; jj < JT; ++jj) {
            const double dx = sx[jj] - xi, dy = sy[jj] - yi, dz = sz[jj] - zi;
            double r = fma(dx, dx, eps2);
            r = fma(dy, dy, r);
            r = fma(dz, dz, r);
            double w = sm[jj] * rsqrt_f64(r);
            if (EPS0) w = (r == 0.0) ? 0.0 : w;
            w = (j0 + jj == i) ? 0.0 : w;
            pot += w;
        }
        __syncthreads();
    }
    double v = ok ? m[i] * pot : 0.0;
    __shared__ double red[BLOCK / 32];
    v = warp_sum(v);
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    if (tid == 0) {
        double s = 0.0;
        for (int w = 0; w < BLOCK / 32; ++w) s += red[w];
        part[blockIdx.x] = s;
    }
}

// Final, single-block and ordered: out[13] in diagnostics.csv order.
__global__ void diagnostics_final_kernel(int n_mom, const double* mom_part, int n_pot,
                                         const double* pot_part, double G, double* out) {
    __shared__ double sums[12];
    const int c = threadIdx.x;
    if (c < 11) {
        double s = 0.0;
        for (int b = 0; b < n_mom; ++b) s += mom_part[(size_t)b * 11 + c];
        sums[c] = s;
    } else if (c == 11) {
        double s = 0.0;
        for (int b = 0; b < n_pot; ++b) s += pot_part[b];
        sums[11] = s;
    }
    __syncthreads();
    if (c == 0) {
        const double M = sums[0];
        const double pe = -0.5 * G * sums[11];
        out[0] = M;
        out[1] = sums[1];
        out[2] = pe;
        out[3] = sums[1] + pe;
        out[4] = sums[2];
        out[5] = sums[3];
        out[6] = sums[4];
        out[7] = M > 0.0 ? sums[5] / M : sums[5];
        out[8] = M > 0.0 ? sums[6] / M : sums[6];
        out[9] = M > 0.0 ? sums[7] / M : sums[7];
        out[10] = sums[8];
        out[11] = sums[9];
        out[12] = sums[10];
    }
}

constexpr int kPotBlock = 128;
constexpr int kPotJT = 256;

int grid_for(int64_t n, int block, int cap) {
    int64_t g = (n + block - 1) / block;
    if (g > cap) g = cap;
    return g < 1 ? 1 : (int)g;
}

}  // namespace

cudaError_t launch_kick(int64_t n, double* vx, double* vy, double* vz, const double* ax,
                        const double* ay, const double* az, double dt, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    kick_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, st>>>(n, vx, vy, vz, ax, ay, az, dt);
    return cudaGetLastError();
}

cudaError_t launch_drift(int64_t n, double* x, double* y, double* z, const double* vx,
                         const double* vy, const double* vz, double dt, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    drift_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, st>>>(n, x, y, z, vx, vy, vz, dt);
    return cudaGetLastError();
}

cudaError_t launch_kick_drift(int64_t n, double* x, double* y, double* z, double* vx,
                              double* vy, double* vz, const double* ax, const double* ay,
                              const double* az, double kdt, double ddt, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    kick_drift_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, st>>>(n, x, y, z, vx, vy, vz, ax,
                                                                  ay, az, kdt, ddt);
    return cudaGetLastError();
}

size_t diagnostics_scratch_bytes(int64_t n) {
    const int nm = grid_for(n, kMomBlock, 148 * 4);
    const int np = grid_for(n, kPotBlock, 1 << 30);
    return ((size_t)nm * 11 + (size_t)np + 16) * sizeof(double);
}

cudaError_t launch_diagnostics(int64_t n, const double* x, const double* y, const double* z,
                               const double* vx, const double* vy, const double* vz,
                               const double* m, double G, double eps2, double* scratch,
                               double* out13, cudaStream_t st) {
    const int nm = grid_for(n, kMomBlock, 148 * 4);
    const int np = grid_for(n, kPotBlock, 1 << 30);
    double* mom = scratch;
    double* pot = scratch + (size_t)nm * 11;
    if (n <= 0) {
        cudaError_t e = cudaMemsetAsync(out13, 0, 13 * sizeof(double), st);
        return e;
    }
    moments_kernel<<<nm, kMomBlock, 0, st>>>(n, x, y, z, vx, vy, vz, m, mom);
    if (eps2 < 1e-200)
        potential_kernel<kPotBlock, kPotJT, true><<<np, kPotBlock, 0, st>>>(n, x, y, z, m, eps2, pot);
    else
        potential_kernel<kPotBlock, kPotJT, false><<<np, kPotBlock, 0, st>>>(n, x, y, z, m, eps2, pot);
    diagnostics_final_kernel<<<1, 32, 0, st>>>(nm, mom, np, pot, G, out13);
    return cudaGetLastError();
}

}  // namespace gx
