// batch.cu -- persistent kernel for ensembles of independent systems of uneven size.
//
// No reference counterpart: the reference runs one system per process.  Instance b owns
// the bodies offsets[b] .. offsets[b+1] of one concatenated SoA state and only interacts
// with itself.  The work is a list of items (instance, target tile), sorted on the host by
// decreasing cost (instance size; longest-processing-time order).  A grid of resident CTAs
// takes items from an atomic ticket counter until the list is exhausted -- there is no
// waiting between CTAs -- and runs the same per-tile arithmetic as the one-system kernels
// (force_tile.cuh), with the closing half-kick fused into the epilogue.
#include "batch.cuh"
#include "force_tile.cuh"

#include <mutex>

namespace gx {
namespace {

template <int MODE, int BLOCK, int IPT, int JT, bool EPS0, bool TP = false, int UNROLL = 4>
__global__ void __launch_bounds__(BLOCK) batch_force_kernel(const BatchArgs b) {
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(b.counter, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= b.n_items) return;
        const int2 w = b.items[it];
        const int64_t off = b.offsets[w.x];
        const int64_t nb = b.offsets[w.x + 1] - off;
        ForceArgs a;
        a.x = b.x + off;
        a.y = b.y + off;
        a.z = b.z + off;
        a.m = b.m + off;
        a.n_src = nb;
        a.tgt_idx = nullptr;
        a.t_begin = 0;
        a.n_tgt = nb;
        a.j_chunk = nb;
        a.nsplit = 1;
        a.ax = b.ax + off;
        a.ay = b.ay + off;
        a.az = b.az + off;
        a.part = nullptr;
        a.vx = b.vx ? b.vx + off : nullptr;
        a.vy = b.vy ? b.vy + off : nullptr;
        a.vz = b.vz ? b.vz + off : nullptr;
        a.kick_dt = b.kick_dt;
        a.G = b.G;
        a.eps2 = b.eps2;
        a.eps2f = b.eps2f;
        const int64_t t0 = (int64_t)w.y * (BLOCK * IPT);
        if constexpr (MODE == kMixed && TP)
            mixed_tp_tile<BLOCK, IPT, JT, EPS0, UNROLL>(a, t0, 0);
        else if constexpr (MODE == kMixed)
            mixed_tile<BLOCK, IPT, JT, true, EPS0>(a, t0, 0);
        else
            f64_tile<BLOCK, IPT, JT, EPS0>(a, t0, 0);
    }
}

// Per-item potential partial sum_t m_t sum_{j != t} m_j / s_tj of one tile (FP64).
template <int BLOCK, int JT>
__global__ void __launch_bounds__(BLOCK) batch_potential_kernel(const BatchArgs b, int tile,
                                                                double* part) {
    __shared__ __align__(16) double sx[JT];
    __shared__ __align__(16) double sy[JT];
    __shared__ __align__(16) double sz[JT];
    __shared__ __align__(16) double sm[JT];
    __shared__ double red[BLOCK / 32];
    const int it = blockIdx.x;
    const int2 w = b.items[it];
    const int64_t off = b.offsets[w.x];
    const int64_t nb = b.offsets[w.x + 1] - off;
    double acc = 0.0;
    for (int64_t t0 = (int64_t)w.y * tile; t0 < min(nb, (int64_t)(w.y + 1) * tile); t0 += BLOCK) {
        const int64_t i = t0 + threadIdx.x;
        const bool ok = i < min(nb, (int64_t)(w.y + 1) * tile);
        const int64_t bi = off + (ok ? i : t0);
        const double xi = b.x[bi], yi = b.y[bi], zi = b.z[bi];
        double pot = 0.0;
        for (int64_t j0 = 0; j0 < nb; j0 += JT) {
            for (int r = threadIdx.x; r < JT; r += BLOCK) {
                const int64_t j = j0 + r;
                const bool in = j < nb;
                sx[r] = in ? b.x[off + j] : 0.0;
                sy[r] = in ? b.y[off + j] : 0.0;
                sz[r] = in ? b.z[off + j] : 0.0;
                sm[r] = in ? b.m[off + j] : 0.0;
            }
            __syncthreads();
            for (int r = 0; r < JT; ++r) {
                const double dx = sx[r] - xi, dy = sy[r] - yi, dz = sz[r] - zi;
                double s = fma(dx, dx, b.eps2);
                s = fma(dy, dy, s);
                s = fma(dz, dz, s);
                double v = sm[r] * rsqrt_f64(s);
                v = (s == 0.0 || j0 + r == i) ? 0.0 : v;
                pot += v;
            }
            __syncthreads();
        }
        if (ok) acc += b.m[bi] * pot;
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < BLOCK / 32; ++q) s += red[q];
        part[it] = s;
    }
}

// One CTA per instance: the 11 O(N) moments, then the ordered sum of the instance's
// potential partials, written as 13 diagnostics values.
__global__ void __launch_bounds__(256) batch_moments_kernel(const BatchArgs b, const double* vx,
                                                            const double* vy, const double* vz,
                                                            const int* item_first,
                                                            const int* item_count,
                                                            const double* pot_part, double* out) {
    const int inst = blockIdx.x;
    const int64_t off = b.offsets[inst], nb = b.offsets[inst + 1] - off;
    double acc[11];
#pragma unroll
    for (int c = 0; c < 11; ++c) acc[c] = 0.0;
    for (int64_t k = threadIdx.x; k < nb; k += 256) {
        const int64_t i = off + k;
        const double mi = b.m[i], X = b.x[i], Y = b.y[i], Z = b.z[i], U = vx[i], V = vy[i], W = vz[i];
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
    __shared__ double red[11][8];
#pragma unroll
    for (int c = 0; c < 11; ++c) {
        const double v = warp_sum(acc[c]);
        if ((threadIdx.x & 31) == 0) red[c][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s[11];
        for (int c = 0; c < 11; ++c) {
            s[c] = 0.0;
            for (int q = 0; q < 8; ++q) s[c] += red[c][q];
        }
        double pe = 0.0;
        for (int q = 0; q < item_count[inst]; ++q) pe += pot_part[item_first[inst] + q];
        pe *= -0.5 * b.G;
        double* o = out + (size_t)inst * 13;
        const double M = s[0];
        o[0] = M;
        o[1] = s[1];
        o[2] = pe;
        o[3] = s[1] + pe;
        o[4] = s[2];
        o[5] = s[3];
        o[6] = s[4];
        o[7] = M > 0.0 ? s[5] / M : s[5];
        o[8] = M > 0.0 ? s[6] / M : s[6];
        o[9] = M > 0.0 ? s[7] / M : s[7];
        o[10] = s[8];
        o[11] = s[9];
        o[12] = s[10];
    }
}

#define BMIX(B, I, J, E) {kMixed, B, I, J, E, (const void*)&batch_force_kernel<kMixed, B, I, J, E>}
#define BMTP(B, I, J, E) {kMixed, B, I, J, E, (const void*)&batch_force_kernel<kMixed, B, I, J, E, true>}
#define BMTPU(B, I, J, U) {kMixed, B, I, J, 0, (const void*)&batch_force_kernel<kMixed, B, I, J, false, true, U>}
#define BF64(B, I, J, E) {kF64, B, I, J, E, (const void*)&batch_force_kernel<kF64, B, I, J, E>}

const BatchVariant kBatchVariants[] = {
    BMTPU(256, 6, 512, 8), BMTPU(128, 8, 512, 8), BMTP(128, 8, 512, false), BMTP(256, 4, 512, false),
    BMIX(128, 8, 512, false), BMTPU(64, 8, 256, 8), BMIX(64, 4, 256, false),
    BMIX(256, 4, 512, true),
    BF64(256, 2, 256, false), BF64(128, 2, 256, false), BF64(64, 2, 128, false),
    BF64(256, 2, 256, true),
};
constexpr int kNumBatchVariants = sizeof(kBatchVariants) / sizeof(kBatchVariants[0]);
constexpr int kPotTile = 256;

}  // namespace

const BatchVariant* batch_variants(int* count) {
    *count = kNumBatchVariants;
    return kBatchVariants;
}

int batch_variant_ids(int precision, int eps0, int* ids, int max_ids) {
    int c = 0;
    for (int i = 0; i < kNumBatchVariants; ++i) {
        if (kBatchVariants[i].precision != precision || kBatchVariants[i].eps0 != eps0) continue;
        if (c < max_ids) ids[c] = i;
        ++c;
    }
    return c;
}

int batch_occupancy(const BatchVariant& v) {
    static std::mutex mu;
    static int cache[32] = {0};
    const int idx = (int)(&v - kBatchVariants);
    std::lock_guard<std::mutex> lock(mu);
    if (idx >= 0 && idx < 32 && cache[idx] > 0) return cache[idx];
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, v.fn, v.block, 0) != cudaSuccess || nb < 1) nb = 1;
    if (idx >= 0 && idx < 32) cache[idx] = nb;
    return nb;
}

cudaError_t batch_force_launch(const BatchVariant& v, const BatchArgs& args, int grid,
                               cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(args.counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    BatchArgs a = args;
    void* params[] = {(void*)&a};
    return cudaLaunchKernel(v.fn, dim3(grid), dim3(v.block), params, 0, st);
}

int batch_potential_tile() { return kPotTile; }

cudaError_t batch_diagnostics_launch(const BatchArgs& pot_args, int n_pot_items,
                                     int n_instances, const double* vx, const double* vy,
                                     const double* vz, const int* item_first,
                                     const int* item_count, double* pot_part, double* out,
                                     cudaStream_t st) {
    if (n_pot_items > 0)
        batch_potential_kernel<128, 256><<<n_pot_items, 128, 0, st>>>(pot_args, kPotTile, pot_part);
    batch_moments_kernel<<<n_instances, 256, 0, st>>>(pot_args, vx, vy, vz, item_first, item_count,
                                                      pot_part, out);
    return cudaGetLastError();
}

}  // namespace gx
