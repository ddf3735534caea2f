// force.cu -- one-system direct-sum kernels (one CTA per target tile and source chunk,
// chunk-minor), the ordered j-split reduction (fused into the last CTA of each tile, or a
// second kernel) and the table of compiled variants.  The arithmetic lives in
// force_tile.cuh.
#include "force_tile.cuh"

#include <mutex>

namespace gx {
namespace {

// Ordered reduction of the j-split partial sums, then G and the epilogue (the unfused path).
__global__ void __launch_bounds__(256) force_reduce_kernel(const ForceArgs a) {
    const int64_t t = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (t >= a.n_tgt) return;
    double s[3] = {0.0, 0.0, 0.0};
    for (int c = 0; c < a.nsplit; ++c) {
        const size_t base = (size_t)c * 3 * (size_t)a.n_tgt + (size_t)t;
        s[0] += a.part[base];
        s[1] += a.part[base + (size_t)a.n_tgt];
        s[2] += a.part[base + 2 * (size_t)a.n_tgt];
    }
    write_result(a, t, target_body(a, t), a.G * s[0], a.G * s[1], a.G * s[2]);
}

// Fused reduction, run by every CTA after its tile body has written its partial sums: the
// CTA that takes the tile's last ticket adds the tile's nsplit partials in chunk order --
// the sums force_reduce_kernel forms -- and writes the results.  Each thread fences its
// own partial stores before the ticket is taken; the last CTA reads the partials from L2
// (ld.global.cg), so no stale L1 line can be seen.  No CTA waits for another.
template <int BLOCK, int IPT>
__device__ __forceinline__ void finish_tile(const ForceArgs& a, const int64_t tile, const int64_t t0) {
    if (a.nsplit <= 1 || !a.tile_count) return;
    __shared__ unsigned s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(&a.tile_count[tile], 1u) == (unsigned)a.nsplit - 1u;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const int64_t t = t0 + k * BLOCK + threadIdx.x;
        if (t >= a.n_tgt) continue;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (int c = 0; c < a.nsplit; ++c) {
            const size_t base = (size_t)c * 3 * (size_t)a.n_tgt + (size_t)t;
            s0 += __ldcg(a.part + base);
            s1 += __ldcg(a.part + base + (size_t)a.n_tgt);
            s2 += __ldcg(a.part + base + 2 * (size_t)a.n_tgt);
        }
        write_result(a, t, target_body(a, t), a.G * s0, a.G * s1, a.G * s2);
    }
    if (threadIdx.x == 0) a.tile_count[tile] = 0u;
}

template <int BLOCK, int IPT, int JT, bool PACKED, bool EPS0>
__global__ void __launch_bounds__(BLOCK) force_mixed_kernel(const ForceArgs a) {
    const int64_t tile = blockIdx.x / a.nsplit;
    mixed_tile<BLOCK, IPT, JT, PACKED, EPS0>(a, tile * (BLOCK * IPT), (int)(blockIdx.x % a.nsplit));
    finish_tile<BLOCK, IPT>(a, tile, tile * (BLOCK * IPT));
}

template <int BLOCK, int IPT, int JT, bool EPS0, int MINB, int UNROLL = 4>
__global__ void __launch_bounds__(BLOCK, MINB) force_mixed_tp_kernel(const ForceArgs a) {
    const int64_t tile = blockIdx.x / a.nsplit;
    mixed_tp_tile<BLOCK, IPT, JT, EPS0, UNROLL>(a, tile * (BLOCK * IPT), (int)(blockIdx.x % a.nsplit));
    finish_tile<BLOCK, IPT>(a, tile, tile * (BLOCK * IPT));
}

template <int BLOCK, int IPT, int JT, bool EPS0>
__global__ void __launch_bounds__(BLOCK) force_f64_kernel(const ForceArgs a) {
    const int64_t tile = blockIdx.x / a.nsplit;
    f64_tile<BLOCK, IPT, JT, EPS0>(a, tile * (BLOCK * IPT), (int)(blockIdx.x % a.nsplit));
    finish_tile<BLOCK, IPT>(a, tile, tile * (BLOCK * IPT));
}

template <int BLOCK, int JT>
__global__ void __launch_bounds__(BLOCK) force_exact_kernel(const ForceArgs a) {
    exact_tile<BLOCK, JT>(a, (int64_t)blockIdx.x * BLOCK);
}

#define MIXED(B, I, J, P, E) {kMixed, B, I, J, P, E, (const void*)&force_mixed_kernel<B, I, J, P, E>}
#define MIXTP(B, I, J, E, MB) {kMixed, B, I, J, 2, E, (const void*)&force_mixed_tp_kernel<B, I, J, E, MB>}
#define MIXTPU(B, I, J, MB, U) {kMixed, B, I, J, 2, 0, (const void*)&force_mixed_tp_kernel<B, I, J, false, MB, U>}
#define F64(B, I, J, E) {kF64, B, I, J, 0, E, (const void*)&force_f64_kernel<B, I, J, E>}
#define EXACT(B, J) {kF64Exact, B, 1, J, 0, 1, (const void*)&force_exact_kernel<B, J>}

const ForceVariant kVariants[] = {
    // mixed, targets packed (fastest at N = 2^20; the first entry is the untuned default)
    MIXTPU(256, 6, 512, 1, 8),
    MIXTPU(128, 8, 512, 1, 8),
    MIXTPU(128, 6, 512, 2, 16),
    MIXTP(128, 8, 512, false, 1),
    MIXTPU(256, 4, 512, 2, 16),
    MIXTPU(64, 8, 256, 1, 8),
    // mixed, sources packed; the scalar entry measures what packing buys
    MIXED(128, 8, 512, true, false),
    MIXED(64, 4, 256, true, false),
    MIXED(256, 4, 512, false, false),
    // softening 0
    MIXED(256, 4, 512, true, true),
    MIXED(64, 4, 256, true, true),
    F64(256, 2, 256, false),
    F64(128, 2, 256, false),
    F64(256, 1, 256, false),
    F64(128, 4, 256, false),
    F64(64, 2, 128, false),
    F64(256, 2, 256, true),
    F64(64, 2, 128, true),
    EXACT(128, 256),
    EXACT(64, 128),
};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

}  // namespace

const ForceVariant* force_variants(int* count) {
    *count = kNumVariants;
    return kVariants;
}

int force_variant_ids(int precision, int eps0, int* ids, int max_ids) {
    int c = 0;
    for (int i = 0; i < kNumVariants; ++i) {
        const ForceVariant& v = kVariants[i];
        if (v.precision != precision) continue;
        if (precision != kF64Exact && v.eps0 != eps0) continue;
        if (c < max_ids) ids[c] = i;
        ++c;
    }
    return c;
}

int64_t force_tiles(const ForceVariant& v, int64_t n_tgt) {
    const int64_t tile = (int64_t)v.block * v.ipt;
    return (n_tgt + tile - 1) / tile;
}

cudaError_t force_launch(const ForceVariant& v, const ForceArgs& args, cudaStream_t stream) {
    if (args.n_tgt <= 0) return cudaSuccess;
    const int ns = v.precision == kF64Exact ? 1 : args.nsplit;
    const int64_t blocks = force_tiles(v, args.n_tgt) * ns;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    ForceArgs a = args;
    void* params[] = {(void*)&a};
    cudaError_t e = cudaLaunchKernel(v.fn, dim3((unsigned)blocks), dim3(v.block), params, 0, stream);
    if (e != cudaSuccess || args.nsplit <= 1 || args.tile_count) return e;
    force_reduce_kernel<<<(unsigned)((args.n_tgt + 255) / 256), 256, 0, stream>>>(a);
    return cudaGetLastError();
}

int force_occupancy(const ForceVariant& v) {
    static std::mutex mu;
    static int cache[64] = {0};
    const int idx = (int)(&v - kVariants);
    std::lock_guard<std::mutex> lock(mu);
    if (idx >= 0 && idx < 64 && cache[idx] > 0) return cache[idx];
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, v.fn, v.block, 0) != cudaSuccess || nb < 1) nb = 1;
    if (idx >= 0 && idx < 64) cache[idx] = nb;
    return nb;
}

}  // namespace gx
