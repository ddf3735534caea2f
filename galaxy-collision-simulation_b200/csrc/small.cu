// small.cu -- the kick-drift-kick loop of a small system in ONE cooperative launch.
//
// For n up to a few thousand bodies a step is a few microseconds of arithmetic, so a loop of
// separate launches (kick-drift, force) is bound by launch latency.  Here every CTA of a
// cooperative grid stays resident for all steps:
//   * every warp owns up to TPW target bodies for the whole launch (global warp w owns
//     w, w + W, w + 2W, ...) and keeps their position, velocity and acceleration in
//     registers;
//   * a step is: opening kick + drift of the owned bodies (integrator.cpp:7-17 rounding),
//     positions stored to one of two global buffers, one grid barrier, the force on every
//     owned target from all n bodies of that buffer (staged through shared memory, read
//     with ld.global.cg so no stale L1 line of an earlier step is seen), closing kick;
//   * one barrier per step suffices: step s reads buffer s & 1 and writes buffer (s+1) & 1,
//     so a buffer is overwritten only after the next barrier, which every CTA reaches after
//     its reads of that buffer are done.
// Two arithmetic forms:
//   * kF64 -- the pair term of the tiled FP64 kernel (refined hardware rsqrt, FMA); the
//     lanes of a warp split the sources (lane l takes j = l mod 32) and a butterfly of
//     shuffles adds the 32 partial sums (every lane ends with the same bits);
//   * kF64Exact -- the reference's operation order (direct_solver.cpp:8-23, 59-83): lane l
//     computes the contribution of source j0 + l into shared memory, and lane c (c < 3)
//     adds component c of the 32 contributions in ascending j order into one running sum,
//     so each target is summed exactly as compute_direct_accelerations_for_targets sums it.  The skipped self pair
//     and the s2 == 0 pair add +0.0, which leaves the running sum unchanged: it starts at
//     +0.0 and, in round-to-nearest, a sum is -0.0 only when both addends are -0.0.
// The grid barrier is an arrival counter and a generation word in global memory; a CTA
// waits on the generation with ld.acquire for at most a.timeout_ns (and 2^30 polls), after
// which it sets the status word and the whole launch stops early: the state arrays are then
// left as they were before the launch and the host reports GX_ERR_TIMEOUT.  The test hook
// a.stall_step makes CTA 0 leave without arriving, so that the others' waits run out.
#include "gx_device.cuh"
#include "precision.cuh"
#include "small.cuh"

#include <atomic>

namespace gx {
namespace {

constexpr int kSmallThreads = 256;
constexpr int kSmallWarps = kSmallThreads / 32;
constexpr int kSmallJT = 512;  // sources staged per shared-memory pass
constexpr size_t kSmallHeader = 256;  // barrier words + status, then the position buffers
std::atomic<int> g_small_tpw{0};      // 0: chosen from n; 1, 2 or 4: forced (measurement)
std::atomic<int> g_small_wpt{0};      // 0: chosen; 1 or 2 warps per target: forced (measurement)

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void red_release_add_u32(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid-wide barrier; false on every thread of the CTA when the launch has to stop.
// `gen` (thread 0 only) is the generation this CTA waits to see pass.  One returning atomic
// per CTA (the arrival); the last arrival resets the counter with a plain store and, after a
// fence, releases the others with a non-returning release add on the generation word, so no
// second returning round trip to L2 sits on the path.  A status set by a CTA that gave up is seen by the others at their
// next wait (polled every 256 loads); the launch then ends within one barrier.
__device__ bool grid_barrier(const SmallArgs& a, unsigned& gen) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();  // after the CTA barrier: the CTA's position stores before its arrival
        const unsigned arrived = atomicAdd(&a.bar[0], 1u);
        if (arrived == gridDim.x - 1) {
            *(volatile unsigned*)&a.bar[0] = 0u;  // nobody arrives again before the release below
            __threadfence();  // every arrival seen through the counter, before the release
            red_release_add_u32(&a.bar[1], 1u);
        } else {
            const unsigned long long t0 = global_ns();
            unsigned polls = 0;
            while (ld_acquire_u32(&a.bar[1]) == gen) {
                if ((++polls & 255u) == 0) {
                    if (polls >= (1u << 30) || global_ns() - t0 > a.timeout_ns ||
                        *(volatile int*)a.status) {
                        ok = 0;
                        break;
                    }
                }
            }
        }
        if (!ok) atomicExch(a.status, 1);
        gen += 1;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// WPT warps per target slot (FP64 form): the slot's sources are split over its warps and the
// warps' sums are added in warp order through shared memory, so each warp has half (a
// quarter) of the dependent pair terms to run per step.  256 x WPT threads per CTA.
template <int PREC, int TPW, bool EPS0, int WPT>
__global__ void __launch_bounds__(kSmallThreads * WPT, 1) small_steps_kernel(const SmallArgs a) {
    constexpr int kBlock = kSmallThreads * WPT;
    static_assert(PREC == kF64 || WPT == 1, "the exact form sums each target in one warp");
    __shared__ double s_part[WPT > 1 ? kSmallWarps * WPT * TPW * 3 : 1];
    __shared__ __align__(16) double sx[kSmallJT];
    __shared__ __align__(16) double sy[kSmallJT];
    __shared__ __align__(16) double sz[kSmallJT];
    __shared__ __align__(16) double sm[kSmallJT];
    // exact form: each warp's 32 contributions (3 doubles each) per owned target
    __shared__ double s_con_all[PREC == kF64Exact ? kSmallWarps * TPW * 96 : 1];
    double* const s_con = s_con_all + (PREC == kF64Exact ? (threadIdx.x >> 5) * TPW * 96 : 0);
    const int lane = threadIdx.x & 31;
    const int n = a.n;
    const int total_warps = gridDim.x * kSmallWarps;  // target slots of the grid
    const int slot = (threadIdx.x >> 5) / WPT, part = (threadIdx.x >> 5) % WPT;
    const int w = blockIdx.x * kSmallWarps + slot;
    const double h = 0.5 * a.dt, dt = a.dt, G = a.G, e2 = a.eps2;

    int T[TPW];
    double X[TPW], Y[TPW], Z[TPW], U[TPW], V[TPW], W[TPW], AX[TPW], AY[TPW], AZ[TPW];
#pragma unroll
    for (int k = 0; k < TPW; ++k) {
        T[k] = w + k * total_warps;
        const int t = T[k] < n ? T[k] : 0;
        X[k] = a.x[t]; Y[k] = a.y[t]; Z[k] = a.z[t];
        U[k] = a.vx[t]; V[k] = a.vy[t]; W[k] = a.vz[t];
        AX[k] = a.ax[t]; AY[k] = a.ay[t]; AZ[k] = a.az[t];
    }
    unsigned gen = 0;
    if (threadIdx.x == 0) gen = ld_acquire_u32(&a.bar[1]);

    for (int64_t s = 0; s < a.steps; ++s) {
        double* px = a.buf + (size_t)((s & 1) * 3) * n;
        double* py = px + n;
        double* pz = py + n;
        // opening kick (dt/2) and drift (dt) of the owned bodies
#pragma unroll
        for (int k = 0; k < TPW; ++k) {
            if (T[k] >= n) continue;
            U[k] = dadd(U[k], dmul(AX[k], h));
            V[k] = dadd(V[k], dmul(AY[k], h));
            W[k] = dadd(W[k], dmul(AZ[k], h));
            X[k] = dadd(X[k], dmul(U[k], dt));
            Y[k] = dadd(Y[k], dmul(V[k], dt));
            Z[k] = dadd(Z[k], dmul(W[k], dt));
            if (lane == 0 && part == 0) {
                px[T[k]] = X[k];
                py[T[k]] = Y[k];
                pz[T[k]] = Z[k];
            }
        }
        if (s == a.stall_step && blockIdx.x == 0) return;
        if (!grid_barrier(a, gen)) return;

        double fx[TPW], fy[TPW], fz[TPW];
#pragma unroll
        for (int k = 0; k < TPW; ++k) fx[k] = fy[k] = fz[k] = 0.0;
        for (int j0 = 0; j0 < n; j0 += kSmallJT) {
            const int cnt = min(kSmallJT, n - j0);
            for (int jj = threadIdx.x; jj < cnt; jj += kBlock) {
                sx[jj] = __ldcg(px + j0 + jj);
                sy[jj] = __ldcg(py + j0 + jj);
                sz[jj] = __ldcg(pz + j0 + jj);
                sm[jj] = __ldg(a.m + j0 + jj);
            }
            __syncthreads();
            if constexpr (PREC == kF64) {
#pragma unroll 4
                for (int jj = part * 32 + lane; jj < cnt; jj += 32 * WPT) {
                    const double qx = sx[jj], qy = sy[jj], qz = sz[jj], qm = sm[jj];
#pragma unroll
                    for (int k = 0; k < TPW; ++k) {
                        if (T[k] >= n) continue;
                        const double dx = qx - X[k], dy = qy - Y[k], dz = qz - Z[k];
                        double r = fma(dx, dx, e2);
                        r = fma(dy, dy, r);
                        r = fma(dz, dz, r);
                        double y = rsqrt_f64(r);
                        if (EPS0) y = (r == 0.0) ? 0.0 : y;
                        const double wgt = qm * (y * y * y);
                        fx[k] = fma(dx, wgt, fx[k]);
                        fy[k] = fma(dy, wgt, fy[k]);
                        fz[k] = fma(dz, wgt, fz[k]);
                    }
                }
            } else {
                // lane l computes the contribution of source jb + l for each owned target into
                // the warp's shared slots; then lane c (c < 3) adds component c of the 32
                // contributions in ascending j, one running sum per target (fx holds it)
                for (int jb = 0; jb < cnt; jb += 32) {
                    const int jj = jb + lane;
                    const int lim = min(32, cnt - jb);
#pragma unroll
                    for (int k = 0; k < TPW; ++k) {
                        double cx = 0.0, cy = 0.0, cz = 0.0;
                        if (T[k] < n && jj < cnt && j0 + jj != T[k]) {
                            const double rx = dsub(sx[jj], X[k]), ry = dsub(sy[jj], Y[k]), rz = dsub(sz[jj], Z[k]);
                            const double s2 = dadd(dadd(dadd(dmul(rx, rx), dmul(ry, ry)), dmul(rz, rz)), e2);
                            if (s2 != 0.0) {
                                const double inv = __ddiv_rn(1.0, __dsqrt_rn(s2));
                                const double inv3 = dmul(dmul(inv, inv), inv);
                                const double scale = dmul(dmul(G, sm[jj]), inv3);
                                cx = dmul(rx, scale);
                                cy = dmul(ry, scale);
                                cz = dmul(rz, scale);
                            }
                        }
                        double* slot = s_con + (k * 32 + lane) * 3;
                        slot[0] = cx;
                        slot[1] = cy;
                        slot[2] = cz;
                    }
                    __syncwarp();
                    if (lane < 3) {
                        for (int q = 0; q < lim; ++q) {
#pragma unroll
                            for (int k = 0; k < TPW; ++k) fx[k] = dadd(fx[k], s_con[(k * 32 + q) * 3 + lane]);
                        }
                    }
                    __syncwarp();
                }
            }
            __syncthreads();
        }
        // results and the closing kick (dt/2)
        if constexpr (PREC == kF64) {
#pragma unroll
            for (int k = 0; k < TPW; ++k) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    fx[k] += __shfl_xor_sync(0xffffffffu, fx[k], o);
                    fy[k] += __shfl_xor_sync(0xffffffffu, fy[k], o);
                    fz[k] += __shfl_xor_sync(0xffffffffu, fz[k], o);
                }
                if constexpr (WPT > 1) {
                    double* mine = s_part + ((slot * WPT + part) * TPW + k) * 3;
                    if (lane == 0) {
                        mine[0] = fx[k];
                        mine[1] = fy[k];
                        mine[2] = fz[k];
                    }
                }
            }
            if constexpr (WPT > 1) {  // the slot's warps' sums, added in warp order by each of them
                __syncthreads();
#pragma unroll
                for (int k = 0; k < TPW; ++k) {
                    const double* p0 = s_part + ((slot * WPT) * TPW + k) * 3;
                    double sx = p0[0], sy = p0[1], sz = p0[2];
#pragma unroll
                    for (int q = 1; q < WPT; ++q) {
                        const double* pq = p0 + q * TPW * 3;
                        sx += pq[0];
                        sy += pq[1];
                        sz += pq[2];
                    }
                    fx[k] = sx;
                    fy[k] = sy;
                    fz[k] = sz;
                }
            }
#pragma unroll
            for (int k = 0; k < TPW; ++k) {
                AX[k] = G * fx[k];
                AY[k] = G * fy[k];
                AZ[k] = G * fz[k];
            }
        } else {
#pragma unroll
            for (int k = 0; k < TPW; ++k) {  // lane c holds component c
                AX[k] = __shfl_sync(0xffffffffu, fx[k], 0);
                AY[k] = __shfl_sync(0xffffffffu, fx[k], 1);
                AZ[k] = __shfl_sync(0xffffffffu, fx[k], 2);
            }
        }
#pragma unroll
        for (int k = 0; k < TPW; ++k) {
            if (T[k] >= n) continue;
            U[k] = dadd(U[k], dmul(AX[k], h));
            V[k] = dadd(V[k], dmul(AY[k], h));
            W[k] = dadd(W[k], dmul(AZ[k], h));
        }
    }
    if (lane == 0 && part == 0) {
#pragma unroll
        for (int k = 0; k < TPW; ++k) {
            const int t = T[k];
            if (t >= n) continue;
            a.x[t] = X[k]; a.y[t] = Y[k]; a.z[t] = Z[k];
            a.vx[t] = U[k]; a.vy[t] = V[k]; a.vz[t] = W[k];
            a.ax[t] = AX[k]; a.ay[t] = AY[k]; a.az[t] = AZ[k];
        }
    }
}

template <int PREC, bool EPS0, int WPT>
const void* pick(int tpw) {
    switch (tpw) {
        case 1: return (const void*)&small_steps_kernel<PREC, 1, EPS0, WPT>;
        case 2: return (const void*)&small_steps_kernel<PREC, 2, EPS0, WPT>;
        default: return (const void*)&small_steps_kernel<PREC, 4, EPS0, WPT>;
    }
}

}  // namespace

void small_set_targets_per_warp(int tpw) { g_small_tpw.store(tpw == 1 || tpw == 2 || tpw == 4 ? tpw : 0); }
void small_set_warps_per_target(int wpt) { g_small_wpt.store(wpt == 1 || wpt == 2 ? wpt : 0); }

size_t small_scratch_bytes(int n) { return kSmallHeader + (size_t)6 * (size_t)n * sizeof(double); }

void small_bind_scratch(SmallArgs& a, void* scratch) {
    a.bar = (unsigned*)scratch;
    a.status = (int*)((char*)scratch + 2 * sizeof(unsigned));
    a.buf = (double*)((char*)scratch + kSmallHeader);
}

cudaError_t small_steps_launch(const SmallArgs& a, int precision, bool eps0, int device, cudaStream_t st) {
    if (a.n < 1 || a.n > kSmallMaxBodies || (precision != kF64 && precision != kF64Exact)) return cudaErrorNotSupported;
    if (a.steps <= 0) return cudaSuccess;
    int coop = 0, sms = 0;
    cudaError_t e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
    if (e != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) return e;
    if (!coop) return cudaErrorNotSupported;
    // Shape: targets per warp (tpw) and, in the FP64 form, warps per target (wpt), the first
    // of (1, 2), (1, 1), (2, 2), (2, 1), (4, 2), (4, 1) whose grid is co-resident.  Measured on
    // B200 (steps/s of the FP64 form): n = 1000: 155k at (1, 2), 128k at (1, 1), 111k at
    // (2, 2), 90k at (2, 1); n = 4096: 26.4k at (2, 1) and (2, 2), 18.8k at (4, 1).  Forced
    // shapes (measurement knobs) skip the others.
    const int f_tpw = g_small_tpw.load(), f_wpt = g_small_wpt.load();
    const void* fn = nullptr;
    int blocks = 0, threads = 0;
    for (int tpw : {1, 2, 4}) {
        if (f_tpw && tpw != f_tpw) continue;
        for (int wpt : {2, 1}) {
            if (precision == kF64Exact ? wpt != 1 : (f_wpt && wpt != f_wpt)) continue;  // exact: one warp
            const void* g;
            if (precision == kF64Exact) g = pick<kF64Exact, true, 1>(tpw);
            else if (wpt == 2) g = eps0 ? pick<kF64, true, 2>(tpw) : pick<kF64, false, 2>(tpw);
            else g = eps0 ? pick<kF64, true, 1>(tpw) : pick<kF64, false, 1>(tpw);
            const int b = (a.n + kSmallWarps * tpw - 1) / (kSmallWarps * tpw);
            int occ = 0;
            if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, g, kSmallThreads * wpt, 0)) != cudaSuccess)
                return e;
            if ((int64_t)occ * sms < b) continue;
            fn = g;
            blocks = b;
            threads = kSmallThreads * wpt;
            break;
        }
        if (fn) break;
    }
    if (!fn) return cudaErrorNotSupported;
    if ((e = cudaMemsetAsync(a.bar, 0, 4 * sizeof(unsigned), st)) != cudaSuccess) return e;
    SmallArgs args = a;
    void* params[] = {(void*)&args};
    return cudaLaunchCooperativeKernel(fn, dim3((unsigned)blocks), dim3(threads), params, 0, st);
}

}  // namespace gx
