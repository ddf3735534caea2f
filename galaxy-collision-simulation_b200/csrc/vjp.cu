// vjp.cu -- vector-Jacobian product of the direct accelerations (the adjoint kernel).
//
// No reference counterpart (the reference has no gradients).  With
//     a_k = G sum_{j != k} m_j d s^-3/2,   d = x_j - x_k,   s = |d|^2 + eps^2,
// and a cotangent l_k on a_k, L = sum_k l_k . a_k has
//     dL/dx_k = G sum_j [ s^-3/2 A - 3 s^-5/2 (A . d) d ],  A = m_k l_j - m_j l_k,
//     dL/dm_k = -G sum_j s^-3/2 (l_j . d),
// which is a gather over j with the forward kernel's tiling: the sources stage
// (x_j, m_j, l_j) -- 7 words -- in shared memory and each thread keeps IPT targets.
// A self pair has d = 0 and A = 0, so it adds exactly zero when eps > 0.
// Forms: FP64 (refined rsqrt) and mixed (FP32 pair arithmetic on offsets from a per-tile
// FP64 origin, per-tile compensated accumulation).  A j-split with ordered reduction keeps
// small systems spread over all SMs.
#include "gx_device.cuh"
#include "vjp.cuh"

#include <cfloat>
#include <type_traits>

namespace gx {
namespace {

template <int BLOCK, int IPT, int JT, bool MIXED, bool EPS0>
__global__ void __launch_bounds__(BLOCK) vjp_kernel(const VjpArgs a) {
    static_assert(JT % BLOCK == 0, "tile shape");
    using T = typename std::conditional<MIXED, float, double>::type;
    __shared__ __align__(16) T sx[JT];
    __shared__ __align__(16) T sy[JT];
    __shared__ __align__(16) T sz[JT];
    __shared__ __align__(16) T sm[JT];
    __shared__ __align__(16) T sl[3][JT];
    __shared__ double sred[6][BLOCK / 32];

    const int tid = threadIdx.x;
    const int64_t t0 = (int64_t)blockIdx.x * (BLOCK * IPT);
    int64_t idx[IPT];
    double bx[IPT], by[IPT], bz[IPT];
    double org[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const int64_t t = t0 + k * BLOCK + tid;
        idx[k] = t < a.n ? t : t0;
        bx[k] = a.x[idx[k]];
        by[k] = a.y[idx[k]];
        bz[k] = a.z[idx[k]];
    }
    if (MIXED) {
        double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            lo[0] = fmin(lo[0], bx[k]); hi[0] = fmax(hi[0], bx[k]);
            lo[1] = fmin(lo[1], by[k]); hi[1] = fmax(hi[1], by[k]);
            lo[2] = fmin(lo[2], bz[k]); hi[2] = fmax(hi[2], bz[k]);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            lo[c] = warp_min(lo[c]);
            hi[c] = warp_max(hi[c]);
        }
        if ((tid & 31) == 0)
            for (int c = 0; c < 3; ++c) {
                sred[c][tid >> 5] = lo[c];
                sred[3 + c][tid >> 5] = hi[c];
            }
        __syncthreads();
        for (int c = 0; c < 3; ++c) {
            double l = sred[c][0], h = sred[3 + c][0];
            for (int w = 1; w < BLOCK / 32; ++w) {
                l = fmin(l, sred[c][w]);
                h = fmax(h, sred[3 + c][w]);
            }
            org[c] = 0.5 * (l + h);
        }
    }
    T xk[IPT], yk[IPT], zk[IPT], mk[IPT], lk[IPT][3];
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        xk[k] = (T)(bx[k] - org[0]);
        yk[k] = (T)(by[k] - org[1]);
        zk[k] = (T)(bz[k] - org[2]);
        mk[k] = (T)a.m[idx[k]];
        lk[k][0] = (T)a.lx[idx[k]];
        lk[k][1] = (T)a.ly[idx[k]];
        lk[k][2] = (T)a.lz[idx[k]];
    }
    // Accumulators: gx, gy, gz, h (gm = -G h).
    double acc[IPT][4];
    CompF comp[IPT][4];
#pragma unroll
    for (int k = 0; k < IPT; ++k)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            acc[k][c] = 0.0;
            comp[k][c].init();
        }
    const T e2 = MIXED ? (T)a.eps2f : (T)a.eps2;
    const int64_t jb = (int64_t)blockIdx.y * a.j_chunk;
    const int64_t je = min(a.n, jb + a.j_chunk);
    for (int64_t j0 = jb; j0 < je; j0 += JT) {
#pragma unroll
        for (int r = 0; r < JT / BLOCK; ++r) {
            const int jj = r * BLOCK + tid;
            const int64_t j = j0 + jj;
            const bool in = j < je;
            sx[jj] = in ? (T)(a.x[j] - org[0]) : (T)0;
            sy[jj] = in ? (T)(a.y[j] - org[1]) : (T)0;
            sz[jj] = in ? (T)(a.z[j] - org[2]) : (T)0;
            sm[jj] = in ? (T)a.m[j] : (T)0;
            sl[0][jj] = in ? (T)a.lx[j] : (T)0;
            sl[1][jj] = in ? (T)a.ly[j] : (T)0;
            sl[2][jj] = in ? (T)a.lz[j] : (T)0;
        }
        __syncthreads();
        T p[IPT][4];
#pragma unroll
        for (int k = 0; k < IPT; ++k)
#pragma unroll
            for (int c = 0; c < 4; ++c) p[k][c] = (T)0;
#pragma unroll 2
        for (int jj = 0; jj < JT; ++jj) {
            const T qx = sx[jj], qy = sy[jj], qz = sz[jj], qm = sm[jj];
            const T l0 = sl[0][jj], l1 = sl[1][jj], l2 = sl[2][jj];
#pragma unroll
            for (int k = 0; k < IPT; ++k) {
                const T dx = qx - xk[k], dy = qy - yk[k], dz = qz - zk[k];
                T s = dx * dx + e2;
                s = dy * dy + s;
                s = dz * dz + s;
                T y;
                if constexpr (MIXED) y = rsqrt_f32(s);
                else y = rsqrt_f64(s);
                if (EPS0) y = (s == (T)0) ? (T)0 : y;
                const T y2 = y * y;
                const T i3 = y2 * y;
                const T i5 = i3 * y2;
                const T ljd = l0 * dx + l1 * dy + l2 * dz;
                const T lkd = lk[k][0] * dx + lk[k][1] * dy + lk[k][2] * dz;
                const T A0 = mk[k] * l0 - qm * lk[k][0];
                const T A1 = mk[k] * l1 - qm * lk[k][1];
                const T A2 = mk[k] * l2 - qm * lk[k][2];
                const T B = mk[k] * ljd - qm * lkd;
                const T c3 = (T)3 * i5 * B;
                p[k][0] += i3 * A0 - c3 * dx;
                p[k][1] += i3 * A1 - c3 * dy;
                p[k][2] += i3 * A2 - c3 * dz;
                p[k][3] += i3 * ljd;
            }
        }
#pragma unroll
        for (int k = 0; k < IPT; ++k)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                if constexpr (MIXED) comp[k][c].add((float)p[k][c]);
                else acc[k][c] += (double)p[k][c];
            }
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const int64_t t = t0 + k * BLOCK + tid;
        if (t >= a.n) continue;
        double v[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) v[c] = MIXED ? comp[k][c].value() : acc[k][c];
        if (a.nsplit == 1) {
            a.gx[t] = a.G * v[0];
            a.gy[t] = a.G * v[1];
            a.gz[t] = a.G * v[2];
            if (a.gm) a.gm[t] = -a.G * v[3];
        } else {
            const size_t base = (size_t)blockIdx.y * 4 * (size_t)a.n + (size_t)t;
#pragma unroll
            for (int c = 0; c < 4; ++c) a.part[base + (size_t)c * (size_t)a.n] = v[c];
        }
    }
}

__global__ void vjp_reduce_kernel(const VjpArgs a) {
    const int64_t t = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (t >= a.n) return;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int c = 0; c < a.nsplit; ++c) {
        const size_t base = (size_t)c * 4 * (size_t)a.n + (size_t)t;
        for (int q = 0; q < 4; ++q) s[q] += a.part[base + (size_t)q * (size_t)a.n];
    }
    a.gx[t] = a.G * s[0];
    a.gy[t] = a.G * s[1];
    a.gz[t] = a.G * s[2];
    if (a.gm) a.gm[t] = -a.G * s[3];
}

template <int BLOCK, int IPT, int JT, bool MIXED>
cudaError_t launch_shape(const VjpArgs& a, bool eps0, cudaStream_t st) {
    const int64_t tile = (int64_t)BLOCK * IPT;
    dim3 grid((unsigned)((a.n + tile - 1) / tile), (unsigned)a.nsplit);
    if (eps0)
        vjp_kernel<BLOCK, IPT, JT, MIXED, true><<<grid, BLOCK, 0, st>>>(a);
    else
        vjp_kernel<BLOCK, IPT, JT, MIXED, false><<<grid, BLOCK, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace

int vjp_tile(int precision) { return precision == kMixed ? 256 * 2 : 128 * 2; }
int vjp_jt(int precision) { return precision == kMixed ? 512 : 256; }

cudaError_t launch_vjp(const VjpArgs& a, int precision, cudaStream_t st) {
    if (a.n <= 0) return cudaSuccess;
    cudaError_t e;
    if (precision == kMixed)
        e = launch_shape<256, 2, 512, true>(a, a.eps2f < 1e-24f, st);
    else
        e = launch_shape<128, 2, 256, false>(a, a.eps2 < 1e-200, st);
    if (e != cudaSuccess || a.nsplit <= 1) return e;
    vjp_reduce_kernel<<<(unsigned)((a.n + 255) / 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace gx
