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

// Mixed precision, two TARGETS per packed .f32x2 lane pair (sources pre-duplicated in shared
// memory as (x,x,y,y) (z,z,m,m) (l0,l0,l1,l1) (l2,l2,-,-)).  Per source and target pair: 31
// packed FP32 instructions + 2 MUFU rsqrt.  The two gradient terms are accumulated apart,
// G = sum s^-3/2 A and W = sum s^-5/2 (A.d) d, and combined as G - 3W in the epilogue (FP64).
template <int BLOCK, int IPT, int JT, bool EPS0>
__global__ void __launch_bounds__(BLOCK) vjp_mixed_tp_kernel(const VjpArgs a) {
    static_assert(JT % BLOCK == 0 && IPT % 2 == 0, "tile shape");
    constexpr int NP = IPT / 2;
    __shared__ __align__(16) float4 sS[JT][4];
    __shared__ double sred[6][BLOCK / 32];

    const int tid = threadIdx.x;
    const int64_t t0 = (int64_t)blockIdx.x * (BLOCK * IPT);
    int64_t idx[IPT];
    double bx[IPT], by[IPT], bz[IPT];
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const int64_t t = t0 + k * BLOCK + tid;
        idx[k] = t < a.n ? t : t0;
        bx[k] = a.x[idx[k]];
        by[k] = a.y[idx[k]];
        bz[k] = a.z[idx[k]];
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
    double org[3];
    for (int c = 0; c < 3; ++c) {
        double l = sred[c][0], h = sred[3 + c][0];
        for (int w = 1; w < BLOCK / 32; ++w) {
            l = fmin(l, sred[c][w]);
            h = fmax(h, sred[3 + c][w]);
        }
        org[c] = 0.5 * (l + h);
    }
    // target-pair constants
    f2 XK[NP], YK[NP], ZK[NP], MK[NP], NL0[NP], NL1[NP], NL2[NP];
#pragma unroll
    for (int q = 0; q < NP; ++q) {
        const int k0 = 2 * q, k1 = 2 * q + 1;
        XK[q] = pk2(__double2float_rn(bx[k0] - org[0]), __double2float_rn(bx[k1] - org[0]));
        YK[q] = pk2(__double2float_rn(by[k0] - org[1]), __double2float_rn(by[k1] - org[1]));
        ZK[q] = pk2(__double2float_rn(bz[k0] - org[2]), __double2float_rn(bz[k1] - org[2]));
        MK[q] = pk2(__double2float_rn(a.m[idx[k0]]), __double2float_rn(a.m[idx[k1]]));
        NL0[q] = pk2(-__double2float_rn(a.lx[idx[k0]]), -__double2float_rn(a.lx[idx[k1]]));
        NL1[q] = pk2(-__double2float_rn(a.ly[idx[k0]]), -__double2float_rn(a.ly[idx[k1]]));
        NL2[q] = pk2(-__double2float_rn(a.lz[idx[k0]]), -__double2float_rn(a.lz[idx[k1]]));
    }
    // compensated per-target accumulators: G (3), W (3), H (1)
    CompF acc[IPT][7];
#pragma unroll
    for (int k = 0; k < IPT; ++k)
#pragma unroll
        for (int c = 0; c < 7; ++c) acc[k][c].init();
    const f2 E2 = pk2(a.eps2f, a.eps2f);
    const f2 Z0 = pk2(0.f, 0.f);
    const int64_t jb = (int64_t)blockIdx.y * a.j_chunk;
    const int64_t je = min(a.n, jb + a.j_chunk);
    for (int64_t j0 = jb; j0 < je; j0 += JT) {
#pragma unroll
        for (int r = 0; r < JT / BLOCK; ++r) {
            const int jj = r * BLOCK + tid;
            const int64_t j = j0 + jj;
            float qx = 0.f, qy = 0.f, qz = 0.f, qm = 0.f, l0 = 0.f, l1 = 0.f, l2 = 0.f;
            if (j < je) {
                qx = __double2float_rn(a.x[j] - org[0]);
                qy = __double2float_rn(a.y[j] - org[1]);
                qz = __double2float_rn(a.z[j] - org[2]);
                qm = __double2float_rn(a.m[j]);
                l0 = __double2float_rn(a.lx[j]);
                l1 = __double2float_rn(a.ly[j]);
                l2 = __double2float_rn(a.lz[j]);
            }
            sS[jj][0] = make_float4(qx, qx, qy, qy);
            sS[jj][1] = make_float4(qz, qz, qm, qm);
            sS[jj][2] = make_float4(l0, l0, l1, l1);
            sS[jj][3] = make_float4(l2, l2, 0.f, 0.f);
        }
        __syncthreads();
        f2 G[NP][3], W[NP][3], H[NP];
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            G[q][0] = G[q][1] = G[q][2] = Z0;
            W[q][0] = W[q][1] = W[q][2] = Z0;
            H[q] = Z0;
        }
#pragma unroll 2
        for (int jj = 0; jj < JT; ++jj) {
            f2 X, Y, Z, M, L0, L1, L2, U;
            lds_v2b64(reinterpret_cast<const float*>(&sS[jj][0]), X, Y);
            lds_v2b64(reinterpret_cast<const float*>(&sS[jj][1]), Z, M);
            lds_v2b64(reinterpret_cast<const float*>(&sS[jj][2]), L0, L1);
            lds_v2b64(reinterpret_cast<const float*>(&sS[jj][3]), L2, U);
#pragma unroll
            for (int q = 0; q < NP; ++q) {
                const f2 dX = sub2(X, XK[q]), dY = sub2(Y, YK[q]), dZ = sub2(Z, ZK[q]);
                f2 S = fma2(dX, dX, E2);
                S = fma2(dY, dY, S);
                S = fma2(dZ, dZ, S);
                float s0, s1;
                upk2(S, s0, s1);
                float y0 = rsqrt_f32(s0), y1 = rsqrt_f32(s1);
                if (EPS0) {
                    y0 = (s0 == 0.f) ? 0.f : y0;
                    y1 = (s1 == 0.f) ? 0.f : y1;
                }
                const f2 Yv = pk2(y0, y1);
                const f2 Y2 = mul2(Yv, Yv);
                const f2 I3 = mul2(Y2, Yv);
                const f2 I5 = mul2(I3, Y2);
                f2 LJD = mul2(L0, dX);                  // l_j . d
                LJD = fma2(L1, dY, LJD);
                LJD = fma2(L2, dZ, LJD);
                f2 NLKD = mul2(NL0[q], dX);              // -(l_k . d)
                NLKD = fma2(NL1[q], dY, NLKD);
                NLKD = fma2(NL2[q], dZ, NLKD);
                const f2 A0 = fma2(MK[q], L0, mul2(M, NL0[q]));  // m_k l_j - m_j l_k
                const f2 A1 = fma2(MK[q], L1, mul2(M, NL1[q]));
                const f2 A2 = fma2(MK[q], L2, mul2(M, NL2[q]));
                const f2 B = fma2(MK[q], LJD, mul2(M, NLKD));     // A . d
                const f2 C = mul2(I5, B);
                G[q][0] = fma2(I3, A0, G[q][0]);
                G[q][1] = fma2(I3, A1, G[q][1]);
                G[q][2] = fma2(I3, A2, G[q][2]);
                W[q][0] = fma2(C, dX, W[q][0]);
                W[q][1] = fma2(C, dY, W[q][1]);
                W[q][2] = fma2(C, dZ, W[q][2]);
                H[q] = fma2(I3, LJD, H[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            float v0, v1;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                upk2(G[q][c], v0, v1);
                acc[2 * q][c].add(v0);
                acc[2 * q + 1][c].add(v1);
                upk2(W[q][c], v0, v1);
                acc[2 * q][3 + c].add(v0);
                acc[2 * q + 1][3 + c].add(v1);
            }
            upk2(H[q], v0, v1);
            acc[2 * q][6].add(v0);
            acc[2 * q + 1][6].add(v1);
        }
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const int64_t t = t0 + k * BLOCK + tid;
        if (t >= a.n) continue;
        double v[4];
#pragma unroll
        for (int c = 0; c < 3; ++c) v[c] = acc[k][c].value() - 3.0 * acc[k][3 + c].value();
        v[3] = acc[k][6].value();
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

template <int BLOCK, int IPT, int JT>
cudaError_t launch_mixed_tp(const VjpArgs& a, bool eps0, cudaStream_t st) {
    const int64_t tile = (int64_t)BLOCK * IPT;
    dim3 grid((unsigned)((a.n + tile - 1) / tile), (unsigned)a.nsplit);
    if (eps0)
        vjp_mixed_tp_kernel<BLOCK, IPT, JT, true><<<grid, BLOCK, 0, st>>>(a);
    else
        vjp_mixed_tp_kernel<BLOCK, IPT, JT, false><<<grid, BLOCK, 0, st>>>(a);
    return cudaGetLastError();
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

int vjp_tile(int precision) { return precision == kMixed ? 128 * 4 : 128 * 2; }
int vjp_jt(int precision) { return precision == kMixed ? 256 : 256; }

VjpShape vjp_shape(int precision) {
    static int occ[2] = {0, 0};
    const int k = precision == kMixed ? 1 : 0;
    if (occ[k] == 0) {
        int nb = 0;
        const cudaError_t e = k ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                      &nb, vjp_mixed_tp_kernel<128, 4, 256, false>, 128, 0)
                                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                      &nb, vjp_kernel<128, 2, 256, false, false>, 128, 0);
        if (e != cudaSuccess || nb < 1) {
            cudaGetLastError();
            nb = 1;
        }
        occ[k] = nb;
    }
    return k ? VjpShape{128, 4, 256, occ[1]} : VjpShape{128, 2, 256, occ[0]};
}

cudaError_t launch_vjp(const VjpArgs& a, int precision, cudaStream_t st) {
    if (a.n <= 0) return cudaSuccess;
    cudaError_t e;
    if (precision == kMixed)
        e = launch_mixed_tp<128, 4, 256>(a, a.eps2f < 1e-24f, st);
    else
        e = launch_shape<128, 2, 256, false>(a, a.eps2 < 1e-200, st);
    if (e != cudaSuccess || a.nsplit <= 1) return e;
    vjp_reduce_kernel<<<(unsigned)((a.n + 255) / 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace gx
