// force_tile.cuh -- per-tile bodies of the direct-sum kernels, shared by the one-system
// kernels (force.cu) and the persistent batched kernels (batch.cu).
//
// Pair term of the reference (cpp/direct/direct_solver.cpp:8-23, cpp/cuda/cuda_solver.cu:63-106):
//     a_i = G * sum_{j != i} m_j (x_j - x_i) / (|x_j - x_i|^2 + eps^2)^(3/2)
//
// A tile is BLOCK*IPT consecutive target ordinals [t0, t0 + BLOCK*IPT) held in registers
// (IPT per thread); the sources of one chunk stream through shared memory JT at a time and
// every shared-memory load of a source is reused by IPT targets.  Three arithmetic forms:
//   * mixed  -- sources are staged as FP32 offsets from an FP64 origin (the centre of the
//               bounding box of the tile's targets); the pair term runs in FP32 (12 FP32
//               FMA-pipe operations + 1 MUFU rsqrt per interaction), two sources per
//               packed .f32x2 instruction; the per-j-tile FP32 partial sums are folded into a
//               compensated (TwoSum) accumulator; the result is FP64.
//   * f64    -- FP64 pair term with a refined hardware rsqrt (17 FP64 pipe operations).
//   * exact  -- FP64 with the reference's operation order, IEEE sqrt and division and no
//               contraction; j ascending, i == j skipped: bit-identical to
//               compute_direct_accelerations_for_targets (direct_solver.cpp:59-83).
// A self pair (same body as target and source) has a zero offset and so adds exactly 0
// when eps > 0; with eps == 0 the eps0 variants select s == 0 pairs away, as the
// reference's `if (s2 == 0.0)` does.
//
// Every function here contains __syncthreads(): call it with block-uniform arguments.
#pragma once

#include "force.cuh"
#include "gx_device.cuh"

#include <cfloat>

namespace gx {


// Body index of target ordinal t.  An index-list entry outside [0, n_src) (device index
// arrays are not checked on the host) is replaced by body 0 for the loads, and
// write_result() stores NaN for that target instead of its sum.
__device__ __forceinline__ bool target_ok(const ForceArgs& a, int64_t t) {
    if (!a.tgt_idx) return true;
    const int64_t i = a.tgt_idx[t];
    return i >= 0 && i < a.n_src;
}

__device__ __forceinline__ int64_t target_body(const ForceArgs& a, int64_t t) {
    if (!a.tgt_idx) return a.t_begin + t;
    const int64_t i = a.tgt_idx[t];
    return (i >= 0 && i < a.n_src) ? i : 0;
}

// Final FP64 result of target t (body index `body`): store, then the optional closing kick
// v += a*dt in the reference's rounding (integrator.cpp:7-11, no contraction).
__device__ __forceinline__ void write_result(const ForceArgs& a, int64_t t, int64_t body,
                                             double fx, double fy, double fz) {
    if (!target_ok(a, t)) {
        a.ax[t] = a.ay[t] = a.az[t] = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    a.ax[t] = fx;
    a.ay[t] = fy;
    a.az[t] = fz;
    if (a.vx) {
        a.vx[body] = dadd(a.vx[body], dmul(fx, a.kick_dt));
        a.vy[body] = dadd(a.vy[body], dmul(fy, a.kick_dt));
        a.vz[body] = dadd(a.vz[body], dmul(fz, a.kick_dt));
    }
}

__device__ __forceinline__ void write_partial(const ForceArgs& a, int chunk, int64_t t, double sx,
                                              double sy, double sz) {
    const size_t base = (size_t)chunk * 3 * (size_t)a.n_tgt + (size_t)t;
    a.part[base] = sx;
    a.part[base + (size_t)a.n_tgt] = sy;
    a.part[base + 2 * (size_t)a.n_tgt] = sz;
}


// ---------------------------------------------------------------------------------------
// Mixed precision.
// ---------------------------------------------------------------------------------------
template <int BLOCK, int IPT, int JT, bool PACKED, bool EPS0>
__device__ __forceinline__ void mixed_tile(const ForceArgs& a, const int64_t t0, const int chunk) {
    static_assert(JT % BLOCK == 0 && JT % 4 == 0 && BLOCK % 32 == 0, "tile shape");
    constexpr int NW = BLOCK / 32;
    __shared__ __align__(16) float sx[JT];
    __shared__ __align__(16) float sy[JT];
    __shared__ __align__(16) float sz[JT];
    __shared__ __align__(16) float sm[JT];
    __shared__ double sred[6][NW];

    const int tid = threadIdx.x;
    const int64_t first_body = target_body(a, t0);

    double bx[IPT], by[IPT], bz[IPT];
    int64_t body[IPT];
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const int64_t t = t0 + k * BLOCK + tid;
        body[k] = t < a.n_tgt ? target_body(a, t) : first_body;
        bx[k] = a.x[body[k]];
        by[k] = a.y[body[k]];
        bz[k] = a.z[body[k]];
        lo[0] = fmin(lo[0], bx[k]); hi[0] = fmax(hi[0], bx[k]);
        lo[1] = fmin(lo[1], by[k]); hi[1] = fmax(hi[1], by[k]);
        lo[2] = fmin(lo[2], bz[k]); hi[2] = fmax(hi[2], bz[k]);
    }
    // Origin of the tile: centre of the bounding box of its targets (padding lanes repeat
    // a real target, so they do not widen the box).
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        lo[c] = warp_min(lo[c]);
        hi[c] = warp_max(hi[c]);
    }
    if ((tid & 31) == 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            sred[c][tid >> 5] = lo[c];
            sred[3 + c][tid >> 5] = hi[c];
        }
    }
    __syncthreads();
    double org[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double l = sred[c][0], h = sred[3 + c][0];
#pragma unroll
        for (int w = 1; w < NW; ++w) {
            l = fmin(l, sred[c][w]);
            h = fmax(h, sred[3 + c][w]);
        }
        org[c] = 0.5 * (l + h);
    }

    float xi[IPT], yi[IPT], zi[IPT];
    CompF cx[IPT], cy[IPT], cz[IPT];
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        xi[k] = __double2float_rn(bx[k] - org[0]);
        yi[k] = __double2float_rn(by[k] - org[1]);
        zi[k] = __double2float_rn(bz[k] - org[2]);
        cx[k].init();
        cy[k].init();
        cz[k].init();
    }

    const int64_t jb = (int64_t)chunk * a.j_chunk;
    const int64_t je = min(a.n_src, jb + a.j_chunk);
    const float e2 = a.eps2f;

    for (int64_t j0 = jb; j0 < je; j0 += JT) {
#pragma unroll
        for (int r = 0; r < JT / BLOCK; ++r) {
            const int jj = r * BLOCK + tid;
            const int64_t j = j0 + jj;
            float qx = 0.f, qy = 0.f, qz = 0.f, qm = 0.f;
            if (j < je) {
                qx = __double2float_rn(a.x[j] - org[0]);
                qy = __double2float_rn(a.y[j] - org[1]);
                qz = __double2float_rn(a.z[j] - org[2]);
                qm = __double2float_rn(a.m[j]);
            }
            sx[jj] = qx;
            sy[jj] = qy;
            sz[jj] = qz;
            sm[jj] = qm;
        }
        __syncthreads();

        if constexpr (PACKED) {
            f2 XI[IPT], YI[IPT], ZI[IPT], PX[IPT], PY[IPT], PZ[IPT];
            const f2 E2 = pk2(e2, e2);
            const f2 Z0 = pk2(0.f, 0.f);
#pragma unroll
            for (int k = 0; k < IPT; ++k) {
                XI[k] = pk2(xi[k], xi[k]);
                YI[k] = pk2(yi[k], yi[k]);
                ZI[k] = pk2(zi[k], zi[k]);
                PX[k] = Z0;
                PY[k] = Z0;
                PZ[k] = Z0;
            }
#pragma unroll 2
            for (int jj = 0; jj < JT; jj += 4) {
                f2 X[2], Y[2], Z[2], M[2];
                lds_v2b64(sx + jj, X[0], X[1]);
                lds_v2b64(sy + jj, Y[0], Y[1]);
                lds_v2b64(sz + jj, Z[0], Z[1]);
                lds_v2b64(sm + jj, M[0], M[1]);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
#pragma unroll
                    for (int k = 0; k < IPT; ++k) {
                        const f2 dX = sub2(X[h], XI[k]);
                        const f2 dY = sub2(Y[h], YI[k]);
                        const f2 dZ = sub2(Z[h], ZI[k]);
                        f2 R = fma2(dX, dX, E2);
                        R = fma2(dY, dY, R);
                        R = fma2(dZ, dZ, R);
                        float r0, r1;
                        upk2(R, r0, r1);
                        float i0 = rsqrt_f32(r0), i1 = rsqrt_f32(r1);
                        if (EPS0) {
                            i0 = (r0 == 0.f) ? 0.f : i0;
                            i1 = (r1 == 0.f) ? 0.f : i1;
                        }
                        const f2 I = pk2(i0, i1);
                        f2 T = mul2(I, I);
                        T = mul2(T, I);
                        const f2 W = mul2(M[h], T);
                        PX[k] = fma2(dX, W, PX[k]);
                        PY[k] = fma2(dY, W, PY[k]);
                        PZ[k] = fma2(dZ, W, PZ[k]);
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < IPT; ++k) {
                float l0, l1;
                upk2(PX[k], l0, l1);
                cx[k].add(l0 + l1);
                upk2(PY[k], l0, l1);
                cy[k].add(l0 + l1);
                upk2(PZ[k], l0, l1);
                cz[k].add(l0 + l1);
            }
        } else {
            float px[IPT], py[IPT], pz[IPT];
#pragma unroll
            for (int k = 0; k < IPT; ++k) px[k] = py[k] = pz[k] = 0.f;
#pragma unroll 4
            for (int jj = 0; jj < JT; ++jj) {
                const float qx = sx[jj], qy = sy[jj], qz = sz[jj], qm = sm[jj];
#pragma unroll
                for (int k = 0; k < IPT; ++k) {
                    const float dx = qx - xi[k], dy = qy - yi[k], dz = qz - zi[k];
                    float r = fmaf(dx, dx, e2);
                    r = fmaf(dy, dy, r);
                    r = fmaf(dz, dz, r);
                    float iv = rsqrt_f32(r);
                    if (EPS0) iv = (r == 0.f) ? 0.f : iv;
                    const float w = qm * (iv * iv * iv);
                    px[k] = fmaf(dx, w, px[k]);
                    py[k] = fmaf(dy, w, py[k]);
                    pz[k] = fmaf(dz, w, pz[k]);
                }
            }
#pragma unroll
            for (int k = 0; k < IPT; ++k) {
                cx[k].add(px[k]);
                cy[k].add(py[k]);
                cz[k].add(pz[k]);
            }
        }
        __syncthreads();
    }

#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const int64_t t = t0 + k * BLOCK + tid;
        if (t >= a.n_tgt) continue;
        if (a.nsplit == 1)
            write_result(a, t, body[k], a.G * cx[k].value(), a.G * cy[k].value(), a.G * cz[k].value());
        else
            write_partial(a, chunk, t, cx[k].value(), cy[k].value(), cz[k].value());
    }
}

// ---------------------------------------------------------------------------------------
// Mixed precision, targets packed: the same arithmetic as mixed_tile, but each packed
// .f32x2 instruction serves two TARGETS against one source.  Sources are staged in shared
// memory already duplicated ((x, x, y, y), (z, z, m, m): two 16-byte loads per source), so a
// target pair keeps one 64-bit register per coordinate and per accumulator instead of two:
// 6 registers fewer per target, which buys occupancy or more targets per thread.
// ---------------------------------------------------------------------------------------
template <int BLOCK, int IPT, int JT, bool EPS0, int UNROLL = 4>
__device__ __forceinline__ void mixed_tp_tile(const ForceArgs& a, const int64_t t0, const int chunk) {
    static_assert(JT % BLOCK == 0 && BLOCK % 32 == 0 && IPT % 2 == 0, "tile shape");
    constexpr int NW = BLOCK / 32;
    constexpr int NP = IPT / 2;
    __shared__ __align__(16) float4 sA[JT];  // (x, x, y, y)
    __shared__ __align__(16) float4 sB[JT];  // (z, z, m, m)
    __shared__ double sred[6][NW];

    const int tid = threadIdx.x;
    const int64_t first_body = target_body(a, t0);
    double bx[IPT], by[IPT], bz[IPT];
    int64_t body[IPT];
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const int64_t t = t0 + k * BLOCK + tid;
        body[k] = t < a.n_tgt ? target_body(a, t) : first_body;
        bx[k] = a.x[body[k]];
        by[k] = a.y[body[k]];
        bz[k] = a.z[body[k]];
        lo[0] = fmin(lo[0], bx[k]); hi[0] = fmax(hi[0], bx[k]);
        lo[1] = fmin(lo[1], by[k]); hi[1] = fmax(hi[1], by[k]);
        lo[2] = fmin(lo[2], bz[k]); hi[2] = fmax(hi[2], bz[k]);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        lo[c] = warp_min(lo[c]);
        hi[c] = warp_max(hi[c]);
    }
    if ((tid & 31) == 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            sred[c][tid >> 5] = lo[c];
            sred[3 + c][tid >> 5] = hi[c];
        }
    }
    __syncthreads();
    double org[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double l = sred[c][0], h = sred[3 + c][0];
#pragma unroll
        for (int w = 1; w < NW; ++w) {
            l = fmin(l, sred[c][w]);
            h = fmax(h, sred[3 + c][w]);
        }
        org[c] = 0.5 * (l + h);
    }

    f2 XI[NP], YI[NP], ZI[NP];
    CompF cx[IPT], cy[IPT], cz[IPT];
#pragma unroll
    for (int q = 0; q < NP; ++q) {
        XI[q] = pk2(__double2float_rn(bx[2 * q] - org[0]), __double2float_rn(bx[2 * q + 1] - org[0]));
        YI[q] = pk2(__double2float_rn(by[2 * q] - org[1]), __double2float_rn(by[2 * q + 1] - org[1]));
        ZI[q] = pk2(__double2float_rn(bz[2 * q] - org[2]), __double2float_rn(bz[2 * q + 1] - org[2]));
    }
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        cx[k].init();
        cy[k].init();
        cz[k].init();
    }

    const int64_t jb = (int64_t)chunk * a.j_chunk;
    const int64_t je = min(a.n_src, jb + a.j_chunk);
    const f2 E2 = pk2(a.eps2f, a.eps2f);
    const f2 Z0 = pk2(0.f, 0.f);

    for (int64_t j0 = jb; j0 < je; j0 += JT) {
#pragma unroll
        for (int r = 0; r < JT / BLOCK; ++r) {
            const int jj = r * BLOCK + tid;
            const int64_t j = j0 + jj;
            float qx = 0.f, qy = 0.f, qz = 0.f, qm = 0.f;
            if (j < je) {
                qx = __double2float_rn(a.x[j] - org[0]);
                qy = __double2float_rn(a.y[j] - org[1]);
                qz = __double2float_rn(a.z[j] - org[2]);
                qm = __double2float_rn(a.m[j]);
            }
            sA[jj] = make_float4(qx, qx, qy, qy);
            sB[jj] = make_float4(qz, qz, qm, qm);
        }
        __syncthreads();
        f2 PX[NP], PY[NP], PZ[NP];
#pragma unroll
        for (int q = 0; q < NP; ++q) PX[q] = PY[q] = PZ[q] = Z0;
#pragma unroll UNROLL
        for (int jj = 0; jj < JT; ++jj) {
            f2 X, Y, Z, M;
            lds_v2b64(reinterpret_cast<const float*>(&sA[jj]), X, Y);
            lds_v2b64(reinterpret_cast<const float*>(&sB[jj]), Z, M);
#pragma unroll
            for (int q = 0; q < NP; ++q) {
                const f2 dX = sub2(X, XI[q]);
                const f2 dY = sub2(Y, YI[q]);
                const f2 dZ = sub2(Z, ZI[q]);
                f2 R = fma2(dX, dX, E2);
                R = fma2(dY, dY, R);
                R = fma2(dZ, dZ, R);
                float r0, r1;
                upk2(R, r0, r1);
                float i0 = rsqrt_f32(r0), i1 = rsqrt_f32(r1);
                if (EPS0) {
                    i0 = (r0 == 0.f) ? 0.f : i0;
                    i1 = (r1 == 0.f) ? 0.f : i1;
                }
                const f2 I = pk2(i0, i1);
                f2 T = mul2(I, I);
                T = mul2(T, I);
                const f2 W = mul2(M, T);
                PX[q] = fma2(dX, W, PX[q]);
                PY[q] = fma2(dY, W, PY[q]);
                PZ[q] = fma2(dZ, W, PZ[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            float p0, p1;
            upk2(PX[q], p0, p1);
            cx[2 * q].add(p0);
            cx[2 * q + 1].add(p1);
            upk2(PY[q], p0, p1);
            cy[2 * q].add(p0);
            cy[2 * q + 1].add(p1);
            upk2(PZ[q], p0, p1);
            cz[2 * q].add(p0);
            cz[2 * q + 1].add(p1);
        }
        __syncthreads();
    }

#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const int64_t t = t0 + k * BLOCK + tid;
        if (t >= a.n_tgt) continue;
        if (a.nsplit == 1)
            write_result(a, t, body[k], a.G * cx[k].value(), a.G * cy[k].value(), a.G * cz[k].value());
        else
            write_partial(a, chunk, t, cx[k].value(), cy[k].value(), cz[k].value());
    }
}

// ---------------------------------------------------------------------------------------
// FP64 with a refined hardware rsqrt.
// ---------------------------------------------------------------------------------------
template <int BLOCK, int IPT, int JT, bool EPS0>
__device__ __forceinline__ void f64_tile(const ForceArgs& a, const int64_t t0, const int chunk) {
    static_assert(JT % BLOCK == 0 && JT % 2 == 0, "tile shape");
    __shared__ __align__(16) double sx[JT];
    __shared__ __align__(16) double sy[JT];
    __shared__ __align__(16) double sz[JT];
    __shared__ __align__(16) double sm[JT];

    const int tid = threadIdx.x;
    const int64_t first_body = target_body(a, t0);
    double xi[IPT], yi[IPT], zi[IPT], fx[IPT], fy[IPT], fz[IPT];
    int64_t body[IPT];
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const int64_t t = t0 + k * BLOCK + tid;
        body[k] = t < a.n_tgt ? target_body(a, t) : first_body;
        xi[k] = a.x[body[k]];
        yi[k] = a.y[body[k]];
        zi[k] = a.z[body[k]];
        fx[k] = fy[k] = fz[k] = 0.0;
    }
    const int64_t jb = (int64_t)chunk * a.j_chunk;
    const int64_t je = min(a.n_src, jb + a.j_chunk);
    const double e2 = a.eps2;

    for (int64_t j0 = jb; j0 < je; j0 += JT) {
#pragma unroll
        for (int r = 0; r < JT / BLOCK; ++r) {
            const int jj = r * BLOCK + tid;
            const int64_t j = j0 + jj;
            const bool in = j < je;
            sx[jj] = in ? a.x[j] : 0.0;
            sy[jj] = in ? a.y[j] : 0.0;
            sz[jj] = in ? a.z[j] : 0.0;
            sm[jj] = in ? a.m[j] : 0.0;
        }
        __syncthreads();
#pragma unroll 4
        for (int jj = 0; jj < JT; ++jj) {
            const double qx = sx[jj], qy = sy[jj], qz = sz[jj], qm = sm[jj];
#pragma unroll
            for (int k = 0; k < IPT; ++k) {
                const double dx = qx - xi[k], dy = qy - yi[k], dz = qz - zi[k];
                double r = fma(dx, dx, e2);
                r = fma(dy, dy, r);
                r = fma(dz, dz, r);
                double y = rsqrt_f64(r);
                if (EPS0) y = (r == 0.0) ? 0.0 : y;
                const double w = qm * (y * y * y);
                fx[k] = fma(dx, w, fx[k]);
                fy[k] = fma(dy, w, fy[k]);
                fz[k] = fma(dz, w, fz[k]);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const int64_t t = t0 + k * BLOCK + tid;
        if (t >= a.n_tgt) continue;
        if (a.nsplit == 1)
            write_result(a, t, body[k], a.G * fx[k], a.G * fy[k], a.G * fz[k]);
        else
            write_partial(a, chunk, t, fx[k], fy[k], fz[k]);
    }
}

// ---------------------------------------------------------------------------------------
// FP64 in the reference's operation order (bit-identical to direct_solver.cpp:59-83).
// ---------------------------------------------------------------------------------------
template <int BLOCK, int JT>
__device__ __forceinline__ void exact_tile(const ForceArgs& a, const int64_t t0) {
    static_assert(JT % BLOCK == 0, "tile shape");
    __shared__ double sx[JT];
    __shared__ double sy[JT];
    __shared__ double sz[JT];
    __shared__ double sm[JT];
    const int tid = threadIdx.x;
    const int64_t t = t0 + tid;
    const int64_t body = target_body(a, t < a.n_tgt ? t : t0);
    const double xi = a.x[body], yi = a.y[body], zi = a.z[body];
    const double G = a.G, e2 = a.eps2;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int64_t j0 = 0; j0 < a.n_src; j0 += JT) {
#pragma unroll
        for (int r = 0; r < JT / BLOCK; ++r) {
            const int jj = r * BLOCK + tid;
            const int64_t j = j0 + jj;
            if (j < a.n_src) {
                sx[jj] = a.x[j];
                sy[jj] = a.y[j];
                sz[jj] = a.z[j];
                sm[jj] = a.m[j];
            }
        }
        __syncthreads();
        const int cnt = (int)min((int64_t)JT, a.n_src - j0);
        for (int jj = 0; jj < cnt; ++jj) {
            if (j0 + jj == body) continue;
            const double rx = dsub(sx[jj], xi), ry = dsub(sy[jj], yi), rz = dsub(sz[jj], zi);
            const double s2 = dadd(dadd(dadd(dmul(rx, rx), dmul(ry, ry)), dmul(rz, rz)), e2);
            if (s2 == 0.0) {  // softened_acceleration returns {} and the caller adds it
                fx = dadd(fx, 0.0);
                fy = dadd(fy, 0.0);
                fz = dadd(fz, 0.0);
                continue;
            }
            const double inv = __ddiv_rn(1.0, __dsqrt_rn(s2));
            const double inv3 = dmul(dmul(inv, inv), inv);
            const double scale = dmul(dmul(G, sm[jj]), inv3);
            fx = dadd(fx, dmul(rx, scale));
            fy = dadd(fy, dmul(ry, scale));
            fz = dadd(fz, dmul(rz, scale));
        }
        __syncthreads();
    }
    if (t < a.n_tgt) write_result(a, t, body, fx, fy, fz);
}

}  // namespace gx
