// p2p.cu -- FMM near-field (P2P) leaf kernel.
//
// Replaces the near loop of FastMultipoleSolver::evaluate_particle
// (cpp/fmm/fmm_solver.cpp:295-310): for every body i of a target leaf, the pair terms of
// all bodies j != i of the leaf's near leaves, in near-list order and leaf body order.
//
// One CTA per target leaf.  The bodies of the near leaves are gathered (by index, from the
// SoA state) into shared memory JT at a time.  In the fast forms each target is served by
// L adjacent lanes (L = 8, 4, 2, 1 for leaves of <= 16, 32, 64, more bodies) that split the
// staged sources and are combined with warp shuffles at the end, so small leaves still
// fill the CTA.  The exact form uses one lane per target and walks the sources in the
// reference's order starting from the incoming acceleration (the far field), which makes
// it bit-identical to the reference's evaluate_particle.
#include "gx_device.cuh"
#include "p2p.cuh"

namespace gx {
namespace {

constexpr int kP2PBlock = 128;
constexpr int kP2PJT = 256;

__device__ __forceinline__ int lanes_for(int nt) {
    return nt <= 16 ? 8 : nt <= 32 ? 4 : nt <= 64 ? 2 : 1;
}

template <int MODE, bool EPS0>
__global__ void __launch_bounds__(kP2PBlock) p2p_kernel(const P2PArgs a) {
    __shared__ __align__(16) double sxd[kP2PJT];
    __shared__ __align__(16) double syd[kP2PJT];
    __shared__ __align__(16) double szd[kP2PJT];
    __shared__ __align__(16) double smd[kP2PJT];
    __shared__ int sidx[kP2PJT];

    const int leaf = blockIdx.x;
    const int tid = threadIdx.x;
    const int tb = a.leaf_off[leaf];
    const int nt = a.leaf_off[leaf + 1] - tb;
    if (nt <= 0) return;  // block-uniform: an empty row has no targets
    const int nb = a.near_off[leaf], ne = a.near_off[leaf + 1];
    const int L = (MODE == kF64Exact) ? 1 : lanes_for(nt);
    const int slots = kP2PBlock / L;
    const int slot = tid / L, lane = tid % L;
    // Origin of the mixed form: the leaf's first body (near sources are close to it).
    const int first = a.leaf_part[tb];
    const double ox = a.x[first], oy = a.y[first], oz = a.z[first];

    for (int pass = 0; pass * slots < nt; ++pass) {
        const int t = pass * slots + slot;
        const bool ok = t < nt;
        const int i = ok ? a.leaf_part[tb + t] : first;
        const double xi = a.x[i], yi = a.y[i], zi = a.z[i];
        const float xf = __double2float_rn(xi - ox), yf = __double2float_rn(yi - oy),
                    zf = __double2float_rn(zi - oz);
        double fx = 0.0, fy = 0.0, fz = 0.0;
        if (MODE == kF64Exact && ok) {
            fx = a.ax[i];
            fy = a.ay[i];
            fz = a.az[i];
        }
        CompF cx, cy, cz;
        cx.init();
        cy.init();
        cz.init();

        int fill = 0;
        auto compute = [&](int cnt) {
            if (MODE == kF64Exact) {
                for (int jj = 0; jj < cnt; ++jj) {
                    if (sidx[jj] == i) continue;
                    const double rx = dsub(sxd[jj], xi), ry = dsub(syd[jj], yi), rz = dsub(szd[jj], zi);
                    const double s2 = dadd(dadd(dadd(dmul(rx, rx), dmul(ry, ry)), dmul(rz, rz)), a.eps2);
                    if (s2 == 0.0) {
                        fx = dadd(fx, 0.0);
                        fy = dadd(fy, 0.0);
                        fz = dadd(fz, 0.0);
                        continue;
                    }
                    const double inv = __ddiv_rn(1.0, __dsqrt_rn(s2));
                    const double inv3 = dmul(dmul(inv, inv), inv);
                    const double scale = dmul(dmul(a.G, smd[jj]), inv3);
                    fx = dadd(fx, dmul(rx, scale));
                    fy = dadd(fy, dmul(ry, scale));
                    fz = dadd(fz, dmul(rz, scale));
                }
            } else if (MODE == kF64) {
                for (int jj = lane; jj < cnt; jj += L) {
                    const double dx = sxd[jj] - xi, dy = syd[jj] - yi, dz = szd[jj] - zi;
                    double r = fma(dx, dx, a.eps2);
                    r = fma(dy, dy, r);
                    r = fma(dz, dz, r);
                    double y = rsqrt_f64(r);
                    if (EPS0) y = (r == 0.0 || sidx[jj] == i) ? 0.0 : y;
                    const double w = smd[jj] * (y * y * y);
                    fx = fma(dx, w, fx);
                    fy = fma(dy, w, fy);
                    fz = fma(dz, w, fz);
                }
            } else {
                float px = 0.f, py = 0.f, pz = 0.f;
                const float* sxf = reinterpret_cast<const float*>(sxd);
                const float* syf = reinterpret_cast<const float*>(syd);
                const float* szf = reinterpret_cast<const float*>(szd);
                const float* smf = reinterpret_cast<const float*>(smd);
                for (int jj = lane; jj < cnt; jj += L) {
                    const float dx = sxf[jj] - xf, dy = syf[jj] - yf, dz = szf[jj] - zf;
                    float r = fmaf(dx, dx, a.eps2f);
                    r = fmaf(dy, dy, r);
                    r = fmaf(dz, dz, r);
                    float iv = rsqrt_f32(r);
                    if (EPS0) iv = (r == 0.f || sidx[jj] == i) ? 0.f : iv;
                    const float w = smf[jj] * (iv * iv * iv);
                    px = fmaf(dx, w, px);
                    py = fmaf(dy, w, py);
                    pz = fmaf(dz, w, pz);
                }
                cx.add(px);
                cy.add(py);
                cz.add(pz);
            }
        };
        auto stage = [&](int slot_base, int j) {
            sidx[slot_base] = j;
            if (MODE == kMixed) {
                float* sxf = reinterpret_cast<float*>(sxd);
                float* syf = reinterpret_cast<float*>(syd);
                float* szf = reinterpret_cast<float*>(szd);
                float* smf = reinterpret_cast<float*>(smd);
                sxf[slot_base] = __double2float_rn(a.x[j] - ox);
                syf[slot_base] = __double2float_rn(a.y[j] - oy);
                szf[slot_base] = __double2float_rn(a.z[j] - oz);
                smf[slot_base] = __double2float_rn(a.m[j]);
            } else {
                sxd[slot_base] = a.x[j];
                syd[slot_base] = a.y[j];
                szd[slot_base] = a.z[j];
                smd[slot_base] = a.m[j];
            }
        };

        for (int q = nb; q < ne; ++q) {
            const int s = a.near_leaf[q];
            const int sb = a.leaf_off[s];
            const int ns = a.leaf_off[s + 1] - sb;
            int o = 0;
            while (o < ns) {
                const int take = min(ns - o, kP2PJT - fill);
                for (int c = tid; c < take; c += kP2PBlock) stage(fill + c, a.leaf_part[sb + o + c]);
                fill += take;
                o += take;
                if (fill == kP2PJT) {
                    __syncthreads();
                    compute(fill);
                    __syncthreads();
                    fill = 0;
                }
            }
        }
        if (fill > 0) {
            __syncthreads();
            compute(fill);
            __syncthreads();
        }

        if (MODE == kF64Exact) {
            if (ok) {
                a.ax[i] = fx;
                a.ay[i] = fy;
                a.az[i] = fz;
            }
        } else {
            if (MODE == kMixed) {
                fx = cx.value();
                fy = cy.value();
                fz = cz.value();
            }
            // Combine the L lanes of this target (adjacent lanes of one warp).
            for (int o = L >> 1; o > 0; o >>= 1) {
                fx += __shfl_xor_sync(0xffffffffu, fx, o);
                fy += __shfl_xor_sync(0xffffffffu, fy, o);
                fz += __shfl_xor_sync(0xffffffffu, fz, o);
            }
            if (ok && lane == 0) {
                a.ax[i] = a.ax[i] + a.G * fx;
                a.ay[i] = a.ay[i] + a.G * fy;
                a.az[i] = a.az[i] + a.G * fz;
            }
        }
    }
}

}  // namespace

cudaError_t launch_p2p(const P2PArgs& a, int precision, cudaStream_t st) {
    if (a.n_leaves <= 0) return cudaSuccess;
    const bool eps0 = precision == kMixed ? (a.eps2f < 1e-24f) : (a.eps2 < 1e-200);
    dim3 grid((unsigned)a.n_leaves);
    if (precision == kF64Exact)
        p2p_kernel<kF64Exact, false><<<grid, kP2PBlock, 0, st>>>(a);
    else if (precision == kF64)
        eps0 ? p2p_kernel<kF64, true><<<grid, kP2PBlock, 0, st>>>(a)
             : p2p_kernel<kF64, false><<<grid, kP2PBlock, 0, st>>>(a);
    else
        eps0 ? p2p_kernel<kMixed, true><<<grid, kP2PBlock, 0, st>>>(a)
             : p2p_kernel<kMixed, false><<<grid, kP2PBlock, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace gx
