// fmm.cu -- FMM far field on the device: leaf moments (P2M), the upward pass (M2M) and
// the multipole evaluation at every target (M2P).
//
// Moments.  FastMultipoleSolver::p2m_m2m / compute_multipole_moments
// (cpp/fmm/fmm_solver.cpp:157-208) with add_multipole_point / add_multipole_shifted_child
// (cpp/fmm/multipole.cpp:218-252) are restated with the reference's operations in the
// reference's order and no contraction (dadd/dmul), so masses, centres of mass and the 31
// moments of every node are bit-identical to the reference's (for masses >= 0).  One warp
// per node; lane k owns moment 4 + k.  Leaves first, then one launch per tree level,
// deepest first.
//
// M2P.  multipole_acceleration (multipole.cpp:254-296) builds the degree-4 Taylor
// polynomial of (d + u)_c |d + u|_eps^-3 in the source offset u by truncated polynomial
// products and contracts it with the moments.  Those Taylor coefficients are the
// Cartesian derivatives of the softened potential phi(r) = (r.r + eps^2)^-1/2:
//     a_c = -G sum_k 1/k! M^(k)_{i1..ik} d^(k+1) phi / dr_i1..dr_ik dr_c  at r = d,
// with d = centre of mass - target and M^(k) the raw k-th moment tensor (M^(0) = mass,
// M^(1) = 0 about the centre of mass).  Writing g_n = (-1)^n (2n-1)!! s^-(2n+1)/2,
// s = d.d + eps^2, the derivative tensors are sums of g_n times products of d's and
// Kronecker deltas, and the contraction per order is
//     k=0: -m g1 d
//     k=2: -1/2  [ g3 M[dd] d + g2 (tr M d + 2 M[d]) ]
//     k=3: -1/6  [ g4 O[ddd] d + g3 (3 (w.d) d + 3 O[dd]) + 3 g2 w ]
//     k=4: -1/24 [ g5 H[dddd] d + g4 (6 T2[dd] d + 4 H[ddd]) + g3 (3 tr2 d + 12 T2[d]) ]
// (w, T2, tr2 are the traces stored in the node record).  This is the same polynomial,
// evaluated in about 170 FP64 operations per (target, node) pair instead of the
// reference's polynomial algebra; only rounding differs.  Moments of degree above the
// effective order are left out exactly as evaluate_component does (:205-216).
#include "fmm.cuh"
#include "gx_device.cuh"

#include <algorithm>
#include <atomic>

namespace gx {
namespace {

constexpr int kMomBlock = 256;  // 8 warps, one node each
constexpr int kM2PBlock = 128;

// binomial (multipole.cpp:57-76) for n <= 4.
constexpr int binom4(int n, int k) {
    return (k < 0 || k > n) ? 0 : (k == 0 || k == n) ? 1 : n == 2 ? 2 : n == 3 ? 3 : (k == 2 ? 6 : 4);
}

constexpr int kMaxShiftTerms = 12;  // (2+1)(1+1)(1+1): the most multi-indices below a degree-4 one

// Index tables, evaluated at compile time.  Moment slot k (0..34) is the reference's
// exponent order (multipole.cpp:16-26): degree ascending, then the x exponent descending,
// then the y exponent descending.  For every moment alpha of degree 2..4 (slot 4 + a) the
// terms of add_multipole_shifted_child (multipole.cpp:227-252) in the reference's beta
// order: beta <= alpha componentwise, degree-1 betas left out (their moment is 0 about the
// child's centre of mass, and adding the zero product never changes a sum that starts at
// +0), each with the binomial product and the exponents of the shift.
struct MomentTables {
    int ex[35] = {}, ey[35] = {}, ez[35] = {};
    int nterm[31] = {};
    double bin[31][kMaxShiftTerms] = {};
    int kb[31][kMaxShiftTerms] = {}, dx[31][kMaxShiftTerms] = {}, dy[31][kMaxShiftTerms] = {},
        dz[31][kMaxShiftTerms] = {};
};

constexpr MomentTables make_moment_tables() {
    MomentTables t;
    int k = 0;
    for (int d = 0; d <= 4; ++d)
        for (int x = d; x >= 0; --x)
            for (int y = d - x; y >= 0; --y) {
                t.ex[k] = x;
                t.ey[k] = y;
                t.ez[k] = d - x - y;
                ++k;
            }
    for (int a = 0; a < 31; ++a) {
        const int ka = 4 + a, ax = t.ex[ka], ay = t.ey[ka], az = t.ez[ka];
        int n = 0;
        for (int b = 0; b < 35; ++b) {
            const int bx = t.ex[b], by = t.ey[b], bz = t.ez[b];
            if (bx > ax || by > ay || bz > az || bx + by + bz == 1) continue;
            t.bin[a][n] = (double)(binom4(ax, bx) * binom4(ay, by) * binom4(az, bz));
            t.kb[a][n] = b;
            t.dx[a][n] = ax - bx;
            t.dy[a][n] = ay - by;
            t.dz[a][n] = az - bz;
            ++n;
        }
        t.nterm[a] = n;
    }
    return t;
}

__device__ const MomentTables kTab = make_moment_tables();

// Traces of the moments (record slots 35..45) from slots 4..34.
__device__ __forceinline__ void write_traces(double* r) {
    r[kRecTrQ] = r[4] + r[7] + r[9];
    r[kRecW + 0] = r[10] + r[13] + r[15];
    r[kRecW + 1] = r[11] + r[16] + r[18];
    r[kRecW + 2] = r[12] + r[17] + r[19];
    const double txx = r[20] + r[23] + r[25], tyy = r[23] + r[30] + r[32], tzz = r[25] + r[32] + r[34];
    r[kRecT2 + 0] = txx;
    r[kRecT2 + 1] = r[21] + r[26] + r[28];
    r[kRecT2 + 2] = r[22] + r[27] + r[29];
    r[kRecT2 + 3] = tyy;
    r[kRecT2 + 4] = r[24] + r[31] + r[33];
    r[kRecT2 + 5] = tzz;
    r[kRecTr2] = txx + tyy + tzz;
}

// v^e for e in 0..4 as pow_int (multipole.cpp:43-49) computes it: 1.0 times v, e times
// (the first product is exact).
struct Pow4 {
    double p1, p2, p3, p4;
    __device__ __forceinline__ explicit Pow4(double v) : p1(v), p2(dmul(v, v)), p3(dmul(p2, v)), p4(dmul(p3, v)) {}
    __device__ __forceinline__ double operator()(int e) const {
        return e == 0 ? 1.0 : (e == 1 ? p1 : (e == 2 ? p2 : (e == 3 ? p3 : p4)));
    }
};

// Leaf moments: p2m_m2m leaf branch (fmm_solver.cpp:162-167, 180-181) and
// compute_multipole_moments leaf branch (:187-193).  One warp per node; internal nodes
// return.  The leaf's bodies are staged 32 at a time in shared memory; every lane then
// runs the reference's sequential sums over them (lane k for moment 4 + k).  A massless
// leaf gets its cell centre as centre of mass, as in the reference.
__global__ void __launch_bounds__(kMomBlock) fmm_leaf_kernel(const FmmArgs a) {
    __shared__ double s_b[kMomBlock / 32][4][32];
    const int wl = threadIdx.x >> 5;
    const int w = (int)((blockIdx.x * (unsigned)kMomBlock + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (w >= fmm_nodes(a) || a.node_child[w] >= 0) return;
    const int b = a.node_beg[w], e = a.node_end[w];
    double* r = a.rec + (size_t)w * kFmmRec;
    double(*sb)[32] = s_b[wl];
    auto stage = [&](int k0) {
        __syncwarp();
        if (k0 + lane < e) {
            const int i = a.perm[k0 + lane];
            sb[0][lane] = a.x[i];
            sb[1][lane] = a.y[i];
            sb[2][lane] = a.z[i];
            sb[3][lane] = a.m[i];
        }
        __syncwarp();
        return min(32, e - k0);
    };
    double mass = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
    for (int k0 = b; k0 < e; k0 += 32) {
        const int cnt = stage(k0);
#pragma unroll 4
        for (int q = 0; q < cnt; ++q) {
            const double mi = sb[3][q];
            mass = dadd(mass, mi);
            wx = dadd(wx, dmul(sb[0][q], mi));
            wy = dadd(wy, dmul(sb[1][q], mi));
            wz = dadd(wz, dmul(sb[2][q], mi));
        }
    }
    const bool pos = mass > 0.0;
    const double cx = pos ? __ddiv_rn(wx, mass) : a.node_cx[w];
    const double cy = pos ? __ddiv_rn(wy, mass) : a.node_cy[w];
    const double cz = pos ? __ddiv_rn(wz, mass) : a.node_cz[w];
    const int ks = lane < 31 ? 4 + lane : 0;
    const int ex = kTab.ex[ks], ey = kTab.ey[ks], ez = kTab.ez[ks];
    double v = 0.0;
    for (int k0 = b; k0 < e; k0 += 32) {
        const int cnt = stage(k0);
#pragma unroll 4
        for (int q = 0; q < cnt; ++q) {
            const Pow4 px(dsub(sb[0][q], cx)), py(dsub(sb[1][q], cy)), pz(dsub(sb[2][q], cz));
            const double mono = dmul(dmul(px(ex), py(ey)), pz(ez));
            v = dadd(v, dmul(sb[3][q], mono));
        }
    }
    if (lane < 31) {
        r[4 + lane] = v;
    } else {
        r[0] = cx;
        r[1] = cy;
        r[2] = cz;
        r[kRecMass] = mass;
    }
    __syncwarp();
    if (lane == 0) write_traces(r);
}

// Internal node: p2m_m2m (fmm_solver.cpp:168-181) over the children in octant order, then
// add_multipole_shifted_child per child (multipole.cpp:227-252).  One CTA per node: the 8
// children's records are staged in shared memory, warp c computes child c's shifted
// contribution to every moment (lane a for moment 4 + a), and warp 0 adds the 8
// contributions in child order, as the reference does.  A massless child adds exact zeros
// to every sum in the reference and is skipped here (masses are >= 0).
// All threads of the CTA call it for the same node w (it holds CTA barriers).
__device__ __forceinline__ void m2m_node(const FmmArgs& a, const int w, double (*s_child)[kRecTrQ],
                                         double (*s_val)[32]) {
    const int c0 = a.node_child[w];
    if (c0 < 0) return;
    const int tid = threadIdx.x, c = tid >> 5, lane = tid & 31;
    for (int k = tid; k < 8 * kRecTrQ; k += 256)
        s_child[k / kRecTrQ][k % kRecTrQ] = __ldcg(&a.rec[(size_t)(c0 + k / kRecTrQ) * kFmmRec + k % kRecTrQ]);
    __syncthreads();
    double mass = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
    for (int q = 0; q < 8; ++q) {
        const double cm = s_child[q][kRecMass];
        if (!(cm > 0.0)) continue;
        mass = dadd(mass, cm);
        wx = dadd(wx, dmul(s_child[q][0], cm));
        wy = dadd(wy, dmul(s_child[q][1], cm));
        wz = dadd(wz, dmul(s_child[q][2], cm));
    }
    const bool pos = mass > 0.0;
    const double cx = pos ? __ddiv_rn(wx, mass) : a.node_cx[w];
    const double cy = pos ? __ddiv_rn(wy, mass) : a.node_cy[w];
    const double cz = pos ? __ddiv_rn(wz, mass) : a.node_cz[w];
    const double* cr = s_child[c];
    const double cm = cr[kRecMass];
    if (lane < 31 && cm > 0.0) {
        const Pow4 px(dsub(cr[0], cx)), py(dsub(cr[1], cy)), pz(dsub(cr[2], cz));
        // The terms are independent until the sum: the loop runs to the table's bound with the
        // lane's own count as a predicate, so the loads and products of later terms overlap the
        // additions, which stay in the reference's order.
        const int nt = kTab.nterm[lane];
        double value = 0.0;
#pragma unroll
        for (int q = 0; q < kMaxShiftTerms; ++q) {
            if (q < nt) {
                const double sf = dmul(dmul(dmul(kTab.bin[lane][q], px(kTab.dx[lane][q])), py(kTab.dy[lane][q])),
                                       pz(kTab.dz[lane][q]));
                if (sf != 0.0) {
                    const int kb = kTab.kb[lane][q];
                    value = dadd(value, dmul(sf, kb == 0 ? cm : cr[kb]));
                }
            }
        }
        s_val[c][lane] = value;
    }
    __syncthreads();
    if (c == 0) {
        double* r = a.rec + (size_t)w * kFmmRec;
        if (lane < 31) {
            double total = 0.0;
            for (int q = 0; q < 8; ++q)
                if (s_child[q][kRecMass] > 0.0) total = dadd(total, s_val[q][lane]);
            r[4 + lane] = total;
        } else {
            r[0] = cx;
            r[1] = cy;
            r[2] = cz;
            r[kRecMass] = mass;
        }
        __syncwarp();
        if (lane == 0) write_traces(r);
    }
    __syncthreads();  // the staging arrays are free for the next node
}

__global__ void __launch_bounds__(256) fmm_m2m_kernel(const FmmArgs a, int lb) {
    __shared__ double s_child[8][kRecTrQ];
    __shared__ double s_val[8][32];
    m2m_node(a, lb + blockIdx.x, s_child, s_val);
}

// Every internal node in one launch, without a barrier per level.  Blocks take the nodes
// from a ticket counter in decreasing index order; levels are numbered top down, so a node
// comes after all its children.  A block waits (thread c for child c) until the flag of each
// internal child is set, computes the node as above and sets its own flag.  A block only
// waits for nodes whose tickets were taken before its own, by blocks already running, so the
// wait always ends; it is bounded all the same (timeout_ns of the global timer), and a wait
// that gives up sets bit 0 of err[0] and err[1] (the evaluation is then redone).  Child
// records are read through L2 (__ldcg), since another SM wrote them in this launch.
__device__ __forceinline__ unsigned long long m2m_clock() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__global__ void __launch_bounds__(256) fmm_m2m_tree_kernel(const FmmArgs a, int* ticket, int* ready, int* err,
                                                           unsigned long long timeout_ns) {
    __shared__ double s_child[8][kRecTrQ];
    __shared__ double s_val[8][32];
    __shared__ int s_t;
    const int nn = fmm_nodes(a);
    for (;;) {
        if (threadIdx.x == 0) s_t = atomicAdd(ticket, 1);
        __syncthreads();
        const int t = s_t;
        __syncthreads();
        if (t >= nn) return;
        const int w = nn - 1 - t;
        const int c0 = a.node_child[w];
        if (c0 < 0) continue;  // a leaf: fmm_leaf_kernel wrote it
        if (threadIdx.x < 8 && a.node_child[c0 + threadIdx.x] >= 0) {
            const int* f = ready + c0 + threadIdx.x;
            const unsigned long long t0 = m2m_clock();
            int v = 0;
            for (unsigned it = 0;; ++it) {
                asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(f) : "memory");
                if (v) break;
                if ((it & 255) == 255 && m2m_clock() - t0 > timeout_ns) {
                    atomicOr(err, 1);
                    atomicOr(err + 1, 1);
                    break;
                }
            }
        }
        __syncthreads();
        m2m_node(a, w, s_child, s_val);  // ends with a block barrier
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(ready + w), "r"(1) : "memory");
    }
}

__device__ __forceinline__ double rsqrt_t(double s) { return rsqrt_f64(s); }
__device__ __forceinline__ float rsqrt_t(float s) { return rsqrt_f32(s); }

// One far node's contribution at one target (without the factor G), from the offset d =
// centre of mass - target and the node's values r[k] = record slot k (k >= 3).  T = double
// is the FP64 far field; T = float the mixed-precision one (d taken in FP64, then rounded).
template <int P, typename T>
__device__ __forceinline__ void m2p_terms(const T* __restrict__ r, const T dx, const T dy, const T dz, const T eps2,
                                          T& fx, T& fy, T& fz) {
    const T s = dx * dx + dy * dy + dz * dz + eps2;
    if (s == T(0)) return;  // h0 == 0 (multipole.cpp:272-275)
    const T ri = rsqrt_t(s);
    const T r2 = ri * ri;
    const T g1 = -ri * r2;
    T cd = -r[kRecMass] * g1;  // coefficient of d
    T vx = T(0), vy = T(0), vz = T(0);
    if (P >= 2) {
        const T g2 = T(-3.0) * g1 * r2, g3 = T(-5.0) * g2 * r2;
        const T mx = r[4] * dx + r[5] * dy + r[6] * dz;
        const T my = r[5] * dx + r[7] * dy + r[8] * dz;
        const T mz = r[6] * dx + r[8] * dy + r[9] * dz;
        const T mdd = dx * mx + dy * my + dz * mz;
        cd -= T(0.5) * (g3 * mdd + g2 * r[kRecTrQ]);
        vx -= g2 * mx;
        vy -= g2 * my;
        vz -= g2 * mz;
        if (P >= 4) {
            const T g4 = T(-7.0) * g3 * r2, g5 = T(-9.0) * g4 * r2;
            // degree-2 monomials of d weighted 2/nu!
            const T qxx = dx * dx, qxy = T(2.0) * dx * dy, qxz = T(2.0) * dx * dz, qyy = dy * dy,
                    qyz = T(2.0) * dy * dz, qzz = dz * dz;
            const T ox = r[10] * qxx + r[11] * qxy + r[12] * qxz + r[13] * qyy + r[14] * qyz + r[15] * qzz;
            const T oy = r[11] * qxx + r[13] * qxy + r[14] * qxz + r[16] * qyy + r[17] * qyz + r[18] * qzz;
            const T oz = r[12] * qxx + r[14] * qxy + r[15] * qxz + r[17] * qyy + r[18] * qyz + r[19] * qzz;
            const T oddd = dx * ox + dy * oy + dz * oz;
            const T wd = r[kRecW] * dx + r[kRecW + 1] * dy + r[kRecW + 2] * dz;
            cd -= g4 * oddd * T(1.0 / 6.0) + T(0.5) * g3 * wd;
            vx -= T(0.5) * (g3 * ox + g2 * r[kRecW]);
            vy -= T(0.5) * (g3 * oy + g2 * r[kRecW + 1]);
            vz -= T(0.5) * (g3 * oz + g2 * r[kRecW + 2]);
            // degree-3 monomials of d weighted 6/mu!
            const T cxxx = qxx * dx, cxxy = T(3.0) * qxx * dy, cxxz = T(3.0) * qxx * dz, cxyy = T(3.0) * dx * qyy,
                    cxyz = T(3.0) * qxy * dz, cxzz = T(3.0) * dx * qzz, cyyy = qyy * dy, cyyz = T(3.0) * qyy * dz,
                    cyzz = T(3.0) * dy * qzz, czzz = qzz * dz;
            const T hx = r[20] * cxxx + r[21] * cxxy + r[22] * cxxz + r[23] * cxyy + r[24] * cxyz + r[25] * cxzz +
                         r[26] * cyyy + r[27] * cyyz + r[28] * cyzz + r[29] * czzz;
            const T hy = r[21] * cxxx + r[23] * cxxy + r[24] * cxxz + r[26] * cxyy + r[27] * cxyz + r[28] * cxzz +
                         r[30] * cyyy + r[31] * cyyz + r[32] * cyzz + r[33] * czzz;
            const T hz = r[22] * cxxx + r[24] * cxxy + r[25] * cxxz + r[27] * cxyy + r[28] * cxyz + r[29] * cxzz +
                         r[31] * cyyy + r[32] * cyyz + r[33] * cyzz + r[34] * czzz;
            const T hdddd = dx * hx + dy * hy + dz * hz;
            const T* Tq = r + kRecT2;  // xx xy xz yy yz zz
            const T tx2 = Tq[0] * dx + Tq[1] * dy + Tq[2] * dz;
            const T ty2 = Tq[1] * dx + Tq[3] * dy + Tq[4] * dz;
            const T tz2 = Tq[2] * dx + Tq[4] * dy + Tq[5] * dz;
            const T tdd = dx * tx2 + dy * ty2 + dz * tz2;
            cd -= g5 * hdddd * T(1.0 / 24.0) + T(0.25) * g4 * tdd + T(0.125) * g3 * r[kRecTr2];
            const T k4 = g4 * T(1.0 / 6.0), k3 = T(0.5) * g3;
            vx -= k4 * hx + k3 * tx2;
            vy -= k4 * hy + k3 * ty2;
            vz -= k4 * hz + k3 * tz2;
        }
    }
    fx += cd * dx + vx;
    fy += cd * dy + vy;
    fz += cd * dz + vz;
}

// A staged record at one target: the FP64 record, or the mixed record (kRec32 layout).
template <int P>
__device__ __forceinline__ void m2p_one(const double* __restrict__ r, double tx, double ty, double tz, double eps2,
                                        double& fx, double& fy, double& fz) {
    m2p_terms<P, double>(r, r[0] - tx, r[1] - ty, r[2] - tz, eps2, fx, fy, fz);
}
template <int P>
__device__ __forceinline__ void m2p_one(const float* __restrict__ r, double tx, double ty, double tz, float eps2,
                                        float& fx, float& fy, float& fz) {
    const double* com = reinterpret_cast<const double*>(r);
    m2p_terms<P, float>(r + 3, (float)(com[0] - tx), (float)(com[1] - ty), (float)(com[2] - tz), eps2, fx, fy, fz);
}

// The mixed-precision records (kRec32) from the FP64 ones, one thread per node.
__global__ void __launch_bounds__(256) fmm_rec32_kernel(const FmmArgs a) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k >= fmm_nodes(a)) return;
    const double* r = a.rec + (size_t)k * kFmmRec;
    float* o = a.rec32 + (size_t)k * kRec32;
    double* oc = reinterpret_cast<double*>(o);
    oc[0] = r[0];
    oc[1] = r[1];
    oc[2] = r[2];
    for (int q = kRecMass; q <= kRecTr2; ++q) o[q + 3] = __double2float_rn(r[q]);
    for (int q = kRecTr2 + 4; q < kRec32; ++q) o[q] = 0.0f;
}

// Shared-memory stride of a staged node record, in elements: slots 0..45 of an FP64 record
// (16-byte multiple), or a whole mixed record.
template <typename T>
__host__ __device__ constexpr int stage_stride() { return sizeof(T) == 8 ? 46 : kRec32; }
constexpr int kM2PSub = 64;     // node records per shared-memory buffer
constexpr int kM2PStages = 2;   // buffers in the cp.async ring
template <typename T>
constexpr size_t m2p_dyn_smem() { return (size_t)kM2PStages * kM2PSub * stage_stride<T>() * sizeof(T); }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Work item = (target leaf, up to kM2PChunk far nodes).  The item's node records stream
// through a ring of kM2PStages shared-memory buffers: while the block evaluates one, cp.async
// fills the next ones.  Thread t evaluates target t % W against nodes t / W, t / W + S, ...
// of each buffer (W = the leaf's targets, at most one block; S = block / W node slots, so at
// most W - 1 threads idle); a buffer is filled with a multiple of S records, so every slot
// evaluates the same number of nodes between barriers.  The S partial sums of a target are
// added in slot order, so results do not depend on scheduling.
template <int P, typename T>
__global__ void __launch_bounds__(kM2PBlock) fmm_m2p_kernel(const FmmArgs a) {
    // record elements the order reads, staged in 16-byte pieces
    constexpr bool F64 = sizeof(T) == 8;
    constexpr int kElems = F64 ? (P == 0 ? 4 : P == 2 ? kRecTrQ + 1 : 46) : (P == 0 ? 7 : P == 2 ? kRecTrQ + 4 : kRecTr2 + 4);
    constexpr int PIECES = (kElems * (int)sizeof(T) + 15) / 16;
    constexpr int kPer = 16 / (int)sizeof(T);  // elements per piece
    constexpr int kStride = stage_stride<T>();
    constexpr int kGlobal = F64 ? kFmmRec : kRec32;  // record stride in global memory
    const T* rec = F64 ? reinterpret_cast<const T*>(a.rec) : reinterpret_cast<const T*>(a.rec32);
    const T eps2 = F64 ? (T)a.eps2 : (T)a.eps2f;
    extern __shared__ __align__(16) unsigned char s_raw[];
    T* s_dyn = reinterpret_cast<T*>(s_raw);
    __shared__ double s_red[kM2PBlock * 3];
    __shared__ int s_last;
    const int tid = threadIdx.x;
    if (a.overflow && *a.overflow) return;
    const int n_items = fmm_items(a);
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const M2PItem w = a.items[it];
        const int cnt = w.fe - w.fb;
        const int tb = a.leaf_off[w.leaf], nt = a.leaf_off[w.leaf + 1] - tb;
        const int W = min(nt, kM2PBlock);
        const int S = kM2PBlock / W;
        const int q = tid / W, tl = tid - q * W;
        const int R = S <= kM2PSub ? S * (kM2PSub / S) : kM2PSub;  // records per buffer
        const int nsub = (cnt + R - 1) / R;
        // fills buffer sc % kM2PStages with records sc * R ..; one commit group per call, empty
        // past the end, so that the waits below count groups uniformly
        auto stage = [&](int sc) {
            if (sc < nsub) {
                T* buf = s_dyn + (sc % kM2PStages) * (kM2PSub * kStride);
                const int j0 = sc * R, m = min(R, cnt - j0);
                for (int k = tid; k < m * PIECES; k += kM2PBlock) {
                    const int j = k / PIECES, pc = k - j * PIECES;
                    const T* src = rec + (size_t)a.far_node[w.fb + j0 + j] * kGlobal + kPer * pc;
                    cp_async16(buf + j * kStride + kPer * pc, src);
                }
            }
            cp_async_commit();
        };
        for (int t0 = 0; t0 < nt; t0 += W) {
            const int t = t0 + tl;
            T fx = T(0), fy = T(0), fz = T(0);
            int i = -1;
            double tx = 0.0, ty = 0.0, tz = 0.0;
            if (q < S && t < nt) {
                i = a.leaf_part[tb + t];
                if (i >= a.t_begin && i < a.t_end) {
                    tx = a.x[i];
                    ty = a.y[i];
                    tz = a.z[i];
                } else {
                    i = -1;
                }
            }
            for (int sc = 0; sc < kM2PStages - 1; ++sc) stage(sc);
            for (int sc = 0; sc < nsub; ++sc) {
                stage(sc + kM2PStages - 1);  // into the buffer released at the end of sc - 1
                cp_async_wait<kM2PStages - 1>();
                __syncthreads();
                const T* buf = s_dyn + (sc % kM2PStages) * (kM2PSub * kStride);
                const int m = min(R, cnt - sc * R);
                if (i >= 0)
                    for (int j = q; j < m; j += S) m2p_one<P>(buf + j * kStride, tx, ty, tz, eps2, fx, fy, fz);
                __syncthreads();  // a later stage() overwrites this buffer
            }
            cp_async_wait<0>();  // the empty trailing groups
            s_red[tid * 3 + 0] = (double)fx;
            s_red[tid * 3 + 1] = (double)fy;
            s_red[tid * 3 + 2] = (double)fz;
            __syncthreads();
            if (q == 0 && i >= 0) {
                double sx = 0.0, sy = 0.0, sz = 0.0;
                for (int k = 0; k < S; ++k) {
                    const int o = (k * W + tl) * 3;
                    sx += s_red[o];
                    sy += s_red[o + 1];
                    sz += s_red[o + 2];
                }
                if (w.nchunks == 1) {
                    a.ax[i] = a.ax[i] + a.G * sx;
                    a.ay[i] = a.ay[i] + a.G * sy;
                    a.az[i] = a.az[i] + a.G * sz;
                } else {
                    const size_t o = (size_t)(w.scratch + (int64_t)w.chunk * nt + t) * 3;
                    a.scratch[o] = sx;
                    a.scratch[o + 1] = sy;
                    a.scratch[o + 2] = sz;
                }
            }
            __syncthreads();
        }
        if (w.nchunks > 1) {
            // The CTA that completes the leaf's last chunk adds the partials in chunk order.
            __threadfence();
            __syncthreads();
            if (tid == 0) s_last = (atomicAdd(&a.done[w.leaf], 1) == w.nchunks - 1);
            __syncthreads();
            if (s_last) {
                __threadfence();
                for (int t = tid; t < nt; t += kM2PBlock) {
                    const int i = a.leaf_part[tb + t];
                    if (i < a.t_begin || i >= a.t_end) continue;
                    double sx = 0.0, sy = 0.0, sz = 0.0;
                    for (int c = 0; c < w.nchunks; ++c) {
                        const size_t o = (size_t)(w.scratch + (int64_t)c * nt + t) * 3;
                        sx += __ldcg(&a.scratch[o]);
                        sy += __ldcg(&a.scratch[o + 1]);
                        sz += __ldcg(&a.scratch[o + 2]);
                    }
                    a.ax[i] = a.ax[i] + a.G * sx;
                    a.ay[i] = a.ay[i] + a.G * sy;
                    a.az[i] = a.az[i] + a.G * sz;
                }
            }
            __syncthreads();
        }
    }
}

template <int P, typename T>
cudaError_t launch_m2p_order(const FmmArgs& a, cudaStream_t st) {
    // the shared-memory opt-in is a per-device setting of the kernel
    static std::atomic<unsigned long long> set_on{0};
    constexpr size_t smem = m2p_dyn_smem<T>();
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(set_on.load() & bit)) {
        e = cudaFuncSetAttribute(fmm_m2p_kernel<P, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        set_on.fetch_or(bit);
    }
    fmm_m2p_kernel<P, T><<<std::min(a.n_items, 1 << 20), kM2PBlock, smem, st>>>(a);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_m2p_type(const FmmArgs& a, cudaStream_t st) {
    switch (a.order) {
        case 0: return launch_m2p_order<0, T>(a, st);
        case 2: return launch_m2p_order<2, T>(a, st);
        default: return launch_m2p_order<4, T>(a, st);
    }
}

}  // namespace

int fmm_effective_order(int expansion_order) {
    int p = std::min(4, std::max(0, expansion_order));
    if (p == 1 || p == 3) ++p;
    return p;
}

cudaError_t launch_fmm_moments_tree(const FmmArgs& a, int* ticket, int* ready, int* err, int sms, cudaStream_t st) {
    constexpr int wpb = kMomBlock / 32;
    if (a.n_nodes == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(ready, 0, (size_t)a.n_nodes * sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ticket, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    fmm_leaf_kernel<<<(a.n_nodes + wpb - 1) / wpb, kMomBlock, 0, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int grid = std::min(a.n_nodes, sms * 8);
    fmm_m2m_tree_kernel<<<grid, 256, 0, st>>>(a, ticket, ready, err, 1000000000ull);
    return cudaGetLastError();
}

// ax += nx, ay += ny, az += nz: the near field, computed into its own arrays while the far
// field ran, added to it (one rounding, as when the near kernel adds to the far field).
__global__ void __launch_bounds__(256) fmm_add_near_kernel(int64_t n, double* ax, double* ay, double* az,
                                                           const double* nx, const double* ny, const double* nz) {
    for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256) {
        ax[i] = ax[i] + nx[i];
        ay[i] = ay[i] + ny[i];
        az[i] = az[i] + nz[i];
    }
}

cudaError_t launch_fmm_add_near(int64_t n, double* ax, double* ay, double* az, const double* nx, const double* ny,
                                const double* nz, int sms, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int64_t blocks = std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8);
    fmm_add_near_kernel<<<(unsigned)blocks, 256, 0, st>>>(n, ax, ay, az, nx, ny, nz);
    return cudaGetLastError();
}

cudaError_t launch_fmm_moments(const FmmArgs& a, const int32_t* level_off_host, int n_levels, cudaStream_t st) {
    constexpr int wpb = kMomBlock / 32;
    if (a.n_nodes == 0) return cudaSuccess;
    fmm_leaf_kernel<<<(a.n_nodes + wpb - 1) / wpb, kMomBlock, 0, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    for (int d = n_levels - 1; d >= 0; --d) {
        const int lb = level_off_host[d], le = level_off_host[d + 1];
        if (le <= lb) continue;
        fmm_m2m_kernel<<<le - lb, 256, 0, st>>>(a, lb);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_fmm_m2p(const FmmArgs& a, bool mixed, cudaStream_t st) {
    if (a.n_items == 0) return cudaSuccess;
    if (!mixed) return launch_m2p_type<double>(a, st);
    fmm_rec32_kernel<<<(a.n_nodes + 255) / 256, 256, 0, st>>>(a);
    const cudaError_t e = cudaGetLastError();
    return e != cudaSuccess ? e : launch_m2p_type<float>(a, st);
}

}  // namespace gx
