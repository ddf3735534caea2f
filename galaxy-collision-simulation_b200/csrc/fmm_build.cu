// fmm_build.cu -- the reference octree (FastMultipoleSolver::build,
// cpp/fmm/fmm_solver.cpp:48-98) and its interaction lists (:228-277) built on the device.
//
// The reference inserts bodies one at a time; a leaf splits when it would hold more than
// leaf_capacity bodies below max_depth (:133-155).  The resulting tree is the recursive
// 8-way partition in which exactly the nodes with more than leaf_capacity bodies above
// max_depth are split.  A body's octant at every level depends only on its position and on
// the cell centres along its path, which follow the reference's recurrence
// (child centre = centre +- half_width * 0.5, :111-131; octant by >=, :104-109).  So:
//   1. root cell from the bounding box (:62-85);
//   2. every body's path as a 63-bit key, 3 bits per level, level 0 in the top bits;
//   3. a stable radix sort of (key, body): depth-first tree order;
//   4. one CTA walks the levels: a node with more than leaf_capacity bodies splits into 8
//      children whose body ranges are found by binary search on the sorted keys;
//   5. one warp per leaf sorts the leaf's bodies into ascending index order, the order
//      the reference's sums run in.
// Nodes are numbered breadth-first.  Trees that need a split below level 21 (more than
// leaf_capacity nearly coincident bodies) are reported back for the host builder.
//
// Lists: every leaf with mass > 0 is walked with the reference's tests (mass > 0,
// well_separated, leaf) by one warp over a shared-memory stack; a count pass, exclusive
// sums, and a fill pass (near lists sorted into the reference's depth-first order).
#include "fmm_build.cuh"
#include "fmm.cuh"
#include "gx_device.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <thrust/iterator/zip_iterator.h>
#include <thrust/tuple.h>

#include <algorithm>
#include <cfloat>

namespace gx {
namespace {

constexpr int kBboxThreads = 256;
constexpr int kWalkThreads = 128;  // 4 warps, one leaf each
// Shared stack slots per warp: 4 x 1024 x 4 B = 16 KiB per block, plus the 1 KiB the
// runtime reserves per block: 8 blocks (32 warps, the count __launch_bounds__(kWalkThreads, 8)
// sizes the registers for) take 136 KiB, inside the 60% shared-memory carveout walk_kernel
// asks for; the rest of the SM's unified memory stays L1 for the node-record loads (measured
// against 1760 slots at the largest carveout: lists phase 13% faster at N=2^20, leaf 16).
constexpr int kWalkStack = 1024;
// near lists up to this many entries are sorted in the warp's stack buffer (a bitonic network
// pads to a power of two, so the largest power of two that fits kWalkStack / 2 keys)
constexpr int pow2_floor(int v) { return v < 2 ? v : 2 * pow2_floor(v / 2); }
constexpr int kSortCap = pow2_floor(kWalkStack / 2);
constexpr int kStack = 7 * (kKeyLevels + 1) + 8;

__global__ void __launch_bounds__(kBboxThreads) bbox_partial_kernel(const TreeBuildArgs t) {
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (int i = blockIdx.x * kBboxThreads + threadIdx.x; i < t.n; i += gridDim.x * kBboxThreads) {
        const double v[3] = {t.x[i], t.y[i], t.z[i]};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            lo[c] = fmin(lo[c], v[c]);
            hi[c] = fmax(hi[c], v[c]);
        }
    }
    __shared__ double s[6][kBboxThreads / 32];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        lo[c] = warp_min(lo[c]);
        hi[c] = warp_max(hi[c]);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int c = 0; c < 3; ++c) {
            s[c][w] = lo[c];
            s[3 + c][w] = hi[c];
        }
    __syncthreads();
    if (threadIdx.x < 6) {
        double v = s[threadIdx.x][0];
        for (int k = 1; k < kBboxThreads / 32; ++k) v = threadIdx.x < 3 ? fmin(v, s[threadIdx.x][k]) : fmax(v, s[threadIdx.x][k]);
        t.part[blockIdx.x * 6 + threadIdx.x] = v;
    }
}

// Root cell (fmm_solver.cpp:62-85): one block reduces the partial extrema.
__global__ void __launch_bounds__(kBboxThreads) bbox_final_kernel(const TreeBuildArgs t, int blocks) {
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (int b = threadIdx.x; b < blocks; b += kBboxThreads)
        for (int c = 0; c < 3; ++c) {
            lo[c] = fmin(lo[c], t.part[b * 6 + c]);
            hi[c] = fmax(hi[c], t.part[b * 6 + 3 + c]);
        }
    __shared__ double s[6][kBboxThreads / 32];
    for (int c = 0; c < 3; ++c) {
        lo[c] = warp_min(lo[c]);
        hi[c] = warp_max(hi[c]);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int c = 0; c < 3; ++c) {
            s[c][w] = lo[c];
            s[3 + c][w] = hi[c];
        }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int c = 0; c < 3; ++c)
        for (int k = 1; k < kBboxThreads / 32; ++k) {
            s[c][0] = fmin(s[c][0], s[c][k]);
            s[3 + c][0] = fmax(s[3 + c][0], s[3 + c][k]);
        }
    for (int c = 0; c < 3; ++c) t.root[c] = dmul(dadd(s[c][0], s[3 + c][0]), 0.5);
    double hw = dmul(0.5, fmax(fmax(dsub(s[3][0], s[0][0]), dsub(s[4][0], s[1][0])), dsub(s[5][0], s[2][0])));
    hw = fmax(hw, dadd(t.softening, 1.0e-6));
    t.root[3] = dmul(hw, 1.0001);
}

__device__ __forceinline__ int octant_of(double x, double y, double z, double cx, double cy, double cz) {
    return (x >= cx ? 1 : 0) + (y >= cy ? 2 : 0) + (z >= cz ? 4 : 0);
}

// Child centre (subdivide, fmm_solver.cpp:111-131): centre + sign * (half_width * 0.5).
__device__ __forceinline__ double child_centre(double c, double chw, bool up) { return dadd(c, up ? chw : -chw); }

__global__ void __launch_bounds__(256) keys_kernel(const TreeBuildArgs t) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= t.n) return;
    const double x = t.x[i], y = t.y[i], z = t.z[i];
    double cx = t.root[0], cy = t.root[1], cz = t.root[2], hw = t.root[3];
    uint64_t key = 0;
    for (int l = 0; l < kKeyLevels; ++l) {
        const int o = octant_of(x, y, z, cx, cy, cz);
        key |= (uint64_t)o << (3 * (kKeyLevels - 1 - l));
        const double chw = dmul(hw, 0.5);
        cx = child_centre(cx, chw, o & 1);
        cy = child_centre(cy, chw, o & 2);
        cz = child_centre(cz, chw, o & 4);
        hw = chw;
    }
    t.keys[i] = key;
    t.idx[i] = i;
}

// First position p in [b, e) whose octant at shift sh is >= o (octants are non-decreasing
// in a cell's sorted range).
__device__ __forceinline__ int lower_octant(const uint64_t* keys, int b, int e, int sh, int o) {
    while (b < e) {
        const int mid = (b + e) >> 1;
        if ((int)((keys[mid] >> sh) & 7) < o) b = mid + 1;
        else e = mid;
    }
    return b;
}

// The topology in parallel from the sorted path keys.  A node at depth L is a key prefix of
// L octants (key >> 3 (kKeyLevels - L)); it splits when it holds more than cap bodies and
// L < max_depth, and a splitting node's 8 children (all of them, empty ones included) are
// the nodes of depth L + 1.  Nodes are numbered breadth-first with children in octant order,
// i.e. level by level in key-prefix order, so a node's number follows from counts alone:
//   flags[L n + i] = 1 when sorted body i is the first body of a splitting depth-L prefix,
//   E = exclusive scan of flags over all levels (kKeyLevels n + 1 entries, in place),
//   S_L = splitting nodes of depth L = E[(L + 1) n] - E[L n],
//   level_off[L + 1] = level_off[L] + 8 S_(L-1)  (level_off[0] = 0, level_off[1] = 1),
//   the rank of body i's depth-L prefix among the splitting ones = E[L n + i] - E[L n],
//   and its children start at level_off[L + 1] + 8 rank.
// A node's centre is the reference's recurrence (subdivide, fmm_solver.cpp:111-131) walked
// from the root along its prefix -- the same operations in the same order as building level
// by level, so the same bits.  A prefix of depth kKeyLevels that would still split needs a
// deeper key: hdr[2] bit 0 hands the tree to the host builder.  When the sort ordered only
// the first key_levels levels, a prefix of that depth that would split sets hdr[2] bit 2
// instead (the build stops there; the caller redoes it with all levels).

__device__ __forceinline__ uint64_t key_prefix(uint64_t key, int L) {
    const int sh = 3 * (kKeyLevels - L);
    return sh >= 64 ? 0 : key >> sh;
}

// Position one past the last body of the depth-L prefix that starts at sorted body i:
// galloping from i, then a binary search in the last gap (log of the prefix's size).
__device__ __forceinline__ int prefix_end(const uint64_t* keys, int n, int i, int L) {
    const uint64_t p = key_prefix(keys[i], L);
    int lo = i + 1, step = 1;  // keys[lo - 1] has prefix p
    while (lo < n && key_prefix(keys[lo], L) == p) {
        const int nxt = lo + step;
        if (nxt >= n || key_prefix(keys[nxt], L) != p) {
            int b = lo + 1, e = min(nxt, n);  // first mismatch in (lo, nxt]
            while (b < e) {
                const int mid = (b + e) >> 1;
                if (key_prefix(keys[mid], L) == p) b = mid + 1;
                else e = mid;
            }
            return b;
        }
        lo = nxt + 1;
        step <<= 1;
    }
    return lo;
}

__device__ __forceinline__ bool prefix_first(const uint64_t* keys, int i, int L) {
    return i == 0 || key_prefix(keys[i], L) != key_prefix(keys[i - 1], L);
}

// flags[L n + i] = 1 when sorted body i starts a depth-L prefix holding more than cap bodies
// (it does exactly when body i + cap shares the prefix: the keys are sorted) and L < max_depth.
__global__ void __launch_bounds__(256) split_flags_kernel(const TreeBuildArgs t, const uint64_t* keys, int32_t* flags) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i == 0) flags[(size_t)kKeyLevels * t.n] = 0;
    if (i >= t.n) return;
    const int lmax = min(t.max_depth, kKeyLevels + 1);
    const int sorted = t.key_levels > 0 ? t.key_levels : kKeyLevels;  // levels the sort ordered
    const uint64_t key = keys[i];
    const bool big = (int64_t)i + t.cap < (int64_t)t.n;
    const uint64_t far = big ? keys[i + t.cap] : 0;
    for (int L = 0; L <= kKeyLevels; ++L) {
        bool split = false;
        if (L < lmax && big && prefix_first(keys, i, L) && key_prefix(far, L) == key_prefix(key, L)) {
            if (L == kKeyLevels) atomicOr(&t.hdr[2], 1);
            else if (L >= sorted) atomicOr(&t.hdr[2], 4);  // the children need deeper sorted keys
            else split = true;
        }
        if (L < kKeyLevels) flags[(size_t)L * t.n + i] = split ? 1 : 0;
    }
}

// One thread: level offsets, node and level counts from the scanned flags.
__global__ void tree_levels_kernel(const TreeBuildArgs t, const int32_t* E) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const size_t n = (size_t)t.n;
    int64_t off = 1;
    int levels = 1;
    t.level_off[0] = 0;
    t.level_off[1] = 1;
    for (int L = 0; L < kKeyLevels; ++L) {
        const int64_t s = (int64_t)E[(L + 1) * n] - (int64_t)E[L * n];
        if (s == 0) break;
        off += 8 * s;
        t.level_off[L + 2] = off <= 0x7fffffffLL ? (int32_t)off : 0x7fffffff;
        ++levels;
    }
    t.level_off[levels + 1] = t.level_off[levels];
    t.hdr[0] = t.level_off[levels];
    t.hdr[1] = levels;
    if (off > t.capacity) atomicOr(&t.hdr[2], 2);
}

// The splitting nodes in global (level, key) order: split_pos[E[L n + i]] = L n + i.
__global__ void __launch_bounds__(256) split_list_kernel(const TreeBuildArgs t, const int32_t* E, int32_t* split_pos,
                                                         int split_cap) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= t.n) return;
    const size_t n = (size_t)t.n;
    for (int L = 0; L < kKeyLevels; ++L) {
        const int32_t e0 = E[L * n + i];
        if (E[L * n + i + 1] != e0 && e0 < split_cap) split_pos[e0] = L * t.n + i;
    }
}

// Every node starts as a leaf (child -1); the root's record.
__global__ void __launch_bounds__(256) tree_init_kernel(const TreeBuildArgs t) {
    const int nodes = min(t.hdr[0], t.capacity);
    for (int k = blockIdx.x * 256 + threadIdx.x; k < nodes; k += gridDim.x * 256) t.child[k] = -1;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        t.beg[0] = 0;
        t.end[0] = t.n;
        t.cx[0] = t.root[0];
        t.cy[0] = t.root[1];
        t.cz[0] = t.root[2];
        t.hw[0] = t.root[3];
    }
}

// One thread per (splitting node, child octant c): the node's child index (c == 0) and child
// c's record -- its body range by binary search on the octant at depth L inside the node's
// range, its centre by the reference's recurrence walked from the root along the path.
__global__ void __launch_bounds__(256) tree_children_kernel(const TreeBuildArgs t, const uint64_t* keys,
                                                            const int32_t* E, const int32_t* split_pos, int split_cap) {
    if (t.hdr[2] & 2) return;
    const size_t n = (size_t)t.n;
    const int total = min(E[kKeyLevels * n], split_cap);
    for (int q = blockIdx.x * 256 + threadIdx.x; q < 8 * total; q += gridDim.x * 256) {
        const int sidx = q >> 3, c = q & 7;
        const int pos = split_pos[sidx];
        const int L = pos / t.n, i = pos - L * t.n;
        const uint64_t key = keys[i];
        int self = 0;
        if (L > 0) {
            const int parent_rank = E[(L - 1) * n + i + 1] - E[(L - 1) * n] - 1;
            self = t.level_off[L] + 8 * parent_rank + (int)((key >> (3 * (kKeyLevels - L))) & 7);
        }
        const int c0 = t.level_off[L + 1] + 8 * (sidx - E[L * n]);
        if (c == 0) t.child[self] = c0;
        const int e = prefix_end(keys, t.n, i, L);
        const int sh = 3 * (kKeyLevels - 1 - L);
        const int cb = c == 0 ? i : lower_octant(keys, i, e, sh, c);
        const int ce = c == 7 ? e : lower_octant(keys, cb, e, sh, c + 1);
        double cx = t.root[0], cy = t.root[1], cz = t.root[2], hw = t.root[3];
        for (int d = 0; d < L; ++d) {
            const int o = (int)((key >> (3 * (kKeyLevels - 1 - d))) & 7);
            hw = dmul(hw, 0.5);
            cx = child_centre(cx, hw, o & 1);
            cy = child_centre(cy, hw, o & 2);
            cz = child_centre(cz, hw, o & 4);
        }
        const double chw = dmul(hw, 0.5);
        t.beg[c0 + c] = cb;
        t.end[c0 + c] = ce;
        t.cx[c0 + c] = child_centre(cx, chw, c & 1);
        t.cy[c0 + c] = child_centre(cy, chw, c & 2);
        t.cz[c0 + c] = child_centre(cz, chw, c & 4);
        t.hw[c0 + c] = chw;
    }
}

__global__ void __launch_bounds__(256) gather_perm_kernel(const int32_t* idx_sorted, int32_t* perm, int n) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i < n) perm[i] = idx_sorted[i];
}

// Leaf order: one warp per leaf puts the leaf's bodies in ascending index order (the
// reference's particle_indices order): each body's new place is the number of smaller
// indices in the leaf, written to t.idx and copied back.
__global__ void __launch_bounds__(256) leaf_sort_kernel(const TreeBuildArgs t, int n_nodes) {
    const int w = (int)((blockIdx.x * 256u + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (t.hdr[2] != 0 || w >= min(n_nodes, t.hdr[0]) || t.child[w] >= 0) return;
    const int b = t.beg[w], e = t.end[w];
    if (e - b < 2) return;
    for (int i = b + lane; i < e; i += 32) {
        const int v = t.perm[i];
        int r = 0;
        for (int q = b; q < e; ++q) r += t.perm[q] < v;
        t.idx[b + r] = v;
    }
    __syncwarp();
    for (int i = b + lane; i < e; i += 32) t.perm[i] = t.idx[i];
}

__device__ __forceinline__ double node_mass(const double* rec, int k) { return rec[(size_t)k * kFmmRec + kRecMass]; }

// Nodes of the tree: the count on the device when the host did not read it (a.n_nodes is
// then the capacity of the node arrays).
__device__ __forceinline__ int list_nodes(const TreeListArgs& a) {
    if (!a.cnt_nodes) return a.n_nodes;
    return a.cnt_nodes[2] ? 0 : min(a.cnt_nodes[0], a.n_nodes);  // header {nodes, levels, flags}
}

// Node k has mass > 0: from the massive-body counts when given, else from its record.
__device__ __forceinline__ bool node_massive(const TreeListArgs& a, int k) {
    if (a.mprefix) return a.mprefix[a.end[k]] > a.mprefix[a.beg[k]];
    return node_mass(a.rec, k) > 0.0;
}

// mflag[k] = body at tree position k has mass > 0 (k < n), mflag[n] = 0; a mass < 0 or NaN
// (whose node sums the counts cannot stand for) raises the overflow words.
__global__ void __launch_bounds__(256) massive_flags_kernel(const TreeListArgs a, int32_t* mflag) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k > a.n) return;
    if (k == a.n) {
        mflag[k] = 0;
        return;
    }
    const double mk = a.m[a.perm[k]];
    mflag[k] = mk > 0.0 ? 1 : 0;
    if (!(mk >= 0.0)) {
        if (a.overflow) *a.overflow = 1;
        if (a.overflow_sticky) atomicOr(a.overflow_sticky, 3);
    }
}

// Marks the first body position of every leaf with mass > 0 and the bodies it keeps.
__global__ void __launch_bounds__(256) leaf_mark_kernel(const TreeListArgs a) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k >= list_nodes(a) || a.child[k] >= 0 || !node_massive(a, k)) return;
    const int b = a.beg[k], e = a.end[k];
    a.start_flag[b] = 1;
    for (int p = b; p < e; ++p) a.keep[p] = 1;
}

__global__ void __launch_bounds__(256) leaf_emit_kernel(const TreeListArgs a) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k >= list_nodes(a) || a.child[k] >= 0 || !node_massive(a, k)) return;
    const int b = a.beg[k], e = a.end[k];
    const int o = a.start_ord[b];
    a.leaf_node[o] = k;
    a.node_leaf[k] = o;
    a.leaf_off[o] = a.newpos[b];
    a.leaf_off[o + 1] = a.newpos[e];
    for (int p = b; p < e; ++p) a.leaf_part[a.newpos[p]] = a.perm[p];
}

__global__ void __launch_bounds__(256) walk_pack_kernel(const TreeListArgs a) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k >= list_nodes(a)) return;
    WalkNode w;
    w.cx = a.cx[k];
    w.cy = a.cy[k];
    w.cz = a.cz[k];
    w.hw = a.hw[k];
    w.mass = node_massive(a, k) ? 1.0 : 0.0;  // the walk only asks whether it is > 0
    w.child = a.child[k];
    w.beg = a.beg[k];
    w.end = a.end[k];
    w.mask = 0;
    if (w.child >= 0)
        for (int c = 0; c < 8; ++c) w.mask |= (node_massive(a, w.child + c) ? 1 : 0) << c;
    a.wn[k] = w;
}

// well_separated (fmm_solver.cpp:228-241): 2 (hw_t + hw_s) / dist < theta, dist != 0, with
// the reference's operations.  The reference's quotient is within 1.5 ulp of the exact
// num / sqrt(r2), so wherever num^2 and theta^2 r2 (each within a few ulp) differ by more
// than 1e-12 relative the squares give the same answer without the square root and the
// division; only near-ties, and magnitudes where the squares could overflow or underflow,
// take the reference's own operations.
__device__ __forceinline__ bool well_separated(const WalkNode& T, const WalkNode& S, double theta) {
    const double dx = dsub(S.cx, T.cx), dy = dsub(S.cy, T.cy), dz = dsub(S.cz, T.cz);
    const double r2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
    if (r2 == 0.0) return false;  // dist == 0
    const double num = dmul(2.0, dadd(T.hw, S.hw));
    const double lhs = dmul(num, num), rhs = dmul(dmul(theta, theta), r2);
    if (theta > 0.0 && rhs > 1e-290 && rhs < 1e290 && lhs < 1e290) {
        if (lhs < dmul(rhs, 1.0 - 1e-12)) return true;
        if (lhs > dmul(rhs, 1.0 + 1e-12)) return false;
    }
    return __ddiv_rn(num, __dsqrt_rn(r2)) < theta;
}

// One node of the walk (build_leaf_interactions, fmm_solver.cpp:254-277): 1 far, 2 near,
// 3 expand, 0 massless.
__device__ __forceinline__ int classify(const WalkNode& T, int t, const WalkNode& S, int s, double theta) {
    if (!(S.mass > 0.0)) return 0;
    if (s != t && well_separated(T, S, theta)) return 1;
    return S.child < 0 ? 2 : 3;
}

// One warp sorts the distinct keys v[0 .. n) ascending and writes the low 32 bits of each to
// out in that order: a bitonic sort in the shared buffer buf (kWalkStack / 2 slots) when the
// list fits, else every key's rank (the number of smaller keys) computed from global memory.
__device__ void sort_into(const uint64_t* v, int n, uint64_t* buf, int lane, int32_t* out) {
    if (n <= kSortCap) {
        int P = 1;
        while (P < n) P <<= 1;
        for (int i = lane; i < P; i += 32) buf[i] = i < n ? v[i] : ~0ull;
        __syncwarp();
        for (int k = 2; k <= P; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = lane; i < P; i += 32) {
                    const int m = i ^ j;
                    if (m > i) {
                        const uint64_t x = buf[i], y = buf[m];
                        if ((x > y) == ((i & k) == 0)) {
                            buf[i] = y;
                            buf[m] = x;
                        }
                    }
                }
                __syncwarp();
            }
        for (int i = lane; i < n; i += 32) out[i] = (int32_t)(uint32_t)buf[i];
        __syncwarp();
        return;
    }
    for (int i = lane; i < n; i += 32) {
        const uint64_t key = v[i];
        int r = 0;
        for (int q = 0; q < n; ++q) r += v[q] < key;
        out[r] = (int32_t)(uint32_t)key;
    }
}

// Every leaf with mass > 0, one warp each: the walk of build_leaf_interactions from the
// root, with a shared-memory stack the warp pops 32 nodes at a time (each lane classifies
// one node; expanded nodes push their children with mass > 0).  The fill pass writes each far node
// where the walk meets it (the far list holds the reference's nodes in the walk's own,
// deterministic order; only the summation order of the far field depends on it) and each
// near leaf as its ordinal, then sorts the near list into the reference's depth-first order
// (leaf ordinals are depth-first numbers), which the near field's exact form relies on.  When the stack would overflow, every lane finishes its share of
// the pending nodes depth first with a private stack.
template <bool FILL>
__global__ void __launch_bounds__(kWalkThreads, 8) walk_kernel(const TreeListArgs a) {
    constexpr int W = kWalkThreads / 32;
    __shared__ __align__(16) int s_stk[W][kWalkStack];
    if (FILL && a.overflow && *a.overflow) return;
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int l = blockIdx.x * W + wid;
    const int n_leaves = a.start_ord[a.n];
    if (l >= n_leaves) return;
    const int t = a.leaf_node[l];
    const WalkNode T = a.wn[t];
    const int fo = FILL ? a.far_off[l] : 0, no = FILL ? a.near_off[l] : 0;
    const unsigned lt = (1u << lane) - 1u;
    int* stk = s_stk[wid];
    int nf = 0, nn = 0, top = 1, pend = -1, pmask = 0, pchild = 0;
    long long nsrc = 0;  // count pass: bodies of the near leaves found by this lane
    if (lane == 0) stk[0] = 0;
    __syncwarp();
    while (top > 0) {
        const int take = min(32, top), base = top - take;
        int s = -1, cls = 0;
        WalkNode S;
        if (lane < take) {
            s = stk[base + lane];
            S = a.wn[s];
            cls = classify(T, t, S, s, a.theta);
        }
        __syncwarp();
        top = base;
        const unsigned mf = __ballot_sync(0xffffffffu, cls == 1);
        const unsigned mn = __ballot_sync(0xffffffffu, cls == 2);
        const unsigned me = __ballot_sync(0xffffffffu, cls == 3);
        if (FILL) {
            if (cls == 1) {
                const int pos = fo + nf + __popc(mf & lt);
                a.far_node[pos] = s;
            }
            if (cls == 2) a.near_key[no + nn + __popc(mn & lt)] = (uint32_t)a.node_leaf[s];
        } else if (cls == 2) {
            nsrc += S.end - S.beg;
        }
        nf += __popc(mf);
        nn += __popc(mn);
        // expanded nodes push their massive children (massless ones would be skipped anyway)
        const int mine = cls == 3 ? __popc(S.mask) : 0;
        int at = mine;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, at, o);
            if (lane >= o) at += u;
        }
        const int add = __shfl_sync(0xffffffffu, at, 31);
        if (top + add > kWalkStack) {
            pend = cls == 3 ? s : -1;
            pmask = cls == 3 ? S.mask : 0;
            pchild = cls == 3 ? S.child : 0;
            break;
        }
        if (cls == 3) {
            at = top + at - mine;
            for (int c = 7; c >= 0; --c)
                if (S.mask >> c & 1) stk[at++] = S.child + c;
        }
        top += add;
        __syncwarp();
    }
    if (top > 0 || __any_sync(0xffffffffu, pend >= 0)) {
        // overflow: each lane walks its pending children and its share of the stack depth
        // first with a private stack -- once to count, and in the fill pass once more to
        // write at the lane's place (lanes in order), so the list order is deterministic
        int st[kStack];
        auto lane_walk = [&](bool write, int fpos, int npos, int& lf, int& ln) {
            lf = ln = 0;
            for (int i = lane - 32; i < top; i += 32) {
                int sp = 0;
                if (i < 0) {
                    if (pend < 0) continue;
                    for (int c = 7; c >= 0; --c)
                        if (pmask >> c & 1) st[sp++] = pchild + c;
                } else {
                    st[sp++] = stk[i];
                }
                while (sp > 0) {
                    const int s = st[--sp];
                    const WalkNode S = a.wn[s];
                    const int cls = classify(T, t, S, s, a.theta);
                    if (cls == 1) {
                        if (write) a.far_node[fpos + lf] = s;
                        ++lf;
                    } else if (cls == 2) {
                        if (write) a.near_key[npos + ln] = (uint32_t)a.node_leaf[s];
                        else nsrc += S.end - S.beg;
                        ++ln;
                    } else if (cls == 3) {
                        for (int c = 7; c >= 0; --c)
                            if (S.mask >> c & 1) st[sp++] = S.child + c;
                    }
                }
            }
        };
        int lf, ln;
        lane_walk(false, 0, 0, lf, ln);
        int ef = lf, en = ln;  // inclusive prefix sums over the lanes
        for (int o = 1; o < 32; o <<= 1) {
            const int uf = __shfl_up_sync(0xffffffffu, ef, o), un = __shfl_up_sync(0xffffffffu, en, o);
            if (lane >= o) {
                ef += uf;
                en += un;
            }
        }
        if (FILL) {
            int lf2, ln2;
            nsrc = 0;
            lane_walk(true, fo + nf + ef - lf, no + nn + en - ln, lf2, ln2);
        }
        nf += __shfl_sync(0xffffffffu, ef, 31);
        nn += __shfl_sync(0xffffffffu, en, 31);
    }
    if constexpr (FILL) {
        // the near list into the reference's depth-first order (leaf ordinals are depth-first
        // numbers)
        __syncwarp();
        if (nn <= kSortCap) {
            sort_into(a.near_key + no, nn, reinterpret_cast<uint64_t*>(stk), lane, a.near_leaf + no);
        } else if (lane == 0) {
            a.long_leaf[atomicAdd(a.long_count, 1)] = l;  // sorted by long_sort_kernel
        }
    } else {
        for (int o = 16; o > 0; o >>= 1) nsrc += __shfl_xor_sync(0xffffffffu, nsrc, o);
        if (lane != 0) return;
        a.far_cnt[l] = nf;
        a.near_cnt[l] = nn;
        // far-field work items: only leaves with a target in range
        const int tb = a.leaf_off[l], te = a.leaf_off[l + 1];
        bool any = false;
        for (int k = tb; k < te && !any; ++k) any = a.leaf_part[k] >= a.t_begin && a.leaf_part[k] < a.t_end;
        const int nch = (any && nf > 0) ? (nf + kM2PChunk - 1) / kM2PChunk : 0;
        const int slots = nch > 1 ? nch * (te - tb) : 0;
        a.item_cnt[l] = nch;
        a.slot_cnt[l] = slots;
        atomicAdd(&a.totals[0], (unsigned long long)nf);
        atomicAdd(&a.totals[1], (unsigned long long)nn);
        atomicAdd(&a.totals[2], (unsigned long long)nch);
        atomicAdd(&a.totals[3], (unsigned long long)slots);
        atomicAdd(&a.totals[4], (unsigned long long)nf * (unsigned long long)(te - tb));
        atomicAdd(&a.totals[5], (unsigned long long)nsrc * (unsigned long long)(te - tb));
    }
}

// Near lists longer than a warp's buffer: one CTA per list.  Runs of kLongSort ordinals
// are sorted by a bitonic network in shared memory and written back in place; each ordinal's
// final place is then the sum over the runs of the number of smaller ordinals in the run
// (binary searches; the ordinals are distinct).
constexpr int kLongSort = 8192;
__global__ void __launch_bounds__(1024) long_sort_kernel(const TreeListArgs a) {
    __shared__ uint32_t s_key[kLongSort];
    const int n_long = *a.long_count;
    for (int q = blockIdx.x; q < n_long; q += gridDim.x) {
        const int l = a.long_leaf[q];
        const int no = a.near_off[l], n = a.near_off[l + 1] - no;
        uint64_t* v = a.near_key + no;
        const int runs = (n + kLongSort - 1) / kLongSort;
        for (int r = 0; r < runs; ++r) {
            const int b = r * kLongSort, m = min(kLongSort, n - b);
            int P = 1;
            while (P < m) P <<= 1;
            for (int i = threadIdx.x; i < P; i += 1024) s_key[i] = i < m ? (uint32_t)v[b + i] : 0xffffffffu;
            __syncthreads();
            for (int k = 2; k <= P; k <<= 1)
                for (int j = k >> 1; j > 0; j >>= 1) {
                    for (int i = threadIdx.x; i < P; i += 1024) {
                        const int mm = i ^ j;
                        if (mm > i) {
                            const uint32_t x = s_key[i], y = s_key[mm];
                            if ((x > y) == ((i & k) == 0)) {
                                s_key[i] = y;
                                s_key[mm] = x;
                            }
                        }
                    }
                    __syncthreads();
                }
            if (runs == 1) {
                for (int i = threadIdx.x; i < m; i += 1024) a.near_leaf[no + i] = (int32_t)s_key[i];
            } else {
                for (int i = threadIdx.x; i < m; i += 1024) v[b + i] = s_key[i];
            }
            __syncthreads();
        }
        if (runs == 1) continue;
        __threadfence_block();
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += 1024) {
            const uint64_t key = v[i];
            int pos = 0;
            for (int r = 0; r < runs; ++r) {
                int lo = r * kLongSort, hi = min(n, lo + kLongSort);
                const int base = lo;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (v[mid] < key) lo = mid + 1;
                    else hi = mid;
                }
                pos += lo - base;
            }
            a.near_leaf[no + pos] = (int32_t)(uint32_t)key;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) items_kernel(const TreeListArgs a, int n_leaves) {
    const int l = blockIdx.x * 256 + threadIdx.x;
    if (l >= min(n_leaves, a.start_ord[a.n]) || (a.overflow && *a.overflow)) return;
    const int nch = a.item_cnt[l];
    const int fb = a.far_off[l], fe = a.far_off[l + 1];
    M2PItem* items = (M2PItem*)a.items;
    for (int c = 0; c < nch; ++c) {
        M2PItem it;
        it.leaf = l;
        it.fb = fb + c * kM2PChunk;
        it.fe = min(fe, it.fb + kM2PChunk);
        it.chunk = c;
        it.nchunks = nch;
        it.pad = 0;
        it.scratch = nch > 1 ? a.slot_off[l] : 0;
        items[a.item_off[l] + c] = it;
    }
}

// Far-field items, largest first (cost = targets x nodes): fewer long items at the tail.
// Sort keys: the cost of the real items (n_real of them, from the device count when given) on
// a log scale with four steps per octave (1..127, 7 bits: one radix pass), 0 for the rest of
// the capacity, so that the real items come first, largest first.  The order only balances
// the blocks' work: a leaf's partial sums are added in chunk order whatever it is.
__global__ void __launch_bounds__(256) item_cost_kernel(const M2PItem* items, const int32_t* leaf_off, int n,
                                                        const unsigned long long* n_real, const int* overflow,
                                                        uint32_t* cost, int32_t* idx) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k >= n) return;
    const int real = (overflow && *overflow) ? 0 : n_real ? (int)min(*n_real, (unsigned long long)n) : n;
    uint32_t c = 0;
    if (k < real) {
        const M2PItem it = items[k];
        const uint32_t v = min((uint32_t)(leaf_off[it.leaf + 1] - leaf_off[it.leaf]) * (uint32_t)(it.fe - it.fb) + 1u,
                               0x7fffffffu);
        const int msb = 31 - __clz(v);
        c = v < 4u ? v : (uint32_t)(msb * 4 + ((v >> (msb - 2)) & 3));
    }
    cost[k] = c;
    idx[k] = k;
}

// Marks an overflow when a list or item pool reserved by capacity is too small for this
// evaluation's totals, or the topology build could not complete on the device.
__global__ void pool_check_kernel(const TreeListArgs a, const int32_t* tree_hdr) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const unsigned long long* t = a.totals;
    if (a.need) {
        atomicMax(&a.need[0], (unsigned long long)(tree_hdr[0] > 0 ? tree_hdr[0] : 0));
        for (int k = 0; k < 4; ++k) atomicMax(&a.need[1 + k], t[k]);
        // levels of the tree; a tree cut short by too few sorted key levels asks for all
        atomicMax(&a.need[5], (unsigned long long)(tree_hdr[2] & 4 ? kKeyLevels : max(tree_hdr[1], 0)));
    }
    if (t[0] > (unsigned long long)a.far_cap || t[1] > (unsigned long long)a.near_cap ||
        t[2] > (unsigned long long)a.item_cap || t[3] > (unsigned long long)a.slot_cap || tree_hdr[2] != 0) {
        *a.overflow = 1;
        if (a.overflow_sticky) atomicOr(a.overflow_sticky, tree_hdr[2] & 1 ? 3 : 1);  // bit 1: too deep
    }
}

__global__ void __launch_bounds__(256) item_gather_kernel(const M2PItem* items, const int32_t* idx, int n,
                                                          M2PItem* out) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k < n) out[k] = items[idx[k]];
}

size_t scan_bytes(int count) {
    size_t b = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b, (const int32_t*)nullptr, (int32_t*)nullptr, count);
    return b;
}

// The four per-leaf counts of the list pass (far, near, work items, partial-sum slots)
// scanned together: one exclusive scan of 4-tuples, element-wise sums.
using Count4 = thrust::tuple<int32_t, int32_t, int32_t, int32_t>;
struct Sum4 {
    __host__ __device__ Count4 operator()(const Count4& a, const Count4& b) const {
        return Count4(thrust::get<0>(a) + thrust::get<0>(b), thrust::get<1>(a) + thrust::get<1>(b),
                      thrust::get<2>(a) + thrust::get<2>(b), thrust::get<3>(a) + thrust::get<3>(b));
    }
};

cudaError_t scan4(void* temp, size_t& bytes, const int32_t* const cnt[4], int32_t* const off[4], int count,
                  cudaStream_t st) {
    auto in = thrust::make_zip_iterator(thrust::make_tuple(cnt[0], cnt[1], cnt[2], cnt[3]));
    auto out = thrust::make_zip_iterator(thrust::make_tuple(off[0], off[1], off[2], off[3]));
    return cub::DeviceScan::ExclusiveScan(temp, bytes, in, out, Sum4{}, Count4(0, 0, 0, 0), count, st);
}

size_t scan4_bytes(int count) {
    size_t b = 0;
    const int32_t* cnt[4] = {nullptr, nullptr, nullptr, nullptr};
    int32_t* off[4] = {nullptr, nullptr, nullptr, nullptr};
    scan4(nullptr, b, cnt, off, count, nullptr);
    return b;
}

}  // namespace

// Temporary storage of launch_tree_build: the split flags / their scan (kKeyLevels n + 1 ints),
// the list of splitting nodes (at most kKeyLevels (n / (cap + 1) + 1): the depth-L prefixes that
// split hold more than cap bodies each and are disjoint), then the radix sort's or the scan's
// own storage (one after the other, sharing the space).
namespace {
int split_capacity(int32_t n, int64_t cap) {
    const int64_t c = (int64_t)kKeyLevels * ((int64_t)n / (std::max<int64_t>(cap, 0) + 1) + 1);
    return (int)std::min<int64_t>(c, 0x7fffffff);
}
}  // namespace

size_t tree_build_temp_bytes(int32_t n, int64_t cap) {
    size_t b = 0;
    cub::DoubleBuffer<uint64_t> k(nullptr, nullptr);
    cub::DoubleBuffer<int32_t> v(nullptr, nullptr);
    cub::DeviceRadixSort::SortPairs(nullptr, b, k, v, n, 0, 3 * kKeyLevels);
    size_t sb = 0;
    const int items = kKeyLevels * n + 1;
    cub::DeviceScan::ExclusiveSum(nullptr, sb, (int32_t*)nullptr, (int32_t*)nullptr, items);
    const size_t flags = ((size_t)items * sizeof(int32_t) + 255) & ~(size_t)255;
    const size_t splits = ((size_t)split_capacity(n, cap) * sizeof(int32_t) + 255) & ~(size_t)255;
    return flags + splits + std::max((b + 255) & ~(size_t)255, sb);
}

cudaError_t launch_tree_build(const TreeBuildArgs& t, void* temp, size_t temp_bytes, cudaStream_t st) {
    const int items = kKeyLevels * t.n + 1;
    const size_t flag_bytes = ((size_t)items * sizeof(int32_t) + 255) & ~(size_t)255;
    const int split_cap = split_capacity(t.n, t.cap);
    const size_t split_bytes = ((size_t)split_cap * sizeof(int32_t) + 255) & ~(size_t)255;
    int32_t* flags = (int32_t*)temp;
    int32_t* split_pos = (int32_t*)((char*)temp + flag_bytes);
    void* work = (char*)temp + flag_bytes + split_bytes;
    size_t work_bytes = temp_bytes - flag_bytes - split_bytes;
    cudaError_t e = cudaMemsetAsync(t.hdr, 0, 3 * sizeof(int32_t), st);
    if (e != cudaSuccess) return e;
    bbox_partial_kernel<<<kBboxBlocks, kBboxThreads, 0, st>>>(t);
    bbox_final_kernel<<<1, kBboxThreads, 0, st>>>(t, kBboxBlocks);
    keys_kernel<<<(t.n + 255) / 256, 256, 0, st>>>(t);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    cub::DoubleBuffer<uint64_t> k(t.keys, t.keys_alt);
    cub::DoubleBuffer<int32_t> v(t.idx, t.perm);
    const int sorted = t.key_levels > 0 ? std::min(t.key_levels, kKeyLevels) : kKeyLevels;
    if ((e = cub::DeviceRadixSort::SortPairs(work, work_bytes, k, v, t.n, 3 * (kKeyLevels - sorted), 3 * kKeyLevels,
                                             st)) != cudaSuccess)
        return e;
    if (v.Current() != t.perm) gather_perm_kernel<<<(t.n + 255) / 256, 256, 0, st>>>(v.Current(), t.perm, t.n);
    split_flags_kernel<<<(t.n + 255) / 256, 256, 0, st>>>(t, k.Current(), flags);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    work_bytes = temp_bytes - flag_bytes - split_bytes;
    if ((e = cub::DeviceScan::ExclusiveSum(work, work_bytes, flags, flags, items, st)) != cudaSuccess) return e;
    tree_levels_kernel<<<1, 32, 0, st>>>(t, flags);
    split_list_kernel<<<(t.n + 255) / 256, 256, 0, st>>>(t, flags, split_pos, split_cap);
    tree_init_kernel<<<148 * 4, 256, 0, st>>>(t);
    tree_children_kernel<<<148 * 8, 256, 0, st>>>(t, k.Current(), flags, split_pos, split_cap);
    return cudaGetLastError();
}

cudaError_t launch_tree_leaf_order(const TreeBuildArgs& t, int32_t n_nodes, void* temp, size_t temp_bytes,
                                   cudaStream_t st) {
    (void)temp;
    (void)temp_bytes;
    leaf_sort_kernel<<<(n_nodes + 7) / 8, 256, 0, st>>>(t, n_nodes);
    return cudaGetLastError();
}

size_t tree_list_temp_bytes(int32_t n, int32_t n_nodes) {
    return std::max({scan_bytes(n + 1), scan_bytes(n_nodes + 1), scan4_bytes(n_nodes + 1)});
}

// Both walk kernels prefer a 60% shared-memory carveout (8 blocks of 17 KiB; the rest is L1).
static cudaError_t walk_carveout() {
    static cudaError_t once = [] {
        cudaError_t e = cudaFuncSetAttribute(walk_kernel<false>, cudaFuncAttributePreferredSharedMemoryCarveout, 60);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(walk_kernel<true>, cudaFuncAttributePreferredSharedMemoryCarveout, 60);
        return e;
    }();
    return once;
}

cudaError_t launch_tree_lists_count(const TreeListArgs& a, void* temp, size_t temp_bytes, cudaStream_t st) {
    cudaError_t e;
    const size_t nb = (size_t)(a.n + 1) * sizeof(int32_t), lb = (size_t)(a.n_nodes + 1) * sizeof(int32_t);
    if ((e = cudaMemsetAsync(a.start_flag, 0, nb, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(a.keep, 0, nb, st)) != cudaSuccess) return e;
    for (int32_t* p : {a.far_cnt, a.near_cnt, a.item_cnt, a.slot_cnt})
        if ((e = cudaMemsetAsync(p, 0, lb, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(a.totals, 0, 6 * sizeof(unsigned long long), st)) != cudaSuccess) return e;
    const int gn = (a.n_nodes + 255) / 256;
    leaf_mark_kernel<<<gn, 256, 0, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    size_t tb = temp_bytes;
    if ((e = cub::DeviceScan::ExclusiveSum(temp, tb, a.start_flag, a.start_ord, a.n + 1, st)) != cudaSuccess) return e;
    tb = temp_bytes;
    if ((e = cub::DeviceScan::ExclusiveSum(temp, tb, a.keep, a.newpos, a.n + 1, st)) != cudaSuccess) return e;
    leaf_emit_kernel<<<gn, 256, 0, st>>>(a);
    walk_pack_kernel<<<gn, 256, 0, st>>>(a);
    if ((e = walk_carveout()) != cudaSuccess) return e;
    walk_kernel<false><<<(a.n_nodes + kWalkThreads / 32 - 1) / (kWalkThreads / 32), kWalkThreads, 0, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int32_t* const cnt[4] = {a.far_cnt, a.near_cnt, a.item_cnt, a.slot_cnt};
    int32_t* const off[4] = {a.far_off, a.near_off, a.item_off, a.slot_off};
    tb = temp_bytes;
    return scan4(temp, tb, cnt, off, a.n_nodes + 1, st);
}

cudaError_t launch_tree_massive(const TreeListArgs& a, void* temp, size_t temp_bytes, cudaStream_t st) {
    // the flags go to start_flag (free until the list pass clears it), the counts to mprefix
    massive_flags_kernel<<<(a.n + 256) / 256, 256, 0, st>>>(a, a.start_flag);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    size_t tb = temp_bytes;
    return cub::DeviceScan::ExclusiveSum(temp, tb, a.start_flag, a.mprefix, a.n + 1, st);
}

cudaError_t launch_pool_check(const TreeListArgs& a, const int32_t* tree_hdr, cudaStream_t st) {
    pool_check_kernel<<<1, 32, 0, st>>>(a, tree_hdr);
    return cudaGetLastError();
}

cudaError_t launch_tree_lists_fill(const TreeListArgs& a, int32_t n_leaves, cudaStream_t st) {
    if (n_leaves == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(a.long_count, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    walk_kernel<true><<<(n_leaves + kWalkThreads / 32 - 1) / (kWalkThreads / 32), kWalkThreads, 0, st>>>(a);
    long_sort_kernel<<<296, 1024, 0, st>>>(a);
    items_kernel<<<(n_leaves + 255) / 256, 256, 0, st>>>(a, n_leaves);
    return cudaGetLastError();
}

size_t item_order_temp_bytes(int32_t n_items) {
    size_t b = 0;
    cub::DoubleBuffer<uint32_t> k(nullptr, nullptr);
    cub::DoubleBuffer<int32_t> v(nullptr, nullptr);
    cub::DeviceRadixSort::SortPairsDescending(nullptr, b, k, v, n_items);
    return b;
}

cudaError_t launch_item_order(const M2PItem* items, const int32_t* leaf_off, int32_t n_items,
                              const unsigned long long* n_real, const int* overflow, uint32_t* cost,
                              uint32_t* cost_alt, int32_t* idx, int32_t* idx_alt, void* temp, size_t temp_bytes,
                              M2PItem* out, cudaStream_t st) {
    if (n_items == 0) return cudaSuccess;
    const int g = (n_items + 255) / 256;
    item_cost_kernel<<<g, 256, 0, st>>>(items, leaf_off, n_items, n_real, overflow, cost, idx);
    cub::DoubleBuffer<uint32_t> k(cost, cost_alt);
    cub::DoubleBuffer<int32_t> v(idx, idx_alt);
    cudaError_t e = cub::DeviceRadixSort::SortPairsDescending(temp, temp_bytes, k, v, n_items, 0, 7, st);
    if (e != cudaSuccess) return e;
    item_gather_kernel<<<g, 256, 0, st>>>(items, v.Current(), n_items, out);
    return cudaGetLastError();
}

}  // namespace gx
